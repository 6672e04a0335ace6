// FP32-mixed instances of the godunov tile kernel: slopes, trace and Riemann
// fluxes in FP32 (contracted, fast division); conservative->primitive and the
// conservative accumulation into unew stay FP64.
#define RB_TILE_REAL float
#define RB_TILE_IS_MIXED 1
#define RB_TILE_LAUNCH launch_tile_mixed
#define RB_TILE_SMEM tile_smem_mixed
#define RB_STREAM_LAUNCH launch_stream_mixed
#define RB_STREAM_SMEM stream_smem_mixed
#define RB_BATCH_LAUNCH launch_batch_mixed
#include "tile_instances.inc"
