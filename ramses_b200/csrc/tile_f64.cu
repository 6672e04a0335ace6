// FP64 drop-in instances of the godunov tile kernel. Compiled with
// --fmad=false: no multiply-add is contracted, so every flux and update is
// bit-identical to the reference's operation order.
#define RB_TILE_REAL double
#define RB_TILE_IS_MIXED 0
#define RB_TILE_LAUNCH launch_tile_f64
#define RB_TILE_SMEM tile_smem_f64
#define RB_STREAM_LAUNCH launch_stream_f64
#define RB_STREAM_SMEM stream_smem_f64
#define RB_BATCH_LAUNCH launch_batch_f64
#include "tile_instances.inc"
