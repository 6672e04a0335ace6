// tile_launch.h -- host-side launch interface of the godunov tile kernel for
// the two compute precisions (separate translation units so that the FP64
// unit is compiled without multiply-add contraction).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "rb_types.h"

namespace rb {

struct TileArgs;

struct TileShape {
  int tx, ty, tz;   // tile size in cells (even)
  int nthreads;     // CTA size
};

// Supported tile shapes, indexed by shape id.
constexpr int kNumTileShapes = 5;
constexpr TileShape kTileShapes[kNumTileShapes] = {
    {2, 2, 2, 64},    // one oct: the reference's per-oct stencil
    {4, 4, 4, 128},
    {8, 4, 4, 256},
    {8, 8, 4, 256},
    {8, 8, 8, 256},
};

size_t tile_smem_f64(int shape);
size_t tile_smem_mixed(int shape);
cudaError_t launch_tile_f64(int shape, const TileArgs& a, int grid, cudaStream_t s);
cudaError_t launch_tile_mixed(int shape, const TileArgs& a, int grid, cudaStream_t s);

// z-streaming kernel of complete levels: column shape (TX x TY cells) and the
// number of CTAs per SM the register allocation is bounded for. Shapes 5 and
// 6 are the FP32-mixed kernel of stream2_kernel.cuh (HLLC, minmod or moncen,
// MUSCL-Hancock only: stream2_supports).
struct StreamArgs;
constexpr int kNumStreamShapes = 7;
constexpr int kStreamShapes[kNumStreamShapes][3] = {{8, 8, 1}, {16, 8, 1}, {16, 16, 1}, {16, 8, 2}, {8, 8, 4},
                                                    {16, 8, 3}, {16, 8, 2}};
constexpr bool kStreamShapeV2[kNumStreamShapes] = {false, false, false, false, false, true, true};
inline bool stream2_supports(const rb_hydro_params& hp) {
  return hp.riemann == RB_RIEMANN_HLLC && (hp.slope_type == 1 || hp.slope_type == 2) &&
         hp.scheme == RB_SCHEME_MUSCL && hp.difmag <= 0.0 && !hp.pressure_fix;
}
cudaError_t launch_stream_f64(int shape, const StreamArgs& a, int grid, cudaStream_t s);
cudaError_t launch_stream_mixed(int shape, const StreamArgs& a, int grid, cudaStream_t s);
size_t stream_smem_f64(int shape);
size_t stream_smem_mixed(int shape);
// batched z-streaming step over many problems (serving)
struct BatchDesc;
cudaError_t launch_batch_f64(int shape, const rb_hydro_params& hp, const BatchDesc* desc, const int32_t* item_off,
                             int nprob, int grid, cudaStream_t s);
cudaError_t launch_batch_mixed(int shape, const rb_hydro_params& hp, const BatchDesc* desc,
                               const int32_t* item_off, int nprob, int grid, cudaStream_t s);

}  // namespace rb
