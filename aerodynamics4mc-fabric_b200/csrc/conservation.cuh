// FP64 mass/momentum sums of a context's streamed state.
#pragma once

#include <cuda_runtime.h>

#include "d3q27_inplace.cuh"

namespace aero {

constexpr int kConservationThreads = 256;
constexpr int kConservationMaxBlocks = 1184;  // 148 SMs x 8

// Blocks the first stage uses for `cells` cells (= partial-sum slots; the
// scratch buffer holds 4 doubles per block).
int conservation_blocks(long long cells);

// out[0..3] = sum rho, sum rho ux, sum rho uy, sum rho uz over fluid cells
// (device pointers; partials: scratch of 4 * conservation_blocks(cells) doubles).
// direct: g already holds the streamed state (no pull).
cudaError_t launch_conservation_ab(int nx, int ny, int nz, const float* g, const uint32_t* flags,
                                   const uint8_t* obstacle, const float* ref_p, const FaceParams* face,
                                   double* partials, double* out, cudaStream_t s, int direct = 0);
cudaError_t launch_conservation_ip(int variant, const void* f, const IpArgs& a, double* partials, double* out,
                                   cudaStream_t s);

}  // namespace aero
