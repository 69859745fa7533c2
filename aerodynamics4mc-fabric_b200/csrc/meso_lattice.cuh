// D3Q19 mesoscale lattice and population storage policies, shared by the
// reference-order kernels (meso_exact.cu) and the packed two-cell step
// (meso_fast.cu).
#pragma once

#include <cuda_fp16.h>

#include "inplace27.cuh"

namespace aero {
namespace meso {

// lattice (native/src/aero_lbm_mesoscale.cpp:146-174): rest, 6 faces, 12 edges
__host__ __device__ constexpr int mcx(int q) {
    return (q == 1 || q == 7 || q == 9 || q == 11 || q == 13) ? 1 : ((q == 2 || q == 8 || q == 10 || q == 12 || q == 14) ? -1 : 0);
}
__host__ __device__ constexpr int mcy(int q) {
    return (q == 3 || q == 7 || q == 10 || q == 15 || q == 17) ? 1 : ((q == 4 || q == 8 || q == 9 || q == 16 || q == 18) ? -1 : 0);
}
__host__ __device__ constexpr int mcz(int q) {
    return (q == 5 || q == 11 || q == 14 || q == 15 || q == 18) ? 1 : ((q == 6 || q == 12 || q == 13 || q == 16 || q == 17) ? -1 : 0);
}
__host__ __device__ constexpr int mopp(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }
// same x and z component, opposite y component (specular reflection at the lid)
__host__ __device__ constexpr int mmirror(int q) {
    return q == 3 ? 4 : q == 4 ? 3 : q == 7 ? 9 : q == 9 ? 7 : q == 8 ? 10 : q == 10 ? 8
         : q == 15 ? 18 : q == 18 ? 15 : q == 16 ? 17 : q == 17 ? 16 : q;
}
static_assert(mcx(mmirror(7)) == 1 && mcy(mmirror(7)) == -1 && mcz(mmirror(16)) == -1 && mcy(mmirror(16)) == 1, "mirror");

__device__ __forceinline__ float mw(int q) { return q == 0 ? 1.0f / 3.0f : (q < 7 ? 1.0f / 18.0f : 1.0f / 36.0f); }
// Storage of one population: FP32 as is, FP16 deviations
// h = (f - w_q) * S / w_q with a per-grid power-of-two scale S, or the same
// deviation in 16-bit fixed point with S = 32767 / d_max (see StoreI16Dev).
struct MesoF32 {
    using T = float;
    __device__ __forceinline__ static float load(const float* __restrict__ p, int, float) { return __ldg(p); }
    __device__ __forceinline__ static void store(float* __restrict__ p, int, float v, float) { *p = v; }
};
struct MesoF16 {
    using T = __half;
    __device__ __forceinline__ static float load(const __half* __restrict__ p, int q, float inv_scale) {
        return fmaf(__half2float(__ldg(p)), mw(q) * inv_scale, mw(q));
    }
    __device__ __forceinline__ static void store(__half* __restrict__ p, int q, float v, float scale) {
        *p = __float2half_rn(fmaf(v, scale * (1.0f / mw(q)), -scale));
    }
};

struct MesoI16 {
    using T = short;
    __device__ __forceinline__ static float load(const short* __restrict__ p, int q, float inv_scale) {
        return fmaf((float)__ldg(p), mw(q) * inv_scale, mw(q));
    }
    __device__ __forceinline__ static void store(short* __restrict__ p, int q, float v, float scale) {
        *p = sat_round_s16(fmaf(v, scale * (1.0f / mw(q)), -scale));
    }
};

}  // namespace meso
}  // namespace aero
