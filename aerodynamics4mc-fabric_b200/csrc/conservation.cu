// Global mass and momentum sums of a context's streamed state, in FP64.
//
// Each thread pulls one cell's 27 incoming populations (the state the next
// step collides; solids excluded), forms rho and rho*u in FP32 as the step
// does, and accumulates them in double. Warp sums use shuffles, block sums go
// through shared memory, and each block writes its four partial sums to a
// scratch buffer; a second single-block kernel reduces the partials into the
// four outputs. Both launches are stream-ordered, so the result is ready when
// the stream reaches it.
#include "conservation.cuh"
#include "ip_launch.h"

namespace aero {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of 4 doubles; result valid in thread 0.
__device__ __forceinline__ void block_sum4(double (&v)[4]) {
    __shared__ double sh[4][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) sh[k][warp] = v[k];
    }
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            double t = lane < nw ? sh[k][lane] : 0.0;
            v[k] = warp_sum(t);
        }
    }
}

__device__ __forceinline__ void accumulate_cell(const float (&f)[27], double (&acc)[4]) {
    RawMoments m;
    raw_moments27<false>(f, m);
    acc[0] += (double)m.r000;
    acc[1] += (double)m.r100;
    acc[2] += (double)m.r010;
    acc[3] += (double)m.r001;
}

__global__ void conservation_ab_kernel(int nx, int ny, int nz, const float* __restrict__ g,
                                       const uint32_t* __restrict__ flags, const uint8_t* __restrict__ obstacle,
                                       const float* __restrict__ ref_p, const FaceParams* __restrict__ F,
                                       double* __restrict__ partials, int direct) {
    const long long cells = (long long)nx * ny * nz;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x; cell < cells;
         cell += (long long)gridDim.x * blockDim.x) {
        const uint32_t w = flags[cell];
        if (w & kFlagSelfSolid) continue;
        const int z = (int)(cell % nz), y = (int)((cell / nz) % ny), x = (int)(cell / ((long long)ny * nz));
        float f[27];
        if (direct) {  // g holds the streamed state itself (after a halo exchange)
#pragma unroll
            for (int q = 0; q < 27; ++q) f[q] = g[(long long)q * cells + cell];
        } else {
            const PullView v{g, obstacle, ref_p, F, cells, nx, ny, nz};
            pull27(v, w, cell, x, y, z, f);
        }
        accumulate_cell(f, acc);
    }
    block_sum4(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) partials[(long long)blockIdx.x * 4 + k] = acc[k];
    }
}

template <class S>
__global__ void conservation_ip_kernel(const typename S::T* __restrict__ f, IpArgs a, double* __restrict__ partials) {
    const PadGeom G = a.g;
    const long long cells = (long long)G.nx * G.ny * G.nz;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x; cell < cells;
         cell += (long long)gridDim.x * blockDim.x) {
        const uint32_t w = a.flags_prev[cell];
        if (w & kFlagSelfSolid) continue;
        int x, y, z;
        cell_coords(G, cell, x, y, z);
        const int own = pad_index(G, x, y, z);
        const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
        float fl[27];
        ip_pull<S>(f, a, G, o, own, w, a.parity, fl);
        accumulate_cell(fl, acc);
    }
    block_sum4(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) partials[(long long)blockIdx.x * 4 + k] = acc[k];
    }
}

__global__ void reduce_partials_kernel(const double* __restrict__ partials, int n, double* __restrict__ out) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] += partials[(long long)i * 4 + k];
    }
    block_sum4(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) out[k] = acc[k];
    }
}

int conservation_blocks(long long cells) {
    const long long want = (cells + kConservationThreads - 1) / kConservationThreads;
    return (int)(want < kConservationMaxBlocks ? (want > 0 ? want : 1) : kConservationMaxBlocks);
}

cudaError_t launch_conservation_ab(int nx, int ny, int nz, const float* g, const uint32_t* flags,
                                   const uint8_t* obstacle, const float* ref_p, const FaceParams* face,
                                   double* partials, double* out, cudaStream_t s, int direct) {
    const int blocks = conservation_blocks((long long)nx * ny * nz);
    conservation_ab_kernel<<<blocks, kConservationThreads, 0, s>>>(nx, ny, nz, g, flags, obstacle, ref_p, face, partials,
                                                                   direct);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    reduce_partials_kernel<<<1, 256, 0, s>>>(partials, blocks, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_conservation_ip(int variant, const void* f, const IpArgs& a, double* partials, double* out,
                                   cudaStream_t s) {
    const int blocks = conservation_blocks((long long)a.g.nx * a.g.ny * a.g.nz);
    if (variant == kIpF16Fast) {
        conservation_ip_kernel<StoreF16Dev><<<blocks, kConservationThreads, 0, s>>>(static_cast<const __half*>(f), a, partials);
    } else if (variant == kIpI16Fast) {
        conservation_ip_kernel<StoreI16Dev><<<blocks, kConservationThreads, 0, s>>>(static_cast<const short*>(f), a, partials);
    } else {
        conservation_ip_kernel<StoreF32><<<blocks, kConservationThreads, 0, s>>>(static_cast<const float*>(f), a, partials);
    }
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    reduce_partials_kernel<<<1, 256, 0, s>>>(partials, blocks, out);
    count_launch();
    return cudaGetLastError();
}

}  // namespace aero
