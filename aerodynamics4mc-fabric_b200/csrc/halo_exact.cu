// Halo exchange between two overlapping bricks (aero_lbm_exchange_halo_layers_rect,
// native/src/aero_lbm_jni.cpp:8136-8426, 9692-9780): cubic contexts of edge
// n with a halo of h layers and a core of n - 2h; the second context lies at
// offset (ox, oy, oz) in {-1, 0, 1}^3 (not all 0) from the first. Per axis the
// slab is (halo_exchange_slab_bounds, jni.cpp:8201-8264)
//   offset -1: first[h, 2h)       -> second[n-h, n),  second[n-2h, n-h) -> first[0, h)
//   offset  0: first[h, n-h)      -> second[h, n-h),  and back
//   offset +1: first[n-2h, n-h)   -> second[0, h),    second[h, 2h)     -> first[n-h, n)
// and every cell of the slab gets the other context's 27 streamed
// populations (the reference's f) and its temperature.
//
// In-place contexts keep the streamed populations in the incoming slots of
// the next step's parity between calls (the equilibrium-face sources a call
// leaves are pre-filled before anything reads them), so a cell's f is read and written
// through the same slot map the step kernel pulls with (bounce-back bits of
// the last classification). Solid cells of an in-place context keep their
// populations beside the lattice (IpArgs::solid_f, at a canonical parity;
// rest equilibrium while that store does not exist yet), and the exchange
// reads and writes them there. Two-buffer contexts materialise f
// (the pull of their post-collision state) into the spare buffer first; the
// next call then collides f directly. Built with --fmad=false: that pull
// evaluates the face rules (convective outflow, equilibria) operation by
// operation, as the step kernel of the reference-order collision does.
#include "halo.cuh"

#include <algorithm>

#include "d3q27_step.cuh"
#include "inplace27.cuh"

namespace aero {
namespace {

template <class S>
struct IpSide {
    typename S::T* f;
    PadGeom g;
    const uint32_t* flags;
    int parity;
    Fp16Scale sc;
    float* solid_f;
};

template <class S>
__device__ __forceinline__ void halo_ip_cell(const IpSide<S>& src, const IpSide<S>& dst, const HaloSlab& slab, int i) {
    const int n_slab = slab.size[0] * slab.size[1] * slab.size[2];
    if (i >= n_slab) return;
    const int lz = i % slab.size[2], ly = (i / slab.size[2]) % slab.size[1], lx = i / (slab.size[2] * slab.size[1]);
    const int sx = slab.src[0] + lx, sy = slab.src[1] + ly, sz = slab.src[2] + lz;
    const int dx = slab.dst[0] + lx, dy = slab.dst[1] + ly, dz = slab.dst[2] + lz;
    const long long dcell = ((long long)dx * dst.g.ny + dy) * dst.g.nz + dz;
    const uint32_t wd = dst.flags[dcell];
    const bool dst_solid = (wd & kFlagSelfSolid) != 0;
    if (dst_solid && !dst.solid_f) return;  // never-opened solid cells: at rest, like the source would have to be
    const long long scell = ((long long)sx * src.g.ny + sy) * src.g.nz + sz;
    const uint32_t ws = src.flags[scell];
    const bool src_solid = (ws & kFlagSelfSolid) != 0;
    const NeighbourOffsets os = neighbour_offsets(src.g, sx, sy, sz);
    const NeighbourOffsets od = neighbour_offsets(dst.g, dx, dy, dz);
    const int own_s = pad_index(src.g, sx, sy, sz), own_d = pad_index(dst.g, dx, dy, dz);
    const long long scells = (long long)src.g.nx * src.g.ny * src.g.nz, dcells = (long long)dst.g.nx * dst.g.ny * dst.g.nz;
    // all 27 loads first (independent, in flight together), then the stores
    float v[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        v[q] = q_w(q);
        if (!src_solid) {
            int c, d;
            incoming_slot(os, own_s, q, src.parity, (ws >> q) & 1u, c, d);
            v[q] = S::load(src.f + (long long)d * src.g.pcells + c, q, src.sc);
        } else if (src.solid_f) {
            v[q] = src.solid_f[(long long)solid_slot(q, src.parity) * scells + scell];
        }
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        if (dst_solid) {
            dst.solid_f[(long long)solid_slot(q, dst.parity) * dcells + dcell] = v[q];
            continue;
        }
        int c, d;
        incoming_slot(od, own_d, q, dst.parity, (wd >> q) & 1u, c, d);
        S::store(dst.f + (long long)d * dst.g.pcells + c, q, v[q], dst.sc);
    }
}

template <class S>
__global__ void halo_ip_kernel(IpSide<S> src, IpSide<S> dst, HaloSlab slab) {
    halo_ip_cell(src, dst, slab, blockIdx.x * blockDim.x + threadIdx.x);
}

// One job per blockIdx.y (jobs in device memory).
template <class S>
__global__ void halo_ip_batch_kernel(const HaloIpJob* __restrict__ jobs) {
    const HaloIpJob& J = jobs[blockIdx.y];
    const IpSide<S> src{static_cast<typename S::T*>(J.src.f), J.src.g, J.src.flags, J.src.parity, J.src.sc, J.src.solid_f};
    const IpSide<S> dst{static_cast<typename S::T*>(J.dst.f), J.dst.g, J.dst.flags, J.dst.parity, J.dst.sc, J.dst.solid_f};
    halo_ip_cell(src, dst, J.slab, blockIdx.x * blockDim.x + threadIdx.x);
}

// Two-buffer contexts: f = the pull of the post-collision state.
__global__ void materialise_ab_kernel(int nx, int ny, int nz, const float* __restrict__ g, const uint32_t* __restrict__ flags,
                                      const uint8_t* __restrict__ obstacle, const float* __restrict__ ref_p,
                                      const FaceParams* __restrict__ F, float* __restrict__ f_out) {
    const long long cells = (long long)nx * ny * nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    int x, y, z;
    cell_xyz32(cell, ny, nz, x, y, z);
    float f[27];
    const PullView v{g, obstacle, ref_p, F, cells, nx, ny, nz};
    pull27(v, flags[cell], cell, x, y, z, f);
#pragma unroll
    for (int q = 0; q < 27; ++q) f_out[(long long)q * cells + cell] = f[q];
}

// Slab copy of `comps` per-cell components stored component-major
// (populations: 27 x cells; temperature: 1 x cells).
__global__ void halo_soa_kernel(const float* __restrict__ src, float* __restrict__ dst, long long cells, int ny, int nz,
                                int comps, HaloSlab slab) {
    const int n_slab = slab.size[0] * slab.size[1] * slab.size[2];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_slab) return;
    const int lz = i % slab.size[2], ly = (i / slab.size[2]) % slab.size[1], lx = i / (slab.size[2] * slab.size[1]);
    const long long scell = ((long long)(slab.src[0] + lx) * ny + slab.src[1] + ly) * nz + slab.src[2] + lz;
    const long long dcell = ((long long)(slab.dst[0] + lx) * ny + slab.dst[1] + ly) * nz + slab.dst[2] + lz;
    for (int k = 0; k < comps; ++k) dst[(long long)k * cells + dcell] = src[(long long)k * cells + scell];
}

__global__ void halo_soa_batch_kernel(const HaloSoaJob* __restrict__ jobs) {
    const HaloSoaJob& J = jobs[blockIdx.y];
    const HaloSlab& slab = J.slab;
    const int n_slab = slab.size[0] * slab.size[1] * slab.size[2];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_slab) return;
    const int lz = i % slab.size[2], ly = (i / slab.size[2]) % slab.size[1], lx = i / (slab.size[2] * slab.size[1]);
    const long long scell = ((long long)(slab.src[0] + lx) * J.ny + slab.src[1] + ly) * J.nz + slab.src[2] + lz;
    const long long dcell = ((long long)(slab.dst[0] + lx) * J.ny + slab.dst[1] + ly) * J.nz + slab.dst[2] + lz;
    J.dst[dcell] = J.src[scell];
}

unsigned blocks_for(const HaloSlab& s) {
    const long long n = (long long)s.size[0] * s.size[1] * s.size[2];
    return (unsigned)((n + 127) / 128);
}

template <class S>
cudaError_t halo_ip_t(const HaloIpSide& a, const HaloIpSide& b, const HaloSlab& ab, const HaloSlab& ba, cudaStream_t s) {
    const IpSide<S> A{static_cast<typename S::T*>(a.f), a.g, a.flags, a.parity, a.sc, a.solid_f};
    const IpSide<S> B{static_cast<typename S::T*>(b.f), b.g, b.flags, b.parity, b.sc, b.solid_f};
    halo_ip_kernel<S><<<blocks_for(ab), 128, 0, s>>>(A, B, ab);
    count_launch();
    halo_ip_kernel<S><<<blocks_for(ba), 128, 0, s>>>(B, A, ba);
    count_launch();
    return cudaGetLastError();
}

}  // namespace

bool halo_slabs(int n, int halo_layers, int ox, int oy, int oz, HaloSlab& first_to_second, HaloSlab& second_to_first) {
    const int halo = std::max(1, std::min(halo_layers, n / 2 - 1));
    const int core = n - 2 * halo;
    if (core <= 0) return false;
    const int off[3] = {ox, oy, oz};
    for (int k = 0; k < 3; ++k) {
        int fs, sd, ss, fd, sz;
        switch (off[k]) {
            case -1: fs = halo; sd = n - halo; ss = core; fd = 0; sz = halo; break;
            case 0: fs = halo; sd = halo; ss = halo; fd = halo; sz = core; break;
            case 1: fs = core; sd = 0; ss = halo; fd = n - halo; sz = halo; break;
            default: return false;
        }
        first_to_second.src[k] = fs;
        first_to_second.dst[k] = sd;
        second_to_first.src[k] = ss;
        second_to_first.dst[k] = fd;
        first_to_second.size[k] = second_to_first.size[k] = sz;
    }
    return true;
}

cudaError_t launch_halo_ip(int storage, const HaloIpSide& a, const HaloIpSide& b, const HaloSlab& ab, const HaloSlab& ba,
                           cudaStream_t s) {
    if (storage == 0) return halo_ip_t<StoreF32>(a, b, ab, ba, s);
    if (storage == 1) return halo_ip_t<StoreF16Dev>(a, b, ab, ba, s);
    return halo_ip_t<StoreI16Dev>(a, b, ab, ba, s);
}

cudaError_t launch_halo_ip_batch(int storage, const HaloIpJob* jobs, int njobs, int max_slab, cudaStream_t s) {
    if (njobs <= 0 || max_slab <= 0) return cudaSuccess;
    const dim3 grid((unsigned)((max_slab + 127) / 128), (unsigned)njobs);
    if (storage == 0) halo_ip_batch_kernel<StoreF32><<<grid, 128, 0, s>>>(jobs);
    else if (storage == 1) halo_ip_batch_kernel<StoreF16Dev><<<grid, 128, 0, s>>>(jobs);
    else halo_ip_batch_kernel<StoreI16Dev><<<grid, 128, 0, s>>>(jobs);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_halo_soa_batch(const HaloSoaJob* jobs, int njobs, int max_slab, cudaStream_t s) {
    if (njobs <= 0 || max_slab <= 0) return cudaSuccess;
    const dim3 grid((unsigned)((max_slab + 127) / 128), (unsigned)njobs);
    halo_soa_batch_kernel<<<grid, 128, 0, s>>>(jobs);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_materialise_ab(BrickDims d, const float* g, const uint32_t* flags, const uint8_t* obstacle,
                                  const float* ref_p, const FaceParams* face, float* f_out, cudaStream_t s) {
    if (d.cells <= 0) return cudaSuccess;
    materialise_ab_kernel<<<(unsigned)((d.cells + 127) / 128), 128, 0, s>>>(d.nx, d.ny, d.nz, g, flags, obstacle, ref_p,
                                                                             face, f_out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_halo_soa(const float* a, float* b, long long cells, int ny, int nz, int comps, const HaloSlab& ab,
                            cudaStream_t s) {
    halo_soa_kernel<<<blocks_for(ab), 128, 0, s>>>(a, b, cells, ny, nz, comps, ab);
    count_launch();
    return cudaGetLastError();
}

}  // namespace aero
