// In-place step with the populations streamed into shared memory by bulk
// asynchronous copies (cp.async.bulk, completion on an mbarrier): the
// factorised collision on two z-adjacent cells per thread in packed FP32, as
// step_ip2_kernel, but with the next tile's loads in flight while the current
// tile collides.
//
// Work unit: a tile of 64 consecutive cells of one (x, y) line (two per lane
// of one warp). Every incoming population of the tile's cells in direction q
// lies in ONE contiguous run of 64 elements of the population array: slot
// plane dir(q), memory line (x, y) or (x - cx, y - cy) (periodic x / y wrap
// at the line level), z shifted by -cz (the ghost layer absorbs z = -1 and
// z = nz). So a tile is 27 bulk copies (plus the tile's flags, mask,
// temperature and force words), issued by one lane; no register holds a
// load in flight. Each warp runs its own one-deep pipeline: wait for tile t,
// move it from shared memory into registers, issue tile t + warps, collide
// and store tile t.
//
// In-place safety: every slot is read and then written by exactly one cell
// per step (inplace27.cuh), and the copies of a tile read only slots that
// the tile's own cells read, plus at most 15 bytes of alignment slack at
// each end of a run, whose values are never used. Half-way bounce-back
// reads (the parity-flipped slot) come from global memory per lane.
//
// Bricks with a periodic z axis are not handled here (a run would wrap).
//
// Measured on B200 (128^3 terrain brick): 13.5 GLUPS FP32 / 11.5 FP16 against
// 17.6 / 20.4 for step_ip2_kernel's per-thread loads. The per-tile copy
// bookkeeping, the shared-memory pass and the one-deep per-warp pipeline add
// more issue time (~58% more instructions) than the hidden load latency saves,
// so this kernel is opt-in (aero_lbm_b200_set_streamed_step). Per-lane 16-byte
// cp.async chunks instead of bulk copies (AERO_IPA_BULK=0) measured slower.
#pragma once

#include <algorithm>

#include "d3q27_inplace.cuh"

namespace aero {

constexpr int kIpaTile = 64;     // cells per warp tile
constexpr int kIpaWarps = 4;     // warps per block
#ifndef AERO_IPA_MIN_BLOCKS
#define AERO_IPA_MIN_BLOCKS 4
#endif
constexpr int kIpaWaitLimit = 1 << 22;
#ifndef AERO_IPA_BULK
#define AERO_IPA_BULK 1
#endif  // mbarrier polls before a tile is declared lost

// Shared memory of one warp: 16-byte-aligned regions, each large enough for
// a run of kIpaTile elements starting anywhere inside a 16-byte granule.
template <class T>
struct IpaLayout {
    static constexpr int region(int bytes, int elem) { return ((16 - elem + bytes + 15) / 16) * 16; }
    static constexpr int kSeg = region(kIpaTile * (int)sizeof(T), (int)sizeof(T));
    static constexpr int kWord = region(kIpaTile * 4, 4);
    static constexpr int kFlags = 27 * kSeg;
    static constexpr int kObst = kFlags + kWord;
    static constexpr int kTemp = kObst + region(kIpaTile, 1);
    static constexpr int kForce = kTemp + kWord;
    static constexpr int kOffs = kForce + 3 * kWord;  // byte offsets of the runs: 0-26 populations, 27 flags,
                                                      // 28 mask, 29 temperature, 30-32 force
    static constexpr int kBar = kOffs + 48;
    static constexpr int kWarpBytes = kBar + 16;
    static_assert(kSeg % 16 == 0 && kWord % 16 == 0 && kOffs % 16 == 0 && kWarpBytes % 16 == 0, "16-byte regions");
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ipa_bar_init(uint32_t bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void ipa_bar_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool ipa_bar_try(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool ipa_bar_wait(uint32_t bar, uint32_t parity) {
    for (int i = 0; i < kIpaWaitLimit; ++i)
        if (ipa_bar_try(bar, parity)) return true;
    return false;
}

// Byte range [p, p + bytes) rounded out to 16-byte granules: start, size and
// the offset of p inside the copied run.
struct IpaRun {
    const void* src;
    uint32_t bytes;
    uint32_t off;
};
__device__ __forceinline__ IpaRun ipa_run(const void* p, uint32_t bytes) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uintptr_t a0 = a & ~(uintptr_t)15;
    return IpaRun{reinterpret_cast<const void*>(a0), (uint32_t)(((a + bytes + 15) & ~(uintptr_t)15) - a0),
                  (uint32_t)(a - a0)};
}
__device__ __forceinline__ void ipa_copy(uint32_t dst, const IpaRun& r, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(r.src), "r"(r.bytes), "r"(bar)
                 : "memory");
}

struct IpaTilePos {
    int x, y, zs, count;
};
__device__ __forceinline__ IpaTilePos ipa_tile(const PadGeom& G, int t, int tiles_per_line) {
    const int line = t / tiles_per_line;
    IpaTilePos p;
    p.zs = (t - line * tiles_per_line) * kIpaTile;
    p.x = line / G.ny;
    p.y = line - p.x * G.ny;
    p.count = min(kIpaTile, G.nz - p.zs);
    return p;
}

// Incoming run of direction q of a tile (normal pull, no bounce).
template <class S, int kParity>
__device__ __forceinline__ IpaRun ipa_pop_run(const typename S::T* __restrict__ f, const PadGeom& G, const IpaTilePos& p,
                                              int q) {
    const int dir = q == kRest27 ? kRest27 : (kParity == 0 ? q_opp(q) : q);
    int mx = p.x, my = p.y, mz = p.zs;
    if (q != kRest27 && !q_positive(q)) {
        mx = axis_neighbour(p.x, -q_cx(q), G.nx, G.wrap[0]);
        my = axis_neighbour(p.y, -q_cy(q), G.ny, G.wrap[1]);
        mz = p.zs - q_cz(q);
    }
    return ipa_run(f + ((long long)dir * G.pcells + pad_index(G, mx, my, mz)),
                   (uint32_t)p.count * (uint32_t)sizeof(typename S::T));
}

// Post the copies of tile t, one run per lane: lanes 0-26 the population
// runs of directions 0-26, lane 27 the flags, 28 the mask (and the z force
// component), 29 the temperature, 30 / 31 the x / y force components. Each
// lane records its run's byte offset in the warp's table. kBulk: every lane
// posts its run as one cp.async.bulk completing on the warp's mbarrier (the
// expected bytes are registered before lane 0 arrives); otherwise the runs
// are copied in 16-byte cp.async chunks, chunk l of every run by lane l.
// temperature / fx: null when the brick has no buoyancy / force field.
template <class S, int kParity, bool kBulk>
__device__ __forceinline__ void ipa_post(const typename S::T* __restrict__ f, const PadGeom& G, const uint32_t* flags,
                                         const uint8_t* obstacle, const float* temperature, const float* fx,
                                         const float* fy, const float* fz, unsigned char* wbuf, uint32_t bar, int t,
                                         int tiles_per_line, int lane) {
    using L = IpaLayout<typename S::T>;
    const IpaTilePos p = ipa_tile(G, t, tiles_per_line);
    const long long cell0 = ((long long)p.x * G.ny + p.y) * G.nz + p.zs;
    const uint32_t n = (uint32_t)p.count;
    IpaRun r{nullptr, 0u, 0u}, r2{nullptr, 0u, 0u};
    uint32_t dst = 0;
    if (lane < 27) {
        r = ipa_pop_run<S, kParity>(f, G, p, lane);
        dst = lane * L::kSeg;
    } else if (lane == 27) {
        r = ipa_run(flags + cell0, n * 4u);
        dst = L::kFlags;
    } else if (lane == 28) {
        r = ipa_run(obstacle + cell0, n);
        dst = L::kObst;
        if (fz) r2 = ipa_run(fz + cell0, n * 4u);
    } else if (lane == 29) {
        if (temperature) r = ipa_run(temperature + cell0, n * 4u);
        dst = L::kTemp;
    } else {
        const float* src = lane == 30 ? fx : fy;
        if (src) r = ipa_run(src + cell0, n * 4u);
        dst = L::kForce + (lane - 30) * L::kWord;
    }
    unsigned char* offs = wbuf + L::kOffs;
    offs[lane] = (unsigned char)r.off;
    if (lane == 28) offs[32] = (unsigned char)r2.off;
    const uint32_t base = smem_addr(wbuf);
    if (kBulk) {
        if (r.bytes) {
            asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(r.bytes) : "memory");
            ipa_copy(base + dst, r, bar);
        }
        if (r2.bytes) {
            asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(r2.bytes) : "memory");
            ipa_copy(base + L::kForce + 2 * L::kWord, r2, bar);
        }
        __syncwarp();
        if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
    } else {
        const uintptr_t src = reinterpret_cast<uintptr_t>(r.src);
#pragma unroll 1
        for (int k = 0; k < 33; ++k) {
            const int from = k < 32 ? k : 28;
            const uintptr_t s_k = __shfl_sync(0xffffffffu, k < 32 ? src : reinterpret_cast<uintptr_t>(r2.src), from);
            const uint32_t b_k = __shfl_sync(0xffffffffu, k < 32 ? r.bytes : r2.bytes, from);
            const uint32_t d_k = __shfl_sync(0xffffffffu, k < 32 ? dst : (uint32_t)(L::kForce + 2 * L::kWord), from);
            if ((uint32_t)lane * 16u < b_k)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(base + d_k + 16u * lane),
                             "l"(s_k + 16u * lane)
                             : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
}

// Two raw stored values of one direction -> populations.
template <class S>
struct IpaDecode;
template <>
struct IpaDecode<StoreF32> {
    __device__ __forceinline__ static F2 pair(float a, float b, int, const Fp16Scale&) { return f2(a, b); }
};
template <>
struct IpaDecode<StoreF16Dev> {
    __device__ __forceinline__ static F2 pair(__half a, __half b, int q, const Fp16Scale& s) {
        const float w = q_w(q), k = w * s.inv_scale;
        return F2{__ffma2_rn(make_float2(__half2float(a), __half2float(b)), make_float2(k, k), make_float2(w, w))};
    }
};
template <>
struct IpaDecode<StoreI16Dev> {
    __device__ __forceinline__ static F2 pair(short a, short b, int q, const Fp16Scale& s) {
        const float w = q_w(q), k = w * s.inv_scale;
        return F2{__ffma2_rn(make_float2((float)a, (float)b), make_float2(k, k), make_float2(w, w))};
    }
};

template <class S, int kParity>
__global__ void __launch_bounds__(kIpaWarps * 32, AERO_IPA_MIN_BLOCKS)
    step_ipa_kernel(typename S::T* __restrict__ f, IpArgs a, int tiles_per_line, int tiles) {
    using T = typename S::T;
    using L = IpaLayout<T>;
    extern __shared__ __align__(16) unsigned char ipa_smem[];
    const PadGeom& G = a.g;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (t >= tiles) return;  // whole warp
    unsigned char* wbuf = ipa_smem + (threadIdx.x >> 5) * L::kWarpBytes;
    const uint32_t bar = smem_addr(wbuf + L::kBar);
    const float* temp_src = a.cp.enable_buoyancy ? a.cur.temperature : nullptr;
    if (AERO_IPA_BULK && lane == 0) ipa_bar_init(bar);
    __syncwarp();
    ipa_post<S, kParity, AERO_IPA_BULK>(f, G, a.flags_prev, a.obstacle_cur, temp_src, a.force.fx, a.force.fy,
                                        a.force.fz, wbuf, bar, t, tiles_per_line, lane);
    uint32_t phase = 0;
    for (; t < tiles; t += nw) {
#if AERO_IPA_BULK
        if (!ipa_bar_wait(bar, phase)) {
            if (lane == 0) atomicExch(a.fault, 1);
            return;
        }
        phase ^= 1u;
#else
        asm volatile("cp.async.wait_group 0;" ::: "memory");
#endif
        __syncwarp();
        const IpaTilePos p = ipa_tile(G, t, tiles_per_line);
        const int z0 = p.zs + 2 * lane;
        const bool in0 = 2 * lane < p.count, in1 = 2 * lane + 1 < p.count;
        const unsigned char* offs = wbuf + L::kOffs;
        const uint32_t* fw = reinterpret_cast<const uint32_t*>(wbuf + L::kFlags + offs[27]) + 2 * lane;
        const uint8_t* ob = wbuf + L::kObst + offs[28] + 2 * lane;
        const uint32_t w0 = in0 ? fw[0] : kFlagSelfSolid;
        const uint32_t w1 = in1 ? fw[1] : kFlagSelfSolid;
        const bool live0 = !(w0 & kFlagSelfSolid), live1 = !(w1 & kFlagSelfSolid);
        const bool pass0 = live0 && ob[0] != 0;
        const bool pass1 = live1 && ob[1] != 0;
        F2 t2 = f2(0.0f), cfx = f2(0.0f), cfy = f2(0.0f), cfz = f2(0.0f);
        if (a.cp.enable_buoyancy) {
            const float* tp = reinterpret_cast<const float*>(wbuf + L::kTemp + offs[29]) + 2 * lane;
            t2 = f2(in0 ? tp[0] : 0.0f, in1 ? tp[1] : 0.0f);
        }
        if (a.force.fx) {
            const float* px = reinterpret_cast<const float*>(wbuf + L::kForce + offs[30]) + 2 * lane;
            const float* py = reinterpret_cast<const float*>(wbuf + L::kForce + L::kWord + offs[31]) + 2 * lane;
            const float* pz = reinterpret_cast<const float*>(wbuf + L::kForce + 2 * L::kWord + offs[32]) + 2 * lane;
            cfx = f2(in0 ? px[0] : 0.0f, in1 ? px[1] : 0.0f);
            cfy = f2(in0 ? py[0] : 0.0f, in1 ? py[1] : 0.0f);
            cfz = f2(in0 ? pz[0] : 0.0f, in1 ? pz[1] : 0.0f);
        }
        F2 fl[27];
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            const T* r = reinterpret_cast<const T*>(wbuf + q * L::kSeg + offs[q]) + 2 * lane;
            fl[q] = IpaDecode<S>::pair(r[0], r[1], q, a.sc);
        }
        // The copies of the next tile overwrite this warp's buffer: order the
        // reads above before them (generic -> async proxy), then post them.
        if (AERO_IPA_BULK) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (t + nw < tiles)
            ipa_post<S, kParity, AERO_IPA_BULK>(f, G, a.flags_prev, a.obstacle_cur, temp_src, a.force.fx, a.force.fy,
                                                a.force.fz, wbuf, bar, t + nw, tiles_per_line, lane);
        if (!live0 && !live1) {
            if (a.cur.u_last) {
                const long long c0 = ((long long)p.x * G.ny + p.y) * G.nz + z0;
                if (in0) record_u(a.cur, c0, 0.0f, 0.0f, 0.0f);
                if (in1) record_u(a.cur, c0 + 1, 0.0f, 0.0f, 0.0f);
            }
            continue;
        }

        const int x = p.x, y = p.y;
        const long long cell0 = ((long long)x * G.ny + y) * G.nz + z0;
        const int own0 = pad_index(G, x, y, z0);
        const int own1 = own0 + 1;
        const bool flat = no_wrap(G, x, y, z0) && (!in1 || no_wrap(G, x, y, z0 + 1));
        typename S::T* __restrict__ base0 = f + own0;
        // Half-way bounce-back: the parity-flipped slot, from global memory.
        if ((w0 | w1) & 0x7ffffffu) {
            if (flat) {
#pragma unroll
                for (int q = 0; q < 27; ++q) {
                    const int off = in_offset(G, q, kParity, true);
                    if (live0 && ((w0 >> q) & 1u)) fl[q].v.x = S::load(base0 + off, q, a.sc);
                    if (live1 && ((w1 >> q) & 1u)) fl[q].v.y = S::load(base0 + 1 + off, q, a.sc);
                }
            } else {
                const NeighbourOffsets o0 = neighbour_offsets(G, x, y, z0);
                const NeighbourOffsets o1 = neighbour_offsets(G, x, y, in1 ? z0 + 1 : z0);
#pragma unroll
                for (int q = 0; q < 27; ++q) {
                    int c, d;
                    if (live0 && ((w0 >> q) & 1u)) {
                        incoming_slot(o0, own0, q, kParity, true, c, d);
                        fl[q].v.x = S::load(f + (d * G.pcells + c), q, a.sc);
                    }
                    if (live1 && ((w1 >> q) & 1u)) {
                        incoming_slot(o1, own1, q, kParity, true, c, d);
                        fl[q].v.y = S::load(f + (d * G.pcells + c), q, a.sc);
                    }
                }
            }
        }
        bool ok[2];
        F2 uc[3];
        collide27_x2(fl, a.cp, t2, cfx, cfy, cfz, ok, uc);
        record_u2(a.cur, cell0, in1, live0 && !pass0 && ok[0], live1 && !pass1 && ok[1], live0 && !ok[0] && !pass0,
                  live1 && !ok[1] && !pass1, uc);
        if (pass0 || pass1) {
            const NeighbourOffsets o0 = neighbour_offsets(G, x, y, z0);
            const NeighbourOffsets o1 = neighbour_offsets(G, x, y, in1 ? z0 + 1 : z0);
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                int c, d;
                if (pass0) {
                    incoming_slot(o0, own0, q, kParity, (w0 >> q) & 1u, c, d);
                    fl[q].v.x = S::load(f + (d * G.pcells + c), q, a.sc);
                }
                if (pass1) {
                    incoming_slot(o1, own1, q, kParity, (w1 >> q) & 1u, c, d);
                    fl[q].v.y = S::load(f + (d * G.pcells + c), q, a.sc);
                }
            }
        }
        const bool st0 = live0 && (ok[0] || pass0), st1 = live1 && (ok[1] || pass1);
        if (live0 && !ok[0] && !pass0) reseed_push<S>(f, a, cell0, x, y, z0, kParity);
        if (live1 && !ok[1] && !pass1) reseed_push<S>(f, a, cell0 + 1, x, y, z0 + 1, kParity);
        if (flat) {
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                const int off = out_offset(G, q, kParity);
                PairIO<S>::store(base0 + off, base0 + off + 1, st0, st1, q, fl[q], a.sc);
            }
        } else {
            const NeighbourOffsets o0 = neighbour_offsets(G, x, y, z0);
            const NeighbourOffsets o1 = neighbour_offsets(G, x, y, in1 ? z0 + 1 : z0);
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                int c0, d0, c1, d1;
                outgoing_slot(o0, own0, q, kParity, c0, d0);
                outgoing_slot(o1, own1, q, kParity, c1, d1);
                PairIO<S>::store(f + (d0 * G.pcells + c0), f + (d1 * G.pcells + c1), st0, st1, q, fl[q], a.sc);
            }
        }
    }
}

// Launch of the streamed step (persistent grid: as many blocks as fit on the
// device at once). Returns false when the brick is not eligible.
template <class S>
struct IpaLaunch {
    static bool eligible(const IpArgs& a) { return !a.g.wrap[2] && a.fault != nullptr; }
    static cudaError_t step(typename S::T* f, const IpArgs& a, cudaStream_t s) {
        using L = IpaLayout<typename S::T>;
        const int smem = kIpaWarps * L::kWarpBytes;
        static int grid[2] = {0, 0};
        int& gp = grid[a.parity & 1];
        if (gp == 0) {
            int dev = 0, sms = 0, per_sm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaError_t e = a.parity == 0
                                ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step_ipa_kernel<S, 0>, kIpaWarps * 32, smem)
                                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, step_ipa_kernel<S, 1>, kIpaWarps * 32, smem);
            if (e != cudaSuccess) return e;
            gp = std::max(1, sms * std::max(1, per_sm));
        }
        const int tiles_per_line = (a.g.nz + kIpaTile - 1) / kIpaTile;
        const int tiles = a.g.nx * a.g.ny * tiles_per_line;
        const int blocks = std::min(gp, (tiles + kIpaWarps - 1) / kIpaWarps);
        if (a.parity == 0) step_ipa_kernel<S, 0><<<blocks, kIpaWarps * 32, smem, s>>>(f, a, tiles_per_line, tiles);
        else step_ipa_kernel<S, 1><<<blocks, kIpaWarps * 32, smem, s>>>(f, a, tiles_per_line, tiles);
        return cudaGetLastError();
    }
};

}  // namespace aero
