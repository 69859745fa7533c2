// Packed D3Q19 hydrodynamic step: two z-adjacent cells per thread, the TRT
// collision (Smagorinsky on the even rate, Guo body force) in sm_100 packed
// FP32 (FFMA2 / FADD2 / FMUL2), built with multiply-add contraction.
//
// Same scheme and call semantics as meso_hydro_kernel<S, kHydroStep>
// (meso_exact.cu): pull the previous call's post-collision populations with
// the previous call's mask and forcing, collide with this call's mask. It
// differs in arithmetic only: sums skip the zero lattice components, the
// non-equilibrium second moment is the population second moment minus the
// equilibrium's rho (I/3 + u u), and the TRT works on the even / odd halves of
// each direction pair — agreement with the reference-order kernel is to FP32
// rounding, not bit for bit. Interior pairs (no periodic wrap, no open
// boundary) read their 19 slots at launch-uniform offsets; the rest take the
// per-cell pull of the reference-order kernel.
#include <cuda_fp16.h>

#include <type_traits>

#include "collide27_x2.cuh"
#include "d3q27_kernels.cuh"
#include "lattice.cuh"
#include "meso.cuh"
#include "meso_lattice.cuh"

namespace aero {
namespace meso {
namespace {

__device__ __forceinline__ float hfeq_f(int q, float r, float ux, float uy, float uz) {
    const float cu = 3.0f * ((float)mcx(q) * ux + (float)mcy(q) * uy + (float)mcz(q) * uz);
    const float uu = ux * ux + uy * uy + uz * uz;
    return mw(q) * r * (1.0f + cu + 0.5f * cu * cu - 1.5f * uu);
}
__device__ __forceinline__ float clamp_sp(float u) { return fminf(0.35f, fmaxf(-0.35f, u)); }

// Streamed populations of one cell: the pull of meso_hydro_kernel (solid
// cells, interior / ground cells by their classification word, open sides,
// the specular lid and the edge blend).
template <class S>
__device__ __forceinline__ void pull_cell(const HydroArgs& A, const typename S::T* __restrict__ src, long long i, int x,
                                          int y, int z, float (&f)[19]) {
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const long long cells = (long long)nx * ny * nz;
    const uint32_t w = A.flags_prev[i];
    if (w & kHydroSelfSolid) {
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = mw(q);
        return;
    }
    if (!(w & kHydroSlow)) {
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            int sx = x - mcx(q), sz = z - mcz(q);
            if (A.periodic_sides) {
                sx = sx < 0 ? sx + nx : (sx >= nx ? sx - nx : sx);
                sz = sz < 0 ? sz + nz : (sz >= nz ? sz - nz : sz);
            }
            const long long idx = ((w >> q) & 1u) ? (long long)mopp(q) * cells + i
                                                  : (long long)q * cells + ((long long)sx * ny + (y - mcy(q))) * nz + sz;
            f[q] = S::load(src + idx, q, A.inv_scale);
        }
        return;
    }
    int edge = min(min(x, z), min(nx - 1 - x, nz - 1 - z));
    int top = ny - 1 - y;
    if (A.periodic_sides) edge = 1 << 20;
    if (A.free_slip_top) top = 1 << 20;
    const int sponge = min(edge, top);
    float alpha = sponge <= 0 ? 1.0f : (sponge < 2 ? 0.5f : 0.0f);
    if (!A.edge_blend) alpha = 0.0f;
    float bx = 0.0f, by = 0.0f, bz = 0.0f;
    if (alpha > 0.0f || edge <= 0 || top <= 0) {
        const float* F = A.forcing_prev + i * kMesoForcingChannels;
        const float den = fmaxf(1.0e-6f, A.velocity_scale);
        bx = clamp_sp((F[kChBackgroundWindX] + F[kChNestedWindXDelta] + F[kChConvectiveInflowX] + F[kChTornadoWindX]) / den);
        bz = clamp_sp((F[kChBackgroundWindZ] + F[kChNestedWindZDelta] + F[kChConvectiveInflowZ] + F[kChTornadoWindZ]) / den);
        by = clamp_sp((F[kChNestedUpdraft] + F[kChTornadoUpdraft]) / den);
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        int sx = x - mcx(q), sy = y - mcy(q), sz = z - mcz(q);
        if (A.periodic_sides) {
            sx = sx < 0 ? sx + nx : (sx >= nx ? sx - nx : sx);
            sz = sz < 0 ? sz + nz : (sz >= nz ? sz - nz : sz);
        }
        float fv;
        bool bounced = false;
        if (sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz) {
            const long long sc = ((long long)sx * ny + sy) * nz + sz;
            if (A.solid_prev[sc]) {
                fv = S::load(src + (long long)mopp(q) * cells + i, mopp(q), A.inv_scale);
                bounced = true;
            } else {
                fv = S::load(src + (long long)q * cells + sc, q, A.inv_scale);
            }
        } else if (sy < 0) {
            fv = S::load(src + (long long)mopp(q) * cells + i, mopp(q), A.inv_scale);
            bounced = true;
        } else if (A.free_slip_top && sy >= ny && sx >= 0 && sx < nx && sz >= 0 && sz < nz) {
            const long long sc = ((long long)sx * ny + (ny - 1)) * nz + sz;
            if (A.solid_prev[sc]) {
                fv = S::load(src + (long long)mopp(q) * cells + i, mopp(q), A.inv_scale);
                bounced = true;
            } else {
                fv = S::load(src + (long long)mmirror(q) * cells + sc, mmirror(q), A.inv_scale);
            }
        } else {
            fv = hfeq_f(q, 1.0f, bx, by, bz);
        }
        if (alpha > 0.0f && !bounced) fv = (1.0f - alpha) * fv + alpha * hfeq_f(q, 1.0f, bx, by, bz);
        f[q] = fv;
    }
}

// signed sum of the lanes' values over the non-zero components of c_q
template <int q>
__device__ __forceinline__ F2 cdot2(F2 x, F2 y, F2 z) {
    constexpr int cx = mcx(q), cy = mcy(q), cz = mcz(q);
    F2 s;
    bool any = false;
    if (cx != 0) { s = cx > 0 ? x : -x; any = true; }
    if (cy != 0) { s = any ? (cy > 0 ? s + y : s - y) : (cy > 0 ? y : -y); any = true; }
    if (cz != 0) { s = any ? (cz > 0 ? s + z : s - z) : (cz > 0 ? z : -z); any = true; }
    return s;
}

template <int q>
__device__ __forceinline__ float cdot1(float x, float y, float z) {
    return (float)mcx(q) * x + (float)mcy(q) * y + (float)mcz(q) * z;
}

// one direction pair (q, q + 1) of the TRT update
template <int q>
__device__ __forceinline__ void trt_pair(F2 (&f)[19], const HydroRates& H, F2 rho, F2 tux, F2 tuy, F2 tuz, F2 uu, F2 om_e,
                                         F2 pref, F2 uf) {
    constexpr int qo = q + 1;
    const F2 w = f2(mw(q));
    const F2 cu = cdot2<q>(tux, tuy, tuz);
    const F2 wr = w * rho;
    const F2 feq_even = wr * fma2(f2(4.5f) * cu, cu, fma2(f2(-1.5f), uu, f2(1.0f)));
    const F2 feq_odd = (f2(3.0f) * wr) * cu;
    const F2 fev = f2(0.5f) * (f[q] + f[qo]);
    const F2 fod = f2(0.5f) * (f[q] - f[qo]);
    const F2 fep = fev - om_e * (fev - feq_even);
    const F2 fop = fod - f2(H.omega_odd) * (fod - feq_odd);
    F2 A = f2(0.0f), B = f2(0.0f);
    if (H.forced) {
        const float cf = cdot1<q>(H.fx, H.fy, H.fz);
        const F2 pw = pref * w;
        A = pw * fma2(f2(9.0f * cf), cu, f2(-3.0f) * uf);
        B = pw * f2(3.0f * cf);
    }
    f[q] = (fep + fop) + (A + B);
    f[qo] = (fep - fop) + (A - B);
}

// Two adjacent populations of one direction: raw storage words (loaded
// first, decoded after every load of the cell pair has been issued) and the
// decoded values. `aligned`: the first element is at an even index, so both
// come in one 8-byte (FP32) or 4-byte (16-bit) load. Stores always are: the
// pair's own index i0 is even (nz even) and so is every q * cells.
template <class S>
struct MesoPair;
// AERO_MESO_VECTOR_LOADS selects 2-element vector loads for aligned pairs.
// Measured on the 256 x 64 x 256 grid (B200), scalar loads are faster
// (FP16 31.5 against 24.5 GLUPS), so they are the default; stores stay
// vectors.
#ifndef AERO_MESO_VECTOR_LOADS
#define AERO_MESO_VECTOR_LOADS 0
#endif
template <>
struct MesoPair<MesoF32> {
    using Raw = float2;
    __device__ __forceinline__ static Raw raw(const float* p, bool aligned) {
        return (AERO_MESO_VECTOR_LOADS && aligned) ? __ldg(reinterpret_cast<const float2*>(p)) : make_float2(__ldg(p), __ldg(p + 1));
    }
    __device__ __forceinline__ static Raw raw2(const float* p0, const float* p1) { return make_float2(__ldg(p0), __ldg(p1)); }
    __device__ __forceinline__ static F2 decode(Raw r, int, float) { return F2{r}; }
    __device__ __forceinline__ static void store(float* p, int, F2 v, float) { *reinterpret_cast<float2*>(p) = v.v; }
};
template <>
struct MesoPair<MesoF16> {
    using Raw = __half2;
    __device__ __forceinline__ static Raw raw(const __half* p, bool aligned) {
        return (AERO_MESO_VECTOR_LOADS && aligned) ? __ldg(reinterpret_cast<const __half2*>(p)) : __halves2half2(__ldg(p), __ldg(p + 1));
    }
    __device__ __forceinline__ static Raw raw2(const __half* p0, const __half* p1) { return __halves2half2(__ldg(p0), __ldg(p1)); }
    __device__ __forceinline__ static F2 decode(Raw r, int q, float inv_scale) {
        const float w = mw(q), k = w * inv_scale;
        return F2{__ffma2_rn(__half22float2(r), make_float2(k, k), make_float2(w, w))};
    }
    __device__ __forceinline__ static void store(__half* p, int q, F2 v, float scale) {
        const float k = scale * (1.0f / mw(q));
        const float2 h = __ffma2_rn(v.v, make_float2(k, k), make_float2(-scale, -scale));
        *reinterpret_cast<__half2*>(p) = __floats2half2_rn(h.x, h.y);
    }
};
template <>
struct MesoPair<MesoI16> {
    using Raw = short2;
    __device__ __forceinline__ static Raw raw(const short* p, bool aligned) {
        return (AERO_MESO_VECTOR_LOADS && aligned) ? __ldg(reinterpret_cast<const short2*>(p)) : make_short2(__ldg(p), __ldg(p + 1));
    }
    __device__ __forceinline__ static Raw raw2(const short* p0, const short* p1) { return make_short2(__ldg(p0), __ldg(p1)); }
    __device__ __forceinline__ static F2 decode(Raw r, int q, float inv_scale) {
        const float w = mw(q), k = w * inv_scale;
        const unsigned bits = (unsigned)(unsigned short)r.x | ((unsigned)(unsigned short)r.y << 16);
        return F2{__ffma2_rn(s16x2_to_float2(bits), make_float2(k, k), make_float2(w, w))};
    }
    __device__ __forceinline__ static void store(short* p, int q, F2 v, float scale) {
        const float k = scale * (1.0f / mw(q));
        const float2 h = __ffma2_rn(v.v, make_float2(k, k), make_float2(-scale, -scale));
        *reinterpret_cast<short2*>(p) = make_short2(sat_round_s16(h.x), sat_round_s16(h.y));
    }
};

// kWide: 64-bit slot offsets (grids of 19 x cells >= 2^31 elements); else
// the launch-uniform offsets of a direction are 32-bit and every slot address
// is the pair's own address plus one of them.
#ifndef AERO_MESO2_MIN_BLOCKS
#define AERO_MESO2_MIN_BLOCKS 6
#endif
template <class S, bool kWide>
__global__ void __launch_bounds__(128, AERO_MESO2_MIN_BLOCKS) meso_hydro2_kernel(HydroArgs A) {
    using T = typename S::T;
    using Off = typename std::conditional<kWide, long long, int>::type;
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const int z0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (z0 >= nz) return;
    const int y = blockIdx.y, x = blockIdx.z;
    const long long cells = (long long)nx * ny * nz;
    const long long i0 = ((long long)x * ny + y) * nz + z0;
    const T* __restrict__ src = static_cast<const T*>(A.src);
    const uint32_t w0 = A.flags_prev[i0], w1 = A.flags_prev[i0 + 1];
    F2 f[19];
    if (!((w0 | w1) & (kHydroSelfSolid | kHydroSlow))) {
        // i0, cells and nz are even: a pair's normal source is 2-aligned
        // when c_z = 0, its bounce-back source always. Periodic sides wrap the
        // sources: along x for the whole line (both cells alike), along z for
        // the first cell of the line's first pair and the second cell of its
        // last pair only.
        const T* __restrict__ own = src + i0;
        const Off plane = (Off)cells;
        const bool xlo = A.periodic_sides && x == 0, xhi = A.periodic_sides && x == nx - 1;
        const bool zlo = A.periodic_sides && z0 == 0, zhi = A.periodic_sides && z0 + 2 == nz;
        typename MesoPair<S>::Raw raw[19];
        // a warp none of whose lanes bounces back or wraps along z reads
        // every slot at its line-uniform offset
        if (__all_sync(__activemask(), ((w0 | w1) & ((1u << 19) - 1u)) == 0u && !zlo && !zhi)) {
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                Off n0 = (Off)q * plane - (((Off)mcx(q) * ny + mcy(q)) * nz + mcz(q));
                if (mcx(q) == 1 && xlo) n0 += plane;
                if (mcx(q) == -1 && xhi) n0 -= plane;
                raw[q] = MesoPair<S>::raw(own + n0, mcz(q) == 0);
            }
        } else {
#pragma unroll
            for (int q = 0; q < 19; ++q) {
                Off n0 = (Off)q * plane - (((Off)mcx(q) * ny + mcy(q)) * nz + mcz(q));
                if (mcx(q) == 1 && xlo) n0 += plane;
                if (mcx(q) == -1 && xhi) n0 -= plane;
                const Off na = n0 + ((mcz(q) == 1 && zlo) ? (Off)nz : (Off)0);
                const Off nb = n0 - ((mcz(q) == -1 && zhi) ? (Off)nz : (Off)0);
                const Off b0 = (Off)mopp(q) * plane;
                const bool bb0 = (w0 >> q) & 1u, bb1 = (w1 >> q) & 1u;
                const Off o0 = bb0 ? b0 : na, o1 = bb1 ? b0 : nb;
                if (o0 == o1) raw[q] = MesoPair<S>::raw(own + o0, bb0 || mcz(q) == 0);
                else raw[q] = MesoPair<S>::raw2(own + o0, own + o1 + 1);
            }
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = MesoPair<S>::decode(raw[q], q, A.inv_scale);
    } else {
        float a[19], b[19];
        pull_cell<S>(A, src, i0, x, y, z0, a);
        pull_cell<S>(A, src, i0 + 1, x, y, z0 + 1, b);
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = f2(a[q], b[q]);
    }

    // moments
    const F2 rsum = ((((f[0] + f[1]) + (f[2] + f[3])) + ((f[4] + f[5]) + (f[6] + f[7]))) +
                     (((f[8] + f[9]) + (f[10] + f[11])) + ((f[12] + f[13]) + (f[14] + f[15])))) + ((f[16] + f[17]) + f[18]);
    const F2 jx = ((f[1] - f[2]) + (f[7] - f[8])) + ((f[9] - f[10]) + ((f[11] - f[12]) + (f[13] - f[14])));
    const F2 jy = ((f[3] - f[4]) + (f[7] - f[8])) + ((f[10] - f[9]) + ((f[15] - f[16]) + (f[17] - f[18])));
    const F2 jz = ((f[5] - f[6]) + (f[11] - f[12])) + ((f[14] - f[13]) + ((f[15] - f[16]) + (f[18] - f[17])));
    const bool s0 = A.solid_cur[i0] != 0, s1 = A.solid_cur[i0 + 1] != 0;
    const F2 rr = fmax2(rsum, 1.0e-6f);
    const F2 ir = rcp2(rr);
    const F2 live = f2(s0 ? 0.0f : 1.0f, s1 ? 0.0f : 1.0f);
    // solid lanes relax toward rest: rho 1, u 0
    const F2 rho = f2(s0 ? 1.0f : rr.v.x, s1 ? 1.0f : rr.v.y);
    const F2 ux = live * (jx * ir), uy = live * (jy * ir), uz = live * (jz * ir);
    const HydroRates& H = A.h;
    F2 tux = ux, tuy = uy, tuz = uz;
    if (H.forced) {
        const F2 hi = live * (f2(0.5f) * ir);
        tux = fma2(f2(H.fx), hi, tux);
        tuy = fma2(f2(H.fy), hi, tuy);
        tuz = fma2(f2(H.fz), hi, tuz);
    }
    F2 om_e = f2(H.omega_even);
    if (H.enable_sgs && !(s0 && s1)) {
        const F2 sxx = (f[1] + f[2]) + ((f[7] + f[8]) + (f[9] + f[10])) + ((f[11] + f[12]) + (f[13] + f[14]));
        const F2 syy = (f[3] + f[4]) + ((f[7] + f[8]) + (f[9] + f[10])) + ((f[15] + f[16]) + (f[17] + f[18]));
        const F2 szz = (f[5] + f[6]) + ((f[11] + f[12]) + (f[13] + f[14])) + ((f[15] + f[16]) + (f[17] + f[18]));
        const F2 sxy = (f[7] + f[8]) - (f[9] + f[10]);
        const F2 sxz = (f[11] + f[12]) - (f[13] + f[14]);
        const F2 syz = (f[15] + f[16]) - (f[17] + f[18]);
        const F2 third = f2(1.0f / 3.0f);
        const F2 pxx = sxx - rho * fma2(tux, tux, third), pyy = syy - rho * fma2(tuy, tuy, third);
        const F2 pzz = szz - rho * fma2(tuz, tuz, third);
        const F2 pxy = sxy - rho * (tux * tuy), pxz = sxz - rho * (tux * tuz), pyz = syz - rho * (tuy * tuz);
        const F2 qn2 = fma2(pxx, pxx, fma2(pyy, pyy, pzz * pzz)) + f2(2.0f) * fma2(pxy, pxy, fma2(pxz, pxz, pyz * pyz));
        const F2 qn = sqrt2(fmax2(qn2, 0.0f));
        const float nu0 = (H.tau_h - 0.5f) / 3.0f;
        const F2 nut = fmin2(div2(f2(H.smagorinsky_c * H.smagorinsky_c) * qn, fmax2(f2(2.0f * nu0) * rho, 1e-6f)), 5.0f * nu0);
        const F2 om_sgs = rcp2(fma2(f2(3.0f), f2(nu0) + nut, f2(0.5f)));
        om_e = f2(s0 ? H.omega_even : om_sgs.v.x, s1 ? H.omega_even : om_sgs.v.y);
    }
    const F2 uu = fma2(tux, tux, fma2(tuy, tuy, tuz * tuz));
    F2 pref = f2(0.0f), uf = f2(0.0f);
    if (H.forced) {
        pref = live * fma2(f2(-0.5f), om_e, f2(1.0f));
        uf = fma2(tux, f2(H.fx), fma2(tuy, f2(H.fy), tuz * f2(H.fz)));
    }
    {
        const F2 w0r = f2(mw(0)) * rho;
        const F2 feq0 = w0r * fma2(f2(-1.5f), uu, f2(1.0f));
        f[0] = (f[0] - om_e * (f[0] - feq0)) + (pref * f2(mw(0))) * (f2(-3.0f) * uf);
    }
    trt_pair<1>(f, H, rho, tux, tuy, tuz, uu, om_e, pref, uf);
    trt_pair<3>(f, H, rho, tux, tuy, tuz, uu, om_e, pref, uf);
    trt_pair<5>(f, H, rho, tux, tuy, tuz, uu, om_e, pref, uf);
    trt_pair<7>(f, H, rho, tux, tuy, tuz, uu, om_e, pref, uf);
    trt_pair<9>(f, H, rho, tux, tuy, tuz, uu, om_e, pref, uf);
    trt_pair<11>(f, H, rho, tux, tuy, tuz, uu, om_e, pref, uf);
    trt_pair<13>(f, H, rho, tux, tuy, tuz, uu, om_e, pref, uf);
    trt_pair<15>(f, H, rho, tux, tuy, tuz, uu, om_e, pref, uf);
    trt_pair<17>(f, H, rho, tux, tuy, tuz, uu, om_e, pref, uf);
    T* __restrict__ dst = static_cast<T*>(A.dst) + i0;
#pragma unroll
    for (int q = 0; q < 19; ++q) MesoPair<S>::store(dst + (Off)q * (Off)cells, q, f[q], A.scale);
}

}  // namespace
}  // namespace meso

cudaError_t meso_hydro_fast_step(const meso::HydroArgs& a, int storage, cudaStream_t s) {
    if (a.nz % 2) return cudaErrorInvalidValue;
    const int pairs = a.nz / 2;
    const int block = pairs >= 128 ? 128 : ((pairs + 31) / 32) * 32;
    const dim3 grid((unsigned)((pairs + block - 1) / block), (unsigned)a.ny, (unsigned)a.nx);
    const bool wide = 19LL * a.nx * a.ny * a.nz >= (1LL << 31);
    if (storage == kMesoStoreF16) {
        if (wide) meso::meso_hydro2_kernel<meso::MesoF16, true><<<grid, block, 0, s>>>(a);
        else meso::meso_hydro2_kernel<meso::MesoF16, false><<<grid, block, 0, s>>>(a);
    } else if (storage == kMesoStoreI16) {
        if (wide) meso::meso_hydro2_kernel<meso::MesoI16, true><<<grid, block, 0, s>>>(a);
        else meso::meso_hydro2_kernel<meso::MesoI16, false><<<grid, block, 0, s>>>(a);
    } else {
        if (wide) meso::meso_hydro2_kernel<meso::MesoF32, true><<<grid, block, 0, s>>>(a);
        else meso::meso_hydro2_kernel<meso::MesoF32, false><<<grid, block, 0, s>>>(a);
    }
    count_launch();
    return cudaGetLastError();
}

}  // namespace aero
