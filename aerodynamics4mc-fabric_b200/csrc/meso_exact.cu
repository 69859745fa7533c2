// D3Q19 mesoscale step (the L1 grid of the mod): two-relaxation-time
// hydrodynamic and thermal double distributions relaxed toward targets built
// from a 25-channel forcing, pull streaming with bounce-back off solid cells
// and the ground, equilibrium inflow with a two-cell blend at the sides and
// top, macro export (native/src/aero_lbm_mesoscale.cpp:146-738).
//
// Two launches per step: `meso_collide_kernel` (targets + TRT, one thread per
// cell; writes post-collision f and g and the next surface / deep-ground
// temperatures) and `meso_stream_kernel` (pull + boundaries + macro export
// for the cell; writes the new f and g, the ambient field and the output
// state). The collision needs the neighbours' previous temperatures
// (laplacians) and the pull needs the neighbours' post-collision populations,
// so the step has two grid-wide dependencies and cannot be one launch.
// Populations are structure-of-arrays f[q][cell] (the reference stores
// f[cell*19+q]; the layout is internal to both).
//
// This file is built with --fmad=false and every expression keeps the
// reference's operation order (products by the integer lattice components
// included), so the step is bit-identical to the reference CPU step. The
// options the reference does not have (periodic x/z sides, a free-slip lid, a
// uniform Guo body force, a fixed hydrodynamic tau, Smagorinsky on the even
// rate, no edge blend) follow the oracle's restatement and are off by default.
#include <cuda_fp16.h>

#include "d3q27_kernels.cuh"
#include "lattice.cuh"
#include "meso.cuh"
#include "meso_lattice.cuh"

namespace aero {
namespace meso {

__device__ __forceinline__ float fx_(int q) { return (float)mcx(q); }
__device__ __forceinline__ float fy_(int q) { return (float)mcy(q); }
__device__ __forceinline__ float fz_(int q) { return (float)mcz(q); }

// std::max / std::min / std::clamp
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float sclamp(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
__device__ __forceinline__ float clamp_speed(float u) { return sclamp(u, -0.35f, 0.35f); }

// hydro_feq_3d / thermal_feq_3d (native/src/aero_lbm_mesoscale.cpp:254-263)
__device__ __forceinline__ float hfeq(int q, float r, float ux, float uy, float uz) {
    const float cu = 3.0f * (fx_(q) * ux + fy_(q) * uy + fz_(q) * uz);
    const float uu = ux * ux + uy * uy + uz * uz;
    return mw(q) * r * (1.0f + cu + 0.5f * cu * cu - 1.5f * uu);
}
__device__ __forceinline__ float tfeq(int q, float t, float ux, float uy, float uz) {
    const float cu = 3.0f * (fx_(q) * ux + fy_(q) * uy + fz_(q) * uz);
    return mw(q) * t * (1.0f + cu);
}

__device__ __forceinline__ float ch(const float* __restrict__ F, long long cell, int c) {
    return __ldg(F + cell * kMesoForcingChannels + c);
}
__device__ __forceinline__ bool solid_at(const float* __restrict__ F, long long cell) { return ch(F, cell, kChSolidMask) > 0.5f; }
__device__ __forceinline__ float wall_temp(const float* __restrict__ F, long long cell) {
    return ch(F, cell, kChSurfaceTarget) + ch(F, cell, kChNestedSurfaceDelta);
}

template <class Args>
__device__ __forceinline__ long long midx(const Args& A, int x, int y, int z) {
    return ((long long)x * A.ny + y) * A.nz + z;
}
// horizontal (x, z) and vertical (y) laplacians with clamped neighbours
// (native/src/aero_lbm_mesoscale.cpp:335-373)
__device__ __forceinline__ float hlap(const MesoArgs& A, const float* __restrict__ a, int x, int y, int z) {
    const float c = a[midx(A, x, y, z)];
    const float xp = a[midx(A, min(A.nx - 1, x + 1), y, z)], xm = a[midx(A, max(0, x - 1), y, z)];
    const float zp = a[midx(A, x, y, min(A.nz - 1, z + 1))], zm = a[midx(A, x, y, max(0, z - 1))];
    return xp + xm + zp + zm - 4.0f * c;
}
__device__ __forceinline__ float vlap(const MesoArgs& A, const float* __restrict__ a, int x, int y, int z) {
    if (A.ny <= 1) return 0.0f;
    const float c = a[midx(A, x, y, z)];
    const float yp = a[midx(A, x, min(A.ny - 1, y + 1), z)], ym = a[midx(A, x, max(0, y - 1), z)];
    return yp + ym - 2.0f * c;
}

struct Targets {
    float rho, ux, uy, uz, teq, nsurf, ndeep;
};

// compute_cell_targets (native/src/aero_lbm_mesoscale.cpp:393-530)
__device__ __forceinline__ Targets cell_targets(const MesoArgs& A, const float (&f)[19], const float (&g)[19], long long i,
                                                int x, int y, int z) {
    const float* F = A.forcing;
    const float dt = smax(1.0e-3f, A.dt_s);
    const float amb_relax = sclamp(dt / 600.0f, 0.0f, 1.0f);
    const float deep_relax = sclamp(dt / 2400.0f, 0.0f, 1.0f);
    const float surf_relax = sclamp(dt / 300.0f, 0.0f, 1.0f);
    const float wind_relax = sclamp(dt / 60.0f, 0.0f, 1.0f);
    float r = 0.0f, ux = 0.0f, uy = 0.0f, uz = 0.0f, amb = 0.0f;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        r += f[q];
        ux += f[q] * fx_(q);
        uy += f[q] * fy_(q);
        uz += f[q] * fz_(q);
        amb += g[q];
    }
    r = smax(1.0e-6f, r);
    ux /= r;
    uy /= r;
    uz /= r;
    const float amb_t = ch(F, i, kChAmbientTarget) + ch(F, i, kChNestedAmbientDelta);
    const float deep_t = ch(F, i, kChDeepGroundTarget);
    const float surf_t = ch(F, i, kChSurfaceTarget) + ch(F, i, kChNestedSurfaceDelta);
    if (solid_at(F, i)) return Targets{1.0f, 0.0f, 0.0f, 0.0f, surf_t, surf_t, deep_t};
    const float rough = smax(0.0f, ch(F, i, kChRoughness));
    const float conv_h = ch(F, i, kChConvectiveHeating), conv_m = ch(F, i, kChConvectiveMoistening);
    const float conv_x = ch(F, i, kChConvectiveInflowX), conv_z = ch(F, i, kChConvectiveInflowZ);
    const float tor_x = ch(F, i, kChTornadoWindX), tor_z = ch(F, i, kChTornadoWindZ);
    const float tor_h = ch(F, i, kChTornadoHeating), tor_m = ch(F, i, kChTornadoMoistening);
    const float tor_up = ch(F, i, kChTornadoUpdraft), nest_up = ch(F, i, kChNestedUpdraft);
    const float nest_dx = ch(F, i, kChNestedWindXDelta), nest_dz = ch(F, i, kChNestedWindZDelta);
    const float bx = ch(F, i, kChBackgroundWindX) + nest_dx + conv_x + tor_x;
    const float bz = ch(F, i, kChBackgroundWindZ) + nest_dz + conv_z + tor_z;
    const float by = nest_up + tor_up;
    const float hum = sclamp(ch(F, i, kChHumidity) + conv_m + tor_m, 0.0f, 1.0f);
    const int xp = min(A.nx - 1, x + 1), xm = max(0, x - 1), zp = min(A.nz - 1, z + 1), zm = max(0, z - 1);
    const float sx = 0.5f * (ch(F, midx(A, xp, y, z), kChTerrainHeight) - ch(F, midx(A, xm, y, z), kChTerrainHeight));
    const float sz = 0.5f * (ch(F, midx(A, x, y, zp), kChTerrainHeight) - ch(F, midx(A, x, y, zm), kChTerrainHeight));
    const float s_hl = hlap(A, A.surface, x, y, z), s_vl = vlap(A, A.surface, x, y, z);
    const float d_vl = vlap(A, A.deep, x, y, z);
    const float a_hl = hlap(A, A.ambient, x, y, z), a_vl = vlap(A, A.ambient, x, y, z);
    const float deep_i = A.deep[i], surf_i = A.surface[i];
    const float ndeep = deep_i + deep_relax * (deep_t - deep_i) + 0.01f * d_vl;
    const float damp = 1.0f - 0.12f * hum;
    const float nsurf = surf_i + surf_relax * damp * (surf_t - surf_i) + 0.10f * (ndeep - surf_i) + 0.04f * conv_h +
                        0.08f * tor_h + 0.05f * s_hl + 0.025f * s_vl;
    const float den = smax(1.0e-6f, A.velocity_scale);
    const float lx = clamp_speed(bx / den), ly = clamp_speed(by / den), lz = clamp_speed(bz / den);
    const float push = 0.0008f * (nsurf - amb);
    const float nsw = 1.0f - (float)y / smax(1.0f, (float)(A.ny - 1));
    const float lift = 0.0015f * (lx * sx + lz * sz) * nsw;
    const float blift = 0.0009f * (nsurf - amb) * nsw;
    const float steer_x = -0.005f * sx * lz;
    const float steer_z = 0.005f * sz * lx;
    const float drag = sclamp(rough * 0.02f, 0.0f, 0.25f);
    const float tux = clamp_speed(lx + steer_x + push * sx - drag * ux);
    const float tuz = clamp_speed(lz + steer_z + push * sz - drag * uz);
    const float tuy = clamp_speed(ly + lift + blift - drag * uy);
    const float rux = clamp_speed((1.0f - wind_relax) * ux + wind_relax * tux);
    const float ruy = clamp_speed((1.0f - wind_relax) * uy + wind_relax * tuy);
    const float ruz = clamp_speed((1.0f - wind_relax) * uz + wind_relax * tuz);
    const float src = amb_relax * (amb_t - amb) + (0.018f + 0.004f * hum) * (nsurf - amb) + 0.01f * (ndeep - amb) +
                      0.08f * conv_h * (0.5f + 0.5f * hum) + 0.10f * tor_h * (0.45f + 0.55f * hum) + 0.06f * tor_up +
                      0.06f * nest_up + 0.01f * a_hl + 0.02f * a_vl;
    return Targets{r, rux, ruy, ruz, amb + src, nsurf, ndeep};
}

// TRT on the hydrodynamic distribution toward feq(rho, u + F / 2 rho) with
// the Guo source and Smagorinsky on the even rate when enabled
// (native/src/aero_lbm_mesoscale.cpp:573-606 plus the restatement's options).
__device__ __forceinline__ void trt_hydro(const HydroRates& H, const float (&f)[19], float rho, float ux, float uy,
                                          float uz, bool solid, float (&pf)[19]) {
    float om_even = H.omega_even;
    const float om_odd = H.omega_odd;
    float tux = ux, tuy = uy, tuz = uz;
    const bool forced = H.forced && !solid;
    if (forced) {
        tux += 0.5f * H.fx / rho;
        tuy += 0.5f * H.fy / rho;
        tuz += 0.5f * H.fz / rho;
    }
    if (H.enable_sgs && !solid) {
        float pxx = 0.0f, pyy = 0.0f, pzz = 0.0f, pxy = 0.0f, pxz = 0.0f, pyz = 0.0f;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const float ne = f[q] - hfeq(q, rho, tux, tuy, tuz);
            pxx += ne * (float)(mcx(q) * mcx(q));
            pyy += ne * (float)(mcy(q) * mcy(q));
            pzz += ne * (float)(mcz(q) * mcz(q));
            pxy += ne * (float)(mcx(q) * mcy(q));
            pxz += ne * (float)(mcx(q) * mcz(q));
            pyz += ne * (float)(mcy(q) * mcz(q));
        }
        const float qn = sqrtf(pxx * pxx + pyy * pyy + pzz * pzz + 2.0f * (pxy * pxy + pxz * pxz + pyz * pyz));
        const float nu0 = (H.tau_h - 0.5f) / 3.0f;
        const float cs2 = H.smagorinsky_c * H.smagorinsky_c;
        const float nut = smin(cs2 * qn / smax(1e-6f, 2.0f * rho * nu0), 5.0f * nu0);
        om_even = 1.0f / (0.5f + 3.0f * (nu0 + nut));
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        const int qo = mopp(q);
        if (q > qo) continue;
        float sq = 0.0f, sqo = 0.0f;
        if (forced) {
            const float pref = 1.0f - 0.5f * om_even;
            const float cu = fx_(q) * tux + fy_(q) * tuy + fz_(q) * tuz;
            const float cf = fx_(q) * H.fx + fy_(q) * H.fy + fz_(q) * H.fz;
            const float uf = tux * H.fx + tuy * H.fy + tuz * H.fz;
            sq = pref * mw(q) * (3.0f * (cf - uf) + 9.0f * cu * cf);
            sqo = pref * mw(q) * (3.0f * (-cf - uf) + 9.0f * cu * cf);
        }
        if (q == qo) {
            const float fe = hfeq(q, rho, tux, tuy, tuz);
            pf[q] = f[q] - om_even * (f[q] - fe) + sq;
            continue;
        }
        const float fe = hfeq(q, rho, tux, tuy, tuz), feo = hfeq(qo, rho, tux, tuy, tuz);
        const float fev = 0.5f * (f[q] + f[qo]), fod = 0.5f * (f[q] - f[qo]);
        const float feev = 0.5f * (fe + feo), feod = 0.5f * (fe - feo);
        const float fep = fev - om_even * (fev - feev);
        const float fop = fod - om_odd * (fod - feod);
        pf[q] = fep + fop + sq;
        pf[qo] = fep - fop + sqo;
    }
}

// Targets + TRT of both distributions (native/src/aero_lbm_mesoscale.cpp:573-618).
__global__ void __launch_bounds__(128) meso_collide_kernel(MesoArgs A) {
    const long long cells = (long long)A.nx * A.ny * A.nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    int x, y, z;
    cell_xyz32(i, A.ny, A.nz, x, y, z);
    float f[19], g[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        f[q] = A.f[q * cells + i];
        g[q] = A.g[q * cells + i];
    }
    const Targets t = cell_targets(A, f, g, i, x, y, z);
    A.next_deep[i] = t.ndeep;
    A.next_surface[i] = t.nsurf;
    float pf[19];
    trt_hydro(A.h, f, t.rho, t.ux, t.uy, t.uz, solid_at(A.forcing, i), pf);
    const float om_t_even = A.omega_t_even, om_t_odd = A.omega_t_odd;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        A.post_f[q * cells + i] = pf[q];
        const int qo = mopp(q);
        if (q > qo) continue;
        if (q == qo) {
            const float ge = tfeq(q, t.teq, t.ux, t.uy, t.uz);
            A.post_g[q * cells + i] = g[q] - om_t_even * (g[q] - ge);
            continue;
        }
        const float ge = tfeq(q, t.teq, t.ux, t.uy, t.uz), geo = tfeq(qo, t.teq, t.ux, t.uy, t.uz);
        const float gev = 0.5f * (g[q] + g[qo]), god = 0.5f * (g[q] - g[qo]);
        const float geev = 0.5f * (ge + geo), geod = 0.5f * (ge - geo);
        const float gep = gev - om_t_even * (gev - geev);
        const float gop = god - om_t_odd * (god - geod);
        A.post_g[q * cells + i] = gep + gop;
        A.post_g[qo * cells + i] = gep - gop;
    }
}

// Pull streaming, boundaries and macro export
// (native/src/aero_lbm_mesoscale.cpp:620-734).
__global__ void __launch_bounds__(128) meso_stream_kernel(MesoArgs A) {
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const long long cells = (long long)nx * ny * nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    int x, y, z;
    cell_xyz32(i, ny, nz, x, y, z);
    const float* F = A.forcing;
    float* out = A.out_state ? A.out_state + i * kMesoStateChannels : nullptr;
    if (solid_at(F, i)) {
        const float wt = wall_temp(F, i);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            A.f[q * cells + i] = hfeq(q, 1.0f, 0.0f, 0.0f, 0.0f);
            A.g[q * cells + i] = tfeq(q, wt, 0.0f, 0.0f, 0.0f);
        }
        A.ambient[i] = wt;
        if (out) {
            out[0] = wt;
            out[1] = A.next_deep[i];
            out[2] = A.next_surface[i];
            out[3] = 0.0f;
            out[4] = 0.0f;
            out[5] = 0.0f;
        }
        return;
    }
    const float den = smax(1.0e-6f, A.velocity_scale);
    const float bx = clamp_speed((ch(F, i, kChBackgroundWindX) + ch(F, i, kChNestedWindXDelta) + ch(F, i, kChConvectiveInflowX) +
                                  ch(F, i, kChTornadoWindX)) / den);
    const float bz = clamp_speed((ch(F, i, kChBackgroundWindZ) + ch(F, i, kChNestedWindZDelta) + ch(F, i, kChConvectiveInflowZ) +
                                  ch(F, i, kChTornadoWindZ)) / den);
    const float btemp = ch(F, i, kChAmbientTarget) + ch(F, i, kChNestedAmbientDelta);
    const float by = clamp_speed((ch(F, i, kChNestedUpdraft) + ch(F, i, kChTornadoUpdraft)) / den);
    int edge = min(min(x, z), min(nx - 1 - x, nz - 1 - z));
    int top = ny - 1 - y;
    if (A.periodic_sides) edge = 1 << 20;
    if (A.free_slip_top) top = 1 << 20;
    const int sponge = min(edge, top);
    float alpha = sponge <= 0 ? 1.0f : (sponge < 2 ? 0.5f : 0.0f);
    if (!A.edge_blend) alpha = 0.0f;
    float fn[19], gn[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        int sx = x - mcx(q), sy = y - mcy(q), sz = z - mcz(q);
        if (A.periodic_sides) {
            sx = (sx + nx) % nx;
            sz = (sz + nz) % nz;
        }
        float fv, gv;
        bool bounced = false;
        if (sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz) {
            const long long src = midx(A, sx, sy, sz);
            if (solid_at(F, src)) {
                fv = A.post_f[mopp(q) * cells + i];
                gv = tfeq(q, wall_temp(F, src), 0.0f, 0.0f, 0.0f);
                bounced = true;
            } else {
                fv = A.post_f[q * cells + src];
                gv = A.post_g[q * cells + src];
            }
        } else if (sy < 0) {
            fv = A.post_f[mopp(q) * cells + i];
            gv = tfeq(q, wall_temp(F, i), 0.0f, 0.0f, 0.0f);
            bounced = true;
        } else if (A.free_slip_top && sy >= ny && sx >= 0 && sx < nx && sz >= 0 && sz < nz) {
            const long long src = midx(A, sx, ny - 1, sz);
            if (solid_at(F, src)) {
                fv = A.post_f[mopp(q) * cells + i];
                gv = tfeq(q, wall_temp(F, src), 0.0f, 0.0f, 0.0f);
                bounced = true;
            } else {
                fv = A.post_f[mmirror(q) * cells + src];
                gv = A.post_g[mmirror(q) * cells + src];
            }
        } else {
            fv = hfeq(q, 1.0f, bx, by, bz);
            gv = tfeq(q, btemp, bx, by, bz);
        }
        if (alpha > 0.0f && !bounced) {
            const float fb = hfeq(q, 1.0f, bx, by, bz);
            const float gb = tfeq(q, btemp, bx, by, bz);
            fv = (1.0f - alpha) * fv + alpha * fb;
            gv = (1.0f - alpha) * gv + alpha * gb;
        }
        fn[q] = fv;
        gn[q] = gv;
    }
    float r = 0.0f, ux = 0.0f, uy = 0.0f, uz = 0.0f, amb = 0.0f;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        A.f[q * cells + i] = fn[q];
        A.g[q * cells + i] = gn[q];
        r += fn[q];
        ux += fn[q] * fx_(q);
        uy += fn[q] * fy_(q);
        uz += fn[q] * fz_(q);
        amb += gn[q];
    }
    r = smax(1.0e-6f, r);
    ux /= r;
    uy /= r;
    uz /= r;
    A.ambient[i] = amb;
    if (out) {
        const float ms = A.max_speed;
        out[0] = amb;
        out[1] = A.next_deep[i];
        out[2] = A.next_surface[i];
        out[3] = sclamp(ux * A.velocity_scale, -ms, ms);
        out[4] = sclamp(uy * A.velocity_scale, -ms, ms);
        out[5] = sclamp(uz * A.velocity_scale, -ms, ms);
    }
}

// seed_mesoscale_state (native/src/aero_lbm_mesoscale.cpp:298-333)
__global__ void meso_seed_kernel(MesoArgs A) {
    const long long cells = (long long)A.nx * A.ny * A.nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    const float* F = A.forcing;
    const float amb_t = ch(F, i, kChAmbientTarget) + ch(F, i, kChNestedAmbientDelta);
    const float surf_t = ch(F, i, kChSurfaceTarget) + ch(F, i, kChNestedSurfaceDelta);
    const bool s = solid_at(F, i);
    const float bx = ch(F, i, kChBackgroundWindX) + ch(F, i, kChNestedWindXDelta);
    const float bz = ch(F, i, kChBackgroundWindZ) + ch(F, i, kChNestedWindZDelta);
    const float by = ch(F, i, kChNestedUpdraft) + ch(F, i, kChTornadoUpdraft);
    const float den = smax(1.0e-6f, A.velocity_scale);
    const float lx = clamp_speed((s ? 0.0f : bx) / den);
    const float ly = clamp_speed((s ? 0.0f : by) / den);
    const float lz = clamp_speed((s ? 0.0f : bz) / den);
    const float amb = s ? surf_t : amb_t;
    A.ambient[i] = amb;
    A.deep[i] = ch(F, i, kChDeepGroundTarget);
    A.surface[i] = surf_t;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        A.f[q * cells + i] = hfeq(q, 1.0f, lx, ly, lz);
        A.g[q * cells + i] = tfeq(q, amb, lx, ly, lz);
    }
}


// ---------------------------------------------------------------------------
// Hydrodynamic-only step (the mesoscale hydrodynamic distribution without the
// thermal distribution and without target relaxation: the collision relaxes
// toward the cell's own rho and u). One fused launch per call: pull the
// previous call's post-collision populations with the previous call's mask
// and forcing (the reference streams at the end of each call with that call's
// inputs), then collide with this call's mask. The first call collides the
// seeded state; outputs stream the current post-collision state once more.
// Two population buffers; each holds post-collision values.

template <class S, int kMode>
__global__ void __launch_bounds__(256) meso_hydro_kernel(HydroArgs A) {
    using T = typename S::T;
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const long long cells = (long long)nx * ny * nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    int x, y, z;
    cell_xyz32(i, ny, nz, x, y, z);
    const T* __restrict__ src = static_cast<const T*>(A.src);
    float f[19];
    if (kMode == kHydroInit) {
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = S::load(src + q * cells + i, q, A.inv_scale);
    } else if (A.flags_prev[i] & kHydroSelfSolid) {
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = hfeq(q, 1.0f, 0.0f, 0.0f, 0.0f);
    } else if (!(A.flags_prev[i] & kHydroSlow)) {
        // interior (or periodic / ground) cell: every source is known from the
        // classification word, so the 19 loads are independent of each other
        const uint32_t w = A.flags_prev[i];
        long long idx[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            int sx = x - mcx(q), sz = z - mcz(q);
            if (A.periodic_sides) {
                sx = sx < 0 ? sx + nx : (sx >= nx ? sx - nx : sx);
                sz = sz < 0 ? sz + nz : (sz >= nz ? sz - nz : sz);
            }
            idx[q] = ((w >> q) & 1u) ? (long long)mopp(q) * cells + i : (long long)q * cells + midx(A, sx, y - mcy(q), sz);
        }
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = S::load(src + idx[q], q, A.inv_scale);
    } else {
        int edge = min(min(x, z), min(nx - 1 - x, nz - 1 - z));
        int top = ny - 1 - y;
        if (A.periodic_sides) edge = 1 << 20;
        if (A.free_slip_top) top = 1 << 20;
        const int sponge = min(edge, top);
        float alpha = sponge <= 0 ? 1.0f : (sponge < 2 ? 0.5f : 0.0f);
        if (!A.edge_blend) alpha = 0.0f;
        // the inflow wind is read only where a pull can leave the grid through
        // an open side or the open top, or where the edge blend acts
        float bx = 0.0f, by = 0.0f, bz = 0.0f;
        if (alpha > 0.0f || edge <= 0 || top <= 0) {
            const float* F = A.forcing_prev;
            const float den = smax(1.0e-6f, A.velocity_scale);
            bx = clamp_speed((ch(F, i, kChBackgroundWindX) + ch(F, i, kChNestedWindXDelta) + ch(F, i, kChConvectiveInflowX) +
                              ch(F, i, kChTornadoWindX)) / den);
            bz = clamp_speed((ch(F, i, kChBackgroundWindZ) + ch(F, i, kChNestedWindZDelta) + ch(F, i, kChConvectiveInflowZ) +
                              ch(F, i, kChTornadoWindZ)) / den);
            by = clamp_speed((ch(F, i, kChNestedUpdraft) + ch(F, i, kChTornadoUpdraft)) / den);
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
                const long long sc = midx(A, sx, sy, sz);
                if (A.solid_prev[sc]) {
                    fv = S::load(src + mopp(q) * cells + i, mopp(q), A.inv_scale);
                    bounced = true;
                } else {
                    fv = S::load(src + q * cells + sc, q, A.inv_scale);
                }
            } else if (sy < 0) {
                fv = S::load(src + mopp(q) * cells + i, mopp(q), A.inv_scale);
                bounced = true;
            } else if (A.free_slip_top && sy >= ny && sx >= 0 && sx < nx && sz >= 0 && sz < nz) {
                const long long sc = midx(A, sx, ny - 1, sz);
                if (A.solid_prev[sc]) {
                    fv = S::load(src + mopp(q) * cells + i, mopp(q), A.inv_scale);
                    bounced = true;
                } else {
                    fv = S::load(src + mmirror(q) * cells + sc, mmirror(q), A.inv_scale);
                }
            } else {
                fv = hfeq(q, 1.0f, bx, by, bz);
            }
            if (alpha > 0.0f && !bounced) {
                const float fb = hfeq(q, 1.0f, bx, by, bz);
                fv = (1.0f - alpha) * fv + alpha * fb;
            }
            f[q] = fv;
        }
    }
    if (kMode == kHydroOutput) {
        float* o = A.out_state + i * kMesoStateChannels;
        if (A.flags_prev[i] & kHydroSelfSolid) {
            o[0] = 1.0f;
            o[1] = o[2] = o[3] = o[4] = o[5] = 0.0f;
            return;
        }
        float r = 0.0f, ux = 0.0f, uy = 0.0f, uz = 0.0f;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            r += f[q];
            ux += f[q] * fx_(q);
            uy += f[q] * fy_(q);
            uz += f[q] * fz_(q);
        }
        r = smax(1.0e-6f, r);
        ux /= r;
        uy /= r;
        uz /= r;
        const float ms = A.max_speed;
        o[0] = r;
        o[1] = 0.0f;
        o[2] = 0.0f;
        o[3] = sclamp(ux * A.velocity_scale, -ms, ms);
        o[4] = sclamp(uy * A.velocity_scale, -ms, ms);
        o[5] = sclamp(uz * A.velocity_scale, -ms, ms);
        return;
    }
    const bool solid = A.solid_cur[i] != 0;
    float r = 1.0f, ux = 0.0f, uy = 0.0f, uz = 0.0f;
    if (!solid) {
        r = 0.0f;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            r += f[q];
            ux += f[q] * fx_(q);
            uy += f[q] * fy_(q);
            uz += f[q] * fz_(q);
        }
        r = smax(1.0e-6f, r);
        ux /= r;
        uy /= r;
        uz /= r;
    }
    float pf[19];
    trt_hydro(A.h, f, r, ux, uy, uz, solid, pf);
    T* __restrict__ dst = static_cast<T*>(A.dst);
#pragma unroll
    for (int q = 0; q < 19; ++q) S::store(dst + q * cells + i, q, pf[q], A.scale);
}

// Seed of the hydrodynamic-only state: seed_mesoscale_state's populations
// (native/src/aero_lbm_mesoscale.cpp:298-333) and the solid mask.
template <class S>
__global__ void meso_hydro_seed_kernel(const float* __restrict__ F, int nx, int ny, int nz, float velocity_scale,
                                       float scale, typename S::T* __restrict__ dst, uint8_t* __restrict__ solid) {
    const long long cells = (long long)nx * ny * nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    const bool s = solid_at(F, i);
    const float bx = ch(F, i, kChBackgroundWindX) + ch(F, i, kChNestedWindXDelta);
    const float bz = ch(F, i, kChBackgroundWindZ) + ch(F, i, kChNestedWindZDelta);
    const float by = ch(F, i, kChNestedUpdraft) + ch(F, i, kChTornadoUpdraft);
    const float den = smax(1.0e-6f, velocity_scale);
    const float lx = clamp_speed((s ? 0.0f : bx) / den);
    const float ly = clamp_speed((s ? 0.0f : by) / den);
    const float lz = clamp_speed((s ? 0.0f : bz) / den);
    solid[i] = s ? 1 : 0;
#pragma unroll
    for (int q = 0; q < 19; ++q) S::store(dst + q * cells + i, q, hfeq(q, 1.0f, lx, ly, lz), scale);
}

// Pull classification of a mask (see meso_hydro_flags).
__global__ void meso_hydro_flags_kernel(HydroArgs A, const uint8_t* __restrict__ solid, uint32_t* __restrict__ flags) {
    const int nx = A.nx, ny = A.ny, nz = A.nz;
    const long long cells = (long long)nx * ny * nz;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    if (solid[i]) {
        flags[i] = kHydroSelfSolid;
        return;
    }
    int x, y, z;
    cell_xyz32(i, ny, nz, x, y, z);
    int edge = min(min(x, z), min(nx - 1 - x, nz - 1 - z));
    int top = ny - 1 - y;
    if (A.periodic_sides) edge = 1 << 20;
    if (A.free_slip_top) top = 1 << 20;
    const int sponge = min(edge, top);
    bool slow = A.edge_blend && sponge < 2;
    uint32_t w = 0;
    for (int q = 0; q < 19; ++q) {
        int sx = x - mcx(q), sy = y - mcy(q), sz = z - mcz(q);
        if (A.periodic_sides) {
            sx = sx < 0 ? sx + nx : (sx >= nx ? sx - nx : sx);
            sz = sz < 0 ? sz + nz : (sz >= nz ? sz - nz : sz);
        }
        if (sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz) {
            if (solid[midx(A, sx, sy, sz)]) w |= 1u << q;
        } else if (sy < 0) {
            w |= 1u << q;
        } else {
            slow = true;
        }
    }
    flags[i] = w | (slow ? kHydroSlow : 0u);
}

__global__ void meso_mask_kernel(const float* __restrict__ F, long long cells, uint8_t* __restrict__ solid) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cells) solid[i] = solid_at(F, i) ? 1 : 0;
}

}  // namespace meso

cudaError_t meso_launch_seed(const meso::MesoArgs& a, cudaStream_t s) {
    const long long cells = (long long)a.nx * a.ny * a.nz;
    meso::meso_seed_kernel<<<(unsigned)((cells + 127) / 128), 128, 0, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t meso_launch_step(const meso::MesoArgs& a, cudaStream_t s) {
    const long long cells = (long long)a.nx * a.ny * a.nz;
    const unsigned blocks = (unsigned)((cells + 127) / 128);
    meso::meso_collide_kernel<<<blocks, 128, 0, s>>>(a);
    count_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    meso::meso_stream_kernel<<<blocks, 128, 0, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t meso_hydro_seed(const float* forcing, int nx, int ny, int nz, float velocity_scale, int storage, float scale,
                            void* dst, uint8_t* solid, cudaStream_t s) {
    const long long cells = (long long)nx * ny * nz;
    const unsigned blocks = (unsigned)((cells + 255) / 256);
    if (storage == kMesoStoreF16)
        meso::meso_hydro_seed_kernel<meso::MesoF16><<<blocks, 256, 0, s>>>(forcing, nx, ny, nz, velocity_scale, scale,
                                                                           static_cast<__half*>(dst), solid);
    else if (storage == kMesoStoreI16)
        meso::meso_hydro_seed_kernel<meso::MesoI16><<<blocks, 256, 0, s>>>(forcing, nx, ny, nz, velocity_scale, scale,
                                                                           static_cast<short*>(dst), solid);
    else
        meso::meso_hydro_seed_kernel<meso::MesoF32><<<blocks, 256, 0, s>>>(forcing, nx, ny, nz, velocity_scale, scale,
                                                                           static_cast<float*>(dst), solid);
    count_launch();
    return cudaGetLastError();
}

cudaError_t meso_hydro_flags(const meso::HydroArgs& a, const uint8_t* solid, uint32_t* flags, cudaStream_t s) {
    const long long cells = (long long)a.nx * a.ny * a.nz;
    meso::meso_hydro_flags_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(a, solid, flags);
    count_launch();
    return cudaGetLastError();
}

cudaError_t meso_hydro_mask(const float* forcing, long long cells, uint8_t* solid, cudaStream_t s) {
    meso::meso_mask_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(forcing, cells, solid);
    count_launch();
    return cudaGetLastError();
}

template <class S>
static void hydro_dispatch(const meso::HydroArgs& a, int mode, unsigned blocks, int threads, cudaStream_t s) {
    if (mode == kHydroInit)
        meso::meso_hydro_kernel<S, kHydroInit><<<blocks, threads, 0, s>>>(a);
    else if (mode == kHydroStep)
        meso::meso_hydro_kernel<S, kHydroStep><<<blocks, threads, 0, s>>>(a);
    else
        meso::meso_hydro_kernel<S, kHydroOutput><<<blocks, threads, 0, s>>>(a);
}

cudaError_t meso_hydro_launch(const meso::HydroArgs& a, int mode, int storage, int threads, cudaStream_t s) {
    if (threads != 64 && threads != 128 && threads != 256) return cudaErrorInvalidValue;
    const long long cells = (long long)a.nx * a.ny * a.nz;
    const unsigned blocks = (unsigned)((cells + threads - 1) / threads);
    if (storage == kMesoStoreF16)
        hydro_dispatch<meso::MesoF16>(a, mode, blocks, threads, s);
    else if (storage == kMesoStoreI16)
        hydro_dispatch<meso::MesoI16>(a, mode, blocks, threads, s);
    else
        hydro_dispatch<meso::MesoF32>(a, mode, blocks, threads, s);
    count_launch();
    return cudaGetLastError();
}

}  // namespace aero
