// ORACLE — test infrastructure only. Not part of the product.
//
// CPU restatement of the reference's D3Q19 mesoscale step (TRT hydrodynamic
// and thermal double distribution), templated on the arithmetic type: the
// float instantiation reproduces the reference CPU step operation for
// operation (pinned against the reference library in oracle/_ref), the double
// one is the FP64 run of the same scheme. It follows
//   lattice / feq / trt_odd_tau      native/src/aero_lbm_mesoscale.cpp:146-272
//   seed_mesoscale_state             native/src/aero_lbm_mesoscale.cpp:298-333
//   laplacians, terrain gradient     native/src/aero_lbm_mesoscale.cpp:335-391
//   compute_cell_targets             native/src/aero_lbm_mesoscale.cpp:393-530
//   mesoscale_cpu_step               native/src/aero_lbm_mesoscale.cpp:548-738
//   derive_transport                 native/src/aero_lbm_mesoscale.cpp:45-68,
//                                    native/include/aero_lbm_hydro_core.h:109-115,
//                                    native/src/aero_lbm_thermal_core.cpp:5-15
//
// Options the reference does not have (off = the reference step): periodic
// x/z sides, a free-slip (specular) top, a uniform body force (Guo source in
// the hydrodynamic collision), a fixed hydrodynamic tau (the reference clamps
// it to >= 0.58) and Smagorinsky SGS on the even TRT rate.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <memory>
#include <vector>

#include "parallel_for.h"

namespace {

constexpr int Q = 19;
constexpr int kCh = 25;
constexpr int kOut = 6;
constexpr int kCx[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
constexpr int kCy[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
constexpr int kCz[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
constexpr int kOpp[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};

// forcing channels (native/src/aero_lbm_mesoscale.cpp:115-139)
enum {
    kTerrain = 0, kAmbientTarget = 2, kDeepTarget = 3, kSurfaceTarget = 4, kRoughness = 5, kBgX = 6, kBgZ = 7,
    kHumidity = 9, kConvHeat = 10, kConvMoist = 11, kConvInX = 12, kConvInZ = 13, kTorX = 14, kTorZ = 15,
    kTorHeat = 16, kTorMoist = 17, kTorUp = 18, kNestUp = 19, kNestDX = 20, kNestDZ = 21, kNestDAmb = 22,
    kNestDSurf = 23, kSolid = 24
};

}  // namespace

extern "C" {
typedef struct OracleD3Q19Options {
    int periodic_sides;     // x and z wrap instead of equilibrium inflow
    int free_slip_top;      // y = ny is a specular wall instead of equilibrium inflow
    int fixed_tau;          // use tau_hydro below instead of the derived, clamped tau
    int enable_sgs;         // Smagorinsky on the even hydrodynamic rate
    int disable_edge_blend; // no 2-cell equilibrium blend at the sides / top
    int hydro_only;         // hydrodynamic distribution alone: relax toward the cell's own
                            // rho, u (no forcing targets); output (rho, 0, 0, wind)
    double tau_hydro;
    double smagorinsky_c;
    double body_force[3];   // lattice force density (x, y, z; y is up)
} OracleD3Q19Options;

typedef struct OracleD3Q19Transport {
    double velocity_scale;  // m/s per lattice unit
    double tau_shear;       // molecular hydrodynamic tau (before clamps)
    double tau_thermal;     // molecular thermal tau (before clamps)
} OracleD3Q19Transport;
}

namespace {

template <typename T>
struct Meso {
    int nx = 0, ny = 0, nz = 0, cells = 0;
    T w[Q];
    T vscale = T(1), tau_s = T(0.58), tau_t = T(0.58);
    OracleD3Q19Options opt{};
    bool initialized = false;
    std::vector<T> f, g, fn, gn, rho, ambient, deep, surface, wx, wy, wz;

    Meso() {
        w[0] = T(1.0) / T(3.0);
        for (int q = 1; q < 7; ++q) w[q] = T(1.0) / T(18.0);
        for (int q = 7; q < Q; ++q) w[q] = T(1.0) / T(36.0);
    }
    int idx(int x, int y, int z) const { return (x * ny + y) * nz + z; }
    static int di(int cell, int q) { return cell * Q + q; }
    static T clampv(T v, T lo, T hi) { return std::clamp(v, lo, hi); }
    static T clamp_speed(T u) { return std::clamp(u, T(-0.35), T(0.35)); }
    T feq(int q, T r, T ux, T uy, T uz) const {
        const T cu = T(3.0) * (T(kCx[q]) * ux + T(kCy[q]) * uy + T(kCz[q]) * uz);
        const T uu = ux * ux + uy * uy + uz * uz;
        return w[q] * r * (T(1.0) + cu + T(0.5) * cu * cu - T(1.5) * uu);
    }
    T geq(int q, T t, T ux, T uy, T uz) const {
        const T cu = T(3.0) * (T(kCx[q]) * ux + T(kCy[q]) * uy + T(kCz[q]) * uz);
        return w[q] * t * (T(1.0) + cu);
    }
    static T trt_odd(T even_tau) {
        const T d = std::max(T(0.03), even_tau - T(0.5));
        return std::clamp(T(0.5) + T(0.25) / d, T(0.55), T(2.5));
    }
    static bool solid(const float* F, int cell) { return F[cell * kCh + kSolid] > 0.5f; }
    static T wall_temp(const float* F, int cell) { return T(F[cell * kCh + kSurfaceTarget]) + T(F[cell * kCh + kNestDSurf]); }
    T ch(const float* F, int cell, int c) const { return T(F[cell * kCh + c]); }

    void allocate(int nx_, int ny_, int nz_) {
        nx = nx_; ny = ny_; nz = nz_; cells = nx * ny * nz;
        f.assign((size_t)cells * Q, T(0)); g = f; fn = f; gn = f;
        rho.assign(cells, T(1)); ambient.assign(cells, T(0)); deep = ambient; surface = ambient;
        wx = ambient; wy = ambient; wz = ambient;
    }

    void seed(const float* F) {
        for (int i = 0; i < cells; ++i) {
            const T amb_t = ch(F, i, kAmbientTarget) + ch(F, i, kNestDAmb);
            const T surf_t = ch(F, i, kSurfaceTarget) + ch(F, i, kNestDSurf);
            const bool s = solid(F, i);
            const T bx = ch(F, i, kBgX) + ch(F, i, kNestDX);
            const T bz = ch(F, i, kBgZ) + ch(F, i, kNestDZ);
            const T by = ch(F, i, kNestUp) + ch(F, i, kTorUp);
            const T den = std::max(T(1.0e-6), vscale);
            const T lx = clamp_speed((s ? T(0) : bx) / den);
            const T ly = clamp_speed((s ? T(0) : by) / den);
            const T lz = clamp_speed((s ? T(0) : bz) / den);
            rho[i] = T(1);
            ambient[i] = s ? surf_t : amb_t;
            deep[i] = ch(F, i, kDeepTarget);
            surface[i] = surf_t;
            wx[i] = s ? T(0) : bx; wy[i] = s ? T(0) : by; wz[i] = s ? T(0) : bz;
            for (int q = 0; q < Q; ++q) {
                f[di(i, q)] = feq(q, T(1.0), lx, ly, lz);
                g[di(i, q)] = geq(q, ambient[i], lx, ly, lz);
            }
        }
    }

    T hlap(const std::vector<T>& a, int x, int y, int z) const {
        const T c = a[idx(x, y, z)];
        const T xp = a[idx(std::min(nx - 1, x + 1), y, z)], xm = a[idx(std::max(0, x - 1), y, z)];
        const T zp = a[idx(x, y, std::min(nz - 1, z + 1))], zm = a[idx(x, y, std::max(0, z - 1))];
        return xp + xm + zp + zm - T(4.0) * c;
    }
    T vlap(const std::vector<T>& a, int x, int y, int z) const {
        if (ny <= 1) return T(0);
        const T c = a[idx(x, y, z)];
        const T yp = a[idx(x, std::min(ny - 1, y + 1), z)], ym = a[idx(x, std::max(0, y - 1), z)];
        return yp + ym - T(2.0) * c;
    }
    T slope(const float* F, int x, int y, int z, int axis) const {
        const int xp = std::min(nx - 1, x + 1), xm = std::max(0, x - 1);
        const int zp = std::min(nz - 1, z + 1), zm = std::max(0, z - 1);
        if (axis == 0) return T(0.5) * (T(F[idx(xp, y, z) * kCh + kTerrain]) - T(F[idx(xm, y, z) * kCh + kTerrain]));
        return T(0.5) * (T(F[idx(x, y, zp) * kCh + kTerrain]) - T(F[idx(x, y, zm) * kCh + kTerrain]));
    }

    struct Targets { T rho, ux, uy, uz, teq, nsurf, ndeep; };

    // hydro_only: the cell's own moments, no target relaxation.
    Targets own_moments(const float* F, int i) const {
        if (solid(F, i)) return Targets{T(1), T(0), T(0), T(0), T(0), surface[i], deep[i]};
        T r = T(0), ux = T(0), uy = T(0), uz = T(0);
        for (int q = 0; q < Q; ++q) {
            const T fq = f[di(i, q)];
            r += fq;
            ux += fq * T(kCx[q]); uy += fq * T(kCy[q]); uz += fq * T(kCz[q]);
        }
        r = std::max(T(1.0e-6), r);
        ux /= r; uy /= r; uz /= r;
        return Targets{r, ux, uy, uz, T(0), surface[i], deep[i]};
    }

    Targets targets(const float* F, T dt_s, int x, int y, int z) const {
        const int i = idx(x, y, z);
        const T dt = std::max(T(1.0e-3), dt_s);
        const T amb_relax = clampv(dt / T(600.0), T(0), T(1));
        const T deep_relax = clampv(dt / T(2400.0), T(0), T(1));
        const T surf_relax = clampv(dt / T(300.0), T(0), T(1));
        const T wind_relax = clampv(dt / T(60.0), T(0), T(1));
        T r = T(0), ux = T(0), uy = T(0), uz = T(0), amb = T(0);
        for (int q = 0; q < Q; ++q) {
            const T fq = f[di(i, q)];
            r += fq;
            ux += fq * T(kCx[q]); uy += fq * T(kCy[q]); uz += fq * T(kCz[q]);
            amb += g[di(i, q)];
        }
        r = std::max(T(1.0e-6), r);
        ux /= r; uy /= r; uz /= r;
        const T amb_t = ch(F, i, kAmbientTarget) + ch(F, i, kNestDAmb);
        const T deep_t = ch(F, i, kDeepTarget);
        const T surf_t = ch(F, i, kSurfaceTarget) + ch(F, i, kNestDSurf);
        const T rough = std::max(T(0), ch(F, i, kRoughness));
        const T conv_h = ch(F, i, kConvHeat), conv_m = ch(F, i, kConvMoist);
        const T conv_x = ch(F, i, kConvInX), conv_z = ch(F, i, kConvInZ);
        const T tor_x = ch(F, i, kTorX), tor_z = ch(F, i, kTorZ), tor_h = ch(F, i, kTorHeat), tor_m = ch(F, i, kTorMoist);
        const T tor_up = ch(F, i, kTorUp), nest_up = ch(F, i, kNestUp);
        const T nest_dx = ch(F, i, kNestDX), nest_dz = ch(F, i, kNestDZ);
        const T bx = ch(F, i, kBgX) + nest_dx + conv_x + tor_x;
        const T bz = ch(F, i, kBgZ) + nest_dz + conv_z + tor_z;
        const T by = nest_up + tor_up;
        if (solid(F, i)) return Targets{T(1), T(0), T(0), T(0), surf_t, surf_t, deep_t};
        const T hum = clampv(ch(F, i, kHumidity) + conv_m + tor_m, T(0), T(1));
        const T sx = slope(F, x, y, z, 0), sz = slope(F, x, y, z, 1);
        const T s_hl = hlap(surface, x, y, z), s_vl = vlap(surface, x, y, z);
        const T d_vl = vlap(deep, x, y, z);
        const T a_hl = hlap(ambient, x, y, z), a_vl = vlap(ambient, x, y, z);
        const T ndeep = deep[i] + deep_relax * (deep_t - deep[i]) + T(0.01) * d_vl;
        const T damp = T(1.0) - T(0.12) * hum;
        const T nsurf = surface[i] + surf_relax * damp * (surf_t - surface[i]) + T(0.10) * (ndeep - surface[i]) +
                        T(0.04) * conv_h + T(0.08) * tor_h + T(0.05) * s_hl + T(0.025) * s_vl;
        const T den = std::max(T(1.0e-6), vscale);
        const T lx = clamp_speed(bx / den), ly = clamp_speed(by / den), lz = clamp_speed(bz / den);
        const T push = T(0.0008) * (nsurf - amb);
        const T nsw = T(1.0) - T(y) / std::max(T(1.0), T(ny - 1));
        const T lift = T(0.0015) * (lx * sx + lz * sz) * nsw;
        const T blift = T(0.0009) * (nsurf - amb) * nsw;
        const T steer_x = T(-0.005) * sx * lz;
        const T steer_z = T(0.005) * sz * lx;
        const T drag = clampv(rough * T(0.02), T(0), T(0.25));
        const T tux = clamp_speed(lx + steer_x + push * sx - drag * ux);
        const T tuz = clamp_speed(lz + steer_z + push * sz - drag * uz);
        const T tuy = clamp_speed(ly + lift + blift - drag * uy);
        const T rux = clamp_speed((T(1.0) - wind_relax) * ux + wind_relax * tux);
        const T ruy = clamp_speed((T(1.0) - wind_relax) * uy + wind_relax * tuy);
        const T ruz = clamp_speed((T(1.0) - wind_relax) * uz + wind_relax * tuz);
        const T src = amb_relax * (amb_t - amb) + (T(0.018) + T(0.004) * hum) * (nsurf - amb) + T(0.01) * (ndeep - amb) +
                      T(0.08) * conv_h * (T(0.5) + T(0.5) * hum) + T(0.10) * tor_h * (T(0.45) + T(0.55) * hum) +
                      T(0.06) * tor_up + T(0.06) * nest_up + T(0.01) * a_hl + T(0.02) * a_vl;
        return Targets{r, rux, ruy, ruz, amb + src, nsurf, ndeep};
    }

    void step(const float* F, T dt_s, float* out) {
        const T tau_h = opt.fixed_tau ? T(opt.tau_hydro) : clampv(tau_s, T(0.58), T(2.5));
        const T tau_h_odd = trt_odd(tau_h);
        const T om_h_odd = T(1.0) / tau_h_odd;
        const T tau_t = clampv(tau_t_v(), T(0.58), T(2.5));
        const T tau_t_odd = trt_odd(tau_t);
        const T om_t_even = T(1.0) / tau_t;
        const T om_t_odd = T(1.0) / tau_t_odd;
        const T max_speed = T(0.35) * vscale;
        std::vector<T> pf(f.size()), pg(g.size()), ndeep(cells), nsurf(cells);
        const T fx = T(opt.body_force[0]), fy = T(opt.body_force[1]), fz = T(opt.body_force[2]);
        const bool forced = fx != T(0) || fy != T(0) || fz != T(0);
        oracle_par::parallel_for(nx, [&](int x) {
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    const int i = idx(x, y, z);
                    const Targets t = opt.hydro_only ? own_moments(F, i) : targets(F, dt_s, x, y, z);
                    ndeep[i] = t.ndeep;
                    nsurf[i] = t.nsurf;
                    T om_h_even = T(1.0) / tau_h;
                    T tux = t.ux, tuy = t.uy, tuz = t.uz;
                    if (forced && !solid(F, i)) {
                        tux += T(0.5) * fx / t.rho; tuy += T(0.5) * fy / t.rho; tuz += T(0.5) * fz / t.rho;
                    }
                    if (opt.enable_sgs && !solid(F, i)) {
                        // |Pi_neq| from the non-equilibrium second moment of f
                        T pxx = T(0), pyy = T(0), pzz = T(0), pxy = T(0), pxz = T(0), pyz = T(0);
                        for (int q = 0; q < Q; ++q) {
                            const T ne = f[di(i, q)] - feq(q, t.rho, tux, tuy, tuz);
                            pxx += ne * T(kCx[q] * kCx[q]); pyy += ne * T(kCy[q] * kCy[q]); pzz += ne * T(kCz[q] * kCz[q]);
                            pxy += ne * T(kCx[q] * kCy[q]); pxz += ne * T(kCx[q] * kCz[q]); pyz += ne * T(kCy[q] * kCz[q]);
                        }
                        const T qn = std::sqrt(pxx * pxx + pyy * pyy + pzz * pzz + T(2) * (pxy * pxy + pxz * pxz + pyz * pyz));
                        const T nu0 = (tau_h - T(0.5)) / T(3.0);
                        const T cs2 = T(opt.smagorinsky_c) * T(opt.smagorinsky_c);
                        const T nut = std::min(cs2 * qn / std::max(T(1e-6), T(2) * t.rho * nu0), T(5) * nu0);
                        om_h_even = T(1.0) / (T(0.5) + T(3.0) * (nu0 + nut));
                    }
                    for (int q = 0; q < Q; ++q) {
                        const int qo = kOpp[q];
                        if (q > qo) continue;
                        const int d = di(i, q);
                        T sq = T(0), sqo = T(0);
                        if (forced && !solid(F, i)) {
                            const T pref = T(1.0) - T(0.5) * om_h_even;
                            const T cu = T(kCx[q]) * tux + T(kCy[q]) * tuy + T(kCz[q]) * tuz;
                            const T cf = T(kCx[q]) * fx + T(kCy[q]) * fy + T(kCz[q]) * fz;
                            const T uf = tux * fx + tuy * fy + tuz * fz;
                            sq = pref * w[q] * (T(3) * (cf - uf) + T(9) * cu * cf);
                            sqo = pref * w[q] * (T(3) * (-cf - uf) + T(9) * cu * cf);
                        }
                        if (q == qo) {
                            const T fe = feq(q, t.rho, tux, tuy, tuz);
                            const T ge = geq(q, t.teq, t.ux, t.uy, t.uz);
                            pf[d] = f[d] - om_h_even * (f[d] - fe) + sq;
                            pg[d] = g[d] - om_t_even * (g[d] - ge);
                            continue;
                        }
                        const int od = di(i, qo);
                        const T fe = feq(q, t.rho, tux, tuy, tuz), feo = feq(qo, t.rho, tux, tuy, tuz);
                        const T ge = geq(q, t.teq, t.ux, t.uy, t.uz), geo = geq(qo, t.teq, t.ux, t.uy, t.uz);
                        const T fev = T(0.5) * (f[d] + f[od]), fod = T(0.5) * (f[d] - f[od]);
                        const T feev = T(0.5) * (fe + feo), feod = T(0.5) * (fe - feo);
                        const T fep = fev - om_h_even * (fev - feev);
                        const T fop = fod - om_h_odd * (fod - feod);
                        pf[d] = fep + fop + sq;
                        pf[od] = fep - fop + sqo;
                        const T gev = T(0.5) * (g[d] + g[od]), god = T(0.5) * (g[d] - g[od]);
                        const T geev = T(0.5) * (ge + geo), geod = T(0.5) * (ge - geo);
                        const T gep = gev - om_t_even * (gev - geev);
                        const T gop = god - om_t_odd * (god - geod);
                        pg[d] = gep + gop;
                        pg[od] = gep - gop;
                    }
                }
        });
        oracle_par::parallel_for(nx, [&](int x) {
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    const int i = idx(x, y, z);
                    if (solid(F, i)) {
                        const T wt = wall_temp(F, i);
                        for (int q = 0; q < Q; ++q) {
                            fn[di(i, q)] = feq(q, T(1.0), T(0), T(0), T(0));
                            gn[di(i, q)] = geq(q, wt, T(0), T(0), T(0));
                        }
                        continue;
                    }
                    const T den = std::max(T(1.0e-6), vscale);
                    const T bx = clamp_speed((ch(F, i, kBgX) + ch(F, i, kNestDX) + ch(F, i, kConvInX) + ch(F, i, kTorX)) / den);
                    const T bz = clamp_speed((ch(F, i, kBgZ) + ch(F, i, kNestDZ) + ch(F, i, kConvInZ) + ch(F, i, kTorZ)) / den);
                    const T btemp = ch(F, i, kAmbientTarget) + ch(F, i, kNestDAmb);
                    const T by = clamp_speed((ch(F, i, kNestUp) + ch(F, i, kTorUp)) / den);
                    int edge = std::min(std::min(x, z), std::min(nx - 1 - x, nz - 1 - z));
                    int top = ny - 1 - y;
                    if (opt.periodic_sides) edge = 1 << 20;
                    if (opt.free_slip_top) top = 1 << 20;
                    const int sponge = std::min(edge, top);
                    T alpha = sponge <= 0 ? T(1.0) : (sponge < 2 ? T(0.5) : T(0.0));
                    if (opt.disable_edge_blend) alpha = T(0);
                    for (int q = 0; q < Q; ++q) {
                        int sx = x - kCx[q], sy = y - kCy[q], sz = z - kCz[q];
                        if (opt.periodic_sides) {
                            sx = (sx + nx) % nx;
                            sz = (sz + nz) % nz;
                        }
                        const int d = di(i, q);
                        T fv, gv;
                        bool bounced = false;
                        if (sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz) {
                            const int src = idx(sx, sy, sz);
                            if (solid(F, src)) {
                                fv = pf[di(i, kOpp[q])];
                                gv = geq(q, wall_temp(F, src), T(0), T(0), T(0));
                                bounced = true;
                            } else {
                                fv = pf[di(src, q)];
                                gv = pg[di(src, q)];
                            }
                        } else if (sy < 0) {
                            fv = pf[di(i, kOpp[q])];
                            gv = geq(q, wall_temp(F, i), T(0), T(0), T(0));
                            bounced = true;
                        } else if (opt.free_slip_top && sy >= ny && sx >= 0 && sx < nx && sz >= 0 && sz < nz) {
                            // specular reflection at the lid: the population that left the cell
                            // (sx, ny-1, sz) upward with the mirrored velocity
                            int mq = 0;
                            for (int k = 0; k < Q; ++k)
                                if (kCx[k] == kCx[q] && kCy[k] == -kCy[q] && kCz[k] == kCz[q]) mq = k;
                            const int src = idx(sx, ny - 1, sz);
                            if (solid(F, src)) {
                                fv = pf[di(i, kOpp[q])];
                                gv = geq(q, wall_temp(F, src), T(0), T(0), T(0));
                                bounced = true;
                            } else {
                                fv = pf[di(src, mq)];
                                gv = pg[di(src, mq)];
                            }
                        } else {
                            fv = feq(q, T(1.0), bx, by, bz);
                            gv = geq(q, btemp, bx, by, bz);
                        }
                        if (alpha > T(0) && !bounced) {
                            const T fb = feq(q, T(1.0), bx, by, bz);
                            const T gb = geq(q, btemp, bx, by, bz);
                            fv = (T(1.0) - alpha) * fv + alpha * fb;
                            gv = (T(1.0) - alpha) * gv + alpha * gb;
                        }
                        fn[d] = fv;
                        gn[d] = gv;
                    }
                }
        });
        f.swap(fn);
        g.swap(gn);
        deep.swap(ndeep);
        surface.swap(nsurf);
        for (int i = 0; i < cells; ++i) {
            if (solid(F, i)) {
                rho[i] = T(1); ambient[i] = wall_temp(F, i);
                wx[i] = wy[i] = wz[i] = T(0);
                continue;
            }
            T r = T(0), ux = T(0), uy = T(0), uz = T(0), amb = T(0);
            for (int q = 0; q < Q; ++q) {
                const T fq = f[di(i, q)];
                r += fq;
                ux += fq * T(kCx[q]); uy += fq * T(kCy[q]); uz += fq * T(kCz[q]);
                amb += g[di(i, q)];
            }
            r = std::max(T(1.0e-6), r);
            ux /= r; uy /= r; uz /= r;
            rho[i] = r;
            ambient[i] = amb;
            wx[i] = std::clamp(ux * vscale, -max_speed, max_speed);
            wy[i] = std::clamp(uy * vscale, -max_speed, max_speed);
            wz[i] = std::clamp(uz * vscale, -max_speed, max_speed);
        }
        if (out)
            for (int i = 0; i < cells; ++i) {
                float* o = out + (size_t)i * kOut;
                if (opt.hydro_only) {
                    o[0] = float(rho[i]); o[1] = 0.0f; o[2] = 0.0f;
                } else {
                    o[0] = float(ambient[i]); o[1] = float(deep[i]); o[2] = float(surface[i]);
                }
                o[3] = float(wx[i]); o[4] = float(wy[i]); o[5] = float(wz[i]);
            }
    }
    T tau_t_v() const { return tau_t; }
};

struct MesoHandle {
    std::unique_ptr<Meso<float>> f32;
    std::unique_ptr<Meso<double>> f64;
    double dt = 5.0;
};

template <typename T>
void set_transport(Meso<T>& m, const OracleD3Q19Transport& t) {
    m.vscale = T(t.velocity_scale);
    m.tau_s = T(t.tau_shear);
    m.tau_t = T(t.tau_thermal);
}

}  // namespace

extern "C" {

void* oracle_d3q19_create(int nx, int ny, int nz, int precision, const OracleD3Q19Transport* transport,
                          const OracleD3Q19Options* options, double dt_s) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !transport) return nullptr;
    auto* h = new MesoHandle();
    h->dt = dt_s;
    if (precision == 0) {
        h->f32 = std::make_unique<Meso<float>>();
        h->f32->allocate(nx, ny, nz);
        set_transport(*h->f32, *transport);
        if (options) h->f32->opt = *options;
    } else {
        h->f64 = std::make_unique<Meso<double>>();
        h->f64->allocate(nx, ny, nz);
        set_transport(*h->f64, *transport);
        if (options) h->f64->opt = *options;
    }
    return h;
}

void oracle_d3q19_destroy(void* handle) { delete static_cast<MesoHandle*>(handle); }

// One call of aero_lbm_mesoscale_step_context: seeds on the first call,
// writes cells x 6 floats (ambient, deep ground, surface, wind x, y, z).
int oracle_d3q19_step(void* handle, const float* forcing, float* out_state) {
    auto* h = static_cast<MesoHandle*>(handle);
    if (!h || !forcing) return 0;
    if (h->f32) {
        if (!h->f32->initialized) { h->f32->seed(forcing); h->f32->initialized = true; }
        h->f32->step(forcing, float(h->dt), out_state);
    } else {
        if (!h->f64->initialized) { h->f64->seed(forcing); h->f64->initialized = true; }
        h->f64->step(forcing, h->dt, out_state);
    }
    return 1;
}

}  // extern "C"
