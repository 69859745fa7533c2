// Discrete adjoint of the D3Q27 cumulant collision, per cell.
//
// `collide_fwd<T>` is the factorised cumulant collision of the brick step
// (collide27.cuh; the reference's scheme, native/src/aero_lbm_jni.cpp:2209-2413):
// raw moments -> midpoint velocity with buoyancy + body force and the speed
// clamp -> second-order central moments -> Smagorinsky tau -> relaxed
// cumulants with the Gaussian closure for orders 4 and 6 -> separable
// central-to-population map -> conservation fix-up -> Guo source. It is
// written over a scalar type T (float for the forward and the adjoint sweep,
// double for the finite-difference reference runs) and keeps what the
// reverse sweep needs in `CollideTape<T>`.
//
// `collide_vjp<T>` is its reverse mode, written out stage by stage: given the
// adjoint of the 27 post-collision populations it returns the adjoint of the
// 27 pre-collision populations and of the cell's force density (the Jacobian
// transposed times a vector, without forming the Jacobian). Clamps contribute
// the derivative of the branch taken. Both run on the host and the device.
#pragma once

#include <cmath>

#include "collide27.cuh"
#include "lattice.cuh"

namespace aero {
namespace adj {

__host__ __device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__host__ __device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }
__host__ __device__ __forceinline__ float sqrt_t(float a) { return sqrtf(a); }
__host__ __device__ __forceinline__ double sqrt_t(double a) { return sqrt(a); }
template <class T>
__host__ __device__ __forceinline__ T max_t(T a, T b) { return a > b ? a : b; }
template <class T>
__host__ __device__ __forceinline__ T min_t(T a, T b) { return a < b ? a : b; }

template <class T>
__host__ __device__ __forceinline__ T wq(int q) { return T(q_w(q)); }

template <class T>
__host__ __device__ __forceinline__ T feq_t(int q, T rho, T ux, T uy, T uz) {
    const T cu = T(3) * (T(q_cx(q)) * ux + T(q_cy(q)) * uy + T(q_cz(q)) * uz);
    const T uu = ux * ux + uy * uy + uz * uz;
    return wq<T>(q) * rho * (T(1) + cu + T(0.5) * cu * cu - T(1.5) * uu);
}

// d feq(q, rho, u) / d u
template <class T>
__host__ __device__ __forceinline__ void dfeq_du(int q, T rho, T ux, T uy, T uz, T (&d)[3]) {
    const T cx = T(q_cx(q)), cy = T(q_cy(q)), cz = T(q_cz(q));
    const T cu = T(3) * (cx * ux + cy * uy + cz * uz);
    const T k = wq<T>(q) * rho;
    // d/du_a [3 c.u + 4.5 (c.u)^2 - 1.5 u.u] = 3 c_a + 3 cu c_a - 3 u_a
    d[0] = k * (T(3) * cx + cu * T(3) * cx - T(3) * ux);
    d[1] = k * (T(3) * cy + cu * T(3) * cy - T(3) * uy);
    d[2] = k * (T(3) * cz + cu * T(3) * cz - T(3) * uz);
}

// 1-D central -> population map along one axis (see back_line in collide27.cuh).
template <class T>
struct Line {
    __host__ __device__ static void fwd(T m0, T m1, T m2, T u, T& fm, T& f0, T& fp) {
        const T r1 = fma_t(u, m0, m1);
        const T r2 = fma_t(u, r1 + m1, m2);
        fm = T(0.5) * (r2 - r1);
        f0 = m0 - r2;
        fp = T(0.5) * (r1 + r2);
    }
    // adjoint: accumulates into lm0, lm1, lm2, lu
    __host__ __device__ static void rev(T m0, T m1, T u, T lfm, T lf0, T lfp, T& lm0, T& lm1, T& lm2, T& lu) {
        const T r1 = fma_t(u, m0, m1);
        const T lr2 = T(0.5) * lfm - lf0 + T(0.5) * lfp;
        T lr1 = T(-0.5) * lfm + T(0.5) * lfp;
        lm0 += lf0;
        lm2 += lr2;
        lr1 += u * lr2;
        lm1 += u * lr2;
        lu += (r1 + m1) * lr2;
        lm0 += u * lr1;
        lm1 += lr1;
        lu += m0 * lr1;
    }
};

template <class T>
struct CollideTape {
    T rho, rs, ir, r1[3], F[3], bq;
    T uraw[3], u[3], umax_scale;
    bool clamped;
    T c200, c020, c002, c110, c101, c011, eq2;
    T nxx, nyy, nzz, qm, D, nu_tot, tau_s, tau_n, om_o, sd, so, pref;
    bool sgs_on, qpos, d_free, nut_free, nu_free, taus_free, taun_free, sd_free, so_free, pref_free, forced;
    T K[14];  // rs, k200, k020, k002, k110, k101, k011, k220, k202, k022, k211, k121, k112, k222
};

// Indices into CollideTape::K.
enum { K0 = 0, K200, K020, K002, K110, K101, K011, K220, K202, K022, K211, K121, K112, K222 };

// Separable central -> population map of the 14 post-collision central
// moments (x pass over the 9 (b, c) lines, then y, then z).
template <class T>
__host__ __device__ __forceinline__ void back_transform(const T (&K)[14], const T (&u)[3], T (&g)[3][9], T (&h)[27],
                                                        T (&fb)[27]) {
    // (b, c) line -> (m0, m1, m2) along x
    const T Z = T(0);
    const T lines[9][3] = {
        {K[K0], Z, K[K200]},   {Z, K[K101], Z},    {K[K002], Z, K[K202]},
        {Z, K[K110], Z},       {K[K011], Z, K[K211]}, {Z, K[K112], Z},
        {K[K020], Z, K[K220]}, {Z, K[K121], Z},    {K[K022], Z, K[K222]},
    };
#pragma unroll
    for (int bc = 0; bc < 9; ++bc) Line<T>::fwd(lines[bc][0], lines[bc][1], lines[bc][2], u[0], g[0][bc], g[1][bc], g[2][bc]);
#pragma unroll
    for (int ix = 0; ix < 3; ++ix)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            Line<T>::fwd(g[ix][0 * 3 + c], g[ix][1 * 3 + c], g[ix][2 * 3 + c], u[1], h[(ix * 3 + 0) * 3 + c],
                         h[(ix * 3 + 1) * 3 + c], h[(ix * 3 + 2) * 3 + c]);
#pragma unroll
    for (int l = 0; l < 9; ++l) Line<T>::fwd(h[3 * l + 0], h[3 * l + 1], h[3 * l + 2], u[2], fb[3 * l + 0], fb[3 * l + 1], fb[3 * l + 2]);
}

template <class T>
__host__ __device__ __forceinline__ T clamp_t(T v, T lo, T hi) { return min_t(hi, max_t(lo, v)); }
template <class T>
__host__ __device__ __forceinline__ bool inside(T v, T lo, T hi) { return v > lo && v < hi; }

// Forward collision of one fluid cell. `temp` is the cell's temperature
// (buoyancy), (cfx, cfy, cfz) its extra force density.
// kOutput = false fills the tape only (what the reverse sweep needs) and
// leaves fo unset.
template <class T, bool kOutput = true>
__host__ __device__ void collide_fwd(const T (&f)[27], const CollideParams& P, T temp, T cfx, T cfy, T cfz, T (&fo)[27],
                                     CollideTape<T>& s) {
    T r000 = 0, r100 = 0, r010 = 0, r001 = 0, r200 = 0, r020 = 0, r002 = 0, r110 = 0, r101 = 0, r011 = 0;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const T cx = T(q_cx(q)), cy = T(q_cy(q)), cz = T(q_cz(q)), v = f[q];
        r000 += v;
        r100 += cx * v;
        r010 += cy * v;
        r001 += cz * v;
        r200 += cx * cx * v;
        r020 += cy * cy * v;
        r002 += cz * cz * v;
        r110 += cx * cy * v;
        r101 += cx * cz * v;
        r011 += cy * cz * v;
    }
    s.rho = r000;
    s.rs = max_t(T(1e-6), r000);
    s.ir = T(1) / s.rs;
    s.r1[0] = r100; s.r1[1] = r010; s.r1[2] = r001;
    T F[3] = {T(0), T(0), T(0)};
    s.bq = T(0);
    if (P.enable_buoyancy) {
        s.bq = clamp_t(T(P.buoy_beta) * temp, -T(P.buoy_fmax), T(P.buoy_fmax));
        F[P.gravity_axis] += s.rs * s.bq;
    }
    F[0] += T(P.body_force[0]) + cfx;
    F[1] += T(P.body_force[1]) + cfy;
    F[2] += T(P.body_force[2]) + cfz;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        s.F[a] = F[a];
        s.uraw[a] = s.r1[a] * s.ir + T(0.5) * (F[a] * s.ir);
        s.u[a] = s.uraw[a];
    }
    const T s2 = s.uraw[0] * s.uraw[0] + s.uraw[1] * s.uraw[1] + s.uraw[2] * s.uraw[2];
    const T ms = T(P.max_speed);
    s.clamped = s2 > ms * ms;
    s.umax_scale = T(1);
    if (s.clamped) {
        s.umax_scale = ms / sqrt_t(s2);
#pragma unroll
        for (int a = 0; a < 3; ++a) s.u[a] = s.uraw[a] * s.umax_scale;
    }
    const T ux = s.u[0], uy = s.u[1], uz = s.u[2], rho = s.rho;
    s.c200 = fma_t(ux * ux, rho, fma_t(T(-2) * ux, r100, r200));
    s.c020 = fma_t(uy * uy, rho, fma_t(T(-2) * uy, r010, r020));
    s.c002 = fma_t(uz * uz, rho, fma_t(T(-2) * uz, r001, r002));
    s.c110 = fma_t(ux * uy, rho, fma_t(-ux, r010, fma_t(-uy, r100, r110)));
    s.c101 = fma_t(ux * uz, rho, fma_t(-ux, r001, fma_t(-uz, r100, r101)));
    s.c011 = fma_t(uy * uz, rho, fma_t(-uy, r001, fma_t(-uz, r010, r011)));
    s.eq2 = s.rs * T(kCs2f);

    s.sgs_on = P.enable_sgs != 0;
    s.tau_s = T(P.tau_shear_base);
    s.tau_n = T(P.tau_normal_base);
    if (s.sgs_on) {
        s.nxx = s.c200 - s.eq2; s.nyy = s.c020 - s.eq2; s.nzz = s.c002 - s.eq2;
        const T qn2 = s.nxx * s.nxx + s.nyy * s.nyy + s.nzz * s.nzz +
                      T(2) * (s.c110 * s.c110 + s.c101 * s.c101 + s.c011 * s.c011);
        s.qpos = qn2 > T(0);
        s.qm = sqrt_t(max_t(T(0), qn2));
        const T d = T(2) * s.rs * T(P.nu0);
        s.d_free = d > T(1e-6);
        s.D = max_t(T(1e-6), d);
        const T sm = s.qm / s.D;
        const T nut_raw = T(P.sgs_c2) * sm;
        s.nut_free = nut_raw < T(P.sgs_nut_cap);
        const T nut = min_t(nut_raw, T(P.sgs_nut_cap));
        s.nu_tot = T(P.nu0) + nut;
        s.nu_free = inside(s.nu_tot, T(kNuShearMin), T(kNuShearMax));
        const T tau_raw = T(0.5) + T(3) * clamp_t(s.nu_tot, T(kNuShearMin), T(kNuShearMax));
        s.taus_free = inside(tau_raw, T(kTauMin), T(kTauMax));
        s.tau_s = clamp_t(tau_raw, T(kTauMin), T(kTauMax));
        const T taun_raw = T(P.tau_normal_base) + (s.tau_s - T(P.tau_shear_base)) * T(P.sgs_bulk);
        s.taun_free = inside(taun_raw, T(kTauMin), T(kTauMax));
        s.tau_n = clamp_t(taun_raw, T(kTauMin), T(kTauMax));
    }
    s.om_o = T(1) / s.tau_s;
    const T sd_raw = T(1) / s.tau_n;
    s.sd_free = inside(sd_raw, T(0), T(1.95));
    s.sd = clamp_t(sd_raw, T(0), T(1.95));
    s.so_free = inside(s.om_o, T(0), T(1.95));
    s.so = clamp_t(s.om_o, T(0), T(1.95));

    T* K = s.K;
    K[K0] = s.rs;
    K[K200] = s.c200 + s.sd * (s.eq2 - s.c200);
    K[K020] = s.c020 + s.sd * (s.eq2 - s.c020);
    K[K002] = s.c002 + s.sd * (s.eq2 - s.c002);
    K[K110] = (T(1) - s.so) * s.c110;
    K[K101] = (T(1) - s.so) * s.c101;
    K[K011] = (T(1) - s.so) * s.c011;
    const T irs = s.ir;
    K[K220] = (K[K200] * K[K020] + T(2) * K[K110] * K[K110]) * irs;
    K[K202] = (K[K200] * K[K002] + T(2) * K[K101] * K[K101]) * irs;
    K[K022] = (K[K020] * K[K002] + T(2) * K[K011] * K[K011]) * irs;
    K[K211] = (K[K200] * K[K011] + T(2) * K[K110] * K[K101]) * irs;
    K[K121] = (K[K020] * K[K101] + T(2) * K[K110] * K[K011]) * irs;
    K[K112] = (K[K002] * K[K110] + T(2) * K[K101] * K[K011]) * irs;
    K[K222] = (K[K200] * K[K020] * K[K002] + T(2) * K[K110] * K[K110] * K[K002] + T(2) * K[K101] * K[K101] * K[K020] +
               T(2) * K[K011] * K[K011] * K[K200] + T(8) * K[K110] * K[K101] * K[K011]) * irs * irs;

    s.forced = (F[0] != T(0)) || (F[1] != T(0)) || (F[2] != T(0));
    const T omc = clamp_t(s.om_o, T(0), T(1.999));
    s.pref_free = inside(s.om_o, T(0), T(1.999)) && (T(1) - T(0.5) * omc) > T(0);
    s.pref = max_t(T(0), T(1) - T(0.5) * omc);
    if (!kOutput) return;

    T g[3][9], h[27];
    back_transform<T>(s.K, s.u, g, h, fo);

    T m0 = 0, m1x = 0, m1y = 0, m1z = 0;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        m0 += fo[q];
        m1x += T(q_cx(q)) * fo[q];
        m1y += T(q_cy(q)) * fo[q];
        m1z += T(q_cz(q)) * fo[q];
    }
    const T drho = s.rs - m0;
    const T djx = T(3) * (s.rs * ux - m1x), djy = T(3) * (s.rs * uy - m1y), djz = T(3) * (s.rs * uz - m1z);
    const T uf = ux * F[0] + uy * F[1] + uz * F[2];
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const T cx = T(q_cx(q)), cy = T(q_cy(q)), cz = T(q_cz(q));
        T add = drho + (cx * djx + cy * djy + cz * djz);
        if (s.forced) {
            const T cu = cx * ux + cy * uy + cz * uz;
            const T cf = cx * F[0] + cy * F[1] + cz * F[2];
            add += s.pref * (T(9) * cu * cf - T(3) * uf + T(3) * cf);
        }
        fo[q] += wq<T>(q) * add;
    }
}

// Reverse sweep of collide_fwd: lam_out (27) -> lam_in (27, overwritten) and
// lam_F (3, overwritten: adjoint of the cell's total force density, which is
// also that of its extra force density cf).
template <class T>
__host__ __device__ void collide_vjp(const CollideTape<T>& s, const CollideParams& P, const T (&lam_out)[27],
                                     T (&lam_in)[27], T (&lam_F)[3]) {
    const T ux = s.u[0], uy = s.u[1], uz = s.u[2];
    const T* F = s.F;
    T lu[3] = {T(0), T(0), T(0)}, lF[3] = {T(0), T(0), T(0)};
    T lrs = T(0), lrho = T(0), lom = T(0);

    // Guo source and fix-up: fo[q] = fb[q] + w_q (drho + c.dj + pref (9 cu cf - 3 uf + 3 cf))
    T ldrho = T(0), ldj[3] = {T(0), T(0), T(0)}, lpref = T(0);
    const T uf = ux * F[0] + uy * F[1] + uz * F[2];
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const T cx = T(q_cx(q)), cy = T(q_cy(q)), cz = T(q_cz(q));
        const T a = wq<T>(q) * lam_out[q];
        ldrho += a;
        ldj[0] += cx * a; ldj[1] += cy * a; ldj[2] += cz * a;
        if (s.forced) {
            const T cu = cx * ux + cy * uy + cz * uz;
            const T cf = cx * F[0] + cy * F[1] + cz * F[2];
            lpref += a * (T(9) * cu * cf - T(3) * uf + T(3) * cf);
            const T pa = s.pref * a;
            // d/du: 9 cf c - 3 F ; d/dF: 9 cu c - 3 u + 3 c
            lu[0] += pa * (T(9) * cf * cx - T(3) * F[0]);
            lu[1] += pa * (T(9) * cf * cy - T(3) * F[1]);
            lu[2] += pa * (T(9) * cf * cz - T(3) * F[2]);
            lF[0] += pa * (T(9) * cu * cx - T(3) * ux + T(3) * cx);
            lF[1] += pa * (T(9) * cu * cy - T(3) * uy + T(3) * cy);
            lF[2] += pa * (T(9) * cu * cz - T(3) * uz + T(3) * cz);
        }
    }
    if (s.forced && s.pref_free) lom += T(-0.5) * lpref;
    // drho = rs - sum fb ; dj = 3 (rs u - sum c fb)
    lrs += ldrho + T(3) * (ldj[0] * ux + ldj[1] * uy + ldj[2] * uz);
    lu[0] += T(3) * s.rs * ldj[0];
    lu[1] += T(3) * s.rs * ldj[1];
    lu[2] += T(3) * s.rs * ldj[2];
    T lfb[27];
#pragma unroll
    for (int q = 0; q < 27; ++q)
        lfb[q] = lam_out[q] - ldrho - T(3) * (T(q_cx(q)) * ldj[0] + T(q_cy(q)) * ldj[1] + T(q_cz(q)) * ldj[2]);

    // back transform (recompute the x and y passes, then reverse z, y, x)
    T g[3][9], h[27], fb[27];
    back_transform<T>(s.K, s.u, g, h, fb);
    T lh[27];
#pragma unroll
    for (int i = 0; i < 27; ++i) lh[i] = T(0);
#pragma unroll
    for (int l = 0; l < 9; ++l)
        Line<T>::rev(h[3 * l + 0], h[3 * l + 1], uz, lfb[3 * l + 0], lfb[3 * l + 1], lfb[3 * l + 2], lh[3 * l + 0],
                     lh[3 * l + 1], lh[3 * l + 2], lu[2]);
    T lg[3][9];
#pragma unroll
    for (int ix = 0; ix < 3; ++ix)
#pragma unroll
        for (int bc = 0; bc < 9; ++bc) lg[ix][bc] = T(0);
#pragma unroll
    for (int ix = 0; ix < 3; ++ix)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            Line<T>::rev(g[ix][0 * 3 + c], g[ix][1 * 3 + c], uy, lh[(ix * 3 + 0) * 3 + c], lh[(ix * 3 + 1) * 3 + c],
                         lh[(ix * 3 + 2) * 3 + c], lg[ix][0 * 3 + c], lg[ix][1 * 3 + c], lg[ix][2 * 3 + c], lu[1]);
    const T* K = s.K;
    const T Z = T(0);
    const T lines[9][3] = {
        {K[K0], Z, K[K200]},   {Z, K[K101], Z},    {K[K002], Z, K[K202]},
        {Z, K[K110], Z},       {K[K011], Z, K[K211]}, {Z, K[K112], Z},
        {K[K020], Z, K[K220]}, {Z, K[K121], Z},    {K[K022], Z, K[K222]},
    };
    // which K feeds (m0, m1, m2) of each (b, c) line (-1: zero)
    const int slot[9][3] = {
        {K0, -1, K200},   {-1, K101, -1}, {K002, -1, K202},
        {-1, K110, -1},   {K011, -1, K211}, {-1, K112, -1},
        {K020, -1, K220}, {-1, K121, -1}, {K022, -1, K222},
    };
    T lK[14];
#pragma unroll
    for (int i = 0; i < 14; ++i) lK[i] = T(0);
#pragma unroll
    for (int bc = 0; bc < 9; ++bc) {
        T l0 = T(0), l1 = T(0), l2 = T(0);
        Line<T>::rev(lines[bc][0], lines[bc][1], ux, lg[0][bc], lg[1][bc], lg[2][bc], l0, l1, l2, lu[0]);
        if (slot[bc][0] >= 0) lK[slot[bc][0]] += l0;
        if (slot[bc][1] >= 0) lK[slot[bc][1]] += l1;
        if (slot[bc][2] >= 0) lK[slot[bc][2]] += l2;
    }

    // closures of orders 4 and 6
    const T irs = s.ir;
    const T k200 = K[K200], k020 = K[K020], k002 = K[K002], k110 = K[K110], k101 = K[K101], k011 = K[K011];
    T l200 = lK[K200], l020 = lK[K020], l002 = lK[K002], l110 = lK[K110], l101 = lK[K101], l011 = lK[K011];
    T lirs = T(0);
    {
        T l = lK[K220];
        l200 += k020 * irs * l; l020 += k200 * irs * l; l110 += T(4) * k110 * irs * l;
        lirs += (k200 * k020 + T(2) * k110 * k110) * l;
        l = lK[K202];
        l200 += k002 * irs * l; l002 += k200 * irs * l; l101 += T(4) * k101 * irs * l;
        lirs += (k200 * k002 + T(2) * k101 * k101) * l;
        l = lK[K022];
        l020 += k002 * irs * l; l002 += k020 * irs * l; l011 += T(4) * k011 * irs * l;
        lirs += (k020 * k002 + T(2) * k011 * k011) * l;
        l = lK[K211];
        l200 += k011 * irs * l; l011 += k200 * irs * l; l110 += T(2) * k101 * irs * l; l101 += T(2) * k110 * irs * l;
        lirs += (k200 * k011 + T(2) * k110 * k101) * l;
        l = lK[K121];
        l020 += k101 * irs * l; l101 += k020 * irs * l; l110 += T(2) * k011 * irs * l; l011 += T(2) * k110 * irs * l;
        lirs += (k020 * k101 + T(2) * k110 * k011) * l;
        l = lK[K112];
        l002 += k110 * irs * l; l110 += k002 * irs * l; l101 += T(2) * k011 * irs * l; l011 += T(2) * k101 * irs * l;
        lirs += (k002 * k110 + T(2) * k101 * k011) * l;
        l = lK[K222];
        const T Q = k200 * k020 * k002 + T(2) * k110 * k110 * k002 + T(2) * k101 * k101 * k020 + T(2) * k011 * k011 * k200 +
                    T(8) * k110 * k101 * k011;
        const T lQ = irs * irs * l;
        lirs += T(2) * Q * irs * l;
        l200 += (k020 * k002 + T(2) * k011 * k011) * lQ;
        l020 += (k200 * k002 + T(2) * k101 * k101) * lQ;
        l002 += (k200 * k020 + T(2) * k110 * k110) * lQ;
        l110 += (T(4) * k110 * k002 + T(8) * k101 * k011) * lQ;
        l101 += (T(4) * k101 * k020 + T(8) * k110 * k011) * lQ;
        l011 += (T(4) * k011 * k200 + T(8) * k110 * k101) * lQ;
    }
    lrs += lK[K0];
    // ir = 1 / rs (rs >= 1e-6 always, so irs == ir)
    T lir = lirs;

    // relaxation: k_aa = c_aa + sd (eq2 - c_aa); k_ab = (1 - so) c_ab
    T lc200 = (T(1) - s.sd) * l200, lc020 = (T(1) - s.sd) * l020, lc002 = (T(1) - s.sd) * l002;
    T leq2 = s.sd * (l200 + l020 + l002);
    T lsd = (s.eq2 - s.c200) * l200 + (s.eq2 - s.c020) * l020 + (s.eq2 - s.c002) * l002;
    T lc110 = (T(1) - s.so) * l110, lc101 = (T(1) - s.so) * l101, lc011 = (T(1) - s.so) * l011;
    T lso = -(s.c110 * l110 + s.c101 * l101 + s.c011 * l011);
    if (s.so_free) lom += lso;
    T ltaun = s.sd_free ? -lsd / (s.tau_n * s.tau_n) : T(0);
    T ltaus = -lom / (s.tau_s * s.tau_s);
    if (s.sgs_on) {
        if (s.taun_free) ltaus += T(P.sgs_bulk) * ltaun;
        T lnu = (s.taus_free && s.nu_free) ? T(3) * ltaus : T(0);
        // nu_tot = nu0 + min(c2 qm / D, cap)
        const T lsm = s.nut_free ? T(P.sgs_c2) * lnu : T(0);
        const T lqm = lsm / s.D;
        if (s.d_free) lrs += -(s.qm / (s.D * s.D)) * T(2) * T(P.nu0) * lsm;
        if (s.qpos && s.qm > T(0)) {
            const T lqn2 = lqm / (T(2) * s.qm);
            const T lnxx = T(2) * s.nxx * lqn2, lnyy = T(2) * s.nyy * lqn2, lnzz = T(2) * s.nzz * lqn2;
            lc200 += lnxx; lc020 += lnyy; lc002 += lnzz;
            leq2 -= lnxx + lnyy + lnzz;
            lc110 += T(4) * s.c110 * lqn2;
            lc101 += T(4) * s.c101 * lqn2;
            lc011 += T(4) * s.c011 * lqn2;
        }
    }
    lrs += leq2 * T(kCs2f);

    // central moments about u
    const T r100 = s.r1[0], r010 = s.r1[1], r001 = s.r1[2], rho = s.rho;
    T lr100 = T(0), lr010 = T(0), lr001 = T(0);
    lu[0] += (T(2) * ux * rho - T(2) * r100) * lc200;
    lrho += ux * ux * lc200;
    lr100 += T(-2) * ux * lc200;
    lu[1] += (T(2) * uy * rho - T(2) * r010) * lc020;
    lrho += uy * uy * lc020;
    lr010 += T(-2) * uy * lc020;
    lu[2] += (T(2) * uz * rho - T(2) * r001) * lc002;
    lrho += uz * uz * lc002;
    lr001 += T(-2) * uz * lc002;
    lu[0] += (uy * rho - r010) * lc110; lu[1] += (ux * rho - r100) * lc110; lrho += ux * uy * lc110;
    lr010 -= ux * lc110; lr100 -= uy * lc110;
    lu[0] += (uz * rho - r001) * lc101; lu[2] += (ux * rho - r100) * lc101; lrho += ux * uz * lc101;
    lr001 -= ux * lc101; lr100 -= uz * lc101;
    lu[1] += (uz * rho - r001) * lc011; lu[2] += (uy * rho - r010) * lc011; lrho += uy * uz * lc011;
    lr001 -= uy * lc011; lr010 -= uz * lc011;
    const T lr200 = lc200, lr020 = lc020, lr002 = lc002, lr110 = lc110, lr101 = lc101, lr011 = lc011;

    // speed clamp: u = uraw * ms / |uraw|
    T lur[3] = {lu[0], lu[1], lu[2]};
    if (s.clamped) {
        const T n = T(P.max_speed) / s.umax_scale;  // |uraw|
        const T hx = s.uraw[0] / n, hy = s.uraw[1] / n, hz = s.uraw[2] / n;
        const T d = hx * lu[0] + hy * lu[1] + hz * lu[2];
        lur[0] = s.umax_scale * (lu[0] - hx * d);
        lur[1] = s.umax_scale * (lu[1] - hy * d);
        lur[2] = s.umax_scale * (lu[2] - hz * d);
    }
    // uraw_a = r1_a ir + 0.5 F_a ir
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        lir += (s.r1[a] + T(0.5) * F[a]) * lur[a];
        lF[a] += T(0.5) * s.ir * lur[a];
    }
    lr100 += s.ir * lur[0];
    lr010 += s.ir * lur[1];
    lr001 += s.ir * lur[2];
    lrs += -s.ir * s.ir * lir;
    if (P.enable_buoyancy) lrs += s.bq * lF[P.gravity_axis];
    if (s.rho > T(1e-6)) lrho += lrs;
    const T lr000 = lrho;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const T cx = T(q_cx(q)), cy = T(q_cy(q)), cz = T(q_cz(q));
        lam_in[q] = lr000 + cx * lr100 + cy * lr010 + cz * lr001 + cx * cx * lr200 + cy * cy * lr020 + cz * cz * lr002 +
                    cx * cy * lr110 + cx * cz * lr101 + cy * cz * lr011;
    }
    lam_F[0] = lF[0];
    lam_F[1] = lF[1];
    lam_F[2] = lF[2];
}

// Probe observable: u = j / clamp(rho, 0.97, 1.03) of a pulled population set
// (the velocity the brick step outputs, without its sub-1e-7 snapping), and
// its adjoint: lam_f[q] = sum_a lam_u[a] d u_a / d f_q.
template <class T>
__host__ __device__ __forceinline__ void probe_velocity(const T (&f)[27], T (&u)[3], T& rho_c, bool& rho_free) {
    T r = 0, jx = 0, jy = 0, jz = 0;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        r += f[q];
        jx += T(q_cx(q)) * f[q];
        jy += T(q_cy(q)) * f[q];
        jz += T(q_cz(q)) * f[q];
    }
    rho_free = inside(r, T(0.97), T(1.03));
    rho_c = clamp_t(r, T(0.97), T(1.03));
    u[0] = jx / rho_c;
    u[1] = jy / rho_c;
    u[2] = jz / rho_c;
}

template <class T>
__host__ __device__ __forceinline__ void probe_velocity_vjp(const T (&u)[3], T rho_c, bool rho_free, const T (&lam_u)[3],
                                                            T (&lam_f)[27]) {
    const T lr = rho_free ? -(lam_u[0] * u[0] + lam_u[1] * u[1] + lam_u[2] * u[2]) / rho_c : T(0);
#pragma unroll
    for (int q = 0; q < 27; ++q)
        lam_f[q] = (T(q_cx(q)) * lam_u[0] + T(q_cy(q)) * lam_u[1] + T(q_cz(q)) * lam_u[2]) / rho_c + lr;
}

}  // namespace adj
}  // namespace aero
