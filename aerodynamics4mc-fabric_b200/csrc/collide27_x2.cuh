// Two cells per thread: the factorised D3Q27 cumulant collision of
// collide27.cuh in sm_100's packed FP32 arithmetic (FADD2 / FMUL2 / FFMA2:
// two IEEE single-precision operations per issued instruction).
//
// The step kernels are issue-bound (every cell costs ~1.3k instructions,
// ~730 of them FP32 adds, multiplies and fused multiply-adds of the
// collision, against an HBM budget of ~1.2k for FP32 and ~0.6k for FP16
// storage). Those operations are lane-independent: evaluating two cells in
// the two halves of a float2 halves their issue cost. The sequence of
// operations is the scalar collision's, lane by lane (the final fix-up and
// Guo source are regrouped per direction pair); clamps, divisions and square
// roots stay scalar per lane. Each lane reports whether its input was finite
// (the scalar collision's `false`, after which the caller reseeds that cell).
#pragma once

#include "collide27.cuh"

namespace aero {

struct F2 {
    float2 v;
};

__device__ __forceinline__ F2 f2(float a) { return F2{make_float2(a, a)}; }
__device__ __forceinline__ F2 f2(float a, float b) { return F2{make_float2(a, b)}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2{__fmul2_rn(a.v, b.v)}; }
// a - b = fma(b, -1, a): the product is exact, so one rounding like a subtraction
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2{__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)}; }
__device__ __forceinline__ F2 operator-(F2 a) { return F2{__fmul2_rn(a.v, make_float2(-1.0f, -1.0f))}; }
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return F2{__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ F2 fmax2(F2 a, float b) { return f2(fmaxf(a.v.x, b), fmaxf(a.v.y, b)); }
__device__ __forceinline__ F2 fmin2(F2 a, float b) { return f2(fminf(a.v.x, b), fminf(a.v.y, b)); }
__device__ __forceinline__ F2 clamp2(F2 a, float lo, float hi) { return fmin2(fmax2(a, lo), hi); }
__device__ __forceinline__ F2 rcp2(F2 a) { return f2(1.0f / a.v.x, 1.0f / a.v.y); }
__device__ __forceinline__ F2 div2(F2 a, F2 b) { return f2(a.v.x / b.v.x, a.v.y / b.v.y); }
__device__ __forceinline__ F2 sqrt2(F2 a) { return f2(sqrtf(a.v.x), sqrtf(a.v.y)); }

// raw_moments27<true> of collide27.cuh, packed.
__device__ __forceinline__ void raw_moments27_x2(const F2 (&f)[27], F2& r000, F2& r100, F2& r010, F2& r001, F2& r200,
                                                 F2& r020, F2& r002, F2& r110, F2& r101, F2& r011) {
    F2 a0[9], a1[9], a2[9];
#pragma unroll
    for (int l = 0; l < 9; ++l) {
        const F2 fm = f[3 * l + 0], f0 = f[3 * l + 1], fp = f[3 * l + 2];
        a0[l] = (fm + fp) + f0;
        a1[l] = fp - fm;
        a2[l] = fp + fm;
    }
    F2 b00[3], b01[3], b02[3], b10[3], b11[3], b20[3];
#pragma unroll
    for (int ix = 0; ix < 3; ++ix) {
        const int l = 3 * ix;
        b00[ix] = (a0[l] + a0[l + 2]) + a0[l + 1];
        b01[ix] = a0[l + 2] - a0[l];
        b10[ix] = (a1[l] + a1[l + 2]) + a1[l + 1];
        b02[ix] = a0[l + 2] + a0[l];
        b11[ix] = a1[l + 2] - a1[l];
        b20[ix] = (a2[l] + a2[l + 2]) + a2[l + 1];
    }
    r000 = (b00[0] + b00[2]) + b00[1];
    r100 = b00[2] - b00[0];
    r010 = (b01[0] + b01[2]) + b01[1];
    r001 = (b10[0] + b10[2]) + b10[1];
    r200 = b00[2] + b00[0];
    r110 = b01[2] - b01[0];
    r020 = (b02[0] + b02[2]) + b02[1];
    r101 = b10[2] - b10[0];
    r011 = (b11[0] + b11[2]) + b11[1];
    r002 = (b20[0] + b20[2]) + b20[1];
}

// Orders 0 and 1 only.
__device__ __forceinline__ void moments01_x2(const F2 (&f)[27], F2& r000, F2& r100, F2& r010, F2& r001) {
    F2 a0[9], a1[9];
#pragma unroll
    for (int l = 0; l < 9; ++l) {
        a0[l] = (f[3 * l] + f[3 * l + 2]) + f[3 * l + 1];
        a1[l] = f[3 * l + 2] - f[3 * l];
    }
    F2 b00[3], b01[3], b10[3];
#pragma unroll
    for (int ix = 0; ix < 3; ++ix) {
        const int l = 3 * ix;
        b00[ix] = (a0[l] + a0[l + 2]) + a0[l + 1];
        b01[ix] = a0[l + 2] - a0[l];
        b10[ix] = (a1[l] + a1[l + 2]) + a1[l + 1];
    }
    r000 = (b00[0] + b00[2]) + b00[1];
    r100 = b00[2] - b00[0];
    r010 = (b01[0] + b01[2]) + b01[1];
    r001 = (b10[0] + b10[2]) + b10[1];
}

// back_line / back_line_even / back_line_odd of collide27.cuh, packed.
__device__ __forceinline__ void back_line_x2(F2 m0, F2 m1, F2 m2, F2 u, F2& fm, F2& f0, F2& fp) {
    const F2 r1 = fma2(u, m0, m1);
    const F2 r2 = fma2(u, r1 + m1, m2);
    fm = f2(0.5f) * (r2 - r1);
    f0 = m0 - r2;
    fp = f2(0.5f) * (r1 + r2);
}
__device__ __forceinline__ void back_line_even_x2(F2 m0, F2 m2, F2 u, F2& fm, F2& f0, F2& fp) {
    const F2 r1 = u * m0;
    const F2 r2 = fma2(u, r1, m2);
    fm = f2(0.5f) * (r2 - r1);
    f0 = m0 - r2;
    fp = f2(0.5f) * (r1 + r2);
}
__device__ __forceinline__ void back_line_odd_x2(F2 m1, F2 u, F2& fm, F2& f0, F2& fp) {
    fm = (u - f2(0.5f)) * m1;
    f0 = (f2(-2.0f) * u) * m1;
    fp = (u + f2(0.5f)) * m1;
}

// Collide two fluid cells (lanes x and y of every F2) in place. temp: the
// cells' temperatures (read when buoyancy is on); cf*: extra force densities.
// ok[k] = false: lane k's input was not finite; its populations are then
// meaningless and the caller reseeds that cell. u: the velocity the
// collision used (midpoint velocity after the speed clamp), per lane.
__device__ __forceinline__ void collide27_x2(F2 (&f)[27], const CollideParams& P, F2 temp, F2 cfx, F2 cfy, F2 cfz,
                                             bool (&ok)[2], F2 (&u)[3]) {
    F2 r000, r100, r010, r001, r200, r020, r002, r110, r101, r011;
    raw_moments27_x2(f, r000, r100, r010, r001, r200, r020, r002, r110, r101, r011);
    const F2 rho = r000;
    ok[0] = isfinite(rho.v.x);
    ok[1] = isfinite(rho.v.y);
    const F2 rs = fmax2(rho, 1e-6f);
    const F2 ir = rcp2(rs);
    F2 ux = r100 * ir, uy = r010 * ir, uz = r001 * ir;
    F2 fx = f2(0.0f), fy = f2(0.0f), fz = f2(0.0f);
    if (P.enable_buoyancy) {
        const F2 add = rs * clamp2(f2(P.buoy_beta) * temp, -P.buoy_fmax, P.buoy_fmax);
        if (P.gravity_axis == 0) fx = add;
        else if (P.gravity_axis == 1) fy = add;
        else fz = add;
    }
    fx = fx + (f2(P.body_force[0]) + cfx);
    fy = fy + (f2(P.body_force[1]) + cfy);
    fz = fz + (f2(P.body_force[2]) + cfz);
    ux = ux + f2(0.5f) * (fx * ir);
    uy = uy + f2(0.5f) * (fy * ir);
    uz = uz + f2(0.5f) * (fz * ir);
    const F2 s2 = fma2(ux, ux, fma2(uy, uy, uz * uz));
    ok[0] = ok[0] && isfinite(ux.v.x) && isfinite(uy.v.x) && isfinite(uz.v.x) && isfinite(s2.v.x);
    ok[1] = ok[1] && isfinite(ux.v.y) && isfinite(uy.v.y) && isfinite(uz.v.y) && isfinite(s2.v.y);
    const float ms2 = P.max_speed * P.max_speed;
    if (s2.v.x > ms2 || s2.v.y > ms2) {
        const F2 sc = f2(s2.v.x > ms2 ? P.max_speed / sqrtf(s2.v.x) : 1.0f, s2.v.y > ms2 ? P.max_speed / sqrtf(s2.v.y) : 1.0f);
        ux = ux * sc;
        uy = uy * sc;
        uz = uz * sc;
    }
    u[0] = ux;
    u[1] = uy;
    u[2] = uz;

    // second-order central moments about u (binomial shift of the raw moments)
    const F2 c200 = fma2(ux * ux, rho, fma2(f2(-2.0f) * ux, r100, r200));
    const F2 c020 = fma2(uy * uy, rho, fma2(f2(-2.0f) * uy, r010, r020));
    const F2 c002 = fma2(uz * uz, rho, fma2(f2(-2.0f) * uz, r001, r002));
    const F2 c110 = fma2(ux * uy, rho, fma2(-ux, r010, fma2(-uy, r100, r110)));
    const F2 c101 = fma2(ux * uz, rho, fma2(-ux, r001, fma2(-uz, r100, r101)));
    const F2 c011 = fma2(uy * uz, rho, fma2(-uy, r001, fma2(-uz, r010, r011)));

    F2 tau_s = f2(P.tau_shear_base), tau_n = f2(P.tau_normal_base);
    const F2 eq2 = rs * f2(kCs2f);
    if (P.enable_sgs) {
        const F2 nxx = c200 - eq2, nyy = c020 - eq2, nzz = c002 - eq2;
        const F2 qn2 = fma2(nxx, nxx, fma2(nyy, nyy, nzz * nzz)) + f2(2.0f) * fma2(c110, c110, fma2(c101, c101, c011 * c011));
        const F2 qm = sqrt2(fmax2(qn2, 0.0f));
        const F2 sm = div2(qm, fmax2(f2(2.0f) * rs * f2(P.nu0), 1e-6f));
        const F2 nut = fmin2(f2(P.sgs_c2) * sm, P.sgs_nut_cap);
        tau_s = clamp2(f2(0.5f) + f2(3.0f) * clamp2(f2(P.nu0) + nut, kNuShearMin, kNuShearMax), kTauMin, kTauMax);
        tau_n = clamp2(f2(P.tau_normal_base) + (tau_s - f2(P.tau_shear_base)) * f2(P.sgs_bulk), kTauMin, kTauMax);
    }
    const F2 om_o = rcp2(tau_s);
    const F2 sd = clamp2(rcp2(tau_n), 0.0f, 1.95f);
    const F2 so = clamp2(om_o, 0.0f, 1.95f);

    // relaxed second-order cumulants, Gaussian closure of orders 4 and 6
    const F2 k200 = c200 + sd * (eq2 - c200);
    const F2 k020 = c020 + sd * (eq2 - c020);
    const F2 k002 = c002 + sd * (eq2 - c002);
    const F2 oso = f2(1.0f) - so;
    const F2 k110 = oso * c110;
    const F2 k101 = oso * c101;
    const F2 k011 = oso * c011;
    const F2 irs = ir;  // rs >= 1e-6, so 1 / max(1e-6, rs) == ir
    const F2 two = f2(2.0f);
    const F2 k220 = fma2(k200, k020, two * k110 * k110) * irs;
    const F2 k202 = fma2(k200, k002, two * k101 * k101) * irs;
    const F2 k022 = fma2(k020, k002, two * k011 * k011) * irs;
    const F2 k211 = fma2(k200, k011, two * k110 * k101) * irs;
    const F2 k121 = fma2(k020, k101, two * k110 * k011) * irs;
    const F2 k112 = fma2(k002, k110, two * k101 * k011) * irs;
    const F2 k222 = (k200 * k020 * k002 + two * k110 * k110 * k002 + two * k101 * k101 * k020 + two * k011 * k011 * k200 +
                     f2(8.0f) * k110 * k101 * k011) * irs * irs;

    // separable central -> population map: x pass, y pass, z pass
    F2 g[3][9];
    back_line_even_x2(rs, k200, ux, g[0][0], g[1][0], g[2][0]);
    back_line_odd_x2(k110, ux, g[0][3], g[1][3], g[2][3]);
    back_line_even_x2(k020, k220, ux, g[0][6], g[1][6], g[2][6]);
    back_line_odd_x2(k101, ux, g[0][1], g[1][1], g[2][1]);
    back_line_even_x2(k011, k211, ux, g[0][4], g[1][4], g[2][4]);
    back_line_odd_x2(k121, ux, g[0][7], g[1][7], g[2][7]);
    back_line_even_x2(k002, k202, ux, g[0][2], g[1][2], g[2][2]);
    back_line_odd_x2(k112, ux, g[0][5], g[1][5], g[2][5]);
    back_line_even_x2(k022, k222, ux, g[0][8], g[1][8], g[2][8]);
    F2 h[27];
#pragma unroll
    for (int ix = 0; ix < 3; ++ix) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            back_line_x2(g[ix][0 * 3 + c], g[ix][1 * 3 + c], g[ix][2 * 3 + c], uy, h[(ix * 3 + 0) * 3 + c],
                         h[(ix * 3 + 1) * 3 + c], h[(ix * 3 + 2) * 3 + c]);
        }
    }
#pragma unroll
    for (int l = 0; l < 9; ++l) back_line_x2(h[3 * l + 0], h[3 * l + 1], h[3 * l + 2], uz, f[3 * l + 0], f[3 * l + 1], f[3 * l + 2]);

    // conservation fix-up (first-order part of feq(rho, u) - feq(rho_c, u_c))
    F2 m0, m1x, m1y, m1z;
    moments01_x2(f, m0, m1x, m1y, m1z);
    const F2 drho = rs - m0;
    const F2 three = f2(3.0f);
    const F2 djx = three * (rs * ux - m1x), djy = three * (rs * uy - m1y), djz = three * (rs * uz - m1z);

    // Guo source pref * w * (3 (c.F - u.F) + 9 (c.u)(c.F)); lanes without force get pref 0
    const bool forced0 = (fx.v.x != 0.0f) | (fy.v.x != 0.0f) | (fz.v.x != 0.0f);
    const bool forced1 = (fx.v.y != 0.0f) | (fy.v.y != 0.0f) | (fz.v.y != 0.0f);
    const F2 omc = clamp2(om_o, 0.0f, 1.999f);
    const F2 pref_raw = fmax2(f2(1.0f) - f2(0.5f) * omc, 0.0f);
    const F2 pref = f2(forced0 ? pref_raw.v.x : 0.0f, forced1 ? pref_raw.v.y : 0.0f);
    const F2 uf = fma2(ux, fx, fma2(uy, fy, uz * fz));
    // per pair (q, 26 - q), q > 13 (first non-zero component +1): even part
    // A = drho + pref (9 cu cf - 3 uf), odd part B = c_q.(dj + 3 pref F)
    const F2 D = drho - three * pref * uf;
    const F2 p9 = f2(9.0f) * pref;
    const F2 p3 = three * pref;
    const F2 vx = fma2(p3, fx, djx), vy = fma2(p3, fy, djy), vz = fma2(p3, fz, djz);
#pragma unroll
    for (int q = 14; q < 27; ++q) {
        const int cx = q_cx(q), cy = q_cy(q), cz = q_cz(q);
        // signed sums over the non-zero components (no products by +-1 or 0)
        F2 cu, cf, B;
        if (cx) {
            cu = ux; cf = fx; B = vx;
            if (cy > 0) { cu = cu + uy; cf = cf + fy; B = B + vy; }
            if (cy < 0) { cu = cu - uy; cf = cf - fy; B = B - vy; }
            if (cz > 0) { cu = cu + uz; cf = cf + fz; B = B + vz; }
            if (cz < 0) { cu = cu - uz; cf = cf - fz; B = B - vz; }
        } else if (cy) {
            cu = uy; cf = fy; B = vy;
            if (cz > 0) { cu = cu + uz; cf = cf + fz; B = B + vz; }
            if (cz < 0) { cu = cu - uz; cf = cf - fz; B = B - vz; }
        } else {
            cu = uz; cf = fz; B = vz;
        }
        const F2 A = fma2(p9 * cu, cf, D);
        const F2 wq = f2(q_w(q));
        f[q] = fma2(wq, A + B, f[q]);
        f[26 - q] = fma2(wq, A - B, f[26 - q]);
    }
    f[13] = fma2(f2(q_w(13)), D, f[13]);
}

}  // namespace aero
