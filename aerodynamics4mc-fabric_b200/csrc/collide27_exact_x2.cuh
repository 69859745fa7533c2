// Two cells per thread in the reference's exact operation order: the
// collision of collide27_exact.cuh with every add, subtract, multiply and
// fused multiply-add issued as one packed FP32 instruction (add / sub / mul /
// fma .rn.f32x2, sm_100) for the two cells. The packed operations are written
// as inline PTX with an explicit rounding mode, so no compiler pass may fuse,
// reorder or re-associate them; each lane rounds exactly like the scalar IEEE
// operation, and every data-dependent branch of the scalar code becomes a
// per-lane select, so each lane's result is bit-identical to collide27_exact
// on that cell. Divisions, square roots and clamps stay scalar per lane.
#pragma once

#include "collide27_exact.cuh"
#include "collide27_x2.cuh"

namespace aero {
namespace exact {

struct X2 {
    float2 v;
};
struct Mul2;

__device__ __forceinline__ X2 x2(float a) { return X2{make_float2(a, a)}; }
__device__ __forceinline__ X2 x2(float a, float b) { return X2{make_float2(a, b)}; }

// add / sub / fma with an explicit rounding mode.
#define AERO_X2_BINOP(NAME, OP)                                                                                    \
    __device__ __forceinline__ X2 NAME(X2 a, X2 b) {                                                            \
        X2 r;                                                                                                      \
        asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t" OP            \
            " pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"                                                         \
            : "=f"(r.v.x), "=f"(r.v.y)                                                                             \
            : "f"(a.v.x), "f"(a.v.y), "f"(b.v.x), "f"(b.v.y));                                                     \
        return r;                                                                                                  \
    }
AERO_X2_BINOP(operator+, "add.rn.f32x2")
AERO_X2_BINOP(operator-, "sub.rn.f32x2")
#undef AERO_X2_BINOP

__device__ __forceinline__ X2 xfma(X2 a, X2 b, X2 c) {
    X2 r;
    asm("{\n\t.reg .b64 pa, pb, pc, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "mov.b64 pc, {%6, %7};\n\tfma.rn.f32x2 pd, pa, pb, pc;\n\tmov.b64 {%0, %1}, pd;\n\t}"
        : "=f"(r.v.x), "=f"(r.v.y)
        : "f"(a.v.x), "f"(a.v.y), "f"(b.v.x), "f"(b.v.y), "f"(c.v.x), "f"(c.v.y));
    return r;
}

// Product a * b, rounded once. ptxas fuses a packed multiply into a packed
// add that consumes it (one rounding instead of two) even with an explicit
// rounding mode and multiply-add contraction disabled, and it sees through
// an addend it knows to be -0. So the product is issued as fma(a, b, z) with
// z = -0 formed from a run-time value (exact: a*b + -0 == a*b, signed zeros
// included), which no later add can absorb.
struct Mul2 {
    X2 z;
    __device__ __forceinline__ X2 operator()(X2 a, X2 b) const { return xfma(a, b, z); }
};
__device__ __forceinline__ Mul2 make_mul2(int zero_bits) {
    const float z = __int_as_float(zero_bits | (int)0x80000000);
    return Mul2{X2{make_float2(z, z)}};
}
// Negation is exact: per lane.
__device__ __forceinline__ X2 operator-(X2 a) { return x2(-a.v.x, -a.v.y); }

__device__ __forceinline__ X2 sel2(bool a, bool b, X2 x, X2 y) { return x2(a ? x.v.x : y.v.x, b ? x.v.y : y.v.y); }
// std::max(c, v) / std::min(v, c) / std::clamp per lane
__device__ __forceinline__ X2 rmax2(float c, X2 v) { return x2(rmax(c, v.v.x), rmax(c, v.v.y)); }
__device__ __forceinline__ X2 rmin2(X2 v, float c) { return x2(rmin(v.v.x, c), rmin(v.v.y, c)); }
__device__ __forceinline__ X2 rclamp2(X2 v, float lo, float hi) { return x2(rclamp(v.v.x, lo, hi), rclamp(v.v.y, lo, hi)); }
__device__ __forceinline__ X2 div2x(X2 a, X2 b) { return x2(a.v.x / b.v.x, a.v.y / b.v.y); }

template <int A, int B, int C>
__device__ __forceinline__ X2 qsum2(const X2 (&f)[27]) {
    X2 s = x2(0.0f);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        const int cx = q_cx(q), cy = q_cy(q), cz = q_cz(q);
        const int px = A == 0 ? 1 : (A == 1 ? cx : cx * cx);
        const int py = B == 0 ? 1 : (B == 1 ? cy : cy * cy);
        const int pz = C == 0 ? 1 : (C == 2 ? cz * cz : (C == 1 ? cz : 1));
        const int coef = px * py * pz;
        if (coef == 0) continue;
        s = coef > 0 ? s + f[q] : s - f[q];
    }
    return s;
}

// cdot of collide27_exact.cuh: x, y, z components in order, zeros skipped
__device__ __forceinline__ X2 cdot2x(int q, X2 ux, X2 uy, X2 uz) {
    const int cx = q_cx(q), cy = q_cy(q), cz = q_cz(q);
    X2 s = x2(0.0f);
    bool any = false;
    if (cx != 0) { s = cx > 0 ? ux : -ux; any = true; }
    if (cy != 0) { const X2 t = cy > 0 ? uy : -uy; s = any ? s + t : t; any = true; }
    if (cz != 0) { const X2 t = cz > 0 ? uz : -uz; s = any ? s + t : t; any = true; }
    return s;
}

__device__ __forceinline__ X2 feq2x(const Mul2& M, int q, X2 rho, X2 ux, X2 uy, X2 uz, X2 uu) {
    const X2 cu = M(x2(3.0f), cdot2x(q, ux, uy, uz));
    return M(M(x2(q_w(q)), rho), ((x2(1.0f) + cu) + M(M(x2(0.5f), cu), cu)) - M(x2(1.5f), uu));
}

// Collide two fluid cells in place; ok[k] = false: lane k's input was not
// finite (its result is meaningless; the caller reseeds that cell).
__device__ __forceinline__ void collide27_exact_x2_impl(X2 (&f)[27], const CollideParams& P, X2 temp, X2 cfx, X2 cfy,
                                                        X2 cfz, bool (&ok)[2], X2 (&u)[3]) {
    const Mul2 M = make_mul2(P.zero_bits);
    bool bad0 = false, bad1 = false;
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        bad0 |= !isfinite(f[q].v.x);
        bad1 |= !isfinite(f[q].v.y);
    }
    const X2 rho = qsum2<0, 0, 0>(f);
    const X2 mom_x = qsum2<1, 0, 0>(f);
    const X2 mom_y = qsum2<0, 1, 0>(f);
    const X2 mom_z = qsum2<0, 0, 1>(f);
    ok[0] = !bad0 && isfinite(rho.v.x) && isfinite(mom_x.v.x) && isfinite(mom_y.v.x) && isfinite(mom_z.v.x);
    ok[1] = !bad1 && isfinite(rho.v.y) && isfinite(mom_x.v.y) && isfinite(mom_y.v.y) && isfinite(mom_z.v.y);
    const X2 rho_safe = rmax2(1e-6f, rho);
    const X2 inv_rho = x2(1.0f / rho_safe.v.x, 1.0f / rho_safe.v.y);
    X2 ux = M(mom_x, inv_rho);
    X2 uy = M(mom_y, inv_rho);
    X2 uz = M(mom_z, inv_rho);
    ok[0] = ok[0] && isfinite(rho_safe.v.x) && isfinite(inv_rho.v.x) && isfinite(ux.v.x) && isfinite(uy.v.x) && isfinite(uz.v.x);
    ok[1] = ok[1] && isfinite(rho_safe.v.y) && isfinite(inv_rho.v.y) && isfinite(ux.v.y) && isfinite(uy.v.y) && isfinite(uz.v.y);
    X2 fx = x2(0.0f), fy = x2(0.0f), fz = x2(0.0f);
    if (P.enable_buoyancy) {
        const X2 buoy = rclamp2(M(x2(P.buoy_beta), temp), -P.buoy_fmax, P.buoy_fmax);
        const X2 add = M(rho_safe, buoy);
        if (P.gravity_axis == 0) fx = fx + add;
        else if (P.gravity_axis == 1) fy = fy + add;
        else fz = fz + add;
    }
    if (P.body_force[0] != 0.0f || P.body_force[1] != 0.0f || P.body_force[2] != 0.0f) {
        fx = fx + x2(P.body_force[0]);
        fy = fy + x2(P.body_force[1]);
        fz = fz + x2(P.body_force[2]);
    }
    {
        const bool c0 = cfx.v.x != 0.0f || cfy.v.x != 0.0f || cfz.v.x != 0.0f;
        const bool c1 = cfx.v.y != 0.0f || cfy.v.y != 0.0f || cfz.v.y != 0.0f;
        if (c0 || c1) {
            fx = sel2(c0, c1, fx + cfx, fx);
            fy = sel2(c0, c1, fy + cfy, fy);
            fz = sel2(c0, c1, fz + cfz, fz);
        }
    }
    const bool forced0 = (fx.v.x != 0.0f) | (fy.v.x != 0.0f) | (fz.v.x != 0.0f);
    const bool forced1 = (fx.v.y != 0.0f) | (fy.v.y != 0.0f) | (fz.v.y != 0.0f);
    if (forced0 || forced1) {
        ux = sel2(forced0, forced1, ux + M(x2(0.5f), M(fx, inv_rho)), ux);
        uy = sel2(forced0, forced1, uy + M(x2(0.5f), M(fy, inv_rho)), uy);
        uz = sel2(forced0, forced1, uz + M(x2(0.5f), M(fz, inv_rho)), uz);
        ok[0] = ok[0] && isfinite(ux.v.x) && isfinite(uy.v.x) && isfinite(uz.v.x);
        ok[1] = ok[1] && isfinite(ux.v.y) && isfinite(uy.v.y) && isfinite(uz.v.y);
    }
    const X2 speed2 = (M(ux, ux) + M(uy, uy)) + M(uz, uz);
    ok[0] = ok[0] && isfinite(speed2.v.x);
    ok[1] = ok[1] && isfinite(speed2.v.y);
    {
        const float ms2 = P.max_speed * P.max_speed;
        const bool k0 = speed2.v.x > ms2, k1 = speed2.v.y > ms2;
        if (k0 || k1) {
            const X2 sc = x2(k0 ? P.max_speed / sqrtf(speed2.v.x) : 1.0f, k1 ? P.max_speed / sqrtf(speed2.v.y) : 1.0f);
            ux = M(ux, sc);
            uy = M(uy, sc);
            uz = M(uz, sc);
        }
    }

    u[0] = ux;
    u[1] = uy;
    u[2] = uz;
    const X2 r200 = qsum2<2, 0, 0>(f), r020 = qsum2<0, 2, 0>(f), r002 = qsum2<0, 0, 2>(f);
    const X2 r110 = qsum2<1, 1, 0>(f), r101 = qsum2<1, 0, 1>(f), r011 = qsum2<0, 1, 1>(f);

    const X2 sx1 = -ux, sy1 = -uy, sz1 = -uz;
    const X2 sx2 = M(ux, ux), sy2 = M(uy, uy), sz2 = M(uz, uz);
    const X2 two = x2(2.0f);
    const X2 c200 = (M(sx2, rho) + M(M(two, sx1), mom_x)) + r200;
    const X2 c020 = (M(sy2, rho) + M(M(two, sy1), mom_y)) + r020;
    const X2 c002 = (M(sz2, rho) + M(M(two, sz1), mom_z)) + r002;
    const X2 c110 = ((M(M(sx1, sy1), rho) + M(sx1, mom_y)) + M(sy1, mom_x)) + r110;
    const X2 c101 = ((M(M(sx1, sz1), rho) + M(sx1, mom_z)) + M(sz1, mom_x)) + r101;
    const X2 c011 = ((M(M(sy1, sz1), rho) + M(sy1, mom_z)) + M(sz1, mom_y)) + r011;

    const float tau_s_base = P.tau_shear_base, tau_n_base = P.tau_normal_base;
    X2 tau_s = x2(tau_s_base), tau_n = x2(tau_n_base);
    const X2 cs2 = x2(kCs2f);
    if (P.enable_sgs) {
        const float nu0 = P.nu0;
        const X2 nxx = c200 - M(rho_safe, cs2);
        const X2 nyy = c020 - M(rho_safe, cs2);
        const X2 nzz = c002 - M(rho_safe, cs2);
        const X2 q_norm2 = ((M(nxx, nxx) + M(nyy, nyy)) + M(nzz, nzz)) +
                           M(two, (M(c110, c110) + M(c101, c101)) + M(c011, c011));
        const X2 qa = rmax2(0.0f, q_norm2);
        const X2 q_mag = x2(sqrtf(qa.v.x), sqrtf(qa.v.y));
        const X2 s_mag = div2x(q_mag, rmax2(1e-6f, M(M(two, rho_safe), x2(nu0))));
        X2 nu_t = M(x2(P.sgs_c2), s_mag);
        nu_t = rmin2(nu_t, P.sgs_nut_cap);
        tau_s = rclamp2(x2(0.5f) + M(x2(3.0f), rclamp2(x2(nu0) + nu_t, kNuShearMin, kNuShearMax)), kTauMin, kTauMax);
        tau_n = rclamp2(x2(tau_n_base) + M(tau_s - x2(tau_s_base), x2(P.sgs_bulk)), kTauMin, kTauMax);
    }
    const X2 omega_diag = x2(1.0f / tau_n.v.x, 1.0f / tau_n.v.y);
    const X2 omega_off = x2(1.0f / tau_s.v.x, 1.0f / tau_s.v.y);

    X2 K[3][3][3];
    const X2 eq_second = M(rho_safe, cs2);
    const X2 s_diag = rclamp2(omega_diag, 0.0f, 1.95f);
    const X2 s_off = rclamp2(omega_off, 0.0f, 1.95f);
    K[0][0][0] = rho_safe;
    K[2][0][0] = c200 + M(s_diag, eq_second - c200);
    K[0][2][0] = c020 + M(s_diag, eq_second - c020);
    K[0][0][2] = c002 + M(s_diag, eq_second - c002);
    K[1][1][0] = M(x2(1.0f) - s_off, c110);
    K[1][0][1] = M(x2(1.0f) - s_off, c101);
    K[0][1][1] = M(x2(1.0f) - s_off, c011);
    {
        const X2 k200 = K[2][0][0], k020 = K[0][2][0], k002 = K[0][0][2];
        const X2 k110 = K[1][1][0], k101 = K[1][0][1], k011 = K[0][1][1];
        const X2 irm = rmax2(1e-6f, rho_safe);
        const X2 ir = x2(1.0f / irm.v.x, 1.0f / irm.v.y);
        K[2][2][0] = M(M(k200, k020), ir) + M(M(M(two, k110), k110), ir);
        K[2][0][2] = M(M(k200, k002), ir) + M(M(M(two, k101), k101), ir);
        K[0][2][2] = M(M(k020, k002), ir) + M(M(M(two, k011), k011), ir);
        K[2][1][1] = M(M(k200, k011) + M(M(two, k110), k101), ir);
        K[1][2][1] = M(M(k020, k101) + M(M(two, k110), k011), ir);
        K[1][1][2] = M(M(k002, k110) + M(M(two, k101), k011), ir);
        K[2][2][2] = M(M((((M(M(k200, k020), k002) + M(M(M(two, k110), k110), k002)) + M(M(M(two, k101), k101), k020)) +
                          M(M(M(two, k011), k011), k200)) +
                             M(M(M(x2(8.0f), k110), k101), k011),
                         ir),
                       ir);
    }

    const X2 upx[3] = {x2(1.0f), ux, M(ux, ux)};
    const X2 upy[3] = {x2(1.0f), uy, M(uy, uy)};
    const X2 upz[3] = {x2(1.0f), uz, M(uz, uz)};
    // central_to_raw entry R[a][b][c] and raw_to_populations entry fc[q]
    // (collide27_exact.cuh's loops, one entry per call).
    X2 R[3][3][3];
    auto raw = [&](int a, int b, int c) {
        X2 sum = x2(0.0f);
        bool first = true;
#pragma unroll
        for (int p = 0; p <= a; ++p)
#pragma unroll
            for (int qq = 0; qq <= b; ++qq)
#pragma unroll
                for (int r = 0; r <= c; ++r) {
                    if (((p + qq + r) & 1) != 0) continue;
                    X2 t = x2(float(binom2(a, p) * binom2(b, qq) * binom2(c, r)));
                    if (a - p > 0) t = M(t, upx[a - p]);
                    if (b - qq > 0) t = M(t, upy[b - qq]);
                    if (c - r > 0) t = M(t, upz[c - r]);
                    t = M(t, K[p][qq][r]);
                    sum = first ? t : sum + t;
                    first = false;
                }
        R[a][b][c] = sum;
    };
    constexpr float inv1[3][3] = {{0.0f, -0.5f, 0.5f}, {1.0f, 0.0f, -1.0f}, {0.0f, 0.5f, 0.5f}};
    X2 fc[27];
    auto pop = [&](int ix, int iy, int iz) {
        X2 sum = x2(0.0f);
        bool first = true;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float coef = inv1[ix][a] * inv1[iy][b] * inv1[iz][c];
                    if (coef == 0.0f) continue;
                    sum = first ? M(x2(coef), R[a][b][c]) : xfma(x2(coef), R[a][b][c], sum);
                    first = false;
                }
        fc[(ix * 3 + iy) * 3 + iz] = sum;
    };
    // Populations with cx = 0 read only R[0][.][.] and R[2][.][.], the others
    // only R[1][.][.] and R[2][.][.]: form them in that order so that R[0]
    // and R[1] are never live together (fewer registers; same values).
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            raw(0, b, c);
            raw(2, b, c);
        }
#pragma unroll
    for (int iy = 0; iy < 3; ++iy)
#pragma unroll
        for (int iz = 0; iz < 3; ++iz) pop(1, iy, iz);
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) raw(1, b, c);
#pragma unroll
    for (int iy = 0; iy < 3; ++iy)
#pragma unroll
        for (int iz = 0; iz < 3; ++iz) {
            pop(0, iy, iz);
            pop(2, iy, iz);
        }

    const X2 rho_c = qsum2<0, 0, 0>(fc);
    const X2 mx_c = qsum2<1, 0, 0>(fc);
    const X2 my_c = qsum2<0, 1, 0>(fc);
    const X2 mz_c = qsum2<0, 0, 1>(fc);
    const X2 rho_cs = rmax2(1e-6f, rho_c);
    const X2 uxc = div2x(mx_c, rho_cs), uyc = div2x(my_c, rho_cs), uzc = div2x(mz_c, rho_cs);
    const X2 uu = (M(ux, ux) + M(uy, uy)) + M(uz, uz);
    const X2 uuc = (M(uxc, uxc) + M(uyc, uyc)) + M(uzc, uzc);
#pragma unroll
    for (int q = 0; q < 27; ++q)
        fc[q] = fc[q] + (feq2x(M, q, rho_safe, ux, uy, uz, uu) - feq2x(M, q, rho_cs, uxc, uyc, uzc, uuc));

    if (forced0 || forced1) {
        const float inv_cs2 = 1.0f / kCs2f;
        const float inv_cs4 = inv_cs2 * inv_cs2;
        const X2 oc = rclamp2(omega_off, 0.0f, 1.999f);
        const X2 pref = rmax2(0.0f, x2(1.0f) - M(x2(0.5f), oc));
        const X2 u_force = (M(ux, fx) + M(uy, fy)) + M(uz, fz);
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            const X2 cu = cdot2x(q, ux, uy, uz);
            const X2 c_force = cdot2x(q, fx, fy, fz);
            const X2 g = fc[q] + M(M(pref, x2(q_w(q))), M(c_force - u_force, x2(inv_cs2)) + M(M(cu, c_force), x2(inv_cs4)));
            f[q] = sel2(forced0, forced1, g, fc[q]);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 27; ++q) f[q] = fc[q];
    }
}

// Entry point on the step kernels' packed type; u: the velocity each lane's
// collision used (post-clamp midpoint velocity).
__device__ __forceinline__ void collide27_exact_x2(F2 (&f)[27], const CollideParams& P, F2 temp, F2 cfx, F2 cfy, F2 cfz,
                                                   bool (&ok)[2], F2 (&u)[3]) {
    X2 g[27], v[3];
#pragma unroll
    for (int q = 0; q < 27; ++q) g[q] = X2{f[q].v};
    collide27_exact_x2_impl(g, P, X2{temp.v}, X2{cfx.v}, X2{cfy.v}, X2{cfz.v}, ok, v);
#pragma unroll
    for (int q = 0; q < 27; ++q) f[q] = F2{g[q].v};
    u[0] = F2{v[0].v};
    u[1] = F2{v[1].v};
    u[2] = F2{v[2].v};
}

}  // namespace exact
}  // namespace aero
