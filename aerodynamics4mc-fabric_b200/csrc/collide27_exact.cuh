// Per-cell D3Q27 cumulant collision in the reference's exact operation order.
//
// Every floating-point operation of the reference CPU collide
// (native/src/aero_lbm_jni.cpp:2209-2413, with compute_raw_moments 1335-1357,
// compute_central_moments 1359-1382, cumulant_relax_closure 1384-1430,
// central_to_raw 1432-1455, raw_to_populations 1457-1473, feq
// native/src/aero_lbm_hydro_core.cpp:48-52, guo_force_source jni.cpp:1270-1281)
// is performed here in the same order with the same rounding, so the result is
// bit-identical to the reference on IEEE hardware. Rules that keep it so:
//   * this header is compiled only in translation units built with
//     --fmad=false (no multiply-add contraction), except where a product is
//     exact (a power-of-two coefficient), where fmaf gives the same rounding;
//   * terms whose coefficient is zero (c = 0 in a moment, a zero post-collision
//     central moment) are skipped: adding +-0 to a finite non-zero partial sum
//     is the identity, so the sums are unchanged;
//   * only the moments the collision reads are formed (the reference computes
//     all 27 pre-collision central moments but uses the second-order six).
// Flops per cell are about a third of the reference's dense loops; the
// collision is still ALU-heavier than the factorised form (collide27.cuh).
#pragma once

#include "collide27.cuh"

namespace aero {
namespace exact {

// std::max / std::min semantics (argument order matters for NaN and zeros).
__device__ __forceinline__ float rmax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float rmin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float rclamp(float v, float lo, float hi) { return rmin(hi, rmax(lo, v)); }

__host__ __device__ constexpr int cval(int i) { return i - 1; }
__host__ __device__ constexpr int binom2(int n, int k) { return (k < 0 || k > n) ? 0 : ((n <= 1 || k == 0 || k == n) ? 1 : 2); }

// c.u for direction q, summed x, y, z skipping zero components.
__device__ __forceinline__ float cdot(int q, float ux, float uy, float uz) {
    const int cx = q_cx(q), cy = q_cy(q), cz = q_cz(q);
    float s = 0.0f;
    bool any = false;
    if (cx != 0) { s = cx > 0 ? ux : -ux; any = true; }
    if (cy != 0) { const float t = cy > 0 ? uy : -uy; s = any ? s + t : t; any = true; }
    if (cz != 0) { const float t = cz > 0 ? uz : -uz; s = any ? s + t : t; any = true; }
    return s;
}

// feq(q, rho, u) = w rho (1 + cu + 0.5 cu^2 - 1.5 u.u), cu = 3 c.u
__device__ __forceinline__ float feq(int q, float rho, float ux, float uy, float uz, float uu) {
    const float cu = 3.0f * cdot(q, ux, uy, uz);
    return q_w(q) * rho * (1.0f + cu + 0.5f * cu * cu - 1.5f * uu);
}

// Signed sum over q (in q order) of f[q] * cx^a cy^b cz^c, terms with a zero
// coefficient skipped: the reference's raw moment / momentum sums.
template <int A, int B, int C>
__device__ __forceinline__ float qsum(const float (&f)[27]) {
    float s = 0.0f;
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

struct ExactOut {
    float rho, ux, uy, uz;
};

// Collide one fluid cell in place (benchmark-mode reference collide: no fan
// forcing, no edge nudge, no sponge). Returns false, with f untouched, when
// the input is not finite; the caller reseeds the cell.
__device__ __forceinline__ bool collide27_exact(float (&f)[27], const CollideParams& P, const float* temperature,
                                                float cfx, float cfy, float cfz, CollideOut& out,
                                                const CellExtras* ex = nullptr) {
    bool bad = false;
#pragma unroll
    for (int q = 0; q < 27; ++q) bad |= !isfinite(f[q]);
    const float rho = qsum<0, 0, 0>(f);
    const float mom_x = qsum<1, 0, 0>(f);
    const float mom_y = qsum<0, 1, 0>(f);
    const float mom_z = qsum<0, 0, 1>(f);
    if (bad || !isfinite(rho) || !isfinite(mom_x) || !isfinite(mom_y) || !isfinite(mom_z)) return false;
    const float rho_safe = rmax(1e-6f, rho);
    const float inv_rho = 1.0f / rho_safe;
    float ux = mom_x * inv_rho;
    float uy = mom_y * inv_rho;
    float uz = mom_z * inv_rho;
    if (!isfinite(rho_safe) || !isfinite(inv_rho) || !isfinite(ux) || !isfinite(uy) || !isfinite(uz)) return false;
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    if (ex && P.fan_beta > 0.0f && ex->fan_mask > 0.0f) fan_force(*ex, P, rho_safe, ux, uy, uz, fx, fy, fz);
    if (P.enable_buoyancy) {
        const float buoy = rclamp(P.buoy_beta * *temperature, -P.buoy_fmax, P.buoy_fmax);
        const float add = rho_safe * buoy;
        if (P.gravity_axis == 0) fx += add;
        else if (P.gravity_axis == 1) fy += add;
        else fz += add;
    }
    // Body force (absent from the reference; zero keeps it bit-identical).
    if (P.body_force[0] != 0.0f || P.body_force[1] != 0.0f || P.body_force[2] != 0.0f) {
        fx += P.body_force[0]; fy += P.body_force[1]; fz += P.body_force[2];
    }
    if (cfx != 0.0f || cfy != 0.0f || cfz != 0.0f) {
        fx += cfx; fy += cfy; fz += cfz;
    }
    const bool forced = (fx != 0.0f) | (fy != 0.0f) | (fz != 0.0f);
    if (forced) {
        ux += 0.5f * (fx * inv_rho);
        uy += 0.5f * (fy * inv_rho);
        uz += 0.5f * (fz * inv_rho);
        if (!isfinite(ux) || !isfinite(uy) || !isfinite(uz)) return false;
    }
    if (ex && P.state_nudge > 0.0f) {
        // runtime-mode state nudge (jni.cpp:2314-2322)
        const float sn = ex->nudge;
        ux = (1.0f - sn) * ux + sn * ex->ref_x;
        uy = (1.0f - sn) * uy + sn * ex->ref_y;
        uz = (1.0f - sn) * uz + sn * ex->ref_z;
        if (!isfinite(ux) || !isfinite(uy) || !isfinite(uz)) return false;
    }
    const float speed2 = ux * ux + uy * uy + uz * uz;
    if (!isfinite(speed2)) return false;
    if (speed2 > P.max_speed * P.max_speed) {
        const float scale = P.max_speed / sqrtf(speed2);
        ux *= scale; uy *= scale; uz *= scale;
    }
    out.rho = rho; out.ux = ux; out.uy = uy; out.uz = uz; out.reseeded = false;

    // Raw moments read by the second-order central moments (raw000 = rho and
    // raw100/010/001 = momentum are the same sums in the same order).
    const float r200 = qsum<2, 0, 0>(f), r020 = qsum<0, 2, 0>(f), r002 = qsum<0, 0, 2>(f);
    const float r110 = qsum<1, 1, 0>(f), r101 = qsum<1, 0, 1>(f), r011 = qsum<0, 1, 1>(f);

    // Second-order central moments: binomial shift with s = (1, -u, u*u), terms
    // in (p, q, r) loop order, products left to right.
    const float sx1 = -ux, sy1 = -uy, sz1 = -uz;
    const float sx2 = ux * ux, sy2 = uy * uy, sz2 = uz * uz;
    const float c200 = (sx2 * rho + (2.0f * sx1) * mom_x) + r200;
    const float c020 = (sy2 * rho + (2.0f * sy1) * mom_y) + r020;
    const float c002 = (sz2 * rho + (2.0f * sz1) * mom_z) + r002;
    const float c110 = (((sx1 * sy1) * rho + sx1 * mom_y) + sy1 * mom_x) + r110;
    const float c101 = (((sx1 * sz1) * rho + sx1 * mom_z) + sz1 * mom_x) + r101;
    const float c011 = (((sy1 * sz1) * rho + sy1 * mom_z) + sz1 * mom_y) + r011;

    const float tau_s_base = P.tau_shear_base, tau_n_base = P.tau_normal_base;
    float tau_s = tau_s_base, tau_n = tau_n_base;
    if (P.enable_sgs) {
        const float nu0 = P.nu0;
        const float nxx = c200 - rho_safe * kCs2f;
        const float nyy = c020 - rho_safe * kCs2f;
        const float nzz = c002 - rho_safe * kCs2f;
        const float q_norm2 = nxx * nxx + nyy * nyy + nzz * nzz + 2.0f * (c110 * c110 + c101 * c101 + c011 * c011);
        const float q_mag = sqrtf(rmax(0.0f, q_norm2));
        const float s_mag = q_mag / rmax(1e-6f, 2.0f * rho_safe * nu0);
        float nu_t = P.sgs_c2 * s_mag;
        nu_t = rmin(nu_t, P.sgs_nut_cap);
        tau_s = rclamp(0.5f + 3.0f * rclamp(nu0 + nu_t, kNuShearMin, kNuShearMax), kTauMin, kTauMax);
        tau_n = rclamp(tau_n_base + (tau_s - tau_s_base) * P.sgs_bulk, kTauMin, kTauMax);
    }
    const float omega_diag = 1.0f / tau_n;
    const float omega_off = 1.0f / tau_s;

    // cumulant_relax_closure with rho = rho_safe.
    float K[3][3][3];
    const float eq_second = rho_safe * kCs2f;
    const float s_diag = rclamp(omega_diag, 0.0f, 1.95f);
    const float s_off = rclamp(omega_off, 0.0f, 1.95f);
    K[0][0][0] = rho_safe;
    K[2][0][0] = c200 + s_diag * (eq_second - c200);
    K[0][2][0] = c020 + s_diag * (eq_second - c020);
    K[0][0][2] = c002 + s_diag * (eq_second - c002);
    K[1][1][0] = (1.0f - s_off) * c110;
    K[1][0][1] = (1.0f - s_off) * c101;
    K[0][1][1] = (1.0f - s_off) * c011;
    {
        const float k200 = K[2][0][0], k020 = K[0][2][0], k002 = K[0][0][2];
        const float k110 = K[1][1][0], k101 = K[1][0][1], k011 = K[0][1][1];
        const float ir = 1.0f / rmax(1e-6f, rho_safe);
        K[2][2][0] = k200 * k020 * ir + 2.0f * k110 * k110 * ir;
        K[2][0][2] = k200 * k002 * ir + 2.0f * k101 * k101 * ir;
        K[0][2][2] = k020 * k002 * ir + 2.0f * k011 * k011 * ir;
        K[2][1][1] = (k200 * k011 + 2.0f * k110 * k101) * ir;
        K[1][2][1] = (k020 * k101 + 2.0f * k110 * k011) * ir;
        K[1][1][2] = (k002 * k110 + 2.0f * k101 * k011) * ir;
        K[2][2][2] = (k200 * k020 * k002 + 2.0f * k110 * k110 * k002 + 2.0f * k101 * k101 * k020 +
                      2.0f * k011 * k011 * k200 + 8.0f * k110 * k101 * k011) * ir * ir;
    }

    // central_to_raw: R[a][b][c] = sum over non-zero K[p][q][r], (p,q,r) <= (a,b,c),
    // of ((((binom * ux^(a-p)) * uy^(b-q)) * uz^(c-r)) * K[p][q][r]).
    const float upx[3] = {1.0f, ux, ux * ux};
    const float upy[3] = {1.0f, uy, uy * uy};
    const float upz[3] = {1.0f, uz, uz * uz};
    float R[3][3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float sum = 0.0f;
                bool first = true;
#pragma unroll
                for (int p = 0; p <= a; ++p)
#pragma unroll
                    for (int qq = 0; qq <= b; ++qq)
#pragma unroll
                        for (int r = 0; r <= c; ++r) {
                            if (((p + qq + r) & 1) != 0) continue;  // odd-order post-collision moments are zero
                            const float coeff = float(binom2(a, p) * binom2(b, qq) * binom2(c, r));
                            float t = coeff;
                            if (a - p > 0) t = t * upx[a - p];
                            if (b - qq > 0) t = t * upy[b - qq];
                            if (c - r > 0) t = t * upz[c - r];
                            t = t * K[p][qq][r];
                            sum = first ? t : sum + t;
                            first = false;
                        }
                R[a][b][c] = sum;
            }

    // raw_to_populations with the 1-D inverse rows {0,-1/2,1/2}, {1,0,-1}, {0,1/2,1/2}.
    // The coefficient products are powers of two, so coef*R is exact and the
    // fused multiply-add rounds exactly like the reference's multiply then add.
    constexpr float inv1[3][3] = {{0.0f, -0.5f, 0.5f}, {1.0f, 0.0f, -1.0f}, {0.0f, 0.5f, 0.5f}};
    float fc[27];
#pragma unroll
    for (int ix = 0; ix < 3; ++ix)
#pragma unroll
        for (int iy = 0; iy < 3; ++iy)
#pragma unroll
            for (int iz = 0; iz < 3; ++iz) {
                float sum = 0.0f;
                bool first = true;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b)
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const float coef = inv1[ix][a] * inv1[iy][b] * inv1[iz][c];
                            if (coef == 0.0f) continue;
                            sum = first ? coef * R[a][b][c] : fmaf(coef, R[a][b][c], sum);
                            first = false;
                        }
                fc[(ix * 3 + iy) * 3 + iz] = sum;
            }

    // Conservation fix-up.
    const float rho_c = qsum<0, 0, 0>(fc);
    const float mx_c = qsum<1, 0, 0>(fc);
    const float my_c = qsum<0, 1, 0>(fc);
    const float mz_c = qsum<0, 0, 1>(fc);
    const float rho_cs = rmax(1e-6f, rho_c);
    const float uxc = mx_c / rho_cs, uyc = my_c / rho_cs, uzc = mz_c / rho_cs;
    const float uu = ux * ux + uy * uy + uz * uz;
    const float uuc = uxc * uxc + uyc * uyc + uzc * uzc;
#pragma unroll
    for (int q = 0; q < 27; ++q) fc[q] += feq(q, rho_safe, ux, uy, uz, uu) - feq(q, rho_cs, uxc, uyc, uzc, uuc);

    if (forced) {
        const float inv_cs2 = 1.0f / kCs2f;
        const float inv_cs4 = inv_cs2 * inv_cs2;
        const float pref = rmax(0.0f, 1.0f - 0.5f * rclamp(omega_off, 0.0f, 1.999f));
        const float u_force = ux * fx + uy * fy + uz * fz;
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            const float cu = cdot(q, ux, uy, uz);
            const float c_force = cdot(q, fx, fy, fz);
            f[q] = fc[q] + pref * q_w(q) * ((c_force - u_force) * inv_cs2 + cu * c_force * inv_cs4);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 27; ++q) f[q] = fc[q];
    }
    return true;
}

// write_output / extract macro readout in the reference's order
// (jni.cpp:2535-2581): sums in q order, clamped rho, true division.
__device__ __forceinline__ void macro_out_exact(const float (&f)[27], bool solid, float scale, float* o) {
    if (solid) { o[0] = o[1] = o[2] = o[3] = 0.0f; return; }
    bool bad = false;
#pragma unroll
    for (int q = 0; q < 27; ++q) bad |= !isfinite(f[q]);
    float rho = qsum<0, 0, 0>(f);
    float ux = qsum<1, 0, 0>(f), uy = qsum<0, 1, 0>(f), uz = qsum<0, 0, 1>(f);
    if (bad || !isfinite(rho) || !isfinite(ux) || !isfinite(uy) || !isfinite(uz)) {
        o[0] = o[1] = o[2] = o[3] = 0.0f;
        return;
    }
    rho = rclamp(rho, 0.97f, 1.03f);
    ux /= rho; uy /= rho; uz /= rho;
    if (!isfinite(ux) || !isfinite(uy) || !isfinite(uz)) ux = uy = uz = 0.0f;
    if (fabsf(rho - 1.0f) < 1e-6f) rho = 1.0f;
    if (fabsf(ux) < 1e-7f) ux = 0.0f;
    if (fabsf(uy) < 1e-7f) uy = 0.0f;
    if (fabsf(uz) < 1e-7f) uz = 0.0f;
    o[0] = ux * scale;
    o[1] = uy * scale;
    o[2] = uz * scale;
    o[3] = rclamp(rho - 1.0f, -0.03f, 0.03f);
}

}  // namespace exact
}  // namespace aero
