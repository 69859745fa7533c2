// Per-cell D3Q27 cumulant collision, factorised for the GPU.
//
// Same scheme as the reference CPU collide (native/src/aero_lbm_jni.cpp:2209-2413):
//   1. rho, momentum; force = buoyancy along the gravity axis + body force;
//      midpoint velocity u += F / (2 rho); speed clamp.
//   2. second-order central moments about u; Smagorinsky SGS from the
//      non-equilibrium part (jni.cpp:2346-2366).
//   3. relax the second-order cumulants (diagonal at 1/tau_normal, off-diagonal
//      at 1/tau_shear, both <= 1.95), zero the odd orders, Gaussian closure for
//      orders 4 and 6 (jni.cpp:1384-1430).
//   4. back to populations, conservation fix-up with the feq difference
//      (jni.cpp:2376-2394), Guo source with omega_shear (jni.cpp:1270-1281).
//
// The reference evaluates the moment changes as dense 27x27 triple loops
// (about 6k flops per cell). Here the raw moments come from 1-D partial sums
// along z, y, x (only the 10 moments the collision reads), and the inverse
// transform is the separable central->population map applied one axis at a
// time on the 14 non-zero post-collision central moments. Results agree with
// the reference to FP32 rounding, not bit-for-bit.
#pragma once

#include "lattice.cuh"

namespace aero {

struct CollideParams {
    float tau_shear_base;   // effective base shear tau (clamped like the reference)
    float tau_normal_base;  // effective base normal tau
    float nu0;              // max(1e-6, base shear viscosity): SGS reference viscosity
    float sgs_c2;           // Smagorinsky C^2 (reference value 0.025^2)
    float sgs_nut_cap;      // nut <= cap (reference: 5 * nu0)
    float sgs_bulk;         // normal-tau coupling to the SGS shear change (0.3)
    float buoy_beta;        // buoyant acceleration = clamp(beta * T, +-buoy_fmax)
    float buoy_fmax;
    float body_force[3];    // uniform force density on every fluid cell
    float max_speed;        // |u| clamp (reference: 0.5773502 * 0.6)
    int enable_sgs;
    int enable_buoyancy;
    int gravity_axis;       // axis the buoyant force points along (+): 0 x, 1 y, 2 z
    int zero_bits;          // always 0 (value-initialised): a run-time zero for collide27_exact_x2.cuh
    // Game-runtime terms of the reference collide (jni.cpp:2256-2322,
    // 2401-2411); all off in benchmark mode with the default flags.
    int runtime_terms;          // any of them active: the kernels take one cell per thread
    float fan_beta;             // 0.07 with fan forcing (kFanBeta), else 0
    float fan_noise_amp;        // 0.02 (kFanNoiseAmp), 0 with DISABLE_FAN_NOISE
    float fan_target_scale;     // 1 / (m/s per lattice velocity)
    int sponge;                 // sponge toward rest in the 4 outer layers
    float state_nudge;          // runtime mode 0.08: velocity nudge toward the packet state, 8 outer layers
    int nx, ny, nz;             // brick of the call (edge distances)
    unsigned long long step;    // the context's call counter (fan noise)
};

// Per-cell inputs of the runtime terms (filled by the caller when
// CollideParams::runtime_terms is set).
struct CellExtras {
    float fan_mask, fan_x, fan_y, fan_z;  // packet fan channels (mask 0: no fan)
    float noise;                          // fan_noise_amp * hash_signed_noise(cell, step)
    float nudge;                          // state nudge factor of the cell
    float ref_x, ref_y, ref_z;            // packet reference velocity
};

// hash_signed_noise (jni.cpp:1318-1328): splitmix-style 64-bit hash of
// (cell, tick) to a float in [-1, 1].
__host__ __device__ inline float signed_noise(unsigned long long cell, unsigned long long tick) {
    unsigned long long x = cell * 0x9E3779B97F4A7C15ULL ^ tick * 0xD1B54A32D192ED03ULL;
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ULL;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBULL;
    x ^= x >> 31;
    const float u = (float)(x & 0x00FFFFFFULL) * (1.0f / 16777215.0f);
    return 2.0f * u - 1.0f;
}

__device__ __forceinline__ int edge_distance(int x, int y, int z, int nx, int ny, int nz) {
    return min(min(min(x, y), min(z, nx - 1 - x)), min(ny - 1 - y, nz - 1 - z));
}
// effective_runtime_state_nudge (jni.cpp:683-694): base (8 - d)^2 / 64 inside 8 layers
__device__ __forceinline__ float state_nudge_at(const CollideParams& P, int d) {
    if (P.state_nudge <= 0.0f || d >= 8) return 0.0f;
    const float eta = (float)(8 - d) / 8.0f;
    return P.state_nudge * eta * eta;
}
// effective_sponge_alpha (jni.cpp:787-794): 0.03 (4 - d)^2 / 16 inside 4 layers
__device__ __forceinline__ float sponge_alpha_at(const CollideParams& P, int d) {
    if (!P.sponge || d >= 4) return 0.0f;
    const float eta = (float)(4 - d) / 4.0f;
    return fminf(0.95f, fmaxf(0.0f, 0.03f * eta * eta));
}

// Fan force (jni.cpp:2256-2286): push toward the fan's target speed along its
// direction, damp the perpendicular velocity, soften above 0.24.
__device__ __forceinline__ void fan_force(const CellExtras& e, const CollideParams& P, float rs, float ux, float uy,
                                          float uz, float& fx, float& fy, float& fz) {
    const float speed_pre = sqrtf(ux * ux + uy * uy + uz * uz);
    const float fan_norm = sqrtf(e.fan_x * e.fan_x + e.fan_y * e.fan_y + e.fan_z * e.fan_z);
    if (!(fan_norm > 1e-8f)) return;
    const float inv_norm = 1.0f / fan_norm;
    const float noise = 1.0f + e.noise;
    const float target = fminf(0.28f, fmaxf(0.0f, fan_norm * P.fan_target_scale * fmaxf(0.0f, noise)));
    const float nx = e.fan_x * inv_norm, ny = e.fan_y * inv_norm, nz = e.fan_z * inv_norm;
    const float u_para = ux * nx + uy * ny + uz * nz;
    const float px = ux - u_para * nx, py = uy - u_para * ny, pz = uz - u_para * nz;
    const float axial = fmaxf(0.0f, target - u_para);
    float damp = 1.0f;
    if (speed_pre > 0.24f) {
        const float r = (speed_pre - 0.24f) / fmaxf(1e-4f, 0.04f);
        damp = 1.0f / (1.0f + r * r);
    }
    const float beta = e.fan_mask * P.fan_beta * damp;
    fx = beta * rs * (axial * nx - 1.0f * px);
    fy = beta * rs * (axial * ny - 1.0f * py);
    fz = beta * rs * (axial * nz - 1.0f * pz);
}

// Reference clamp constants (jni.cpp:118-132).
constexpr float kNuShearMin = 1.0e-8f;
constexpr float kNuShearMax = (0.95f - 0.5f) / 3.0f;
constexpr float kTauMin = 0.5f + 3.0f * 1.0e-8f;
constexpr float kTauMax = 0.95f;
constexpr float kCs2f = 1.0f / 3.0f;

__device__ __forceinline__ float clampf_dev(float v, float lo, float hi) { return fminf(hi, fmaxf(lo, v)); }

__device__ __forceinline__ float feq27(int q, float rho, float ux, float uy, float uz) {
    const float cu = 3.0f * (float(q_cx(q)) * ux + float(q_cy(q)) * uy + float(q_cz(q)) * uz);
    const float uu = ux * ux + uy * uy + uz * uz;
    return q_w(q) * rho * (1.0f + cu + 0.5f * cu * cu - 1.5f * uu);
}

// Raw-moment sums of a population set: rho, j and the second-order raw
// moments, by 1-D partial sums (z, then y, then x).
struct RawMoments {
    float r000, r100, r010, r001, r200, r020, r002, r110, r101, r011;
};

template <bool kSecondOrder>
__device__ __forceinline__ void raw_moments27(const float (&f)[27], RawMoments& m) {
    float a0[9], a1[9], a2[9];
#pragma unroll
    for (int l = 0; l < 9; ++l) {
        const float fm = f[3 * l + 0], f0 = f[3 * l + 1], fp = f[3 * l + 2];
        a0[l] = (fm + fp) + f0;
        a1[l] = fp - fm;
        if (kSecondOrder) a2[l] = fp + fm;
    }
    float b00[3], b01[3], b02[3], b10[3], b11[3], b20[3];
#pragma unroll
    for (int ix = 0; ix < 3; ++ix) {
        const int l = 3 * ix;
        b00[ix] = (a0[l] + a0[l + 2]) + a0[l + 1];
        b01[ix] = a0[l + 2] - a0[l];
        b10[ix] = (a1[l] + a1[l + 2]) + a1[l + 1];
        if (kSecondOrder) {
            b02[ix] = a0[l + 2] + a0[l];
            b11[ix] = a1[l + 2] - a1[l];
            b20[ix] = (a2[l] + a2[l + 2]) + a2[l + 1];
        }
    }
    m.r000 = (b00[0] + b00[2]) + b00[1];
    m.r100 = b00[2] - b00[0];
    m.r010 = (b01[0] + b01[2]) + b01[1];
    m.r001 = (b10[0] + b10[2]) + b10[1];
    if (kSecondOrder) {
        m.r200 = b00[2] + b00[0];
        m.r110 = b01[2] - b01[0];
        m.r020 = (b02[0] + b02[2]) + b02[1];
        m.r101 = b10[2] - b10[0];
        m.r011 = (b11[0] + b11[2]) + b11[1];
        m.r002 = (b20[0] + b20[2]) + b20[1];
    }
}

// 1-D central -> population map along one axis for a line of central moments
// (m0, m1, m2): raw (m0, m1 + u m0, m2 + 2 u m1 + u^2 m0), then
// f(-1) = (R2 - R1)/2, f(0) = R0 - R2, f(+1) = (R1 + R2)/2.
__device__ __forceinline__ void back_line(float m0, float m1, float m2, float u, float& fm, float& f0, float& fp) {
    const float r1 = fmaf(u, m0, m1);
    const float r2 = fmaf(u, r1 + m1, m2);
    fm = 0.5f * (r2 - r1);
    f0 = m0 - r2;
    fp = 0.5f * (r1 + r2);
}
// Line with m1 = 0.
__device__ __forceinline__ void back_line_even(float m0, float m2, float u, float& fm, float& f0, float& fp) {
    const float r1 = u * m0;
    const float r2 = fmaf(u, r1, m2);
    fm = 0.5f * (r2 - r1);
    f0 = m0 - r2;
    fp = 0.5f * (r1 + r2);
}
// Line with m0 = m2 = 0.
__device__ __forceinline__ void back_line_odd(float m1, float u, float& fm, float& f0, float& fp) {
    fm = (u - 0.5f) * m1;
    f0 = -2.0f * u * m1;
    fp = (u + 0.5f) * m1;
}

// Result of a collision: the cell's macro state for diagnostics/output.
struct CollideOut {
    float rho;  // raw density sum (before the 1e-6 floor)
    float ux, uy, uz;  // midpoint velocity after the speed clamp
    bool reseeded;
};

// Reseed a cell from its reference state (jni.cpp:1724-1750): rho from the
// clamped pressure proxy, velocity clamped to max_speed, populations feq.
__device__ __forceinline__ void reseed27(float (&f)[27], float ref_p, float rux, float ruy, float ruz, float max_speed,
                                         CollideOut& out) {
    const float pr = clampf_dev(isfinite(ref_p) ? ref_p : 0.0f, -0.03f, 0.03f);
    const float rho = clampf_dev(1.0f + pr, 0.97f, 1.03f);
    float ux = isfinite(rux) ? rux : 0.0f, uy = isfinite(ruy) ? ruy : 0.0f, uz = isfinite(ruz) ? ruz : 0.0f;
    const float s2 = ux * ux + uy * uy + uz * uz;
    if (!isfinite(s2) || s2 > max_speed * max_speed) {
        if (!isfinite(s2) || s2 <= 0.0f) {
            ux = uy = uz = 0.0f;
        } else {
            const float sc = max_speed / sqrtf(s2);
            ux *= sc; uy *= sc; uz *= sc;
        }
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) f[q] = feq27(q, rho, ux, uy, uz);
    out.rho = rho; out.ux = ux; out.uy = uy; out.uz = uz; out.reseeded = true;
}

// Reference state of a cell, read only when the cell must be reseeded.
struct ReseedSource {
    const float* ref_p;
    const float* ref_ux;
    const float* ref_uy;
    const float* ref_uz;
    long long cell;
};


// Reseed state of a cell (reseed_cell_from_reference, jni.cpp:1724-1750):
// rho from the clamped pressure proxy, velocity clamped to max_speed.
__device__ __forceinline__ void reseed_state(const ReseedSource& r, float max_speed, float& rho, float& ux, float& uy,
                                             float& uz) {
    const float ref_p = r.ref_p[r.cell];
    const float pr = clampf_dev(isfinite(ref_p) ? ref_p : 0.0f, -0.03f, 0.03f);
    rho = clampf_dev(1.0f + pr, 0.97f, 1.03f);
    const float rux = r.ref_ux[r.cell], ruy = r.ref_uy[r.cell], ruz = r.ref_uz[r.cell];
    ux = isfinite(rux) ? rux : 0.0f;
    uy = isfinite(ruy) ? ruy : 0.0f;
    uz = isfinite(ruz) ? ruz : 0.0f;
    const float s2 = ux * ux + uy * uy + uz * uz;
    if (!isfinite(s2) || s2 > max_speed * max_speed) {
        if (!isfinite(s2) || s2 <= 0.0f) {
            ux = uy = uz = 0.0f;
        } else {
            const float sc = max_speed / sqrtf(s2);
            ux *= sc; uy *= sc; uz *= sc;
        }
    }
}

// Collide one fluid cell in place. `temperature` (the cell's entry of the
// temperature field, or a caller's local value) feeds buoyancy (read only
// when buoyancy is on); cfx/cfy/cfz is an extra per-cell force density (zero
// when unused). Returns false, leaving f untouched, when the input is not
// finite: the caller then reseeds the cell (out of line, see reseed_state).
__device__ __forceinline__ bool collide27(float (&f)[27], const CollideParams& P, const float* temperature,
                                          float cfx, float cfy, float cfz, CollideOut& out,
                                          const CellExtras* ex = nullptr) {
    RawMoments m;
    raw_moments27<true>(f, m);
    const float rho = m.r000;
    // Any non-finite population makes the plain sum rho non-finite.
    if (!isfinite(rho)) return false;
    const float rs = fmaxf(1e-6f, rho);
    const float ir = 1.0f / rs;
    float ux = m.r100 * ir, uy = m.r010 * ir, uz = m.r001 * ir;

    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    if (ex && P.fan_beta > 0.0f && ex->fan_mask > 0.0f) fan_force(*ex, P, rs, ux, uy, uz, fx, fy, fz);
    if (P.enable_buoyancy) {
        const float add = rs * clampf_dev(P.buoy_beta * *temperature, -P.buoy_fmax, P.buoy_fmax);
        if (P.gravity_axis == 0) fx += add;
        else if (P.gravity_axis == 1) fy += add;
        else fz += add;
    }
    fx += P.body_force[0] + cfx;
    fy += P.body_force[1] + cfy;
    fz += P.body_force[2] + cfz;
    ux += 0.5f * (fx * ir);
    uy += 0.5f * (fy * ir);
    uz += 0.5f * (fz * ir);
    if (ex && P.state_nudge > 0.0f) {
        const float sn = ex->nudge;
        ux = (1.0f - sn) * ux + sn * ex->ref_x;
        uy = (1.0f - sn) * uy + sn * ex->ref_y;
        uz = (1.0f - sn) * uz + sn * ex->ref_z;
    }
    const float s2 = ux * ux + uy * uy + uz * uz;
    if (!(isfinite(ux) && isfinite(uy) && isfinite(uz) && isfinite(s2))) return false;
    if (s2 > P.max_speed * P.max_speed) {
        const float sc = P.max_speed / sqrtf(s2);
        ux *= sc; uy *= sc; uz *= sc;
    }
    out.rho = rho; out.ux = ux; out.uy = uy; out.uz = uz; out.reseeded = false;

    // Second-order central moments about u from raw moments (binomial shift).
    const float c200 = fmaf(ux * ux, rho, fmaf(-2.0f * ux, m.r100, m.r200));
    const float c020 = fmaf(uy * uy, rho, fmaf(-2.0f * uy, m.r010, m.r020));
    const float c002 = fmaf(uz * uz, rho, fmaf(-2.0f * uz, m.r001, m.r002));
    const float c110 = fmaf(ux * uy, rho, fmaf(-ux, m.r010, fmaf(-uy, m.r100, m.r110)));
    const float c101 = fmaf(ux * uz, rho, fmaf(-ux, m.r001, fmaf(-uz, m.r100, m.r101)));
    const float c011 = fmaf(uy * uz, rho, fmaf(-uy, m.r001, fmaf(-uz, m.r010, m.r011)));

    float tau_s = P.tau_shear_base, tau_n = P.tau_normal_base;
    const float eq2 = rs * kCs2f;
    if (P.enable_sgs) {
        const float nxx = c200 - eq2, nyy = c020 - eq2, nzz = c002 - eq2;
        const float qn2 = nxx * nxx + nyy * nyy + nzz * nzz + 2.0f * (c110 * c110 + c101 * c101 + c011 * c011);
        const float qm = sqrtf(fmaxf(0.0f, qn2));
        const float sm = qm / fmaxf(1e-6f, 2.0f * rs * P.nu0);
        const float nut = fminf(P.sgs_c2 * sm, P.sgs_nut_cap);
        tau_s = clampf_dev(0.5f + 3.0f * clampf_dev(P.nu0 + nut, kNuShearMin, kNuShearMax), kTauMin, kTauMax);
        tau_n = clampf_dev(P.tau_normal_base + (tau_s - P.tau_shear_base) * P.sgs_bulk, kTauMin, kTauMax);
    }
    const float om_o = 1.0f / tau_s;
    const float sd = clampf_dev(1.0f / tau_n, 0.0f, 1.95f);
    const float so = clampf_dev(om_o, 0.0f, 1.95f);

    // Post-collision central moments (orders 0, 2, 4, 6; odd orders zero).
    const float k200 = c200 + sd * (eq2 - c200);
    const float k020 = c020 + sd * (eq2 - c020);
    const float k002 = c002 + sd * (eq2 - c002);
    const float k110 = (1.0f - so) * c110;
    const float k101 = (1.0f - so) * c101;
    const float k011 = (1.0f - so) * c011;
    const float irs = 1.0f / fmaxf(1e-6f, rs);
    const float k220 = (k200 * k020 + 2.0f * k110 * k110) * irs;
    const float k202 = (k200 * k002 + 2.0f * k101 * k101) * irs;
    const float k022 = (k020 * k002 + 2.0f * k011 * k011) * irs;
    const float k211 = (k200 * k011 + 2.0f * k110 * k101) * irs;
    const float k121 = (k020 * k101 + 2.0f * k110 * k011) * irs;
    const float k112 = (k002 * k110 + 2.0f * k101 * k011) * irs;
    const float k222 = (k200 * k020 * k002 + 2.0f * k110 * k110 * k002 + 2.0f * k101 * k101 * k020 +
                        2.0f * k011 * k011 * k200 + 8.0f * k110 * k101 * k011) * irs * irs;

    // x pass: g[ix][b][c] for the 9 (b, c) lines.
    float g[3][9];  // g[ix][b*3+c]
    back_line_even(rs, k200, ux, g[0][0], g[1][0], g[2][0]);     // (b,c)=(0,0)
    back_line_odd(k110, ux, g[0][3], g[1][3], g[2][3]);          // (1,0)
    back_line_even(k020, k220, ux, g[0][6], g[1][6], g[2][6]);   // (2,0)
    back_line_odd(k101, ux, g[0][1], g[1][1], g[2][1]);          // (0,1)
    back_line_even(k011, k211, ux, g[0][4], g[1][4], g[2][4]);   // (1,1)
    back_line_odd(k121, ux, g[0][7], g[1][7], g[2][7]);          // (2,1)
    back_line_even(k002, k202, ux, g[0][2], g[1][2], g[2][2]);   // (0,2)
    back_line_odd(k112, ux, g[0][5], g[1][5], g[2][5]);          // (1,2)
    back_line_even(k022, k222, ux, g[0][8], g[1][8], g[2][8]);   // (2,2)
    // y pass: h[ix][iy][c]
    float h[27];
#pragma unroll
    for (int ix = 0; ix < 3; ++ix) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            back_line(g[ix][0 * 3 + c], g[ix][1 * 3 + c], g[ix][2 * 3 + c], uy,
                      h[(ix * 3 + 0) * 3 + c], h[(ix * 3 + 1) * 3 + c], h[(ix * 3 + 2) * 3 + c]);
        }
    }
    // z pass: populations.
#pragma unroll
    for (int l = 0; l < 9; ++l) back_line(h[3 * l + 0], h[3 * l + 1], h[3 * l + 2], uz, f[3 * l + 0], f[3 * l + 1], f[3 * l + 2]);

    // Conservation fix-up. The reference adds feq(rho, u) - feq(rho_c, u_c)
    // (jni.cpp:2376-2394), a rounding-level correction; here its first-order
    // part w_q (drho + 3 c.dj), which restores sum f = rho and sum f c = rho u
    // exactly as the reference's does up to O(u * rounding).
    RawMoments mc;
    raw_moments27<false>(f, mc);
    const float drho = rs - mc.r000;
    const float djx = 3.0f * (rs * ux - mc.r100), djy = 3.0f * (rs * uy - mc.r010), djz = 3.0f * (rs * uz - mc.r001);

    // Guo source (jni.cpp:1270-1281): pref*w*(3(c.F - u.F) + 9 (c.u)(c.F)).
    const bool forced = (fx != 0.0f) | (fy != 0.0f) | (fz != 0.0f);
    const float pref = fmaxf(0.0f, 1.0f - 0.5f * clampf_dev(om_o, 0.0f, 1.999f));
    const float uf = ux * fx + uy * fy + uz * fz;

    // Pairs (q, 26 - q) for q < 13, then the rest population.
#pragma unroll
    for (int q = 0; q < 13; ++q) {
        const float cxq = float(q_cx(q)), cyq = float(q_cy(q)), czq = float(q_cz(q));
        const float odd = cxq * djx + cyq * djy + czq * djz;
        float se = 0.0f, so_ = 0.0f;
        if (forced) {
            const float cu = cxq * ux + cyq * uy + czq * uz;
            const float cf = cxq * fx + cyq * fy + czq * fz;
            se = pref * (9.0f * cu * cf - 3.0f * uf);
            so_ = pref * 3.0f * cf;
        }
        const float wq = q_w(q);
        f[q] += wq * ((drho + odd) + (se + so_));
        f[26 - q] += wq * ((drho - odd) + (se - so_));
    }
    {
        const float se = forced ? pref * (-3.0f * uf) : 0.0f;
        f[13] += q_w(13) * (drho + se);
    }
    return true;
}

}  // namespace aero
