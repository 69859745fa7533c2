// Temperature transport fused into the in-place step kernels: the first-order
// branch of the reference's benchmark-mode update (update_temperature_field,
// native/src/aero_lbm_jni.cpp:2049-2143; see thermal.cuh for the formula and
// the face rules), computed by the step kernel for its own cells right before
// their collision, instead of by a separate pass.
//
// A cell's update reads the previous temperature state in its 3x3x3
// neighbourhood and its own previous collision velocity; the step writes the
// new state into the other buffer and the new velocity over the old one. The
// state is double-buffered and the velocity is only read at the cell that
// writes it, so the fused update needs no grid-wide barrier. A block of the
// line launch (one (x, y) line segment of z cells) stages the nine z-rows
// (x + dx, y + dy), dx, dy in {-1, 0, 1}, of the state with the face rules
// resolved (th_neighbour's codes: 0 value, 1 the querying cell's own value,
// 2 own value + Neumann flux) in shared memory. Every product and sum is an
// explicitly rounded intrinsic in the reference's order, so the result is the
// separate pass's (bit-identical), also inside kernels compiled with
// multiply-add contraction.
#pragma once

#include "collide27_exact.cuh"
#include "thermal.cuh"

namespace aero {

struct FusedTransport {
    const float* t;       // state before the update (read-only in the step)
    float* t_next;        // state after the update (the collision's buoyancy field)
    const float* u;       // previous collision velocity, SoA (ux, uy, uz), read at the own cell only
    const float* source;  // per-cell source (clamped to +-0.006 here), or null
    float alpha;          // thermal diffusivity
    ThermalFaces faces;
};

namespace thermal_fused {

// One staged entry (x, y, z) of a brick nx x ny x nz: the face rules of
// th_neighbour / stage_outside (periodic thermal faces wrap, Dirichlet takes
// the clamped face value, Neumann own + flux, other faces and solid cells
// the querying cell's own value).
__device__ __forceinline__ void stage_entry(const FusedTransport& tr, const uint8_t* obstacle, int nx, int ny, int nz,
                                            int x, int y, int z, float& v, unsigned char& code) {
    const ThermalFaces& F = tr.faces;
    if ((x < 0 || x >= nx) && F.kind[x < 0 ? 0 : 1] == kThermalPeriodic) {
        x %= nx;
        if (x < 0) x += nx;
    }
    if ((y < 0 || y >= ny) && F.kind[y < 0 ? 2 : 3] == kThermalPeriodic) {
        y %= ny;
        if (y < 0) y += ny;
    }
    if ((z < 0 || z >= nz) && F.kind[z < 0 ? 4 : 5] == kThermalPeriodic) {
        z %= nz;
        if (z < 0) z += nz;
    }
    int face = -1;
    if (x < 0) face = 0;
    else if (x >= nx) face = 1;
    else if (y < 0) face = 2;
    else if (y >= ny) face = 3;
    else if (z < 0) face = 4;
    else if (z >= nz) face = 5;
    v = 0.0f;
    if (face >= 0) {
        const int kind = F.kind[face];
        if (kind == kThermalDirichlet) {
            code = 0;
            v = exact::rclamp(F.temperature[face], -1.0f, 1.0f);
        } else if (kind == kThermalNeumann) {
            code = 2;
            v = F.heat_flux[face];
        } else {
            code = 1;
        }
        return;
    }
    const long long cell = ((long long)x * ny + y) * nz + z;
    code = obstacle[cell] ? 1 : 0;
    if (!code) v = __ldg(tr.t + cell);
}

// Stage the nine rows of a block's z-segment [z_begin, z_begin + span) plus a
// one-cell halo in z: entry (dx, dy, k) at ((dx + 1) * 3 + dy + 1) * W + k,
// W = span + 2, k = z - z_begin + 1. Every thread of the block takes part.
// Tagged staging (no Neumann face, kOwnTag of thermal.cuh): the code array
// is not read.

template <bool kTagged>
__device__ __forceinline__ void put_entry(float* sv, unsigned char* sc, int i, float v, unsigned char code) {
    if (kTagged) {
        sv[i] = code == 1 ? __uint_as_float(kOwnTag) : v;
    } else {
        sv[i] = v;
        sc[i] = code;
    }
}

// A line whose eight neighbour lines lie inside the brick (the block-uniform
// common case) reads its rows directly: the span's own entries are cells of
// the brick (per entry one mask byte and one temperature, kept for a fluid
// cell), and the 18 z-halo entries (one per thread) take the face rules.
template <bool kTagged>
__device__ __forceinline__ void stage_rows(const FusedTransport& tr, const uint8_t* obstacle, int nx, int ny, int nz, int x,
                                           int y, int z_begin, int span, float* sv, unsigned char* sc) {
    const int W = span + 2;
    if (x > 0 && x < nx - 1 && y > 0 && y < ny - 1) {
#pragma unroll 1
        for (int r = 0; r < 9; ++r) {
            const long long row = ((long long)(x + r / 3 - 1) * ny + (y + r % 3 - 1)) * nz + z_begin - 1;
            const uint8_t* ob = obstacle + row;
            const float* t = tr.t + row;
            for (int k = 1 + threadIdx.x; k <= span; k += blockDim.x) {
                const unsigned char code = ob[k] ? 1 : 0;
                const float v = __ldg(t + k);
                put_entry<kTagged>(sv, sc, r * W + k, code ? 0.0f : v, code);
            }
        }
        for (int i = threadIdx.x; i < 18; i += blockDim.x) {
            const int r = i >> 1, k = (i & 1) ? span + 1 : 0;
            float v;
            unsigned char code;
            stage_entry(tr, obstacle, nx, ny, nz, x + r / 3 - 1, y + r % 3 - 1, z_begin - 1 + k, v, code);
            put_entry<kTagged>(sv, sc, r * W + k, v, code);
        }
        return;
    }
    for (int i = threadIdx.x; i < 9 * W; i += blockDim.x) {
        const int r = i / W, k = i - r * W;
        float v;
        unsigned char code;
        stage_entry(tr, obstacle, nx, ny, nz, x + r / 3 - 1, y + r % 3 - 1, z_begin - 1 + k, v, code);
        put_entry<kTagged>(sv, sc, i, v, code);
    }
}

template <bool kTagged>
__device__ __forceinline__ float at(const float* sv, const unsigned char* sc, int i, float self) {
    const float v = sv[i];
    if (kTagged) return __float_as_uint(v) == kOwnTag ? self : v;
    const int c = sc[i];
    return c == 0 ? v : (c == 1 ? self : exact::rclamp(__fadd_rn(self, v), -1.0f, 1.0f));
}

// th_sample (sample_temperature_trilinear_field, jni.cpp:1910-1945) from
// global memory, for a velocity of a full cell or more (out of line: a
// collision's speed clamp keeps |u| < 1).
static __device__ __noinline__ float sample_far(const FusedTransport tr, const uint8_t* obstacle, int nx, int ny, int nz, float px,
                                         float py, float pz, float self) {
    const int x0 = (int)floorf(px), y0 = (int)floorf(py), z0 = (int)floorf(pz);
    const float fx = __fsub_rn(px, (float)x0), fy = __fsub_rn(py, (float)y0), fz = __fsub_rn(pz, (float)z0);
    float c[8];
#pragma unroll 1
    for (int k = 0; k < 8; ++k) {
        float v;
        unsigned char code;
        stage_entry(tr, obstacle, nx, ny, nz, x0 + (k & 1), y0 + ((k >> 1) & 1), z0 + (k >> 2), v, code);
        c[k] = code == 0 ? v : (code == 1 ? self : exact::rclamp(__fadd_rn(self, v), -1.0f, 1.0f));
    }
    const float c00 = __fadd_rn(c[0], __fmul_rn(__fsub_rn(c[1], c[0]), fx));
    const float c10 = __fadd_rn(c[2], __fmul_rn(__fsub_rn(c[3], c[2]), fx));
    const float c01 = __fadd_rn(c[4], __fmul_rn(__fsub_rn(c[5], c[4]), fx));
    const float c11 = __fadd_rn(c[6], __fmul_rn(__fsub_rn(c[7], c[6]), fx));
    const float c0 = __fadd_rn(c00, __fmul_rn(__fsub_rn(c10, c00), fy));
    const float c1 = __fadd_rn(c01, __fmul_rn(__fsub_rn(c11, c01), fy));
    return __fadd_rn(c0, __fmul_rn(__fsub_rn(c1, c0), fz));
}

// The updated temperature of fluid cell (x, y, z) (update_cell of the
// separate pass): semi-Lagrangian sample at x - u, 6-point Laplacian, source;
// k = z - z_begin + 1 indexes the staged rows.
template <bool kTagged>
__device__ __forceinline__ float update(const FusedTransport& tr, const uint8_t* obstacle, int nx, int ny, int nz,
                                        const float* sv, const unsigned char* sc, int W, int k, int x, int y, int z,
                                        long long cell) {
    const float dt = 1.0f, cooling = 0.0f;
    const int ctr = 4 * W + k;  // row (0, 0)
    const float tc = sv[ctr];
    const float ux = tr.u[cell], uy = tr.u[cell + (long long)nx * ny * nz], uz = tr.u[cell + 2LL * nx * ny * nz];
    const float src = tr.source ? exact::rclamp(__ldg(tr.source + cell), -0.006f, 0.006f) : 0.0f;
    const float px = __fsub_rn((float)x, __fmul_rn(dt, ux));
    const float py = __fsub_rn((float)y, __fmul_rn(dt, uy));
    const float pz = __fsub_rn((float)z, __fmul_rn(dt, uz));
    float adv;
    if (fabsf(ux) < 1.0f && fabsf(uy) < 1.0f && fabsf(uz) < 1.0f) {
        const int x0 = (int)floorf(px), y0 = (int)floorf(py), z0 = (int)floorf(pz);
        const float fx = __fsub_rn(px, (float)x0), fy = __fsub_rn(py, (float)y0), fz = __fsub_rn(pz, (float)z0);
        // corner (x0, y0, z0): rows step by 3 W in x and W in y
        const int b = ((x0 - x + 1) * 3 + (y0 - y + 1)) * W + k + (z0 - z);
        const float c000 = at<kTagged>(sv, sc, b, tc);
        const float c100 = at<kTagged>(sv, sc, b + 3 * W, tc);
        const float c010 = at<kTagged>(sv, sc, b + W, tc);
        const float c110 = at<kTagged>(sv, sc, b + 4 * W, tc);
        const float c001 = at<kTagged>(sv, sc, b + 1, tc);
        const float c101 = at<kTagged>(sv, sc, b + 3 * W + 1, tc);
        const float c011 = at<kTagged>(sv, sc, b + W + 1, tc);
        const float c111 = at<kTagged>(sv, sc, b + 4 * W + 1, tc);
        const float c00 = __fadd_rn(c000, __fmul_rn(__fsub_rn(c100, c000), fx));
        const float c10 = __fadd_rn(c010, __fmul_rn(__fsub_rn(c110, c010), fx));
        const float c01 = __fadd_rn(c001, __fmul_rn(__fsub_rn(c101, c001), fx));
        const float c11 = __fadd_rn(c011, __fmul_rn(__fsub_rn(c111, c011), fx));
        const float c0 = __fadd_rn(c00, __fmul_rn(__fsub_rn(c10, c00), fy));
        const float c1 = __fadd_rn(c01, __fmul_rn(__fsub_rn(c11, c01), fy));
        adv = __fadd_rn(c0, __fmul_rn(__fsub_rn(c1, c0), fz));
    } else {
        adv = sample_far(tr, obstacle, nx, ny, nz, px, py, pz, tc);
    }
    // neighbours in the reference's order: +x, -x, +y, -y, +z, -z
    float t_sum = __fadd_rn(at<kTagged>(sv, sc, ctr + 3 * W, tc), at<kTagged>(sv, sc, ctr - 3 * W, tc));
    t_sum = __fadd_rn(t_sum, at<kTagged>(sv, sc, ctr + W, tc));
    t_sum = __fadd_rn(t_sum, at<kTagged>(sv, sc, ctr - W, tc));
    t_sum = __fadd_rn(t_sum, at<kTagged>(sv, sc, ctr + 1, tc));
    t_sum = __fadd_rn(t_sum, at<kTagged>(sv, sc, ctr - 1, tc));
    const float lap = __fsub_rn(t_sum, __fmul_rn(6.0f, tc));
    const float rate = __fsub_rn(__fadd_rn(__fmul_rn(tr.alpha, lap), src), __fmul_rn(cooling, adv));
    return exact::rclamp(__fadd_rn(adv, __fmul_rn(dt, rate)), -1.0f, 1.0f);
}

// Stage this block's rows and update the given cells of the thread (zs[i] <
// nz, x, y the block's line): the new state is written to t_next and returned
// in tn (0 on cells that are solid in this call). Called by every thread of
// the block, before any of them returns.
template <int kCells>
__device__ __forceinline__ void update_cells(const FusedTransport& tr, const uint8_t* obstacle, int nx, int ny, int nz,
                                             int x, int y, int z_begin, int span, const int (&zs)[kCells],
                                             float (&tn)[kCells], float* sv, unsigned char* sc) {
    const bool tagged = no_neumann(tr.faces);
    if (tagged) stage_rows<true>(tr, obstacle, nx, ny, nz, x, y, z_begin, span, sv, sc);
    else stage_rows<false>(tr, obstacle, nx, ny, nz, x, y, z_begin, span, sv, sc);
    __syncthreads();
    const int W = span + 2;
#pragma unroll
    for (int i = 0; i < kCells; ++i) {
        tn[i] = 0.0f;
        const int z = zs[i];
        if (z >= nz) continue;
        const long long cell = ((long long)x * ny + y) * nz + z;
        if (!obstacle[cell])
            tn[i] = tagged ? update<true>(tr, obstacle, nx, ny, nz, sv, sc, W, z - z_begin + 1, x, y, z, cell)
                           : update<false>(tr, obstacle, nx, ny, nz, sv, sc, W, z - z_begin + 1, x, y, z, cell);
        tr.t_next[cell] = tn[i];
    }
}

}  // namespace thermal_fused
}  // namespace aero
