// Temperature transport kernels (see thermal.cuh). Built with --fmad=false:
// every product and sum rounds separately, in the reference's order.
#include "thermal.cuh"

#include "collide27_exact.cuh"
#include "collide27_exact_x2.cuh"
#include "d3q27_inplace.cuh"
#include "pdl.cuh"

namespace aero {
namespace {

// thermal_field_neighbor_or_self (jni.cpp:1800-1825) with remap_thermal_coords
// (jni.cpp:738-749, 779-785) and thermal_face_for_oob (jni.cpp:761-769).
__device__ __forceinline__ float th_neighbour(const ThermalArgs& a, const float* field, int x, int y, int z, float self) {
    const ThermalFaces& F = a.faces;
    if ((x < 0 || x >= a.nx) && F.kind[x < 0 ? 0 : 1] == kThermalPeriodic) {
        x %= a.nx;
        if (x < 0) x += a.nx;
    }
    if ((y < 0 || y >= a.ny) && F.kind[y < 0 ? 2 : 3] == kThermalPeriodic) {
        y %= a.ny;
        if (y < 0) y += a.ny;
    }
    if ((z < 0 || z >= a.nz) && F.kind[z < 0 ? 4 : 5] == kThermalPeriodic) {
        z %= a.nz;
        if (z < 0) z += a.nz;
    }
    int face = -1;
    if (x < 0) face = 0;
    else if (x >= a.nx) face = 1;
    else if (y < 0) face = 2;
    else if (y >= a.ny) face = 3;
    else if (z < 0) face = 4;
    else if (z >= a.nz) face = 5;
    if (face >= 0) {
        const int kind = F.kind[face];
        if (kind == kThermalDirichlet) return exact::rclamp(F.temperature[face], -1.0f, 1.0f);
        if (kind == kThermalNeumann) return exact::rclamp(self + F.heat_flux[face], -1.0f, 1.0f);
        return self;
    }
    const long long cell = ((long long)x * a.ny + y) * a.nz + z;
    // both loads issued before the test (one round trip, not two)
    const bool solid = a.obstacle[cell] != 0;
    const float v = field[cell];
    return solid ? self : v;
}
__device__ __forceinline__ float th_neighbour(const ThermalArgs& a, int x, int y, int z, float self) {
    return th_neighbour(a, a.t, x, y, z, self);
}

// sample_temperature_trilinear_field (jni.cpp:1910-1945).
__device__ __forceinline__ float th_sample(const ThermalArgs& a, const float* field, float x, float y, float z,
                                           float fallback) {
    const int x0 = (int)floorf(x), y0 = (int)floorf(y), z0 = (int)floorf(z);
    const int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
    const float fx = x - (float)x0, fy = y - (float)y0, fz = z - (float)z0;
    float c000, c100, c010, c110, c001, c101, c011, c111;
    // x0 < nx - 1, not x1 < nx: a non-finite or huge position converts to
    // INT_MAX, where x0 + 1 wraps
    if (x0 >= 0 && x0 < a.nx - 1 && y0 >= 0 && y0 < a.ny - 1 && z0 >= 0 && z0 < a.nz - 1) {
        // every corner inside the brick: the 16 loads issue together, then
        // th_neighbour's solid rule
        const int sy = a.nz, sx = a.ny * a.nz;
        const int b = (x0 * a.ny + y0) * a.nz + z0;
        const int o[8] = {0, sx, sy, sx + sy, 1, sx + 1, sy + 1, sx + sy + 1};
        bool solid[8];
        float v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            solid[k] = a.obstacle[b + o[k]] != 0;
            v[k] = field[b + o[k]];
        }
        c000 = solid[0] ? fallback : v[0];
        c100 = solid[1] ? fallback : v[1];
        c010 = solid[2] ? fallback : v[2];
        c110 = solid[3] ? fallback : v[3];
        c001 = solid[4] ? fallback : v[4];
        c101 = solid[5] ? fallback : v[5];
        c011 = solid[6] ? fallback : v[6];
        c111 = solid[7] ? fallback : v[7];
    } else {
        c000 = th_neighbour(a, field, x0, y0, z0, fallback);
        c100 = th_neighbour(a, field, x1, y0, z0, fallback);
        c010 = th_neighbour(a, field, x0, y1, z0, fallback);
        c110 = th_neighbour(a, field, x1, y1, z0, fallback);
        c001 = th_neighbour(a, field, x0, y0, z1, fallback);
        c101 = th_neighbour(a, field, x1, y0, z1, fallback);
        c011 = th_neighbour(a, field, x0, y1, z1, fallback);
        c111 = th_neighbour(a, field, x1, y1, z1, fallback);
    }
    const float c00 = c000 + (c100 - c000) * fx;
    const float c10 = c010 + (c110 - c010) * fx;
    const float c01 = c001 + (c101 - c001) * fx;
    const float c11 = c011 + (c111 - c011) * fx;
    const float c0 = c00 + (c10 - c00) * fy;
    const float c1 = c01 + (c11 - c01) * fy;
    return c0 + (c1 - c0) * fz;
}

// The update reads the 3x3x3 neighbourhood of each cell (|u| < 1 keeps every
// trilinear corner inside it). A block owns a (kMY y) x (kMZ z) column of the
// brick over a run of consecutive x-planes and walks it in x; each thread owns
// two z-adjacent cells of a plane. Shared memory holds a ring of kRing staged
// planes, each with its y/z halo (two cells wide in z, so that staged z-pairs
// line up with the brick's even cells) and each entry already resolved by
// th_neighbour's rules: code 0 = use the value (a fluid cell's temperature, or
// a Dirichlet face's clamped temperature), 1 = the querying cell's own value
// (solid cell, adiabatic / disabled / inherit face), 2 = own value + the
// stored Neumann flux, clamped. Periodic faces are resolved by staging the
// wrapped cell. Computing plane x reads the ring's planes x-1, x, x+1 while
// plane x+2 is written from registers loaded two planes earlier, so each
// plane's global loads are in flight during two planes of compute.
constexpr int kMZ = 32, kMY = 8;                  // cells of a plane per block: z x y
constexpr int kMTZ = kMZ / 2;                     // threads along z (one per z-pair)
constexpr int kMThreads = kMTZ * kMY;             // 128
constexpr int kPZ = kMZ + 4;                      // staged row: z from zb - 2 to zb + kMZ + 1
constexpr int kRowPairs = kPZ / 2;                // 18
constexpr int kPairs = kRowPairs * (kMY + 2);     // staged z-pairs per plane: 180
constexpr int kPlane = kPZ * (kMY + 2);           // staged entries per plane: 360
constexpr int kRing = 4;                          // staged planes
constexpr int kColumnBlocksPerSM = 7;             // resident column blocks per SM (72 registers)
static_assert(kPairs <= 2 * kMThreads, "two staged pairs per thread and plane");

// Lookups specialise on the brick's faces (launch-uniform): without a Neumann
// face only codes 0 and 1 occur and code 1 entries hold kOwnTag (the code
// array is not read); otherwise any code.
enum TileKind { kTileTagged = 1, kTileAny = 2 };

template <int kKind>
__device__ __forceinline__ float tile_at(const float* sv, const unsigned char* sc, int i, float self) {
    const float v = sv[i];
    if (kKind == kTileTagged) return __float_as_uint(v) == kOwnTag ? self : v;
    const int c = sc[i];
    return c == 0 ? v : (c == 1 ? self : exact::rclamp(self + v, -1.0f, 1.0f));
}

// th_neighbour's rule for a face (the querying cell's value not yet known):
// Dirichlet -> (clamped face temperature, code 0), Neumann -> (heat flux,
// code 2), any other kind -> code 1 (the querying cell's own value).
__device__ __forceinline__ void face_entry(const ThermalFaces& F, int face, float& v, unsigned char& code) {
    const int kind = F.kind[face];
    v = 0.0f;
    code = 1;
    if (kind == kThermalDirichlet) {
        code = 0;
        v = exact::rclamp(F.temperature[face], -1.0f, 1.0f);
    } else if (kind == kThermalNeumann) {
        code = 2;
        v = F.heat_flux[face];
    }
}

// Where a staged entry at (y, z) of an in-brick (or x-wrapped) plane comes
// from, by th_neighbour's rules (periodic axes wrap first, then the first
// face crossed in the order y, z decides): true with off = y' nz + z' of the
// cell to load, or false with the face's (v, code).
__device__ __forceinline__ bool resolve_yz(const ThermalFaces& F, int ny, int nz, int y, int z, int& off, float& v,
                                           unsigned char& code) {
    if ((y < 0 || y >= ny) && F.kind[y < 0 ? 2 : 3] == kThermalPeriodic) {
        y %= ny;
        if (y < 0) y += ny;
    }
    if ((z < 0 || z >= nz) && F.kind[z < 0 ? 4 : 5] == kThermalPeriodic) {
        z %= nz;
        if (z < 0) z += nz;
    }
    off = y * nz + z;
    if (y >= 0 && y < ny && z >= 0 && z < nz) return true;
    face_entry(F, y < 0 ? 2 : (y >= ny ? 3 : (z < 0 ? 4 : 5)), v, code);
    return false;
}

// Plane gx of the staging: the plane to load (gx, or its periodic wrap), or
// -1 with the x face's (v, code) for every entry (x is tested first).
__device__ __forceinline__ int resolve_x(const ThermalFaces& F, int nx, int gx, float& v, unsigned char& code) {
    if (gx >= 0 && gx < nx) return gx;
    if (F.kind[gx < 0 ? 0 : 1] == kThermalPeriodic) {
        gx %= nx;
        return gx < 0 ? gx + nx : gx;
    }
    face_entry(F, gx < 0 ? 0 : 1, v, code);
    return -1;
}

// th_sample for a cell moving a full cell or more per step (never after a
// collision: the speed clamp keeps |u| < 1; only a first call's packet
// velocity can); out of line.
__device__ __noinline__ float th_sample_far(const ThermalArgs& a, float px, float py, float pz, float fallback) {
    return th_sample(a, a.t, px, py, pz, fallback);
}

// runtime_local_turbulent_nu (jni.cpp:1972-2031): 0 next to a solid face
// neighbour; else C^2 |S| (capped at 5 nu0) from central differences of the
// last collision's velocity, a solid or outside neighbour giving the centre's
// value.
__device__ __noinline__ float eddy_nu(const ThermalArgs& a, int x, int y, int z) {
    // the six face neighbours (+x, -x, +y, -y, +z, -z): every mask byte and
    // velocity is loaded before any test (outside neighbours read the cell
    // itself), so the loads are in flight together
    const int off[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    const long long cc = ((long long)x * a.ny + y) * a.nz + z;
    bool inside[6];
    long long nc[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const int p = x + off[i][0], q = y + off[i][1], r = z + off[i][2];
        inside[i] = !(p < 0 || q < 0 || r < 0 || p >= a.nx || q >= a.ny || r >= a.nz);
        nc[i] = inside[i] ? ((long long)p * a.ny + q) * a.nz + r : cc;
    }
    bool solid[6];
    float nv[3][6], sv[3];
#pragma unroll
    for (int i = 0; i < 6; ++i) solid[i] = a.obstacle[nc[i]] != 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float* v = a.u + (long long)k * a.cells;
        sv[k] = v[cc];
#pragma unroll
        for (int i = 0; i < 6; ++i) nv[k][i] = v[nc[i]];
    }
#pragma unroll
    for (int i = 0; i < 6; ++i)
        if (inside[i] && solid[i]) return 0.0f;
    // the neighbour's velocity, the centre's for an outside one (a solid
    // inside neighbour has returned above)
    float d[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float w[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) w[i] = (inside[i] && !solid[i]) ? nv[k][i] : sv[k];
        d[k][0] = 0.5f * (w[0] - w[1]);
        d[k][1] = 0.5f * (w[2] - w[3]);
        d[k][2] = 0.5f * (w[4] - w[5]);
    }
    const float sxx = d[0][0], syy = d[1][1], szz = d[2][2];
    const float sxy = 0.5f * (d[0][1] + d[1][0]);
    const float sxz = 0.5f * (d[0][2] + d[2][0]);
    const float syz = 0.5f * (d[1][2] + d[2][1]);
    const float smag = sqrtf(exact::rmax(0.0f, 2.0f * (sxx * sxx + syy * syy + szz * szz) +
                                                     4.0f * (sxy * sxy + sxz * sxz + syz * syz)));
    float nut = a.sgs_c2 * smag;
    nut = exact::rmin(nut, 5.0f * a.nu0);
    return exact::rmax(0.0f, nut);
}

// ---- BFECC branch (jni.cpp:2050-2135): one thread per cell, line grid.
__device__ __forceinline__ bool th_line_cell(const ThermalArgs& a, int& x, int& y, int& z, int& cell) {
    z = blockIdx.x * blockDim.x + threadIdx.x;
    y = blockIdx.y;
    x = blockIdx.z;
    cell = (x * a.ny + y) * a.nz + z;
    return z < a.nz;
}

// scratch = A_-(T)
__global__ void __launch_bounds__(128) bfecc_forward_kernel(const __grid_constant__ ThermalArgs a) {
    int x, y, z, cell;
    if (!th_line_cell(a, x, y, z, cell)) return;
    if (a.obstacle[cell]) {
        a.scratch[cell] = 0.0f;
        return;
    }
    const float dt = a.dt;
    const float ux = a.u[cell], uy = a.u[a.cells + cell], uz = a.u[2 * a.cells + cell];
    a.scratch[cell] = th_sample(a, a.t, (float)x - dt * ux, (float)y - dt * uy, (float)z - dt * uz, a.t[cell]);
}

// next = clamp(T + (T - A_+(scratch)) / 2)
__global__ void __launch_bounds__(128) bfecc_correct_kernel(const __grid_constant__ ThermalArgs a) {
    int x, y, z, cell;
    if (!th_line_cell(a, x, y, z, cell)) return;
    if (a.obstacle[cell]) {
        a.t_next[cell] = 0.0f;
        return;
    }
    const float dt = a.dt;
    const float tc = a.t[cell];
    const float ux = a.u[cell], uy = a.u[a.cells + cell], uz = a.u[2 * a.cells + cell];
    const float back = th_sample(a, a.scratch, (float)x + dt * ux, (float)y + dt * uy, (float)z + dt * uz, a.scratch[cell]);
    a.t_next[cell] = exact::rclamp(tc + 0.5f * (tc - back), -1.0f, 1.0f);
}

// scratch = clamp(clamp(A_-(next), local bounds of T) + dt (alpha lap T + s))
__global__ void __launch_bounds__(128) bfecc_final_kernel(const __grid_constant__ ThermalArgs a) {
    int x, y, z, cell;
    if (!th_line_cell(a, x, y, z, cell)) return;
    if (a.obstacle[cell]) {
        a.scratch[cell] = 0.0f;
        return;
    }
    const float dt = a.dt, cooling = 0.0f;
    const float tc = a.t[cell];
    const float ux = a.u[cell], uy = a.u[a.cells + cell], uz = a.u[2 * a.cells + cell];
    float adv = th_sample(a, a.t_next, (float)x - dt * ux, (float)y - dt * uy, (float)z - dt * uz, a.t_next[cell]);
    float n0, n1, n2, n3, n4, n5;
    if (x >= 1 && x + 1 < a.nx && y >= 1 && y + 1 < a.ny && z >= 1 && z + 1 < a.nz) {
        // all six face neighbours inside the brick: loads first, then the solid rule
        const int sx = a.ny * a.nz, sy = a.nz;
        const int o[6] = {sx, -sx, sy, -sy, 1, -1};
        bool solid[6];
        float v[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            solid[k] = a.obstacle[cell + o[k]] != 0;
            v[k] = a.t[cell + o[k]];
        }
        n0 = solid[0] ? tc : v[0];
        n1 = solid[1] ? tc : v[1];
        n2 = solid[2] ? tc : v[2];
        n3 = solid[3] ? tc : v[3];
        n4 = solid[4] ? tc : v[4];
        n5 = solid[5] ? tc : v[5];
    } else {
        n0 = th_neighbour(a, x + 1, y, z, tc);
        n1 = th_neighbour(a, x - 1, y, z, tc);
        n2 = th_neighbour(a, x, y + 1, z, tc);
        n3 = th_neighbour(a, x, y - 1, z, tc);
        n4 = th_neighbour(a, x, y, z + 1, tc);
        n5 = th_neighbour(a, x, y, z - 1, tc);
    }
    // local_temperature_bounds (jni.cpp:1883-1908): std::min / std::max in neighbour order
    float lo = tc, hi = tc;
    const float nb[6] = {n0, n1, n2, n3, n4, n5};
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        lo = exact::rmin(lo, nb[i]);
        hi = exact::rmax(hi, nb[i]);
    }
    adv = exact::rclamp(adv, lo, hi);
    const float t_sum = n0 + n1 + n2 + n3 + n4 + n5;
    const float lap = t_sum - 6.0f * tc;
    const float src = a.source ? exact::rclamp(a.source[cell], -0.006f, 0.006f) : 0.0f;
    const float alpha = a.turbulent ? a.alpha + eddy_nu(a, x, y, z) / exact::rmax(1.0e-6f, 0.85f) : a.alpha;
    a.scratch[cell] = exact::rclamp(adv + dt * (alpha * lap + src - cooling * adv), -1.0f, 1.0f);
}

__global__ void thermal_reference_nudge_kernel(ThermalNudgeArgs a) {
    const long long cells = (long long)a.nx * a.ny * a.nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    if (a.obstacle[cell]) {
        a.t[cell] = 0.0f;
        return;
    }
    int x, y, z;
    cell_xyz32(cell, a.ny, a.nz, x, y, z);
    const int d = min(min(min(x, y), min(z, a.nx - 1 - x)), min(a.ny - 1 - y, a.nz - 1 - z));
    if (d >= 8) return;
    const float eta = (float)(8 - d) / 8.0f;
    const float n = a.nudge * eta * eta;
    if (n <= 0.0f) return;
    const float rt = exact::rclamp(a.ref_t[cell], -1.0f, 1.0f);
    const float keep = 1.0f - n;
    a.t[cell] = exact::rclamp(a.t[cell] * keep + rt * n, -1.0f, 1.0f);
}

// The staged z-pairs of one thread (e = 0: pair tid, e = 1: pair tid + 128
// where that is inside the plane) and the registers a plane is fetched into.
// Where each staged entry comes from is resolved once per block (SourceTable):
// most pairs are two aligned in-brick cells loaded as one vector; the others
// (halo entries outside the brick, odd nz) go entry by entry through the table.
struct StageSlots {
    int idx[2];      // entry of the pair's first cell inside a staged plane
    int off[2];      // gy nz + gz of the pair's first cell (vector pairs)
    unsigned flags;  // per pair e (2 bits from bit 2e): valid, vector pair
    __device__ bool valid(int e) const { return (flags >> (2 * e)) & 1u; }
    __device__ bool vec(int e) const { return (flags >> (2 * e + 1)) & 1u; }
};
struct SourceTable {
    int off[kPlane];            // >= 0: y nz + z of the cell an entry loads; < 0: -1 - its face code
    float val[kPlane];          // the face value of an entry with off < 0
};
struct PlaneRegs {
    float t[2][2];
    unsigned m;  // mask byte of cell k of pair e at bit 8 (2 e + k)
    __device__ bool solid(int e, int k) const { return ((m >> (8 * (2 * e + k))) & 0xFFu) != 0; }
};

// Loads plane gxe (resolve_x's result; -1: nothing to load).
__device__ __forceinline__ void fetch_plane(const ThermalArgs& a, const StageSlots& s, const SourceTable& src, int gxe,
                                            PlaneRegs& r) {
    const int base = gxe * a.ny * a.nz;
    r.m = 0;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        r.t[e][0] = r.t[e][1] = 0.0f;
        if (gxe < 0 || !s.valid(e)) continue;
        if (s.vec(e)) {
            const int c = base + s.off[e];
            const float2 t2 = __ldg(reinterpret_cast<const float2*>(a.t + c));
            const unsigned short m2 = __ldg(reinterpret_cast<const unsigned short*>(a.obstacle + c));
            r.t[e][0] = t2.x;
            r.t[e][1] = t2.y;
            r.m |= (unsigned)m2 << (16 * e);
        } else {
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int o = src.off[s.idx[e] + k];
                if (o >= 0) {
                    r.m |= (unsigned)__ldg(a.obstacle + base + o) << (8 * (2 * e + k));
                    r.t[e][k] = __ldg(a.t + base + o);
                }
            }
        }
    }
}

// Stages plane gx (loaded as gxe, or the x face's (xv, xcode) when gxe < 0)
// into its ring slot.
__device__ __forceinline__ void store_plane(const StageSlots& s, const SourceTable& src, int gx, int gxe, float xv,
                                            unsigned char xcode, const PlaneRegs& r, float* sv, unsigned char* sc,
                                            bool tagged) {
    const int slot = (gx & (kRing - 1)) * kPlane;
    const float own_tag = tagged ? __uint_as_float(kOwnTag) : 0.0f;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        if (!s.valid(e)) continue;
        const int i = slot + s.idx[e];
        if (gxe >= 0 && s.vec(e)) {
            const bool s0 = r.solid(e, 0), s1 = r.solid(e, 1);
            *reinterpret_cast<float2*>(sv + i) = make_float2(s0 ? own_tag : r.t[e][0], s1 ? own_tag : r.t[e][1]);
            *reinterpret_cast<uchar2*>(sc + i) = make_uchar2(s0 ? 1 : 0, s1 ? 1 : 0);
            continue;
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int o = src.off[s.idx[e] + k];
            float v;
            unsigned char code;
            if (gxe < 0) {
                v = xv;
                code = xcode;
            } else if (o >= 0) {
                code = r.solid(e, k) ? 1 : 0;
                v = code ? 0.0f : r.t[e][k];
            } else {
                code = (unsigned char)(-1 - o);
                v = src.val[s.idx[e] + k];
            }
            sv[i + k] = (tagged && code == 1) ? own_tag : v;
            sc[i + k] = code;
        }
    }
}

// The velocity and source of the thread's two cells for three planes ahead
// travel by cp.async into a per-thread shared ring (no registers held while
// in flight): slot x % 3, component d (ux, uy, uz, source), one float pair per
// thread. Each plane's copies form one commit group.
constexpr int kMotionSlots = 3;
struct MotionRing {
    float2 v[kMotionSlots][4][kMThreads];
};

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int kPending>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(kPending) : "memory"); }

// Issues the copies of plane x (x <= last plane) and commits them as a group.
__device__ __forceinline__ void issue_motion(const ThermalArgs& a, const bool (&own)[2], bool vec, int x, int yz,
                                             MotionRing& ring, int tid) {
    const int cell = x * a.ny * a.nz + yz;
    const int slot = x % kMotionSlots;
    const int fields = a.source ? 4 : 3;
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        if (d >= fields) break;
        const float* src = (d < 3 ? a.u + d * a.cells : a.source) + cell;
        float2* dst = &ring.v[slot][d][tid];
        if (vec) {
            cp_async8(dst, src);
        } else {
            if (own[0]) cp_async4(&dst->x, src);
            if (own[1]) cp_async4(&dst->y, src + 1);
        }
    }
    cp_async_commit();
}

// Cell k's velocity and clamped source from the ring (its group complete).
__device__ __forceinline__ void read_motion(const ThermalArgs& a, const MotionRing& ring, int x, int tid, int k,
                                            float (&m)[4]) {
    const int slot = x % kMotionSlots;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float2 v = ring.v[slot][d][tid];
        m[d] = k ? v.y : v.x;
    }
    if (a.source) {
        const float2 v = ring.v[slot][3][tid];
        m[3] = exact::rclamp(k ? v.y : v.x, -0.006f, 0.006f);
    } else {
        m[3] = 0.0f;
    }
}

// Staged entry i resolved for a querying cell whose own value is `self`.
template <int kKind>
__device__ __forceinline__ exact::X2 tile_at2(const float* sv, const unsigned char* sc, int i0, int i1, float self0,
                                              float self1) {
    return exact::x2(tile_at<kKind>(sv, sc, i0, self0), tile_at<kKind>(sv, sc, i1, self1));
}
// An aligned staged pair (i even) resolved lane by lane.
template <int kKind>
__device__ __forceinline__ exact::X2 tile_pair(const float* sv, const unsigned char* sc, int i, exact::X2 self) {
    const float2 v = *reinterpret_cast<const float2*>(sv + i);
    if (kKind == kTileTagged)
        return exact::x2(__float_as_uint(v.x) == kOwnTag ? self.v.x : v.x, __float_as_uint(v.y) == kOwnTag ? self.v.y : v.y);
    return tile_at2<kKind>(sv, sc, i, i + 1, self.v.x, self.v.y);
}

// First-order update of the thread's two cells (x, y, z) and (x, y, z+1)
// from the staged planes x-1, x, x+1 (ring offsets pm, p0, pp; ci the first
// cell's entry inside a plane, even), velocities and sources m0 / m1. Every
// add, subtract and multiply of the two cells is one packed FP32 operation
// (exact per lane, the reference's order); a lane whose cell is solid or off
// the brick is computed on whatever its entries hold and discarded by the
// caller. Returns the two new temperatures.
template <int kKind>
__device__ __forceinline__ float2 update_pair(const ThermalArgs& a, const float* sv, const unsigned char* sc, int pm,
                                              int p0, int pp, int ci, int x, int y, int z, const float (&m0)[4],
                                              const float (&m1)[4]) {
    using exact::X2;
    using exact::x2;
    const exact::Mul2 mul = exact::make_mul2(a.zero_bits);
    const int c = p0 + ci;
    const float2 own = *reinterpret_cast<const float2*>(sv + c);
    const X2 tc = x2(own.x, own.y);
    // x - dt u (dt = 1)
    const X2 px = x2((float)x) - x2(m0[0], m1[0]);
    const X2 py = x2((float)y) - x2(m0[1], m1[1]);
    const X2 pz = x2((float)z, (float)(z + 1)) - x2(m0[2], m1[2]);
    const int x00 = (int)floorf(px.v.x), y00 = (int)floorf(py.v.x), z00 = (int)floorf(pz.v.x);
    const int x01 = (int)floorf(px.v.y), y01 = (int)floorf(py.v.y), z01 = (int)floorf(pz.v.y);
    // every corner staged: the lower corner at offset -1 or 0 on each axis
    // (|u| < 1, and the position not rounded up to the next cell)
    const bool near0 = fabsf(m0[0]) < 1.0f && fabsf(m0[1]) < 1.0f && fabsf(m0[2]) < 1.0f &&
                       (unsigned)(x00 - x + 1) <= 1u && (unsigned)(y00 - y + 1) <= 1u && (unsigned)(z00 - z + 1) <= 1u;
    const bool near1 = fabsf(m1[0]) < 1.0f && fabsf(m1[1]) < 1.0f && fabsf(m1[2]) < 1.0f &&
                       (unsigned)(x01 - x + 1) <= 1u && (unsigned)(y01 - y + 1) <= 1u && (unsigned)(z01 - z) <= 1u;
    const X2 fx = px - x2((float)x00, (float)x01);
    const X2 fy = py - x2((float)y00, (float)y01);
    const X2 fz = pz - x2((float)z00, (float)z01);
    // corner (x0, y0, z0) of each lane (a far lane reads its own entry; its
    // sample comes from th_sample_far below)
    const int lo0 = near0 && x00 < x ? pm : p0, hi0 = near0 && x00 < x ? p0 : pp;
    const int lo1 = near1 && x01 < x ? pm : p0, hi1 = near1 && x01 < x ? p0 : pp;
    const int b0 = near0 ? ci + (y00 - y) * kPZ + (z00 - z) : ci;
    const int b1 = near1 ? ci + 1 + (y01 - y) * kPZ + (z01 - z - 1) : ci + 1;
    const X2 c000 = tile_at2<kKind>(sv, sc, lo0 + b0, lo1 + b1, own.x, own.y);
    const X2 c100 = tile_at2<kKind>(sv, sc, hi0 + b0, hi1 + b1, own.x, own.y);
    const X2 c010 = tile_at2<kKind>(sv, sc, lo0 + b0 + kPZ, lo1 + b1 + kPZ, own.x, own.y);
    const X2 c110 = tile_at2<kKind>(sv, sc, hi0 + b0 + kPZ, hi1 + b1 + kPZ, own.x, own.y);
    const X2 c001 = tile_at2<kKind>(sv, sc, lo0 + b0 + 1, lo1 + b1 + 1, own.x, own.y);
    const X2 c101 = tile_at2<kKind>(sv, sc, hi0 + b0 + 1, hi1 + b1 + 1, own.x, own.y);
    const X2 c011 = tile_at2<kKind>(sv, sc, lo0 + b0 + kPZ + 1, lo1 + b1 + kPZ + 1, own.x, own.y);
    const X2 c111 = tile_at2<kKind>(sv, sc, hi0 + b0 + kPZ + 1, hi1 + b1 + kPZ + 1, own.x, own.y);
    const X2 c00 = c000 + mul(c100 - c000, fx);
    const X2 c10 = c010 + mul(c110 - c010, fx);
    const X2 c01 = c001 + mul(c101 - c001, fx);
    const X2 c11 = c011 + mul(c111 - c011, fx);
    const X2 c0 = c00 + mul(c10 - c00, fy);
    const X2 c1 = c01 + mul(c11 - c01, fy);
    X2 adv = c0 + mul(c1 - c0, fz);
    if (!near0) adv.v.x = th_sample_far(a, px.v.x, py.v.x, pz.v.x, own.x);
    if (!near1) adv.v.y = th_sample_far(a, px.v.y, py.v.y, pz.v.y, own.y);
    // six face neighbours in the reference's order: +x, -x, +y, -y, +z, -z
    const X2 sxp = tile_pair<kKind>(sv, sc, pp + ci, tc);
    const X2 sxm = tile_pair<kKind>(sv, sc, pm + ci, tc);
    const X2 syp = tile_pair<kKind>(sv, sc, c + kPZ, tc);
    const X2 sym = tile_pair<kKind>(sv, sc, c - kPZ, tc);
    const X2 szp = x2(tile_at<kKind>(sv, sc, c + 1, own.x), tile_at<kKind>(sv, sc, c + 2, own.y));
    const X2 szm = x2(tile_at<kKind>(sv, sc, c - 1, own.x), tile_at<kKind>(sv, sc, c, own.y));
    const X2 t_sum = sxp + sxm + syp + sym + szp + szm;
    const X2 lap = t_sum - mul(x2(6.0f), tc);
    const X2 src = x2(m0[3], m1[3]);
    // adv + dt (alpha lap + s - cooling adv), dt = 1, cooling = 0
    const X2 t_next = adv + ((mul(x2(a.alpha), lap) + src) - mul(x2(0.0f), adv));
    return make_float2(exact::rclamp(t_next.v.x, -1.0f, 1.0f), exact::rclamp(t_next.v.y, -1.0f, 1.0f));
}

// Thread-constant state of a column walk.
struct ColumnThread {
    StageSlots s;
    bool own[2];   // the thread's cells lie inside the brick
    bool vec;      // both inside and 8-byte aligned (float2 velocity loads and stores)
    int y, z, yz;  // first cell's y, z and y nz + z
    int ci;        // first cell's entry inside a staged plane
    int xl;        // last plane of the column
};

// Plane x of a column: stage x+2 (fetched two planes ago) into the slot the
// last plane freed, fetch x+4 into the same registers, issue x+2's velocity
// copies, compute x from planes x-1..x+1. kTagged: no Neumann face (lookups
// test the own-value tag), else lookups read the code array.
template <bool kTagged>
__device__ __forceinline__ void column_plane(const ThermalArgs& a, const ColumnThread& t, const SourceTable& src,
                                             float* sv, unsigned char* sc, MotionRing& ring, int x, PlaneRegs& r) {
    const int tid = threadIdx.y * kMTZ + threadIdx.x;
    // x-1..x+1 staged; the slot of x+2 (last read for x-1) is free
    __syncthreads();
    if (x + 2 <= t.xl + 1) {
        float xv;
        unsigned char xc;
        const int gxe = resolve_x(a.faces, a.nx, x + 2, xv, xc);
        store_plane(t.s, src, x + 2, gxe, xv, xc, r, sv, sc, kTagged);
    }
    if (x + 4 <= t.xl + 1) {
        float xv;
        unsigned char xc;
        fetch_plane(a, t.s, src, resolve_x(a.faces, a.nx, x + 4, xv, xc), r);
    }
    // the groups of x+1 and x+2 may stay in flight; x's is complete
    if (x + 2 <= t.xl) issue_motion(a, t.own, t.vec, x + 2, t.yz, ring, tid);
    else cp_async_commit();
    cp_async_wait<2>();
    const int pm = ((x - 1) & (kRing - 1)) * kPlane, p0 = (x & (kRing - 1)) * kPlane,
              pp = ((x + 1) & (kRing - 1)) * kPlane;
    float m0[4], m1[4];
    read_motion(a, ring, x, tid, 0, m0);
    read_motion(a, ring, x, tid, 1, m1);
    float2 out = update_pair < kTagged ? kTileTagged : kTileAny > (a, sv, sc, pm, p0, pp, t.ci, x, t.y, t.z, m0, m1);
    // solid now (or off the brick): 0
    const uchar2 solid = *reinterpret_cast<const uchar2*>(sc + p0 + t.ci);
    if (solid.x || !t.own[0]) out.x = 0.0f;
    if (solid.y || !t.own[1]) out.y = 0.0f;
    const int cell = x * a.ny * a.nz + t.yz;
    if (t.vec) {
        *reinterpret_cast<float2*>(a.t_next + cell) = out;
    } else {
        if (t.own[0]) a.t_next[cell] = out.x;
        if (t.own[1]) a.t_next[cell + 1] = out.y;
    }
}

// One x-column of the transport: block (16 z-pairs) x (8 y) threads, tile
// (bx, by) in (z, y), x-planes [bz a.xchunk, bz a.xchunk + a.xchunk). Bricks
// stay below 2^31 cells (32-bit cell indices).
template <bool kTagged>
__device__ __forceinline__ void thermal_column(const ThermalArgs& a, int bx, int by, int bz) {
    __shared__ __align__(16) float sv[kRing * kPlane];
    __shared__ __align__(16) unsigned char sc[kRing * kPlane];
    __shared__ MotionRing ring;
    __shared__ SourceTable src;
    const int zb = bx * kMZ, yb = by * kMY;
    const int xf = bz * a.xchunk;
    const int tid = threadIdx.y * kMTZ + threadIdx.x;
    const bool even = a.pairs != 0;  // z-pairs start on even cells, fields aligned
    ColumnThread t;
    t.xl = min(xf + a.xchunk, a.nx) - 1;
    t.s.flags = 0;
    // the sources of this thread's staged entries (read back only by this thread)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        const int p = tid + e * kMThreads;
        const int row = p / kRowPairs, j = p - row * kRowPairs;
        const int gy = yb + row - 1, gz = zb - 2 + 2 * j;
        t.s.idx[e] = row * kPZ + 2 * j;
        t.s.off[e] = gy * a.nz + gz;
        if (p >= kPairs) continue;
        bool direct = true;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            int off;
            float v = 0.0f;
            unsigned char code = 0;
            const bool in = (unsigned)gy < (unsigned)a.ny && (unsigned)(gz + k) < (unsigned)a.nz;
            const bool load = resolve_yz(a.faces, a.ny, a.nz, gy, gz + k, off, v, code);
            src.off[t.s.idx[e] + k] = load ? off : -1 - (int)code;
            src.val[t.s.idx[e] + k] = v;
            direct = direct && in;
        }
        t.s.flags |= (1u | (even && direct ? 2u : 0u)) << (2 * e);
    }
    t.y = yb + threadIdx.y;
    t.z = zb + 2 * threadIdx.x;
    t.own[0] = t.y < a.ny && t.z < a.nz;
    t.own[1] = t.y < a.ny && t.z + 1 < a.nz;
    t.vec = even && t.own[0] && t.own[1];
    t.yz = t.y * a.nz + t.z;
    t.ci = (threadIdx.y + 1) * kPZ + 2 * threadIdx.x + 2;
    // prologue: planes xf-1, xf, xf+1 staged; xf+2 and xf+3 in registers
    {
        PlaneRegs r3[3];
        float xv[3];
        unsigned char xc[3];
        int gxe[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            gxe[i] = resolve_x(a.faces, a.nx, xf - 1 + i, xv[i], xc[i]);
            fetch_plane(a, t.s, src, gxe[i], r3[i]);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) store_plane(t.s, src, xf - 1 + i, gxe[i], xv[i], xc[i], r3[i], sv, sc, kTagged);
    }
    PlaneRegs ra, rb;
    {
        float xv;
        unsigned char xc;
        if (xf + 2 <= t.xl + 1) fetch_plane(a, t.s, src, resolve_x(a.faces, a.nx, xf + 2, xv, xc), ra);
        if (xf + 3 <= t.xl + 1) fetch_plane(a, t.s, src, resolve_x(a.faces, a.nx, xf + 3, xv, xc), rb);
    }
    issue_motion(a, t.own, t.vec, xf, t.yz, ring, tid);
    if (xf + 1 <= t.xl) issue_motion(a, t.own, t.vec, xf + 1, t.yz, ring, tid);
    else cp_async_commit();
    // one plane per iteration; the register sets rotate (ra holds plane x+2)
    for (int x = xf; x <= t.xl; ++x) {
        column_plane<kTagged>(a, t, src, sv, sc, ring, x, ra);
        const PlaneRegs r = ra;
        ra = rb;
        rb = r;
    }
    cp_async_wait<0>();  // no copy outlives the block
}

// __grid_constant__: the out-of-line helpers take the arguments by reference
// straight from the parameter space (no per-thread copy to local memory).
template <bool kTagged>
__global__ void __launch_bounds__(kMThreads, kColumnBlocksPerSM) thermal_update_kernel(const __grid_constant__ ThermalArgs a) {
    pdl_trigger();
    pdl_wait();  // launched with launch_pdl after the previous call's step
    thermal_column<kTagged>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// The transport's columns (the first `columns` blocks, numbered z-tile
// fastest; about one wave of resident blocks) and, in the remaining blocks,
// the face pre-fill of an in-place context: two independent passes in one
// launch (the fill writes ghost-layer slots from post-collision populations,
// the transport reads and writes temperature).
template <class S, bool kTagged>
__global__ void __launch_bounds__(kMThreads, kColumnBlocksPerSM) thermal_fill_kernel(const __grid_constant__ ThermalArgs a,
                                                                   typename S::T* __restrict__ f,
                                                                   const __grid_constant__ IpArgs fa, unsigned columns,
                                                                   unsigned gx, unsigned gy) {
    pdl_trigger();
    pdl_wait();  // launched with launch_pdl after the previous call's step
    const unsigned b = blockIdx.x;
    if (b < columns) {
        thermal_column<kTagged>(a, (int)(b % gx), (int)((b / gx) % gy), (int)(b / (gx * gy)));
        return;
    }
    face_fill_cell<S>(f, fa, (b - columns) * kMThreads + threadIdx.y * kMTZ + threadIdx.x);
}

__global__ void thermal_init_kernel(ThermalInitArgs a) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= a.cells) return;
    const bool solid = a.obstacle[cell] != 0;
    float t = a.t[cell];
    if (a.benchmark && fabsf(t) < 1e-8f) t = exact::rclamp(a.initial_temperature, -1.0f, 1.0f);
    else if (!solid) t = exact::rclamp(a.ref_t[cell], -1.0f, 1.0f);
    a.t[cell] = exact::rclamp(t, -1.0f, 1.0f);
    a.u[cell] = solid ? 0.0f : a.ref_ux[cell];
    a.u[a.cells + cell] = solid ? 0.0f : a.ref_uy[cell];
    a.u[2 * a.cells + cell] = solid ? 0.0f : a.ref_uz[cell];
}

}  // namespace

cudaError_t launch_thermal_init(const ThermalInitArgs& a, cudaStream_t s) {
    if (a.cells <= 0) return cudaSuccess;
    thermal_init_kernel<<<(unsigned)((a.cells + 255) / 256), 256, 0, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_thermal_reference_nudge(const ThermalNudgeArgs& a, cudaStream_t s) {
    const long long cells = (long long)a.nx * a.ny * a.nz;
    if (cells <= 0) return cudaSuccess;
    thermal_reference_nudge_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

// The column walk's launch parameters: z-pair loads and stores (8-byte float
// pairs, 2-byte mask pairs) need an even z extent and aligned fields; the
// x-chunk makes the grid one wave of resident blocks where the brick allows.
static ThermalArgs column_args(const ThermalArgs& a, unsigned tiles_yz) {
    ThermalArgs p = a;
    auto al = [](const void* q, uintptr_t n) { return (reinterpret_cast<uintptr_t>(q) & (n - 1)) == 0; };
    p.pairs = (a.nz % 2 == 0) && al(a.t, 8) && al(a.t_next, 8) && al(a.u, 8) && al(a.source, 8) && al(a.obstacle, 2);
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            sms = 148;
    }
    const unsigned slots = (unsigned)sms * kColumnBlocksPerSM;
    const unsigned chunks = max(1u, slots / max(1u, tiles_yz));
    p.xchunk = max(4, (int)((a.nx + chunks - 1) / chunks));
    p.zero_bits = 0;
    return p;
}

cudaError_t launch_thermal_update(const ThermalArgs& a, cudaStream_t s) {
    if (a.cells <= 0) return cudaSuccess;
    if (a.cells >= (1LL << 31)) return cudaErrorInvalidValue;  // 32-bit cell indices
    if (a.bfecc) {
        const int block = a.nz >= 128 ? 128 : ((a.nz + 31) / 32) * 32;
        const dim3 grid((unsigned)((a.nz + block - 1) / block), (unsigned)a.ny, (unsigned)a.nx);
        bfecc_forward_kernel<<<grid, block, 0, s>>>(a);
        count_launch();
        bfecc_correct_kernel<<<grid, block, 0, s>>>(a);
        count_launch();
        bfecc_final_kernel<<<grid, block, 0, s>>>(a);
        count_launch();
        return cudaGetLastError();
    }
    const unsigned gx = (unsigned)((a.nz + kMZ - 1) / kMZ), gy = (unsigned)((a.ny + kMY - 1) / kMY);
    const ThermalArgs ap = column_args(a, gx * gy);
    const dim3 grid(gx, gy, (unsigned)((a.nx + ap.xchunk - 1) / ap.xchunk));
    const cudaError_t e = no_neumann(a.faces) ? launch_pdl(thermal_update_kernel<true>, grid, dim3(kMTZ, kMY), 0, s, ap)
                                              : launch_pdl(thermal_update_kernel<false>, grid, dim3(kMTZ, kMY), 0, s, ap);
    count_launch();
    return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_thermal_update_fill(const ThermalArgs& a, int storage, void* f, const IpArgs& fill, cudaStream_t s) {
    if (a.bfecc || a.cells <= 0 || a.cells >= (1LL << 31)) return cudaErrorInvalidValue;
    const unsigned gx = (unsigned)((a.nz + kMZ - 1) / kMZ), gy = (unsigned)((a.ny + kMY - 1) / kMY);
    const ThermalArgs ap = column_args(a, gx * gy);
    const unsigned columns = gx * gy * (unsigned)((a.nx + ap.xchunk - 1) / ap.xchunk);
    const unsigned fill_blocks = (unsigned)((face_fill_count(fill.g, fill.fill_faces) + kMThreads - 1) / kMThreads);
    const dim3 block(kMTZ, kMY), grid(fill_blocks + columns);
    const bool tagged = no_neumann(a.faces);
#define AERO_THERMAL_FILL(S, T)                                                                                    \
    (tagged ? launch_pdl(thermal_fill_kernel<S, true>, grid, block, 0, s, ap, static_cast<T*>(f), fill, columns, gx, gy) \
            : launch_pdl(thermal_fill_kernel<S, false>, grid, block, 0, s, ap, static_cast<T*>(f), fill, columns, gx, gy))
    cudaError_t e;
    if (storage == 1) e = AERO_THERMAL_FILL(StoreF16Dev, __half);
    else if (storage == 2) e = AERO_THERMAL_FILL(StoreI16Dev, short);
    else e = AERO_THERMAL_FILL(StoreF32, float);
#undef AERO_THERMAL_FILL
    if (e != cudaSuccess) return e;
    count_launch();
    return cudaGetLastError();
}

}  // namespace aero
