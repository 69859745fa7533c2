// Temperature transport kernels (see thermal.cuh). Built with --fmad=false:
// every product and sum rounds separately, in the reference's order.
#include "thermal.cuh"

#include "collide27_exact.cuh"

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
    const float c000 = th_neighbour(a, field, x0, y0, z0, fallback);
    const float c100 = th_neighbour(a, field, x1, y0, z0, fallback);
    const float c010 = th_neighbour(a, field, x0, y1, z0, fallback);
    const float c110 = th_neighbour(a, field, x1, y1, z0, fallback);
    const float c001 = th_neighbour(a, field, x0, y0, z1, fallback);
    const float c101 = th_neighbour(a, field, x1, y0, z1, fallback);
    const float c011 = th_neighbour(a, field, x0, y1, z1, fallback);
    const float c111 = th_neighbour(a, field, x1, y1, z1, fallback);
    const float c00 = c000 + (c100 - c000) * fx;
    const float c10 = c010 + (c110 - c010) * fx;
    const float c01 = c001 + (c101 - c001) * fx;
    const float c11 = c011 + (c111 - c011) * fx;
    const float c0 = c00 + (c10 - c00) * fy;
    const float c1 = c01 + (c11 - c01) * fy;
    return c0 + (c1 - c0) * fz;
}

// The update reads the 3x3x3 neighbourhood of each cell (|u| < 1 keeps every
// trilinear corner inside it). A block stages its tile plus a one-cell halo
// in shared memory, each entry already resolved by th_neighbour's rules:
// code 0 = use the value (a fluid cell's temperature, or a Dirichlet face's
// clamped temperature), 1 = the querying cell's own value (solid cell,
// adiabatic / disabled / inherit face), 2 = own value + the stored Neumann
// flux, clamped. Periodic faces are resolved by staging the wrapped cell.
// Lookups specialise on what the tile holds (block-uniform): only code 0
// (most of the air above a terrain), codes 0 and 1, or any code.
constexpr int kTZ = 32, kTY = 8, kTX = 4;  // cells per block: z x y x x
constexpr int kSY = kTZ + 2, kSX = (kTY + 2) * (kTZ + 2), kTile = (kTX + 2) * kSX;

// kTileTagged: codes 0 and 1 only, code 1 entries hold kOwnTag (bricks
// without a Neumann face; the code array is not read).
enum TileKind { kTileClean = 0, kTileTagged = 1, kTileAny = 2 };

template <int kKind>
__device__ __forceinline__ float tile_at(const float* sv, const unsigned char* sc, int i, float self) {
    const float v = sv[i];
    if (kKind == kTileClean) return v;
    if (kKind == kTileTagged) return __float_as_uint(v) == kOwnTag ? self : v;
    const int c = sc[i];
    return c == 0 ? v : (c == 1 ? self : exact::rclamp(self + v, -1.0f, 1.0f));
}

// One staged entry outside the brick: th_neighbour's rules without the
// querying cell's value (rare path).
__device__ __noinline__ void stage_outside(const ThermalFaces* F, const float* t, const uint8_t* obstacle, int nx, int ny,
                                           int nz, int x, int y, int z, float* v, unsigned char* code) {
    if ((x < 0 || x >= nx) && F->kind[x < 0 ? 0 : 1] == kThermalPeriodic) {
        x %= nx;
        if (x < 0) x += nx;
    }
    if ((y < 0 || y >= ny) && F->kind[y < 0 ? 2 : 3] == kThermalPeriodic) {
        y %= ny;
        if (y < 0) y += ny;
    }
    if ((z < 0 || z >= nz) && F->kind[z < 0 ? 4 : 5] == kThermalPeriodic) {
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
    *v = 0.0f;
    if (face >= 0) {
        const int kind = F->kind[face];
        if (kind == kThermalDirichlet) {
            *code = 0;
            *v = exact::rclamp(F->temperature[face], -1.0f, 1.0f);
        } else if (kind == kThermalNeumann) {
            *code = 2;
            *v = F->heat_flux[face];
        } else {
            *code = 1;
        }
        return;
    }
    const int cell = (x * ny + y) * nz + z;
    *code = obstacle[cell] ? 1 : 0;
    if (!*code) *v = __ldg(t + cell);
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
__global__ void __launch_bounds__(128) bfecc_forward_kernel(ThermalArgs a) {
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
__global__ void __launch_bounds__(128) bfecc_correct_kernel(ThermalArgs a) {
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
__global__ void __launch_bounds__(128) bfecc_final_kernel(ThermalArgs a) {
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
    const float n0 = th_neighbour(a, x + 1, y, z, tc), n1 = th_neighbour(a, x - 1, y, z, tc);
    const float n2 = th_neighbour(a, x, y + 1, z, tc), n3 = th_neighbour(a, x, y - 1, z, tc);
    const float n4 = th_neighbour(a, x, y, z + 1, tc), n5 = th_neighbour(a, x, y, z - 1, tc);
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

template <int kKind>
__device__ __forceinline__ void update_cell(const ThermalArgs& a, const float* sv, const unsigned char* sc, int c, int x,
                                            int y, int z, int cell, const float (&uv)[3], float src) {
    const float dt = 1.0f, cooling = 0.0f;
    const float tc = sv[c];
    const float ux = uv[0], uy = uv[1], uz = uv[2];
    const float px = (float)x - dt * ux, py = (float)y - dt * uy, pz = (float)z - dt * uz;
    float adv;
    if (fabsf(ux) < 1.0f && fabsf(uy) < 1.0f && fabsf(uz) < 1.0f) {
        const int x0 = (int)floorf(px), y0 = (int)floorf(py), z0 = (int)floorf(pz);
        const float fx = px - (float)x0, fy = py - (float)y0, fz = pz - (float)z0;
        const int b = c + (x0 - x) * kSX + (y0 - y) * kSY + (z0 - z);  // corner (x0, y0, z0)
        const float c000 = tile_at<kKind>(sv, sc, b, tc);
        const float c100 = tile_at<kKind>(sv, sc, b + kSX, tc);
        const float c010 = tile_at<kKind>(sv, sc, b + kSY, tc);
        const float c110 = tile_at<kKind>(sv, sc, b + kSX + kSY, tc);
        const float c001 = tile_at<kKind>(sv, sc, b + 1, tc);
        const float c101 = tile_at<kKind>(sv, sc, b + kSX + 1, tc);
        const float c011 = tile_at<kKind>(sv, sc, b + kSY + 1, tc);
        const float c111 = tile_at<kKind>(sv, sc, b + kSX + kSY + 1, tc);
        const float c00 = c000 + (c100 - c000) * fx;
        const float c10 = c010 + (c110 - c010) * fx;
        const float c01 = c001 + (c101 - c001) * fx;
        const float c11 = c011 + (c111 - c011) * fx;
        const float c0 = c00 + (c10 - c00) * fy;
        const float c1 = c01 + (c11 - c01) * fy;
        adv = c0 + (c1 - c0) * fz;
    } else {
        adv = th_sample_far(a, px, py, pz, tc);
    }
    const float t_sum = tile_at<kKind>(sv, sc, c + kSX, tc) + tile_at<kKind>(sv, sc, c - kSX, tc) +
                        tile_at<kKind>(sv, sc, c + kSY, tc) + tile_at<kKind>(sv, sc, c - kSY, tc) +
                        tile_at<kKind>(sv, sc, c + 1, tc) + tile_at<kKind>(sv, sc, c - 1, tc);
    const float lap = t_sum - 6.0f * tc;
    const float t_next = adv + dt * (a.alpha * lap + src - cooling * adv);
    a.t_next[cell] = exact::rclamp(t_next, -1.0f, 1.0f);
}

// Block = (32 z) x (8 y) threads over a kTX x kTY x kTZ tile: each thread
// updates the kTX cells of its (y, z) column. Loads are grouped so that many
// are in flight at once (the kernel is latency-bound). Bricks stay below 2^31
// cells (32-bit cell indices).
__global__ void __launch_bounds__(kTZ * kTY, 4) thermal_update_kernel(ThermalArgs a) {
    __shared__ float sv[kTile];
    __shared__ unsigned char sc[kTile];
    const int zb = blockIdx.x * kTZ, yb = blockIdx.y * kTY, xb = blockIdx.z * kTX;
    const int tid = threadIdx.y * kTZ + threadIdx.x;
    const bool tagged = no_neumann(a.faces);
    // the cells' own velocity and source first: their loads overlap the
    // staging loads instead of following the barrier
    const int z = zb + threadIdx.x, y = yb + threadIdx.y;
    const bool yz_own = y < a.ny && z < a.nz;
    float u[kTX][3], src[kTX];
#pragma unroll
    for (int k = 0; k < kTX; ++k) {
        const int x = xb + k;
        const int cell = (x * a.ny + y) * a.nz + z;
        const bool in = yz_own && x < a.nx;
        u[k][0] = in ? __ldg(a.u + cell) : 0.0f;
        u[k][1] = in ? __ldg(a.u + a.cells + cell) : 0.0f;
        u[k][2] = in ? __ldg(a.u + 2 * a.cells + cell) : 0.0f;
        src[k] = (in && a.source) ? exact::rclamp(__ldg(a.source + cell), -0.006f, 0.006f) : 0.0f;
    }
    int seen = 0;  // bit c: some entry has code c
    // columns (iy, iz) of the halo tile, all kTX + 2 x-planes each
    for (int col = tid; col < kSX; col += kTZ * kTY) {
        const int iy = col / kSY, iz = col - iy * kSY;
        const int gy = yb + iy - 1, gz = zb + iz - 1;
        const bool yz_in = (unsigned)gy < (unsigned)a.ny && (unsigned)gz < (unsigned)a.nz;
        float tv[kTX + 2];
        unsigned char ob[kTX + 2];
#pragma unroll
        for (int ix = 0; ix < kTX + 2; ++ix) {
            const int gx = xb + ix - 1;
            tv[ix] = 0.0f;
            ob[ix] = 0;
            if (yz_in && (unsigned)gx < (unsigned)a.nx) {
                const int cell = (gx * a.ny + gy) * a.nz + gz;
                ob[ix] = __ldg(a.obstacle + cell);
                tv[ix] = __ldg(a.t + cell);
            }
        }
#pragma unroll
        for (int ix = 0; ix < kTX + 2; ++ix) {
            const int gx = xb + ix - 1;
            const int i = ix * kSX + col;
            if (yz_in && (unsigned)gx < (unsigned)a.nx) {
                const unsigned char code = ob[ix] ? 1 : 0;
                sv[i] = code ? (tagged ? __uint_as_float(kOwnTag) : 0.0f) : tv[ix];
                sc[i] = code;
                seen |= 1 << code;
            } else {
                stage_outside(&a.faces, a.t, a.obstacle, a.nx, a.ny, a.nz, gx, gy, gz, &sv[i], &sc[i]);
                if (tagged && sc[i] == 1) sv[i] = __uint_as_float(kOwnTag);
                seen |= 1 << sc[i];
            }
        }
    }
    const int any_neumann = __syncthreads_or(seen & 4);
    const int any_self = __syncthreads_or(seen & 2);
    if (!yz_own) return;
#pragma unroll
    for (int k = 0; k < kTX; ++k) {
        const int x = xb + k;
        if (x >= a.nx) break;
        const int cell = (x * a.ny + y) * a.nz + z;
        const int c = (k + 1) * kSX + (threadIdx.y + 1) * kSY + threadIdx.x + 1;
        if (sc[c] != 0) {  // solid now
            a.t_next[cell] = 0.0f;
            continue;
        }
        if (!any_neumann && !any_self) update_cell<kTileClean>(a, sv, sc, c, x, y, z, cell, u[k], src[k]);
        else if (tagged) update_cell<kTileTagged>(a, sv, sc, c, x, y, z, cell, u[k], src[k]);
        else update_cell<kTileAny>(a, sv, sc, c, x, y, z, cell, u[k], src[k]);
    }
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
    const dim3 grid((unsigned)((a.nz + kTZ - 1) / kTZ), (unsigned)((a.ny + kTY - 1) / kTY), (unsigned)((a.nx + kTX - 1) / kTX));
    thermal_update_kernel<<<grid, dim3(kTZ, kTY), 0, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace aero
