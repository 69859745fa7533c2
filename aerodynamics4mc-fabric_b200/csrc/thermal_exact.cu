// Temperature transport kernels (see thermal.cuh). Built with --fmad=false:
// every product and sum rounds separately, in the reference's order.
#include "thermal.cuh"

#include "collide27_exact.cuh"

namespace aero {
namespace {

// thermal_field_neighbor_or_self (jni.cpp:1800-1825) with remap_thermal_coords
// (jni.cpp:738-749, 779-785) and thermal_face_for_oob (jni.cpp:761-769).
__device__ __forceinline__ float th_neighbour(const ThermalArgs& a, int x, int y, int z, float self) {
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
    if (a.obstacle[cell]) return self;
    return a.t[cell];
}

// sample_temperature_trilinear_field (jni.cpp:1910-1945).
__device__ __forceinline__ float th_sample(const ThermalArgs& a, float x, float y, float z, float fallback) {
    const int x0 = (int)floorf(x), y0 = (int)floorf(y), z0 = (int)floorf(z);
    const int x1 = x0 + 1, y1 = y0 + 1, z1 = z0 + 1;
    const float fx = x - (float)x0, fy = y - (float)y0, fz = z - (float)z0;
    const float c000 = th_neighbour(a, x0, y0, z0, fallback);
    const float c100 = th_neighbour(a, x1, y0, z0, fallback);
    const float c010 = th_neighbour(a, x0, y1, z0, fallback);
    const float c110 = th_neighbour(a, x1, y1, z0, fallback);
    const float c001 = th_neighbour(a, x0, y0, z1, fallback);
    const float c101 = th_neighbour(a, x1, y0, z1, fallback);
    const float c011 = th_neighbour(a, x0, y1, z1, fallback);
    const float c111 = th_neighbour(a, x1, y1, z1, fallback);
    const float c00 = c000 + (c100 - c000) * fx;
    const float c10 = c010 + (c110 - c010) * fx;
    const float c01 = c001 + (c101 - c001) * fx;
    const float c11 = c011 + (c111 - c011) * fx;
    const float c0 = c00 + (c10 - c00) * fy;
    const float c1 = c01 + (c11 - c01) * fy;
    return c0 + (c1 - c0) * fz;
}

// One thread per cell on a line grid (z along the block).
__global__ void __launch_bounds__(128) thermal_update_kernel(ThermalArgs a) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= a.nz) return;
    const int y = blockIdx.y, x = blockIdx.z;
    const long long cell = ((long long)x * a.ny + y) * a.nz + z;
    if (a.obstacle[cell]) {
        a.t_next[cell] = 0.0f;
        return;
    }
    const float dt = 1.0f, cooling = 0.0f;
    const float tc = a.t[cell];
    const float ux = a.u[cell], uy = a.u[a.cells + cell], uz = a.u[2 * a.cells + cell];
    const float adv = th_sample(a, (float)x - dt * ux, (float)y - dt * uy, (float)z - dt * uz, tc);
    const float t_sum = th_neighbour(a, x + 1, y, z, tc) + th_neighbour(a, x - 1, y, z, tc) +
                        th_neighbour(a, x, y + 1, z, tc) + th_neighbour(a, x, y - 1, z, tc) +
                        th_neighbour(a, x, y, z + 1, tc) + th_neighbour(a, x, y, z - 1, tc);
    const float lap = t_sum - 6.0f * tc;
    const float src = a.source ? exact::rclamp(a.source[cell], -0.006f, 0.006f) : 0.0f;
    const float t_next = adv + dt * (a.alpha * lap + src - cooling * adv);
    a.t_next[cell] = exact::rclamp(t_next, -1.0f, 1.0f);
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

cudaError_t launch_thermal_update(const ThermalArgs& a, cudaStream_t s) {
    if (a.cells <= 0) return cudaSuccess;
    const int block = a.nz >= 128 ? 128 : ((a.nz + 31) / 32) * 32;
    const dim3 grid((unsigned)((a.nz + block - 1) / block), (unsigned)a.ny, (unsigned)a.nx);
    thermal_update_kernel<<<grid, block, 0, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace aero
