// FP32 D3Q27 brick step kernels: packet ingest, pull classification,
// fused pull-stream + cumulant collide (two-buffer), macro output.
//
// State convention: a buffer g holds post-collision populations. The
// reference's call order is collide -> stream -> output
// (native/src/aero_lbm_jni.cpp:8480-8507); here one launch performs
// pull-stream (of the previous call's post-collision state, with that call's
// mask and faces) and then collide (with this call's inputs), so every call is
// one fused pass and the output pass reads S(g) with this call's faces.
#include <atomic>
#include <vector>

#include "d3q27_step.cuh"

namespace aero {

namespace {
std::atomic<uint64_t> g_launches{0};
}
uint64_t kernel_launch_count() { return g_launches.load(); }
void count_launch() { g_launches.fetch_add(1); }

namespace {
struct StepTimer {
    bool on = false;
    std::vector<cudaEvent_t> pool;  // begin/end pairs, reused across resets
    size_t used = 0;
};
StepTimer g_timer;
cudaEvent_t timer_event() {
    if (g_timer.used == g_timer.pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        g_timer.pool.push_back(e);
    }
    return g_timer.pool[g_timer.used++];
}
}  // namespace

void step_timer_begin(cudaStream_t s) {
    if (!g_timer.on) return;
    if (cudaEvent_t e = timer_event()) cudaEventRecord(e, s);
}
void step_timer_end(cudaStream_t s) {
    if (!g_timer.on) return;
    if (cudaEvent_t e = timer_event()) cudaEventRecord(e, s);
}
void step_timer_reset(bool on) {
    g_timer.on = on;
    g_timer.used = 0;
}
// Sum of the recorded begin/end intervals (waits for the last event).
bool step_timer_read(double* total_ms, int* launches) {
    double t = 0.0;
    const size_t pairs = g_timer.used / 2;
    if (pairs && cudaEventSynchronize(g_timer.pool[2 * pairs - 1]) != cudaSuccess) return false;
    for (size_t i = 0; i < pairs; ++i) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, g_timer.pool[2 * i], g_timer.pool[2 * i + 1]) != cudaSuccess) return false;
        t += ms;
    }
    *total_ms = t;
    *launches = (int)pairs;
    return true;
}

// ---------------------------------------------------------------- ingest
// Packet semantics of ingest_payload (native/src/aero_lbm_jni.cpp:1671-1694),
// per cell in ingest_cell (d3q27_kernels.cuh).
__global__ void ingest_packet_kernel(const float* __restrict__ packet, int in_ch, long long cells, CellFields out) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    ingest_cell(packet + cell * in_ch, in_ch, cell, out);
}

cudaError_t launch_ingest_packet(const float* packet, int in_channels, BrickDims d, CellFields out, cudaStream_t stream) {
    if (d.cells <= 0) return cudaSuccess;
    const int block = 256;
    const long long grid = (d.cells + block - 1) / block;
    ingest_packet_kernel<<<(unsigned)grid, block, 0, stream>>>(packet, in_channels, d.cells, out);
    count_launch();
    return cudaGetLastError();
}

// Largest reference speed over fluid cells (the per-brick 16-bit storage
// scale of a context whose first inputs were built on the device). Non-
// negative floats order like their bit patterns, so an integer max suffices.
__global__ void max_fluid_speed_kernel(CellFields f, long long cells, unsigned int* out_bits) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float s = 0.0f;
    if (cell < cells && f.obstacle[cell] == 0) {
        const float ux = f.ref_ux[cell], uy = f.ref_uy[cell], uz = f.ref_uz[cell];
        const float s2 = ux * ux + uy * uy + uz * uz;
        if (isfinite(s2)) s = sqrtf(s2);
    }
    for (int o = 16; o > 0; o >>= 1) s = fmaxf(s, __shfl_xor_sync(0xffffffffu, s, o));
    if ((threadIdx.x & 31) == 0 && s > 0.0f) atomicMax(out_bits, __float_as_uint(s));
}

cudaError_t launch_max_fluid_speed(CellFields f, long long cells, unsigned int* out_bits, cudaStream_t stream) {
    if (cells <= 0) return cudaSuccess;
    const int block = 256;
    const long long grid = (cells + block - 1) / block;
    max_fluid_speed_kernel<<<(unsigned)grid, block, 0, stream>>>(f, cells, out_bits);
    count_launch();
    return cudaGetLastError();
}

// Pull classification (see lattice.cuh for the bit layout). Mirrors the
// branch structure of stream_and_bounce (jni.cpp:2415-2452) and
// benchmark_hydrodynamic_boundary_value (jni.cpp:1563-1602). A block stages
// its 32 x 4 x 2 cells' mask with a one-cell halo in shared memory (periodic
// sides wrapped while staging, 2 = outside a non-periodic face), so the 27
// neighbour tests of a cell read shared memory instead of issuing 27
// dependent global loads.
constexpr int kFlagTz = 32, kFlagTy = 4, kFlagTx = 2;
__global__ void __launch_bounds__(kFlagTz * kFlagTy * kFlagTx) build_flags_kernel(
    const uint8_t* __restrict__ obstacle, int nx, int ny, int nz, FaceParams F, uint32_t* __restrict__ flags) {
    constexpr int SZ = kFlagTz + 2, SY = kFlagTy + 2, SX = kFlagTx + 2;
    __shared__ uint8_t tile[SX * SY * SZ];
    const int z0 = blockIdx.x * kFlagTz, y0 = blockIdx.y * kFlagTy, x0 = blockIdx.z * kFlagTx;
    const int tid = (threadIdx.z * kFlagTy + threadIdx.y) * kFlagTz + threadIdx.x;
    for (int i = tid; i < SX * SY * SZ; i += kFlagTz * kFlagTy * kFlagTx) {
        const int tz = i % SZ, ty = (i / SZ) % SY, tx = i / (SZ * SY);
        int gx = x0 + tx - 1, gy = y0 + ty - 1, gz = z0 + tz - 1;
        uint8_t v = 2;
        if (wrap_coord(gx, nx, F.wrap_lo[0], F.wrap_hi[0]) && wrap_coord(gy, ny, F.wrap_lo[1], F.wrap_hi[1]) &&
            wrap_coord(gz, nz, F.wrap_lo[2], F.wrap_hi[2]))
            v = obstacle[((long long)gx * ny + gy) * nz + gz] ? 1 : 0;
        tile[i] = v;
    }
    __syncthreads();
    const int x = x0 + threadIdx.z, y = y0 + threadIdx.y, z = z0 + threadIdx.x;
    if (x >= nx || y >= ny || z >= nz) return;
    const long long cell = ((long long)x * ny + y) * nz + z;
    const int own = ((threadIdx.z + 1) * SY + threadIdx.y + 1) * SZ + threadIdx.x + 1;
    uint32_t w = 0;
    if (tile[own] == 1) {
        w = kFlagSelfSolid;
    } else {
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            const uint8_t v = tile[own - (q_cx(q) * SY + q_cy(q)) * SZ - q_cz(q)];
            if (v == 1) {
                w |= 1u << q;
            } else if (v == 2) {
                // the first axis outside a non-periodic face picks the face (oob_face)
                const int sx = x - q_cx(q), sy = y - q_cy(q), sz = z - q_cz(q);
                int face;
                if ((sx < 0 && !F.wrap_lo[0]) || (sx >= nx && !F.wrap_hi[0])) face = sx < 0 ? kFaceXMin : kFaceXMax;
                else if ((sy < 0 && !F.wrap_lo[1]) || (sy >= ny && !F.wrap_hi[1])) face = sy < 0 ? kFaceYMin : kFaceYMax;
                else face = sz < 0 ? kFaceZMin : kFaceZMax;
                const int kind = F.kind[face];
                if (kind == kHydroBounceBack || (kind == kHydroInheritGame && F.disable_convective)) w |= 1u << q;
                else w |= kFlagFaceSpecial;
            }
        }
    }
    flags[cell] = w;
}

cudaError_t launch_build_flags(const uint8_t* obstacle, BrickDims d, FaceParams face, uint32_t* flags, cudaStream_t stream) {
    if (d.cells <= 0) return cudaSuccess;
    const dim3 block(kFlagTz, kFlagTy, kFlagTx);
    const dim3 grid((unsigned)((d.nz + kFlagTz - 1) / kFlagTz), (unsigned)((d.ny + kFlagTy - 1) / kFlagTy),
                    (unsigned)((d.nx + kFlagTx - 1) / kFlagTx));
    build_flags_kernel<<<grid, block, 0, stream>>>(obstacle, d.nx, d.ny, d.nz, face, flags);
    count_launch();
    return cudaGetLastError();
}

}  // namespace aero
