// Kernels of the device-resident brick-world service. Built with
// --fmad=false: the thermal source and the atlas quantisation are plain
// float products and quotients that must round like the reference's host
// loops (native/src/aero_lbm_simulation_bridge.cpp).
#include "brick_world.cuh"

namespace aero {
namespace bw {

namespace {

constexpr int kBlock = 256;

// decode_client_fan_surface_kind (simulation_bridge.cpp:524-537): surface
// kinds 32..37 blow along -x, +x, -y, +y, -z, +z at 4 m/s.
__device__ __forceinline__ bool decode_fan(uint8_t kind, float& vx, float& vy, float& vz) {
    vx = vy = vz = 0.0f;
    if (kind < 32 || kind > 37) return false;
    const float v = (kind & 1) ? 4.0f : -4.0f;
    const int axis = (kind - 32) >> 1;
    if (axis == 0) vx = v;
    else if (axis == 1) vy = v;
    else vz = v;
    return true;
}

// Flag bits of the warp's cells or-ed together: one atomic per warp.
__device__ __forceinline__ void or_flag(int* flag, int bits) {
    bits = (int)__reduce_or_sync(0xffffffffu, (unsigned)bits);
    if (flag && bits && (threadIdx.x & 31) == 0) atomicOr(flag, bits);
}

__device__ __forceinline__ bool flow_nonzero(const float* f) {
    return fabsf(f[0]) > 1.0e-8f || fabsf(f[1]) > 1.0e-8f || fabsf(f[2]) > 1.0e-8f;
}

// quantize_signed (simulation_bridge.cpp:3122-3128): round-half-away of the
// clamped ratio times 32767; non-finite values publish 0.
__device__ __forceinline__ int16_t quantize(float v, float range) {
    if (!isfinite(v)) return 0;
    float r = __fdiv_rn(v, range);
    r = r < -1.0f ? -1.0f : (1.0f < r ? 1.0f : r);
    return (int16_t)lroundf(__fmul_rn(r, 32767.0f));
}

__global__ void __launch_bounds__(kBlock) fill_kernel(FillArgs a, CellFields out) {
    const long long n = a.n;
    const long long cells = n * n * n;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    float p[kPacketChannels];
#pragma unroll
    for (int c = 0; c < kPacketChannels; ++c) p[c] = 0.0f;
    const bool obstacle = a.st.obstacle[cell] != 0;
    p[kChObstacle] = obstacle ? 1.0f : 0.0f;
    if (!obstacle) {
        float fx, fy, fz;
        if (decode_fan(a.st.surface_kind[cell], fx, fy, fz)) {
            p[1] = 1.0f;
            p[2] = fx;
            p[3] = fy;
            p[4] = fz;
        }
        const int x = (int)(cell / (n * n)), y = (int)((cell / n) % n), z = (int)(cell % n);
        const int L = a.ref_layers;
        const int e = a.ref_flow ? a.exposed : 0;
        const bool use_ref = ((e & 1) && x < L) || ((e & 2) && x >= a.n - L) || ((e & 4) && y < L) ||
                             ((e & 8) && y >= a.n - L) || ((e & 16) && z < L) || ((e & 32) && z >= a.n - L);
        const float* f = (use_ref ? a.ref_flow : a.flow) + cell * kFlowChannels;
        p[kChStateVx] = f[0];
        p[kChStateVy] = f[1];
        p[kChStateVz] = f[2];
        p[kChStateP] = f[3];
        p[kChStateTemp] = (use_ref ? a.ref_air : a.air)[cell];
        const float w = a.st.emitter_power[cell];
        if (w > 0.0f) {
            // temperature_source_from_power_watts (simulation_bridge.cpp:3152-3158)
            const float s = __fdiv_rn(__fmul_rn(w, 0.05f), a.source_denominator);
            p[kChThermalSource] = s < -0.006f ? -0.006f : (0.006f < s ? 0.006f : s);
        }
    }
    ingest_cell(p, kPacketChannels, cell, out);
}

__global__ void __launch_bounds__(kBlock) sync_kernel(SyncArgs a) {
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int bits = 0;
    if (cell < a.cells) {
        float* f = a.flow + cell * kFlowChannels;
        if (a.temperature) a.air[cell] = a.temperature[cell];
        if (a.surface_src && a.surface_src != a.surface) a.surface[cell] = a.surface_src[cell];
        if (flow_nonzero(f)) bits |= kFlagBefore;
        if (a.st.obstacle) {
            if (a.st.obstacle[cell] != 0) {
                f[0] = f[1] = f[2] = f[3] = 0.0f;
                a.air[cell] = 0.0f;
                a.surface[cell] = 0.0f;
            } else if (a.st.open_face_mask[cell] == 0 && a.st.surface_kind[cell] == 0 && !(a.st.emitter_power[cell] > 0.0f)) {
                a.surface[cell] = 0.0f;
            }
        }
        if (flow_nonzero(f)) bits |= kFlagAfter;
    }
    or_flag(a.flag, bits);
}

__global__ void __launch_bounds__(kBlock) publish_kernel(PublishArgs a) {
    const long long res = a.res;
    const long long samples = res * res * res;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= samples) return;
    long long src = i;
    if (a.dense_n > 0) {
        const long long n = a.dense_n;
        const int ax = (int)(i / (res * res)), ay = (int)((i / res) % res), az = (int)(i % res);
        const long long gx = min((long long)n - 1, (long long)ax * a.stride);
        const long long gy = min((long long)n - 1, (long long)ay * a.stride);
        const long long gz = min((long long)n - 1, (long long)az * a.stride);
        src = (gx * n + gy) * n + gz;
    }
    const float* f = a.src + src * kFlowChannels;
    short4 q;
    q.x = quantize(__fmul_rn(f[0], a.velocity_scale), kAtlasVelocityRange);
    q.y = quantize(__fmul_rn(f[1], a.velocity_scale), kAtlasVelocityRange);
    q.z = quantize(__fmul_rn(f[2], a.velocity_scale), kAtlasVelocityRange);
    q.w = quantize(f[3], kAtlasPressureRange);
    reinterpret_cast<short4*>(a.out)[i] = q;
}

unsigned blocks_for(long long count) { return (unsigned)((count + kBlock - 1) / kBlock); }

}  // namespace

cudaError_t launch_fill(const FillArgs& a, const CellFields& out, cudaStream_t s) {
    const long long cells = (long long)a.n * a.n * a.n;
    if (cells <= 0) return cudaSuccess;
    fill_kernel<<<blocks_for(cells), kBlock, 0, s>>>(a, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_sync(const SyncArgs& a, cudaStream_t s) {
    if (a.cells <= 0) return cudaSuccess;
    sync_kernel<<<blocks_for(a.cells), kBlock, 0, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_publish(const PublishArgs& a, cudaStream_t s) {
    const long long samples = (long long)a.res * a.res * a.res;
    if (samples <= 0) return cudaSuccess;
    publish_kernel<<<blocks_for(samples), kBlock, 0, s>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace bw
}  // namespace aero
