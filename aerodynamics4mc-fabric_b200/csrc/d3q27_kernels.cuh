// Kernel interface of the FP32 D3Q27 brick step (device buffers only).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "collide27.cuh"

namespace aero {

// Face configuration the pull of one step uses (a snapshot: the pull of call
// n+1 streams with the faces of call n, as the reference streams at the end of
// call n).
struct FaceParams {
    int kind[6];            // HydroKind per face (x-, x+, y-, y+, z-, z+)
    float velocity[6][3];   // Dirichlet / moving-wall velocity (lattice units)
    float pressure[6];      // pressure-Dirichlet proxy (rho - 1)
    int periodic_mask;      // bit a: axis a wraps (both faces periodic on that side)
    int wrap_lo[3];         // per axis: the min face wraps
    int wrap_hi[3];         // per axis: the max face wraps
    int disable_convective; // INHERIT_GAME faces use bounce-back instead of convective outflow
    float max_speed;
    int cylinder_inlet;     // cylinder preset: the x- velocity face blows the parabolic profile
};

// cylinder_benchmark_inlet_ux (jni.cpp:214-220): 4 u_max s (1 - s) across the
// channel, s = y / max(1, ny - 1); applied to velocity and moving-wall
// sources beyond x- under the cylinder preset (jni.cpp:1536-1545). Rounded
// operation by operation, as the reference evaluates it.
__host__ __device__ inline float cylinder_inlet_ux(int ny, int y, float u_max) {
    const float height = (float)(ny - 1 > 1 ? ny - 1 : 1);
#ifdef __CUDA_ARCH__
    const float denom = fmaxf(__fsub_rn(height, 0.0f), 1.0e-6f);
    const float s = __fdiv_rn(__fsub_rn((float)y, 0.0f), denom);
    if (s < 0.0f || s > 1.0f) return 0.0f;
    return __fmul_rn(__fmul_rn(__fmul_rn(4.0f, u_max), s), __fsub_rn(1.0f, s));
#else
    const float denom = height - 0.0f > 1.0e-6f ? height - 0.0f : 1.0e-6f;
    const float s = ((float)y - 0.0f) / denom;
    if (s < 0.0f || s > 1.0f) return 0.0f;
    return 4.0f * u_max * s * (1.0f - s);
#endif
}

struct BrickDims {
    int nx, ny, nz;
    int pad;
    long long cells;
};

// Input channels of the reference packet (native/src/aero_lbm_jni.cpp:64-81).
constexpr int kChObstacle = 0;
constexpr int kChFanMask = 1;
constexpr int kChFanVx = 2;
constexpr int kChStateVx = 5;
constexpr int kChStateVy = 6;
constexpr int kChStateVz = 7;
constexpr int kChStateP = 8;
constexpr int kChThermalSource = 9;
constexpr int kChStateTemp = 10;

struct CellFields {
    uint8_t* obstacle;    // 1 = solid
    float* ref_ux;
    float* ref_uy;
    float* ref_uz;
    float* ref_p;         // clamped pressure proxy
    float* temperature;   // temperature the collision's buoyancy reads (the transported state, or the packet's field)
    // Temperature transport (null when it is off): the packet's temperature
    // and source channels, and the velocity every collision leaves per cell
    // (SoA ux, uy, uz; 0 on solid cells) for the next call's advection.
    float* ref_temperature = nullptr;
    float* thermal_source = nullptr;
    float* u_last = nullptr;
    long long cells = 0;  // SoA stride of u_last
    // Packet fan channels (mask clamped to [0, 1]; null: fan forcing off).
    float* fan_mask = nullptr;
    float* fan_ux = nullptr;
    float* fan_uy = nullptr;
    float* fan_uz = nullptr;
};

// Velocity a collision leaves for the next call's temperature advection.
__device__ __forceinline__ void record_u(const CellFields& c, long long cell, float ux, float uy, float uz) {
    if (!c.u_last) return;
    c.u_last[cell] = ux;
    c.u_last[c.cells + cell] = uy;
    c.u_last[2 * c.cells + cell] = uz;
}

// One cell of ingest_payload (native/src/aero_lbm_jni.cpp:1671-1694): the
// packet's in_ch channels of this cell (p) into the per-cell fields. Shared by
// the packet ingest kernel and kernels that build a call's inputs on the
// device, so both sanitise and clamp identically.
__device__ __forceinline__ void ingest_cell(const float* p, int in_ch, long long cell, const CellFields& out) {
    const float ob = p[kChObstacle];
    out.obstacle[cell] = ob > 0.5f ? 1 : 0;
    const float vx = p[kChStateVx], vy = p[kChStateVy], vz = p[kChStateVz];
    out.ref_ux[cell] = isfinite(vx) ? vx : 0.0f;
    out.ref_uy[cell] = isfinite(vy) ? vy : 0.0f;
    out.ref_uz[cell] = isfinite(vz) ? vz : 0.0f;
    out.ref_p[cell] = clampf_dev(p[kChStateP], -0.03f, 0.03f);
    if (out.fan_mask) {
        // ingest_payload's fan channels (jni.cpp:1674-1678)
        out.fan_mask[cell] = clampf_dev(p[1], 0.0f, 1.0f);
        out.fan_ux[cell] = isfinite(p[2]) ? p[2] : 0.0f;
        out.fan_uy[cell] = isfinite(p[3]) ? p[3] : 0.0f;
        out.fan_uz[cell] = isfinite(p[4]) ? p[4] : 0.0f;
    }
    const float t = in_ch > kChStateTemp ? p[kChStateTemp] : 0.0f;
    if (out.ref_temperature) {
        // transported temperature: the packet's field is the reference
        // temperature, channel 9 the source (ingest_payload, jni.cpp:1683-1693)
        out.ref_temperature[cell] = clampf_dev(t, -1.0f, 1.0f);
        float src;
        if (in_ch > kChThermalSource) {
            src = clampf_dev(p[kChThermalSource], -0.006f, 0.006f);
        } else {
            // no source channel: the fan-driven source of thermal_source_term
            // (jni.cpp:1783-1797), rounded operation by operation
            const float m = clampf_dev(p[1], 0.0f, 1.0f);
            const float fx = isfinite(p[2]) ? p[2] : 0.0f, fy = isfinite(p[3]) ? p[3] : 0.0f,
                        fz = isfinite(p[4]) ? p[4] : 0.0f;
            const float n = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fy, fy)), __fmul_rn(fz, fz)));
            src = (m > 0.0f && n > 1e-8f) ? __fmul_rn(m, clampf_dev(__fmul_rn(n, 0.0012f), 0.0f, 0.006f)) : 0.0f;
        }
        out.thermal_source[cell] = src;
    } else {
        out.temperature[cell] = clampf_dev(t, -1.0f, 1.0f);
    }
}

// A kernel that writes one call's inputs straight into a context's per-cell
// fields (in place of a host packet's copy and ingest_packet_kernel): the
// device-resident brick service builds its packets this way.
struct DeviceFill {
    cudaError_t (*launch)(const CellFields& out, const BrickDims& d, cudaStream_t s, void* user);
    void* user;
    // the caller guarantees that the obstacle mask this fill writes equals
    // the mask of the context's last call: the pull classification is reused
    // and no cell changes between fluid and solid
    bool mask_unchanged = false;
};

struct ForceField {
    const float* fx;      // optional per-cell force density (SoA); null = none
    const float* fy;
    const float* fz;
};

// Region of a macro output: sample (a, b, c) of the sx x sy x sz result is the
// cell (min(nx - 1, ox + a * stride), ...). A strided atlas has origin 0; a
// sub-box or a point sample has stride 1.
struct OutBox {
    int ox, oy, oz;
    int sx, sy, sz;
    int stride;
    __host__ __device__ long long count() const { return (long long)sx * sy * sz; }
};
inline OutBox strided_box(int nx, int ny, int nz, int stride) {
    return OutBox{0, 0, 0, (nx + stride - 1) / stride, (ny + stride - 1) / stride, (nz + stride - 1) / stride, stride};
}

// Launch helpers (all asynchronous on `stream`; return the launch error).
cudaError_t launch_ingest_packet(const float* packet, int in_channels, BrickDims d, CellFields out, cudaStream_t stream);
// Largest |u| of the fluid cells' reference velocity (fields after an ingest),
// as float bits into *out_bits (cleared first by the caller).
cudaError_t launch_max_fluid_speed(CellFields f, long long cells, unsigned int* out_bits, cudaStream_t stream);
cudaError_t launch_build_flags(const uint8_t* obstacle, BrickDims d, FaceParams face, uint32_t* flags, cudaStream_t stream);
// *_exact: reference-order collision (bit-identical to the reference CPU step);
// *_fast: factorised collision (agrees to FP32 rounding).
cudaError_t launch_init_collide_exact(BrickDims d, CellFields cur, ForceField force, CollideParams cp, float* g_out,
                                      cudaStream_t stream);
cudaError_t launch_init_collide_fast(BrickDims d, CellFields cur, ForceField force, CollideParams cp, float* g_out,
                                     cudaStream_t stream);
cudaError_t launch_step_ab_exact(BrickDims d, const float* g_in, float* g_out, const uint32_t* flags_prev,
                                 const uint8_t* obstacle_prev, const float* ref_p_prev, const FaceParams* face_prev,
                                 CellFields cur, ForceField force, CollideParams cp, cudaStream_t stream);
cudaError_t launch_step_ab_fast(BrickDims d, const float* g_in, float* g_out, const uint32_t* flags_prev,
                                const uint8_t* obstacle_prev, const float* ref_p_prev, const FaceParams* face_prev,
                                CellFields cur, ForceField force, CollideParams cp, cudaStream_t stream);
// Collision of a streamed state held in f_io (the call after a halo exchange).
cudaError_t launch_collide_ab_exact(BrickDims d, float* f_io, CellFields cur, ForceField force, CollideParams cp,
                                    cudaStream_t stream);
cudaError_t launch_collide_ab_fast(BrickDims d, float* f_io, CellFields cur, ForceField force, CollideParams cp,
                                   cudaStream_t stream);
// Macro output of the streamed state S(g): write_output semantics
// (AoS, out_channels per cell; ux,uy,uz scaled; clamp(rho - 1)).
// `face` points to device memory. direct: g already holds the streamed state.
cudaError_t launch_output_ab_exact(BrickDims d, const float* g, const uint32_t* flags, const uint8_t* obstacle,
                                   const float* ref_p, const FaceParams* face, OutBox box, int out_channels,
                                   float velocity_scale, float* out, cudaStream_t stream, int direct = 0);
cudaError_t launch_output_ab_fast(BrickDims d, const float* g, const uint32_t* flags, const uint8_t* obstacle,
                                  const float* ref_p, const FaceParams* face, OutBox box, int out_channels,
                                  float velocity_scale, float* out, cudaStream_t stream, int direct = 0);

uint64_t kernel_launch_count();
void count_launch();
// Optional CUDA-event timing of the brick step kernel launches (off unless
// aero_lbm_b200_kernel_timer enabled it): brackets one launch on stream s.
void step_timer_begin(cudaStream_t s);
void step_timer_end(cudaStream_t s);
void step_timer_reset(bool on);
bool step_timer_read(double* total_ms, int* launches);

}  // namespace aero
