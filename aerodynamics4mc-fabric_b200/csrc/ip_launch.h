// Launchers of the in-place (esoteric pull) kernels, one per storage /
// collision variant; defined in d3q27_exact.cu and d3q27_fast.cu.
#pragma once

#include "ip_launch_t.cuh"

namespace aero {

enum IpVariant { kIpF32Exact = 0, kIpF32Fast = 1, kIpF16Fast = 2, kIpI16Fast = 3 };

cudaError_t ip_init_f32_exact(float* f, const IpArgs& a, cudaStream_t s);
cudaError_t ip_step_f32_exact(float* f, const IpArgs& a, bool transitions, cudaStream_t s);
cudaError_t ip_output_f32_exact(const float* f, const IpArgs& a, OutBox box, int out_ch, float scale, float* out,
                                cudaStream_t s);
cudaError_t ip_init_f32_fast(float* f, const IpArgs& a, cudaStream_t s);
cudaError_t ip_step_f32_fast(float* f, const IpArgs& a, bool transitions, cudaStream_t s);
cudaError_t ip_output_f32_fast(const float* f, const IpArgs& a, OutBox box, int out_ch, float scale, float* out,
                               cudaStream_t s);
cudaError_t ip_init_f16_fast(__half* f, const IpArgs& a, cudaStream_t s);
cudaError_t ip_step_f16_fast(__half* f, const IpArgs& a, bool transitions, cudaStream_t s);
cudaError_t ip_output_f16_fast(const __half* f, const IpArgs& a, OutBox box, int out_ch, float scale, float* out,
                               cudaStream_t s);
cudaError_t ip_init_i16_fast(short* f, const IpArgs& a, cudaStream_t s);
cudaError_t ip_step_i16_fast(short* f, const IpArgs& a, bool transitions, cudaStream_t s);
cudaError_t ip_output_i16_fast(const short* f, const IpArgs& a, OutBox box, int out_ch, float scale, float* out,
                               cudaStream_t s);

cudaError_t ip_fill_f32_exact(float* f, const IpArgs& a, cudaStream_t s);
cudaError_t ip_fill_f32_fast(float* f, const IpArgs& a, cudaStream_t s);
cudaError_t ip_fill_f16_fast(__half* f, const IpArgs& a, cudaStream_t s);
cudaError_t ip_fill_i16_fast(short* f, const IpArgs& a, cudaStream_t s);

// Equilibrium-face pre-fill for the step of parity a.parity (see
// face_fill_ip_kernel); each call leaves one, run before anything reads the
// populations, so that between calls every incoming slot holds the cell's
// streamed population.
inline cudaError_t ip_fill(int v, void* f, const IpArgs& a, cudaStream_t s) {
    if (v == kIpF32Exact) return ip_fill_f32_exact(static_cast<float*>(f), a, s);
    if (v == kIpF32Fast) return ip_fill_f32_fast(static_cast<float*>(f), a, s);
    if (v == kIpI16Fast) return ip_fill_i16_fast(static_cast<short*>(f), a, s);
    return ip_fill_f16_fast(static_cast<__half*>(f), a, s);
}

inline cudaError_t ip_init(int v, void* f, const IpArgs& a, cudaStream_t s) {
    if (v == kIpF32Exact) return ip_init_f32_exact(static_cast<float*>(f), a, s);
    if (v == kIpF32Fast) return ip_init_f32_fast(static_cast<float*>(f), a, s);
    if (v == kIpI16Fast) return ip_init_i16_fast(static_cast<short*>(f), a, s);
    return ip_init_f16_fast(static_cast<__half*>(f), a, s);
}
inline cudaError_t ip_step(int v, void* f, const IpArgs& a, bool transitions, cudaStream_t s) {
    if (v == kIpF32Exact) return ip_step_f32_exact(static_cast<float*>(f), a, transitions, s);
    if (v == kIpF32Fast) return ip_step_f32_fast(static_cast<float*>(f), a, transitions, s);
    if (v == kIpI16Fast) return ip_step_i16_fast(static_cast<short*>(f), a, transitions, s);
    return ip_step_f16_fast(static_cast<__half*>(f), a, transitions, s);
}
inline cudaError_t ip_output(int v, const void* f, const IpArgs& a, OutBox box, int out_ch, float scale, float* out,
                             cudaStream_t s) {
    if (v == kIpF32Exact) return ip_output_f32_exact(static_cast<const float*>(f), a, box, out_ch, scale, out, s);
    if (v == kIpF32Fast) return ip_output_f32_fast(static_cast<const float*>(f), a, box, out_ch, scale, out, s);
    if (v == kIpI16Fast) return ip_output_i16_fast(static_cast<const short*>(f), a, box, out_ch, scale, out, s);
    return ip_output_f16_fast(static_cast<const __half*>(f), a, box, out_ch, scale, out, s);
}

}  // namespace aero
