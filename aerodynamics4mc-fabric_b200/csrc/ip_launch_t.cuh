// Host-side launchers of the in-place (esoteric pull) brick kernels, one
// instantiation per storage / collision variant (d3q27_exact.cu,
// d3q27_fast.cu).
#pragma once

#include <algorithm>

#include "d3q27_async.cuh"

namespace aero {

// The launch-uniform slot offsets of the parity a.parity (IpArgs::off_in,
// off_out) for the packed step's cells without periodic wraps.
inline void fill_slot_offsets(IpArgs& a) {
    for (int q = 0; q < 27; ++q) {
        a.off_in[q][0] = in_offset(a.g, q, a.parity, false);
        a.off_in[q][1] = in_offset(a.g, q, a.parity, true);
        a.off_out[q] = out_offset(a.g, q, a.parity);
    }
}

template <class S, bool kExact>
struct IpLaunch {
    static cudaError_t init(typename S::T* f, const IpArgs& a, cudaStream_t s) {
        const long long cells = (long long)a.g.nx * a.g.ny * a.g.nz;
        init_ip_kernel<S, kExact><<<(unsigned)((cells + 127) / 128), 128, 0, s>>>(f, a);
        count_launch();
        return cudaGetLastError();
    }
    // Pre-fill of equilibrium-face sources; needed when any face is an
    // equilibrium face (velocity, pressure, moving wall).
    static cudaError_t face_fill(typename S::T* f, const IpArgs& a, cudaStream_t s) {
        const long long n = face_fill_count(a.g, a.fill_faces);
        face_fill_ip_kernel<S><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(f, a);
        count_launch();
        return cudaGetLastError();
    }
    static cudaError_t step(typename S::T* f, const IpArgs& a, bool transitions, cudaStream_t s) {
        const long long cells = (long long)a.g.nx * a.g.ny * a.g.nz;
        step_timer_begin(s);
        // the runtime terms (fans, state nudge, sponge) exist in the one-cell kernel only
        const int cpt = a.cp.runtime_terms ? 1 : a.cells_per_thread;
        if (!kExact && cpt == 2 && a.streamed && !a.transport && IpaLaunch<S>::eligible(a)) {
            cudaError_t e = IpaLaunch<S>::step(f, a, s);
            if (e != cudaSuccess) return e;
        } else if (cpt == 2) {
            const int lb = line_block((a.g.nz + 1) / 2);
            const size_t smem = a.transport ? fused_smem_bytes(std::min(2 * lb, a.g.nz)) : 0;
            IpArgs b = a;
            fill_slot_offsets(b);
            const dim3 grid = line_grid(a.g, lb, 2);
            if (a.transport) {
                if (a.parity == 0) step_ip2_kernel<S, kExact, 0, true><<<grid, lb, smem, s>>>(f, b);
                else step_ip2_kernel<S, kExact, 1, true><<<grid, lb, smem, s>>>(f, b);
            } else {
                // may be scheduled under the tail of the transport launch (the kernel waits for it)
                cudaError_t e = a.parity == 0 ? launch_pdl(step_ip2_kernel<S, kExact, 0, false>, grid, dim3(lb), 0, s, f, b)
                                              : launch_pdl(step_ip2_kernel<S, kExact, 1, false>, grid, dim3(lb), 0, s, f, b);
                if (e != cudaSuccess) return e;
            }
        } else {
            const int lb = line_block(a.g.nz);
            const size_t smem = a.transport ? fused_smem_bytes(std::min(lb, a.g.nz)) : 0;
            const dim3 grid = line_grid(a.g, lb);
            if (a.transport) {
                if (a.parity == 0) step_ip_kernel<S, kExact, 0, true><<<grid, lb, smem, s>>>(f, a);
                else step_ip_kernel<S, kExact, 1, true><<<grid, lb, smem, s>>>(f, a);
            } else {
                if (a.parity == 0) step_ip_kernel<S, kExact, 0, false><<<grid, lb, 0, s>>>(f, a);
                else step_ip_kernel<S, kExact, 1, false><<<grid, lb, 0, s>>>(f, a);
            }
        }
        step_timer_end(s);
        count_launch();
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess || !transitions) return e;
        transition_ip_kernel<S, kExact><<<(unsigned)((cells + 127) / 128), 128, 0, s>>>(f, a);
        count_launch();
        return cudaGetLastError();
    }
    static cudaError_t output(const typename S::T* f, const IpArgs& a, OutBox box, int out_ch, float scale, float* out,
                              cudaStream_t s) {
        const long long n = box.count();
        if (n <= 0) return cudaSuccess;
        output_ip_kernel<S, kExact><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(f, a, box, out_ch, scale, out);
        count_launch();
        return cudaGetLastError();
    }
};

}  // namespace aero
