// Per-context operations between or around steps: sparse payload overlays,
// the whole-state shift, temperature sub-box reads, the cylinder benchmark's
// momentum-exchange force.
#pragma once

#include <cuda_runtime.h>

#include "d3q27_kernels.cuh"
#include "inplace27.cuh"

namespace aero {

// apply_sparse_payload_overlays (jni.cpp:1696-1721): overlay i (6 floats:
// vx, vy, vz, p, T, source) replaces the ingested reference fields of cell
// cells[i]; indices outside [0, cells) are skipped. With the temperature
// transport on (thermal 1), T and the source go to the packet reference
// channels; thermal 2 (packets without a source channel) keeps the cells'
// fan-driven source; thermal 0: T is the collision's temperature field (as
// the ingest does).
cudaError_t launch_apply_overlays(const int* cells, const float* values, int count, CellFields f, long long n_cells,
                                  int thermal, cudaStream_t s);

// Shift of a component-major field: dst[k][x] = src[k][x + d] inside the
// brick, else fill (shift_scalar_field / shift_population_field,
// jni.cpp:8067-8130). populations: fill of component q = rest equilibrium.
cudaError_t launch_shift_f32(const float* src, float* dst, BrickDims d, int comps, int dx, int dy, int dz, float fill,
                             bool populations, cudaStream_t s);
cudaError_t launch_shift_u8(const uint8_t* src, uint8_t* dst, BrickDims d, int dx, int dy, int dz, cudaStream_t s);

// Two-buffer layout: f_out[q][x] = the streamed populations (pull of g with
// the last call's classification) of cell x + d, rest equilibrium outside.
cudaError_t launch_shift_materialise_ab(BrickDims d, const float* g, const uint32_t* flags, const uint8_t* obstacle,
                                        const float* ref_p, const FaceParams* face, int dx, int dy, int dz, float* f_out,
                                        cudaStream_t s);

// In-place layout (storage 0 FP32, 1 IEEE-half deviations, 2 fixed point):
// gather the shifted streamed populations into tmp (27 x cells FP32) through
// the old slot map, then, after the classification was rebuilt from the
// shifted mask, scatter them into the incoming slots of the same parity.
struct IpView {
    void* f;
    PadGeom g;
    const uint32_t* flags;
    int parity;
    Fp16Scale sc;
};
cudaError_t launch_ip_gather_shifted(int storage, const IpView& v, int dx, int dy, int dz, float* tmp, cudaStream_t s);
cudaError_t launch_ip_scatter(int storage, const IpView& v, const float* tmp, cudaStream_t s);

// Every population of every cell at rest (feq(q, 1, 0, 0, 0)), 27 x cells.
cudaError_t launch_fill_rest(float* f, long long cells, cudaStream_t s);

// Temperature of a sub-box as aero_lbm_copy_flow_temperature_subrect reads it
// (jni.cpp:9451-9526): 0 on solid cells, else clamp to [-1, 1] with non-finite
// values as 0.
cudaError_t launch_gather_temperature(const float* t, const uint8_t* obstacle, BrickDims d, OutBox box, float* out,
                                      cudaStream_t s);

// compute_benchmark_force (jni.cpp:2454-2492): over fluid cells, directions
// with c_z = 0 whose in-brick neighbour x + c is solid and inside the
// cylinder (cylinder_benchmark_solid_cell, jni.cpp:201-227), accumulate
// 2 f_post[q] c_q in double into out3 (zeroed first); post = the post-collision
// populations (two-buffer state).
cudaError_t launch_cylinder_force(const float* post, const uint8_t* obstacle, BrickDims d, double* out3, cudaStream_t s);

}  // namespace aero
