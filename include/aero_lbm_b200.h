/*
 * aero_lbm_b200 — C ABI of the B200 (sm_100a) lattice-Boltzmann brick step.
 *
 * This header is the drop-in boundary: the entry points below carry the same
 * names, argument meaning, return convention (1 = ok, 0 = error, message via
 * *_last_error) and struct layouts as the reference library's C ABI, so the
 * reference's Java JNI layer, its ctypes tools and its brick runtime can bind
 * this library instead. Each declaration names the reference interface it
 * replaces as file:line in the reference project.
 *
 * Entry points prefixed aero_lbm_b200_* have no reference counterpart; they
 * expose the device-resident paths (batched bricks, FP16 storage, stream
 * selection, conservation sums) that the reference does not have.
 *
 * Struct layouts must stay byte-identical to the reference's
 * (native/include/aero_lbm_capi.h:15-111, native/include/aero_solver_capi.h:12-56).
 */
#ifndef AERO_LBM_B200_H
#define AERO_LBM_B200_H

#include <stdint.h>

#if defined(_WIN32)
#define AERO_LBM_B200_EXPORT __declspec(dllexport)
#else
#define AERO_LBM_B200_EXPORT __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- enums and structs (native/include/aero_lbm_capi.h:15-111) ---- */
enum {
    AERO_LBM_BENCHMARK_ABI_VERSION = 1,
    AERO_LBM_MESOSCALE_ABI_VERSION = 3,
    AERO_LBM_SIMULATION_ABI_VERSION = 1,
    AERO_LBM_MESOSCALE_FORCING_CHANNELS = 25,
    AERO_LBM_MESOSCALE_STATE_CHANNELS = 6,
    AERO_LBM_SIMULATION_FLOW_STATE_CHANNELS = 4,
    AERO_LBM_SIMULATION_PACKED_ATLAS_CHANNELS = 4,
    AERO_LBM_SIMULATION_PLAYER_PROBE_CHANNELS = 6,
    AERO_LBM_SIMULATION_BRICK_RUNTIME_STATUS_FIELDS = 8
};

enum {
    AERO_LBM_REALTIME_SOLVER_AUTO = 0,
    AERO_LBM_REALTIME_SOLVER_CLASSIC_D3Q27 = 1,
    AERO_LBM_REALTIME_SOLVER_COMPACT_EXPERIMENTAL = 2,
    AERO_LBM_REALTIME_SOLVER_D3Q27_FP16_INPLACE_EXPERIMENTAL = 3
};

typedef enum AeroLbmBenchmarkPreset {
    AERO_LBM_BENCHMARK_PRESET_NONE = 0,
    AERO_LBM_BENCHMARK_PRESET_TAYLOR_GREEN_3D = 1,
    AERO_LBM_BENCHMARK_PRESET_LID_DRIVEN_CAVITY_2D = 2,
    AERO_LBM_BENCHMARK_PRESET_LID_DRIVEN_CAVITY_3D = 3,
    AERO_LBM_BENCHMARK_PRESET_CYLINDER_CROSSFLOW_2D = 4,
    AERO_LBM_BENCHMARK_PRESET_DIFFERENTIALLY_HEATED_CAVITY_2D = 5,
    AERO_LBM_BENCHMARK_PRESET_DIFFERENTIALLY_HEATED_CAVITY_3D = 6
} AeroLbmBenchmarkPreset;

typedef enum AeroLbmHydrodynamicBoundaryKind {
    AERO_LBM_HYDRO_BOUNDARY_INHERIT_GAME = 0,
    AERO_LBM_HYDRO_BOUNDARY_PERIODIC = 1,
    AERO_LBM_HYDRO_BOUNDARY_BOUNCE_BACK = 2,
    AERO_LBM_HYDRO_BOUNDARY_MOVING_WALL = 3,
    AERO_LBM_HYDRO_BOUNDARY_VELOCITY_DIRICHLET = 4,
    AERO_LBM_HYDRO_BOUNDARY_PRESSURE_DIRICHLET = 5,
    AERO_LBM_HYDRO_BOUNDARY_CONVECTIVE_OUTFLOW = 6,
    AERO_LBM_HYDRO_BOUNDARY_SYMMETRY = 7
} AeroLbmHydrodynamicBoundaryKind;

typedef enum AeroLbmThermalBoundaryKind {
    AERO_LBM_THERMAL_BOUNDARY_INHERIT_GAME = 0,
    AERO_LBM_THERMAL_BOUNDARY_DISABLED = 1,
    AERO_LBM_THERMAL_BOUNDARY_PERIODIC = 2,
    AERO_LBM_THERMAL_BOUNDARY_ADIABATIC = 3,
    AERO_LBM_THERMAL_BOUNDARY_TEMPERATURE_DIRICHLET = 4,
    AERO_LBM_THERMAL_BOUNDARY_HEAT_FLUX_NEUMANN = 5
} AeroLbmThermalBoundaryKind;

typedef enum AeroLbmBenchmarkFlags {
    AERO_LBM_BENCHMARK_FLAG_DISABLE_FAN_FORCING = 1u << 0,
    AERO_LBM_BENCHMARK_FLAG_DISABLE_FAN_NOISE = 1u << 1,
    AERO_LBM_BENCHMARK_FLAG_DISABLE_SPONGE = 1u << 2,
    AERO_LBM_BENCHMARK_FLAG_DISABLE_CONVECTIVE_OUTFLOW = 1u << 3,
    AERO_LBM_BENCHMARK_FLAG_DISABLE_OBSTACLE_BOUNCE_BLEND = 1u << 4,
    AERO_LBM_BENCHMARK_FLAG_DISABLE_SGS = 1u << 5,
    AERO_LBM_BENCHMARK_FLAG_DISABLE_INTERNAL_THERMAL_SOURCE = 1u << 6,
    AERO_LBM_BENCHMARK_FLAG_DISABLE_BUOYANCY = 1u << 7
} AeroLbmBenchmarkFlags;

typedef struct AeroLbmBoundaryFaceConfig {
    int hydrodynamic_kind;
    int thermal_kind;
    float velocity[3];
    float pressure;
    float temperature;
    float heat_flux;
} AeroLbmBoundaryFaceConfig;

typedef struct AeroLbmBenchmarkConfig {
    uint32_t abi_version;
    uint32_t struct_size;
    uint32_t flags;
    int enabled;
    int preset;
    int reserved0;
    float reynolds_number;
    float rayleigh_number;
    float prandtl_number;
    float mach_number;
    float reference_density;
    float reference_temperature;
    float reference_length;
    float body_force[3];
    float gravity[3];
    float initial_velocity[3];
    float initial_pressure;
    float initial_temperature;
    AeroLbmBoundaryFaceConfig x_min;
    AeroLbmBoundaryFaceConfig x_max;
    AeroLbmBoundaryFaceConfig y_min;
    AeroLbmBoundaryFaceConfig y_max;
    AeroLbmBoundaryFaceConfig z_min;
    AeroLbmBoundaryFaceConfig z_max;
    uint32_t reserved[8];
} AeroLbmBenchmarkConfig;

typedef struct AeroLbmTimingSnapshot {
    uint64_t ticks;
    double last_payload_copy_ms;
    double last_solver_ms;
    double last_readback_ms;
    double last_total_ms;
    double avg_payload_copy_ms;
    double avg_solver_ms;
    double avg_readback_ms;
    double avg_total_ms;
} AeroLbmTimingSnapshot;

/* ---- per-context LBM ABI (native/include/aero_lbm_capi.h:166-302) ---- */

/* native/include/aero_lbm_capi.h:166 (jni.cpp:8625) — square grid init. */
AERO_LBM_B200_EXPORT int aero_lbm_init(int grid_size, int input_channels, int output_channels);
/* native/include/aero_lbm_capi.h:167 — square-grid step. */
AERO_LBM_B200_EXPORT int aero_lbm_step(const float* packet, int grid_size, long long context_key, float* output_flow);
/* native/include/aero_lbm_capi.h:168 (jni.cpp:8592-8624) — global reset of all contexts,
 * input_channels >= 9, output_channels >= 4. */
AERO_LBM_B200_EXPORT int aero_lbm_init_rect(int nx, int ny, int nz, int input_channels, int output_channels);
/* native/include/aero_lbm_capi.h:169 (jni.cpp:8630-8684) — one step from an AoS packet
 * (input_channels floats per cell, cell = (x*ny+y)*nz+z); output_flow may be null. */
AERO_LBM_B200_EXPORT int aero_lbm_step_rect(const float* packet, int nx, int ny, int nz, long long context_key, float* output_flow);
/* native/include/aero_lbm_capi.h:170 — as step_rect, output velocity scaled. */
AERO_LBM_B200_EXPORT int aero_lbm_step_rect_scaled(const float* packet, int nx, int ny, int nz, long long context_key,
                                                   float output_velocity_scale, float* output_flow);
/* native/include/aero_lbm_capi.h:171 (jni.cpp:8534-8582) — step with the resident packet. */
AERO_LBM_B200_EXPORT int aero_lbm_step_rect_cached(int nx, int ny, int nz, long long context_key, float* output_flow);
/* native/include/aero_lbm_capi.h:172 */
AERO_LBM_B200_EXPORT int aero_lbm_step_rect_cached_scaled(int nx, int ny, int nz, long long context_key,
                                                          float output_velocity_scale, float* output_flow);
/* native/include/aero_lbm_capi.h:218 */
AERO_LBM_B200_EXPORT int aero_lbm_has_context(long long context_key);
/* native/include/aero_lbm_capi.h:220 */
AERO_LBM_B200_EXPORT int aero_lbm_context_realtime_cached_initialized(long long context_key);
/* native/include/aero_lbm_capi.h:210-217 (jni.cpp:9623-9691, 8428-8430) — halo
 * exchange between two stepped contexts of the configured cubic grid with
 * max(1, grid_size / 4) halo layers. */
AERO_LBM_B200_EXPORT int aero_lbm_exchange_halo(int grid_size, long long first_context_key, long long second_context_key,
                                                int offset_x, int offset_y, int offset_z);
/* native/include/aero_lbm_capi.h:218-228 (jni.cpp:9693-9790, 8136-8426) — the
 * second context lies at offset (offset_x, offset_y, offset_z) in {-1,0,1}^3
 * (not all 0) from the first; each receives the other's streamed populations
 * and temperature on the slab of halo_layers (clamped to n/2 - 1) layers.
 * Cubic contexts only; returns 1 (no-op) while either context has not
 * stepped; both contexts must use the same storage. */
AERO_LBM_B200_EXPORT int aero_lbm_exchange_halo_layers_rect(int nx, int ny, int nz, int halo_layers,
                                                            long long first_context_key, long long second_context_key,
                                                            int offset_x, int offset_y, int offset_z);
/* native/include/aero_lbm_capi.h:173-182 (jni.cpp:6156-6260, 9905-9960) — block
 * edits on an in-place context that has stepped: the next call's mask is the
 * current one with cell_indices[i] set to solid_values[i] (later entries win),
 * and every patched cell restarts at rest. fan_dir_values must be given and
 * is ignored (no fan model). */
AERO_LBM_B200_EXPORT int aero_lbm_patch_d3q27_f16_static_cells_rect(int nx, int ny, int nz, long long context_key,
                                                                    int patch_count, const int* cell_indices,
                                                                    const uint8_t* solid_values,
                                                                    const uint8_t* fan_dir_values);
/* native/include/aero_lbm_capi.h:183-193 (jni.cpp:6449-6540, 9962-10022) — a
 * boundary-reference shell: fluid cells within shell_layers of the faces in
 * face_mask (bit i: x-, x+, y-, y+, z-, z+) are relaxed after every call made
 * in the FP16 in-place solver mode (3; the reference's FP16 step is the only
 * one that reads the shell) toward the given flow state (flow_channels >= 4: ux, uy, uz, p) with
 * strength relaxation (<= 0.5) x (1 - (layer - 1) / layers)^2. In-place
 * contexts that have stepped; a zero mask, layer count or relaxation clears. */
AERO_LBM_B200_EXPORT int aero_lbm_set_d3q27_f16_boundary_shell_rect(int nx, int ny, int nz, long long context_key,
                                                                    const float* flow_state, int flow_channels,
                                                                    int face_mask, int shell_layers, float relaxation);
/* native/include/aero_lbm_capi.h:194 — remove the shell (1 also without a context). */
AERO_LBM_B200_EXPORT int aero_lbm_clear_d3q27_f16_boundary_shell_rect(long long context_key);
/* native/include/aero_lbm_capi.h:195-205 (jni.cpp:8686-8745, 1696-1721) — a
 * full step whose ingested reference fields are replaced at overlay_count
 * cells before the collision (6 floats per overlay: vx, vy, vz, p, T, source;
 * cell indices outside the brick are skipped). */
AERO_LBM_B200_EXPORT int aero_lbm_step_rect_with_sparse_overlays(const float* packet, int nx, int ny, int nz,
                                                                 long long context_key, const int* overlay_cells,
                                                                 const float* overlay_values, int overlay_count,
                                                                 float* output_flow);
/* native/include/aero_lbm_capi.h:206 (jni.cpp:9603-9616, 8432-8478) — move
 * the whole state by (dx, dy, dz): new cell x holds old cell x + d; cells
 * shifted in from outside are fluid at rest with zero fields. */
AERO_LBM_B200_EXPORT int aero_lbm_shift_context(int grid_size, long long context_key, int dx, int dy, int dz);
/* native/include/aero_lbm_capi.h:208 — always 0: no compact (heuristic)
 * contexts exist in this library. */
AERO_LBM_B200_EXPORT int aero_lbm_context_compact_initialized(long long context_key);
/* native/include/aero_lbm_capi.h:230-239 (jni.cpp:8899-8947) — raw
 * temperature state of one cell. */
AERO_LBM_B200_EXPORT int aero_lbm_sample_temperature_point_rect(int nx, int ny, int nz, long long context_key, int sample_x,
                                                                int sample_y, int sample_z, float* out_temperature);
/* native/include/aero_lbm_capi.h:240-249 (jni.cpp:8949-9244) — write_output
 * of one cell (4 floats, velocity unscaled). */
AERO_LBM_B200_EXPORT int aero_lbm_sample_flow_point_rect(int nx, int ny, int nz, long long context_key, int sample_x,
                                                         int sample_y, int sample_z, float* out_flow);
/* native/include/aero_lbm_capi.h:259-272 (jni.cpp:9451-9526) — flow (4 floats
 * per cell) and temperature (0 on solids, clamped to [-1, 1]) of a sub-box,
 * x outermost. */
AERO_LBM_B200_EXPORT int aero_lbm_copy_flow_temperature_subrect(int nx, int ny, int nz, long long context_key, int offset_x,
                                                                int offset_y, int offset_z, int copy_nx, int copy_ny,
                                                                int copy_nz, float* out_flow, float* out_temperature);
/* native/include/aero_lbm_capi.h:275 (jni.cpp:10259-10267, 2454-2492) — the
 * last call's momentum-exchange force on the cylinder (cylinder preset only,
 * else 0). */
AERO_LBM_B200_EXPORT int aero_lbm_get_last_force(long long context_key, float* out_fx, float* out_fy, float* out_fz);
/* native/include/aero_lbm_capi.h:281 (jni.cpp:5436-5457) — device bytes per
 * category, the reference's key set. */
AERO_LBM_B200_EXPORT const char* aero_lbm_memory_info(void);
/* native/include/aero_lbm_capi.h:241 */
AERO_LBM_B200_EXPORT int aero_lbm_get_temperature_state_rect(int nx, int ny, int nz, long long context_key, float* out_temperature);
/* native/include/aero_lbm_capi.h:262 (jni.cpp:9246-9450) — sample every stride cells
 * (min(n-1, a*stride)), 4 floats per atlas cell; value_count must equal ceil(n/stride)^3*4. */
AERO_LBM_B200_EXPORT int aero_lbm_extract_flow_atlas_rect(int nx, int ny, int nz, long long context_key, int stride,
                                                          float* out_flow_atlas, int value_count);
/* native/include/aero_lbm_capi.h:285 (jni.cpp:9528) — stride-1 flow state, 4 floats per cell. */
AERO_LBM_B200_EXPORT int aero_lbm_get_flow_state_rect(int nx, int ny, int nz, long long context_key, float* out_flow);
/* native/include/aero_lbm_capi.h:286 */
AERO_LBM_B200_EXPORT int aero_lbm_set_temperature_state_rect(int nx, int ny, int nz, long long context_key, const float* temperature);
/* native/include/aero_lbm_capi.h:288 */
AERO_LBM_B200_EXPORT void aero_lbm_release_context(long long context_key);
/* native/include/aero_lbm_capi.h:289 */
AERO_LBM_B200_EXPORT void aero_lbm_shutdown(void);
/* native/include/aero_lbm_capi.h:290-292 */
AERO_LBM_B200_EXPORT const char* aero_lbm_runtime_info(void);
AERO_LBM_B200_EXPORT const char* aero_lbm_last_error(void);
AERO_LBM_B200_EXPORT const char* aero_lbm_timing_info(void);
/* native/include/aero_lbm_capi.h:294 */
AERO_LBM_B200_EXPORT void aero_lbm_reset_timing(void);
/* native/include/aero_lbm_capi.h:295 */
AERO_LBM_B200_EXPORT void aero_lbm_set_realtime_solver_mode(int solver_mode);
/* native/include/aero_lbm_capi.h:296 — waits for all queued device work. */
AERO_LBM_B200_EXPORT int aero_lbm_finish(void);
/* native/include/aero_lbm_capi.h:297 */
AERO_LBM_B200_EXPORT int aero_lbm_get_timing_snapshot(AeroLbmTimingSnapshot* out_snapshot);

/* ---- benchmark/boundary configuration (native/include/aero_lbm_capi.h:698-703) ---- */
AERO_LBM_B200_EXPORT void aero_lbm_benchmark_default_config(AeroLbmBenchmarkConfig* out_config);
AERO_LBM_B200_EXPORT int aero_lbm_benchmark_default_preset_config(int preset, AeroLbmBenchmarkConfig* out_config);
AERO_LBM_B200_EXPORT int aero_lbm_benchmark_set_config(const AeroLbmBenchmarkConfig* config);
AERO_LBM_B200_EXPORT int aero_lbm_benchmark_get_config(AeroLbmBenchmarkConfig* out_config);
AERO_LBM_B200_EXPORT void aero_lbm_benchmark_reset_config(void);
AERO_LBM_B200_EXPORT const char* aero_lbm_benchmark_info(void);

/* ---- device-resident extensions (no reference counterpart) ---- */

/* Queue all kernels of this library on `stream` (a cudaStream_t; null = the
 * library's own stream). */
AERO_LBM_B200_EXPORT void aero_lbm_b200_set_stream(void* stream);
/* Number of kernels this library has launched since load. */
AERO_LBM_B200_EXPORT unsigned long long aero_lbm_b200_launch_count(void);
/* CUDA-event timing of the in-place step kernel launches alone (the
 * population stream-collide kernel, without the face pre-fill, temperature
 * transport or transition kernels): on != 0 starts a new record, 0 stops.
 * kernel_time waits for the last recorded launch and returns the summed
 * device time and the number of launches timed. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_kernel_timer(int on);
AERO_LBM_B200_EXPORT int aero_lbm_b200_kernel_time(double* total_ms, int* launches);
/* Advance a context `steps` times with its resident inputs, no host copies and
 * no synchronisation (the device-resident form of step_rect_cached). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_advance_rect(long long context_key, int steps);
/* Select the streaming scheme of a context: 0 automatic (in-place when every
 * face is local), 1 two-buffer pull, 2 in-place esoteric pull. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_set_streaming_mode(int mode);
/* Global mass and momentum of a context's current streamed state (the
 * populations the next step collides), summed in FP64 over fluid cells:
 * out4 = {sum rho, sum rho ux, sum rho uy, sum rho uz}. Uses a per-context
 * device scratch buffer (allocated on first use) for the block partial sums;
 * synchronises the library stream. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_conservation_sums(long long context_key, double* out4);
/* Allocation-free form of aero_lbm_b200_conservation_sums, for callers that
 * cannot call cudaMalloc (a real-time tick thread that must not stall on an
 * allocation that synchronises the device; an embedding with a fixed device
 * memory budget). No counterpart in the reference. Its scratch is a static
 * 256 KiB device array, so contexts of at most 2,097,152 cells (128^3) are
 * accepted; larger ones return 0 with an error. Call it with the context's
 * device current (another current device is rejected with an error). The
 * first call on a device looks up the array's address; make it before any
 * stream capture. Calls share the array: overlapping calls on the GPU race. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_conservation_sums_noalloc(long long context_key, double* out4);
/* FP32 collision arithmetic: 0 = the reference's operation order, no
 * multiply-add contraction (bit-identical to the reference CPU step; default),
 * 1 = factorised moment transforms with contraction (same scheme, fewer flops,
 * agrees to FP32 rounding per step). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_set_collision_mode(int mode);
/* Launch shape of the in-place step: 2 = two z-adjacent cells per thread with
 * the collision in sm_100 packed FP32 (default), 1 = one cell per thread. With
 * the reference-order collision both shapes are bit-identical; with the
 * factorised one they agree to FP32 rounding. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_set_cells_per_thread(int cells_per_thread);
/* Temperature transport before every collision (the reference's
 * benchmark-mode update: first-order semi-Lagrangian advection by the
 * previous collision's velocity, diffusion, the packet's source channel,
 * thermal faces; native/src/aero_lbm_jni.cpp:2049-2143): -1 = whenever
 * buoyancy is enabled (default; the only case where it changes the flow),
 * 1 = always (the temperature state then evolves exactly like the
 * reference's also without buoyancy), 0 = never (the packet's temperature
 * channel is the buoyancy field of each call). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_set_thermal_transport(int mode);
/* In-place step with the factorised collision, two cells per thread, on a
 * brick whose z axis is not periodic: 1 = each warp streams its next 64-cell
 * tile into shared memory with bulk asynchronous copies while it collides the
 * current one, 0 = per-thread loads (default; faster on B200). Same
 * arithmetic, bit-identical results. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_set_streamed_step(int on);
/* Where the first-order temperature transport of in-place contexts runs:
 * 0 (default) as a separate pass before the step; 1 inside the step kernel,
 * each cell updating its own temperature right before its collision. Same
 * arithmetic, bit-identical results; the heated-cavity and game-runtime
 * (BFECC) transports always run as separate passes. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_set_fused_transport(int on);
/* Restore every aero_lbm_b200_set_* tuning knob (streaming mode, collision
 * mode, cells per thread, thermal transport, streamed step, fused transport,
 * 16-bit format, physics overrides) to its default. */
AERO_LBM_B200_EXPORT void aero_lbm_b200_reset_tuning(void);
/* Format of the 16-bit deviation storage chosen by
 * aero_lbm_set_realtime_solver_mode(3), for contexts created afterwards:
 * 1 = 16-bit fixed point of (f - w) * S / w with S = 32767 / d_max (default:
 * uniform resolution, within 1e-3 of the max speed of an FP64 run after 1000
 * steps of a 128^3 terrain brick), 0 = IEEE half of the same deviation with a
 * power-of-two per-brick S (about 2e-3 on that brick). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_set_fp16_format(int format);
/* Per-cell force density field for a context (3 x cells floats, SoA order
 * fx[cells], fy[cells], fz[cells]; host pointer; null clears). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_set_force_field(long long context_key, const float* force_soa, int value_count);
/* Smagorinsky constant C (reference hard-codes 0.025) and buoyancy
 * coefficient/axis (reference: beta from its runtime constants, +y). A
 * negative value keeps the reference default. */
AERO_LBM_B200_EXPORT void aero_lbm_b200_set_physics_overrides(float smagorinsky_c, float buoyancy_beta, int gravity_axis);

/* ---- batched bricks (no reference counterpart: the reference steps bricks one
 * aero_lbm_step_rect call at a time, native/src/aero_lbm_simulation_bridge.cpp:1092-1166) ----
 * Many independent bricks of uneven sizes, each with its own mask, relaxation
 * time, body force and storage precision, advanced by one persistent launch
 * per tick, with a stride-s packed int16 velocity publish per tick. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_create(long long* out_handle);
/* precision 0 = fp32, 1 = fp16 deviation storage; obstacle: cells bytes (or
 * null); init_velocity_soa: 3 x cells floats (or null = rest); tau in
 * (0.5, 0.95]; body_force: 3 floats (force density) or null; face_kinds: 6
 * AeroLbmHydrodynamicBoundaryKind values, periodic or bounce-back only (null =
 * all periodic). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_add_brick(long long handle, int nx, int ny, int nz, int precision,
                                                       const uint8_t* obstacle, const float* init_velocity_soa,
                                                       float tau, const float* body_force, const int* face_kinds,
                                                       int* out_index);
/* Allocate device state and the work list; velocity_scale = dx/dt used to
 * convert published velocities to m/s before quantisation. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_finalize(long long handle, int publish_stride, float velocity_scale);
/* use_graph: replay ticks from a captured CUDA graph; publish: run the
 * stride-s publish after every tick. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_set_options(long long handle, int use_graph, int publish);
/* Queue `ticks` ticks on the library stream (no synchronisation). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_tick(long long handle, int ticks);
/* Time launch shapes on the live bricks (trial ticks are real ticks) and keep
 * the fastest; reports the choice and its time per tick. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_autotune(long long handle, int trial_ticks, int* out_threads,
                                                      int* out_blocks_per_sm, float* out_ms_per_tick);
/* Cells, algorithmic population bytes per tick, atlas records, work units and
 * ticks done so far (autotuning trials included). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_info(long long handle, long long* out_cells, double* out_bytes_per_tick,
                                                  int* out_atlas_records, int* out_units, long long* out_ticks);
/* Packed int16 atlas of one brick from the last published tick (4 values per
 * atlas cell, quantised like aero_lbm_simulation_copy_brick_world_packed_flow_atlas). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_copy_atlas(long long handle, int brick, int16_t* out, int value_count);
/* Flow state of one brick (cells x 4 floats, write_output semantics, scale 1). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_copy_flow(long long handle, int brick, float* out, int value_count);
AERO_LBM_B200_EXPORT void aero_lbm_b200_batch_destroy(long long handle);
AERO_LBM_B200_EXPORT const char* aero_lbm_b200_batch_last_error(void);

/* ---- D3Q19 mesoscale ABI (native/include/aero_lbm_capi.h:124-150, 286-301;
 *      native/src/aero_lbm_mesoscale.cpp:1397-1510) ---- */

/* native/include/aero_lbm_capi.h:124 — mesoscale grid (y up). */
typedef struct AeroLbmMesoscaleConfig {
    uint32_t abi_version;
    uint32_t struct_size;
    int nx;
    int ny;
    int nz;
    float dx_m;
    float dt_s;
    float molecular_nu_m2_s;
    float prandtl_air;
    float turbulent_prandtl;
    float reference_density_kg_m3;
    float ambient_air_temperature_k;
    float deep_ground_temperature_k;
    float background_wind_m_s[3];
    uint32_t reserved[8];
} AeroLbmMesoscaleConfig;

/* native/include/aero_lbm_capi.h:143 */
typedef struct AeroLbmMesoscaleTransport {
    float velocity_scale_m_s_per_lattice;
    float nu_molecular_lattice;
    float alpha_molecular_lattice;
    float tau_shear_molecular;
    float tau_thermal_molecular;
} AeroLbmMesoscaleTransport;

/* native/include/aero_lbm_capi.h:286 (mesoscale.cpp:1399) — 32 x 4 x 32, dx 64 m, dt 5 s, ... */
AERO_LBM_B200_EXPORT void aero_lbm_mesoscale_default_config(AeroLbmMesoscaleConfig* out_config);
/* native/include/aero_lbm_capi.h:287 (mesoscale.cpp:1420) — lattice transport of a config. */
AERO_LBM_B200_EXPORT int aero_lbm_mesoscale_derive_transport(const AeroLbmMesoscaleConfig* config,
                                                             AeroLbmMesoscaleTransport* out_transport);
/* native/include/aero_lbm_capi.h:291 (mesoscale.cpp:1436) — keys count up from 1. */
AERO_LBM_B200_EXPORT int aero_lbm_mesoscale_create_context(const AeroLbmMesoscaleConfig* config, long long* out_context_key);
/* native/include/aero_lbm_capi.h:295 (mesoscale.cpp:1452) — one step: forcing is cells x 25
 * floats, out_state cells x 6 (ambient K, deep ground K, surface K, wind x, y, z m/s). The
 * first call (and the first after a shape change) seeds from the forcing. Synchronous. */
AERO_LBM_B200_EXPORT int aero_lbm_mesoscale_step_context(long long context_key, const AeroLbmMesoscaleConfig* config,
                                                         const float* forcing, float* out_state);
/* native/include/aero_lbm_capi.h:301 (mesoscale.cpp:1500) */
AERO_LBM_B200_EXPORT void aero_lbm_mesoscale_release_context(long long context_key);

/* B200 extension: options of the mesoscale step the reference does not have.
 * All zero = the reference step. hydro_only runs the hydrodynamic
 * distribution alone (relaxation toward the cell's own rho, u; no thermal
 * distribution, no forcing targets; output channels rho, 0, 0, wind) in one
 * fused pull + collide launch per call, with FP32 populations (storage 0,
 * bit-identical to the restatement) or FP16 deviations (storage 1). */
typedef struct AeroLbmB200MesoscaleOptions {
    int periodic_sides;      /* x and z wrap */
    int free_slip_top;       /* specular lid at y = ny */
    int fixed_tau;           /* use tau_hydro instead of the derived, clamped tau */
    int enable_sgs;          /* Smagorinsky on the even hydrodynamic rate */
    int disable_edge_blend;  /* no 2-cell equilibrium blend at open sides / top */
    int hydro_only;
    double tau_hydro;
    double smagorinsky_c;
    double body_force[3];    /* lattice force density (Guo source), y up */
    int storage;             /* hydro_only: 0 FP32, 1 FP16 deviations, 2 16-bit fixed-point deviations */
    int threads;             /* hydro_only: block size 64, 128 or 256 (0 = 256) */
    int collision;           /* hydro_only: 0 reference order (FP32 bit-identical to the restatement),
                                1 two cells per thread in packed FP32 (nz even; agrees to FP32 rounding) */
    int reserved;
} AeroLbmB200MesoscaleOptions;

AERO_LBM_B200_EXPORT void aero_lbm_b200_mesoscale_default_options(AeroLbmB200MesoscaleOptions* out_options);
/* Set a context's options; the context re-seeds at its next step. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_mesoscale_set_options(long long context_key, const AeroLbmB200MesoscaleOptions* options);
/* `steps` more steps with the forcing of the last step call, on the library
 * stream, without output or synchronisation (device-resident stepping). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_mesoscale_advance(long long context_key, int steps);
/* The output state of the current step (cells x 6); synchronises. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_mesoscale_read_state(long long context_key, float* out_state);
/* Cells and algorithmic population bytes per step of a context (after its first step). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_mesoscale_info(long long context_key, long long* out_cells, double* out_bytes_per_step);

/* ---- B200 extension: discrete adjoint of the brick step (no counterpart in
 *      the reference). A brick with a static mask and temperature field is run
 *      forward `steps` calls from the equilibrium at the inflow vector; the loss
 *      is the squared velocity mismatch at probe cells after the last call, and
 *      its gradient with respect to the per-cell body-force field and the inflow
 *      vector comes from the reverse sweep, with states checkpointed every
 *      `checkpoint_every` calls and recomputed per segment. ---- */
typedef struct AeroLbmB200AdjointConfig {
    int nx;
    int ny;
    int nz;
    int face_kind[6];      /* x-, x+, y-, y+, z-, z+: 1 periodic, 2 bounce-back, 4 velocity (feq at the inflow) */
    float tau;             /* shear (and normal) relaxation time */
    float smagorinsky_c;   /* 0 = no SGS */
    float buoyancy_beta;   /* g*beta along +z from the temperature field; 0 = off */
    int steps;             /* forward calls */
    int checkpoint_every;  /* K (1 = keep every state) */
    int reserved;
} AeroLbmB200AdjointConfig;

AERO_LBM_B200_EXPORT void aero_lbm_b200_adjoint_default_config(AeroLbmB200AdjointConfig* out_config);
/* obstacle: cells bytes (1 = solid); temperature: cells floats or null. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_create(const AeroLbmB200AdjointConfig* config, const uint8_t* obstacle,
                                                      const float* temperature, long long* out_handle);
/* Probe cell indices ((x*ny+y)*nz+z, fluid cells) and their target velocities (count x 3, lattice units). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_set_probes(long long handle, int count, const int* cells, const float* targets);
/* Forward run: loss and probe velocities (count x 3). force_soa: 3 x cells or null; inflow: 3.
 * precision 0 = the FP32 model the gradient is taken of, 1 = the same model in FP64. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_forward(long long handle, const float* force_soa, const float* inflow,
                                                       int precision, double* out_loss, float* out_probe_u);
/* Loss and gradients (FP64): out_grad_force 3 x cells (SoA) or null, out_grad_inflow 3. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_gradient(long long handle, const float* force_soa, const float* inflow,
                                                        double* out_loss, double* out_grad_force, double* out_grad_inflow);
/* Device ms per call of the last gradient run, and its wall ms. forward: the forward run with its
 * checkpoints. The reverse sweep recomputes each segment's states on a second stream while the previous
 * segment is reversed; recompute: the time the reverse stream waited for recomputed states (the part not
 * hidden under reverse launches); reverse: the time of the reverse launches. recompute + reverse is the
 * sweep's device time. */
AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_timing(long long handle, double* out_forward_ms_per_step,
                                                      double* out_recompute_ms_per_step, double* out_reverse_ms_per_step,
                                                      double* out_total_ms);
AERO_LBM_B200_EXPORT void aero_lbm_b200_adjoint_destroy(long long handle);
AERO_LBM_B200_EXPORT const char* aero_lbm_b200_adjoint_last_error(void);
/* One cell's collision and its vector-Jacobian product, on the host CPU (precision 0 float, 1 double). */
AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_collide_vjp_host(int precision, const AeroLbmB200AdjointConfig* config,
                                                                const double* f_in, double temperature,
                                                                const double* cell_force, const double* lam_out,
                                                                double* f_out, double* lam_in, double* lam_force);

/* ---- brick-world service ABI (native/include/aero_lbm_capi.h:151-164, 303-466, 695-696;
 * implemented by native/src/aero_lbm_simulation_bridge.cpp:4562-5535, 6866-7022) ----
 * The entry points the mod's ClientL2Solver reaches through JNI. One service
 * (key 1) holds brick worlds keyed by the caller; each world has one brick
 * size, its bricks are keyed by brick coordinates. Brick state lives on the
 * device between ticks: a tick builds each brick's inputs and refreshes its
 * dynamic state with kernels, and reads back one flag word per brick; the
 * packed atlas is quantised on the device. Regions (server L2), nested
 * feedback, atlases by key and the analysis codec are not part of this
 * library. Return convention as the reference: 1 ok, 0 error (message by
 * aero_lbm_simulation_last_error), counts -1 on error. */
typedef struct AeroLbmWorldDelta {
    int type;
    int x;
    int y;
    int z;
    int data0;
    int data1;
    int data2;
    int data3;
    float value0;
    float value1;
    float value2;
    float value3;
} AeroLbmWorldDelta;

/* capi.h:303-304 */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_create_service(long long* out_service_key);
AERO_LBM_B200_EXPORT void aero_lbm_simulation_release_service(long long service_key);
/* capi.h:305-311 */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_set_focus(long long service_key, int block_x, int block_y, int block_z,
                                                       int radius_blocks);
/* capi.h:312-316: brick deltas (types 1-5, 8 cell patch, 9 queued upload, 10
 * source patch) apply at the world's next step; type 6 drops the world */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_submit_world_deltas(long long service_key, const AeroLbmWorldDelta* deltas,
                                                                 int delta_count);
/* capi.h:317-323 */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_ensure_brick_world_runtime(long long service_key, long long world_key,
                                                                        int brick_size, float dx_meters, float dt_seconds);
/* capi.h:324-328 */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_set_brick_world_solver_mode(long long service_key, long long world_key,
                                                                         int solver_mode);
/* capi.h:329-342 */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_set_brick_world_active_hints(long long service_key, long long world_key,
                                                                          int brick_size, const int* brick_coords,
                                                                          int brick_count);
AERO_LBM_B200_EXPORT int aero_lbm_simulation_set_brick_world_exact_active_hints(long long service_key, long long world_key,
                                                                                int brick_size, const int* brick_coords,
                                                                                int brick_count);
/* capi.h:343-348: status[8] = brick size, bricks, hinted, active,
 * geometry-dirty, forcing-dirty, pending re-init, epoch */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_get_brick_world_runtime_status(long long service_key, long long world_key,
                                                                            int* out_status, int status_count);
/* capi.h:349-353 */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_step_brick_world_runtime(long long service_key, long long world_key,
                                                                      int step_count);
/* capi.h:354-373 */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_get_brick_world_resident_brick_count(long long service_key, long long world_key);
AERO_LBM_B200_EXPORT int aero_lbm_simulation_copy_brick_world_resident_bricks(long long service_key, long long world_key,
                                                                              int* out_coords, int brick_capacity);
AERO_LBM_B200_EXPORT int aero_lbm_simulation_get_brick_world_active_brick_count(long long service_key, long long world_key);
AERO_LBM_B200_EXPORT int aero_lbm_simulation_copy_brick_world_active_bricks(long long service_key, long long world_key,
                                                                            int* out_coords, int brick_capacity);
/* capi.h:374-417 */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_upload_brick_world_static_brick(
    long long service_key, long long world_key, int brick_size, int brick_x, int brick_y, int brick_z,
    const uint8_t* obstacle, const uint8_t* surface_kind, const uint16_t* open_face_mask, const float* emitter_power_watts,
    const uint8_t* face_sky_exposure, const uint8_t* face_direct_exposure);
AERO_LBM_B200_EXPORT int aero_lbm_simulation_upload_brick_world_static_brick_with_sources(
    long long service_key, long long world_key, int brick_size, int brick_x, int brick_y, int brick_z,
    const uint8_t* obstacle, const uint8_t* surface_kind, const uint16_t* open_face_mask, const float* emitter_power_watts,
    const uint8_t* source_fan_dir, const float* source_emitter_power_watts, const uint8_t* face_sky_exposure,
    const uint8_t* face_direct_exposure);
AERO_LBM_B200_EXPORT int aero_lbm_simulation_queue_brick_world_static_brick_upload(
    long long service_key, long long world_key, int brick_size, int brick_x, int brick_y, int brick_z,
    const uint8_t* obstacle, const uint8_t* surface_kind, const uint16_t* open_face_mask, const float* emitter_power_watts,
    const uint8_t* face_sky_exposure, const uint8_t* face_direct_exposure);
/* capi.h:435-456 */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_copy_brick_world_dynamic_brick(long long service_key, long long world_key,
                                                                            int brick_size, int brick_x, int brick_y,
                                                                            int brick_z, float* out_flow_state,
                                                                            float* out_air_temperature,
                                                                            float* out_surface_temperature);
AERO_LBM_B200_EXPORT int aero_lbm_simulation_copy_brick_world_packed_flow_atlas(long long service_key, long long world_key,
                                                                                int brick_size, int brick_x, int brick_y,
                                                                                int brick_z, int sample_stride,
                                                                                int16_t* out_packed_flow,
                                                                                int packed_value_count);
/* capi.h:457-466 (dynamic upload: simulation_bridge.cpp:5412-5477) */
AERO_LBM_B200_EXPORT int aero_lbm_simulation_upload_brick_world_dynamic_brick(long long service_key, long long world_key,
                                                                              int brick_size, int brick_x, int brick_y,
                                                                              int brick_z, const float* flow_state,
                                                                              const float* air_temperature,
                                                                              const float* surface_temperature);
AERO_LBM_B200_EXPORT int aero_lbm_simulation_upload_brick_world_boundary_reference_brick(
    long long service_key, long long world_key, int brick_size, int brick_x, int brick_y, int brick_z,
    const float* flow_state, const float* air_temperature, const float* surface_temperature);
/* capi.h:695-696 */
AERO_LBM_B200_EXPORT const char* aero_lbm_simulation_runtime_info(void);
AERO_LBM_B200_EXPORT const char* aero_lbm_simulation_last_error(void);

/* ---- wind-tunnel ABI (native/include/aero_solver_capi.h:1-115) ---- */
enum {
    AERO_SOLVER_ABI_VERSION = 1,
    AERO_SOLVER_FLOW_CHANNELS = 4,
    AERO_SOLVER_STATUS_OK = 1,
    AERO_SOLVER_STATUS_ERROR = 0
};

typedef enum AeroSolverBoundaryMode {
    AERO_SOLVER_BOUNDARY_WIND_TUNNEL = 1,
    AERO_SOLVER_BOUNDARY_WIND_TUNNEL_PRESSURE_OUTLET = 2,
    AERO_SOLVER_BOUNDARY_CLOSED = 3,
    AERO_SOLVER_BOUNDARY_PERIODIC = 4
} AeroSolverBoundaryMode;

typedef struct AeroGridDesc {
    int nx;
    int ny;
    int nz;
    float dx;
    float dt;
} AeroGridDesc;

typedef struct AeroBoundaryDesc {
    int mode;
    float inlet_vx;
    float inlet_vy;
    float inlet_vz;
    float outlet_pressure;
    float density;
    float viscosity;
} AeroBoundaryDesc;

typedef struct AeroStepInput {
    const uint8_t* solid_mask;
    const float* prev_flow;
    AeroGridDesc grid;
    AeroBoundaryDesc boundary;
    int steps;
} AeroStepInput;

typedef struct AeroStepOutput {
    float* flow_out;
    float max_velocity;
    int status;
} AeroStepOutput;

/* native/include/aero_solver_capi.h:58-109 (aero_solver_capi.cpp:333-587) */
AERO_LBM_B200_EXPORT void aero_solver_default_grid(AeroGridDesc* out_grid);
AERO_LBM_B200_EXPORT void aero_solver_default_boundary(AeroBoundaryDesc* out_boundary);
AERO_LBM_B200_EXPORT int aero_solver_create(int nx, int ny, int nz, float dx, float dt, long long* out_handle);
AERO_LBM_B200_EXPORT int aero_solver_create_with_grid(const AeroGridDesc* grid, long long* out_handle);
AERO_LBM_B200_EXPORT int aero_solver_set_solid_mask(long long handle, const uint8_t* solid_mask, int cell_count);
AERO_LBM_B200_EXPORT int aero_solver_set_flow_state(long long handle, const float* flow, int value_count);
AERO_LBM_B200_EXPORT int aero_solver_step_wind_tunnel(long long handle, const AeroBoundaryDesc* boundary, int steps,
                                                      float* out_flow, int out_value_count);
AERO_LBM_B200_EXPORT int aero_solver_advance_wind_tunnel(long long handle, const AeroBoundaryDesc* boundary, int steps);
AERO_LBM_B200_EXPORT int aero_solver_run_wind_tunnel(const AeroStepInput* input, AeroStepOutput* output);
AERO_LBM_B200_EXPORT void aero_solver_destroy(long long handle);
AERO_LBM_B200_EXPORT const char* aero_solver_last_error(void);
AERO_LBM_B200_EXPORT const char* aero_solver_runtime_info(void);
AERO_LBM_B200_EXPORT int aero_solver_finish(void);

#ifdef __cplusplus
}
#endif

#endif
