// Host runtime of the per-context LBM C ABI: context registry, benchmark /
// boundary configuration, parameter derivation, step dispatch, output.
//
// Behaviour follows the reference runtime (native/src/aero_lbm_jni.cpp):
// contexts keyed by a caller-chosen long long (jni.cpp:516-611), a process
// global boundary configuration (jni.cpp:229-489), the effective-parameter
// rules (jni.cpp:722-1118), init/step/extract entry points (jni.cpp:8592-10368).
// There is no CPU fallback: every path runs the CUDA kernels and reports
// failure through aero_lbm_last_error().
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_fp16.h>

#include "../../include/aero_lbm_b200.h"
#include "d3q27_kernels.cuh"
#include "ip_launch.h"
#include "conservation.cuh"
#include "context_ops.cuh"
#include "edits.cuh"
#include "halo.cuh"
#include "runtime_internal.h"
#include "thermal.cuh"

namespace aero {

// ------------------------------------------------------------------ globals
namespace {

struct RuntimeConfig {
    bool initialized = false;
    int nx = 0, ny = 0, nz = 0;
    int input_channels = 0, output_channels = 0;
    std::string runtime_info = "uninitialized";
};

struct TimingStats {
    uint64_t ticks = 0;
    double last_copy = 0, last_solver = 0, last_readback = 0, last_total = 0;
    double sum_copy = 0, sum_solver = 0, sum_readback = 0, sum_total = 0;
    uint64_t full_packet_steps = 0, cached_steps = 0;
};

RuntimeConfig g_cfg;
std::recursive_mutex g_mutex;  // guards every entry point (the caller is one worker thread)
// Arguments of each context's deferred face pre-fill (Context::fill_pending).
std::unordered_map<const Context*, IpArgs> g_fill_args;
void drop_pending_fill(Context& ctx) {
    ctx.fill_pending = false;
    g_fill_args.erase(&ctx);
}

// Tuning knobs (aero_lbm_b200_set_*), at their defaults; reset_tuning()
// restores exactly these values.
int g_thermal_mode = -1;      // temperature transport: -1 with buoyancy, 0 never (packet field), 1 always
int g_streamed_step = 0;      // factorised two-cell in-place step: bulk-copy streamed kernel where eligible (opt-in)
int g_fused_transport = 0;    // in-place steps compute the first-order temperature transport themselves (opt-in)
int g_cells_per_thread = 2;    // in-place step: 1 one cell per thread, 2 two cells per thread (packed collision)
int g_fp16_format = 1;         // 16-bit storage: 0 IEEE half deviations, 1 fixed-point deviations (default)
std::unordered_map<long long, std::unique_ptr<Context>> g_contexts;
std::string g_last_error;
std::string g_timing_text;
std::string g_bench_text;
TimingStats g_timing;
AeroLbmBenchmarkConfig g_bench{};
bool g_bench_ready = false;
cudaStream_t g_stream = nullptr;
bool g_own_stream = false;
int g_stream_mode = 0;  // 0 auto, 1 two-buffer, 2 in-place
int g_collision_mode = 0;  // 0 reference-order (bit-exact), 1 factorised
float g_smagorinsky_c = -1.0f;
float g_buoyancy_beta_override = -1.0f;
int g_gravity_axis = -1;
int g_realtime_solver_mode = AERO_LBM_REALTIME_SOLVER_AUTO;

using Clock = std::chrono::steady_clock;
double ms_since(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

inline float finite_or(float v, float fb) { return std::isfinite(v) ? v : fb; }
inline float clampf_h(float v, float lo, float hi) { return std::min(hi, std::max(lo, v)); }

// Reference runtime constants (jni.cpp:83-168), evaluated in float.
constexpr float kCs2 = 1.0f / 3.0f;
constexpr float kRuntimeMolecularNu0 = 1.50e-5f * (1.0f / 20.0f) / (1.0f * 1.0f);
constexpr float kNuMin = 1.0e-8f;
constexpr float kNuMax = (0.95f - 0.5f) / 3.0f;
constexpr float kTauMinH = 0.5f + 3.0f * 1.0e-8f;
constexpr float kTauMaxH = 0.95f;
constexpr float kTauNormalGame = 0.5f + 3.0f * kRuntimeMolecularNu0;
constexpr float kSgsCDefault = 0.025f;
constexpr float kSgsNutToNu0Max = 5.0f;
constexpr float kSgsBulkCoupling = 0.30f;
constexpr float kBoussinesqBeta = 9.81f * (1.0f / 300.0f) * 20.0f * ((1.0f / 20.0f) * (1.0f / 20.0f) / 1.0f);
constexpr float kBoussinesqForceMax = 0.02f;
constexpr float kThermalDiffusivity = 0.035f;  // benchmark-mode scalar diffusivity (jni.cpp:154)
constexpr float kMaxSpeed = 0.57735026919f * 0.60f;
constexpr uint32_t kKnownFlags = 0xffu;

AeroLbmBoundaryFaceConfig make_face(int hydro, int thermal) {
    AeroLbmBoundaryFaceConfig f{};
    f.hydrodynamic_kind = hydro;
    f.thermal_kind = thermal;
    return f;
}

void set_all_faces(AeroLbmBenchmarkConfig& c, int hydro, int thermal) {
    c.x_min = c.x_max = c.y_min = c.y_max = c.z_min = c.z_max = make_face(hydro, thermal);
}

// make_default_benchmark_config (jni.cpp:304-338)
AeroLbmBenchmarkConfig default_config() {
    AeroLbmBenchmarkConfig c{};
    c.abi_version = AERO_LBM_BENCHMARK_ABI_VERSION;
    c.struct_size = sizeof(AeroLbmBenchmarkConfig);
    c.flags = AERO_LBM_BENCHMARK_FLAG_DISABLE_FAN_FORCING | AERO_LBM_BENCHMARK_FLAG_DISABLE_FAN_NOISE |
              AERO_LBM_BENCHMARK_FLAG_DISABLE_SPONGE | AERO_LBM_BENCHMARK_FLAG_DISABLE_OBSTACLE_BOUNCE_BLEND |
              AERO_LBM_BENCHMARK_FLAG_DISABLE_SGS;
    c.enabled = 0;
    c.preset = AERO_LBM_BENCHMARK_PRESET_NONE;
    c.reynolds_number = 100.0f;
    c.rayleigh_number = 1.0e5f;
    c.prandtl_number = 0.71f;
    c.mach_number = 0.05f;
    c.reference_density = 1.0f;
    c.reference_temperature = 0.0f;
    c.reference_length = 1.0f;
    c.gravity[1] = -1.0f;
    set_all_faces(c, AERO_LBM_HYDRO_BOUNDARY_INHERIT_GAME, AERO_LBM_THERMAL_BOUNDARY_INHERIT_GAME);
    return c;
}

bool valid_preset(int p) { return p >= AERO_LBM_BENCHMARK_PRESET_NONE && p <= AERO_LBM_BENCHMARK_PRESET_DIFFERENTIALLY_HEATED_CAVITY_3D; }
bool valid_hydro(int k) { return k >= 0 && k <= 7; }
bool valid_thermal(int k) { return k >= 0 && k <= 5; }

void sanitize_face(AeroLbmBoundaryFaceConfig& f) {
    if (!valid_hydro(f.hydrodynamic_kind)) f.hydrodynamic_kind = AERO_LBM_HYDRO_BOUNDARY_INHERIT_GAME;
    if (!valid_thermal(f.thermal_kind)) f.thermal_kind = AERO_LBM_THERMAL_BOUNDARY_INHERIT_GAME;
    for (float& v : f.velocity) v = finite_or(v, 0.0f);
    f.pressure = finite_or(f.pressure, 0.0f);
    f.temperature = finite_or(f.temperature, 0.0f);
    f.heat_flux = finite_or(f.heat_flux, 0.0f);
}

// sanitize_benchmark_config (jni.cpp:408-440)
void sanitize(AeroLbmBenchmarkConfig& c) {
    c.abi_version = AERO_LBM_BENCHMARK_ABI_VERSION;
    c.struct_size = sizeof(AeroLbmBenchmarkConfig);
    c.flags &= kKnownFlags;
    c.enabled = c.enabled != 0 ? 1 : 0;
    if (!valid_preset(c.preset)) c.preset = AERO_LBM_BENCHMARK_PRESET_NONE;
    c.reynolds_number = finite_or(c.reynolds_number, 100.0f);
    c.rayleigh_number = finite_or(c.rayleigh_number, 1.0e5f);
    c.prandtl_number = finite_or(c.prandtl_number, 0.71f);
    c.mach_number = clampf_h(finite_or(c.mach_number, 0.05f), 1.0e-4f, 0.30f);
    c.reference_density = finite_or(c.reference_density, 1.0f);
    c.reference_temperature = finite_or(c.reference_temperature, 0.0f);
    c.reference_length = std::max(1.0e-6f, finite_or(c.reference_length, 1.0f));
    for (float& v : c.body_force) v = finite_or(v, 0.0f);
    c.gravity[0] = finite_or(c.gravity[0], 0.0f);
    c.gravity[1] = finite_or(c.gravity[1], -1.0f);
    c.gravity[2] = finite_or(c.gravity[2], 0.0f);
    for (float& v : c.initial_velocity) v = finite_or(v, 0.0f);
    c.initial_pressure = finite_or(c.initial_pressure, 0.0f);
    c.initial_temperature = finite_or(c.initial_temperature, 0.0f);
    sanitize_face(c.x_min); sanitize_face(c.x_max);
    sanitize_face(c.y_min); sanitize_face(c.y_max);
    sanitize_face(c.z_min); sanitize_face(c.z_max);
}

// apply_benchmark_preset_defaults (jni.cpp:340-407)
AeroLbmBenchmarkConfig preset_config(int preset) {
    AeroLbmBenchmarkConfig c = default_config();
    c.enabled = 1;
    c.preset = preset;
    switch (preset) {
        case AERO_LBM_BENCHMARK_PRESET_TAYLOR_GREEN_3D:
            c.flags |= AERO_LBM_BENCHMARK_FLAG_DISABLE_CONVECTIVE_OUTFLOW | AERO_LBM_BENCHMARK_FLAG_DISABLE_INTERNAL_THERMAL_SOURCE |
                       AERO_LBM_BENCHMARK_FLAG_DISABLE_BUOYANCY;
            set_all_faces(c, AERO_LBM_HYDRO_BOUNDARY_PERIODIC, AERO_LBM_THERMAL_BOUNDARY_DISABLED);
            break;
        case AERO_LBM_BENCHMARK_PRESET_LID_DRIVEN_CAVITY_2D:
        case AERO_LBM_BENCHMARK_PRESET_LID_DRIVEN_CAVITY_3D:
            c.reynolds_number = 1000.0f;
            set_all_faces(c, AERO_LBM_HYDRO_BOUNDARY_BOUNCE_BACK, AERO_LBM_THERMAL_BOUNDARY_ADIABATIC);
            c.y_max = make_face(AERO_LBM_HYDRO_BOUNDARY_MOVING_WALL, AERO_LBM_THERMAL_BOUNDARY_ADIABATIC);
            c.y_max.velocity[0] = 0.10f;
            c.flags |= AERO_LBM_BENCHMARK_FLAG_DISABLE_INTERNAL_THERMAL_SOURCE | AERO_LBM_BENCHMARK_FLAG_DISABLE_BUOYANCY;
            if (preset == AERO_LBM_BENCHMARK_PRESET_LID_DRIVEN_CAVITY_2D) {
                c.z_min = make_face(AERO_LBM_HYDRO_BOUNDARY_PERIODIC, AERO_LBM_THERMAL_BOUNDARY_PERIODIC);
                c.z_max = make_face(AERO_LBM_HYDRO_BOUNDARY_PERIODIC, AERO_LBM_THERMAL_BOUNDARY_PERIODIC);
            }
            break;
        case AERO_LBM_BENCHMARK_PRESET_CYLINDER_CROSSFLOW_2D:
            c.reynolds_number = 100.0f;
            c.flags |= AERO_LBM_BENCHMARK_FLAG_DISABLE_INTERNAL_THERMAL_SOURCE | AERO_LBM_BENCHMARK_FLAG_DISABLE_BUOYANCY;
            set_all_faces(c, AERO_LBM_HYDRO_BOUNDARY_BOUNCE_BACK, AERO_LBM_THERMAL_BOUNDARY_DISABLED);
            c.x_min = make_face(AERO_LBM_HYDRO_BOUNDARY_VELOCITY_DIRICHLET, AERO_LBM_THERMAL_BOUNDARY_DISABLED);
            c.initial_velocity[0] = 0.08f;
            c.x_min.velocity[0] = 1.5f * 0.08f;
            c.x_max = make_face(AERO_LBM_HYDRO_BOUNDARY_CONVECTIVE_OUTFLOW, AERO_LBM_THERMAL_BOUNDARY_DISABLED);
            c.z_min = make_face(AERO_LBM_HYDRO_BOUNDARY_PERIODIC, AERO_LBM_THERMAL_BOUNDARY_PERIODIC);
            c.z_max = make_face(AERO_LBM_HYDRO_BOUNDARY_PERIODIC, AERO_LBM_THERMAL_BOUNDARY_PERIODIC);
            break;
        case AERO_LBM_BENCHMARK_PRESET_DIFFERENTIALLY_HEATED_CAVITY_2D:
        case AERO_LBM_BENCHMARK_PRESET_DIFFERENTIALLY_HEATED_CAVITY_3D:
            c.rayleigh_number = 1.0e5f;
            c.prandtl_number = 0.71f;
            c.mach_number = 0.15f;
            c.flags |= AERO_LBM_BENCHMARK_FLAG_DISABLE_INTERNAL_THERMAL_SOURCE;
            set_all_faces(c, AERO_LBM_HYDRO_BOUNDARY_BOUNCE_BACK, AERO_LBM_THERMAL_BOUNDARY_ADIABATIC);
            c.x_min = make_face(AERO_LBM_HYDRO_BOUNDARY_BOUNCE_BACK, AERO_LBM_THERMAL_BOUNDARY_TEMPERATURE_DIRICHLET);
            c.x_min.temperature = 0.5f;
            c.x_max = make_face(AERO_LBM_HYDRO_BOUNDARY_BOUNCE_BACK, AERO_LBM_THERMAL_BOUNDARY_TEMPERATURE_DIRICHLET);
            c.x_max.temperature = -0.5f;
            if (preset == AERO_LBM_BENCHMARK_PRESET_DIFFERENTIALLY_HEATED_CAVITY_2D) {
                c.z_min = make_face(AERO_LBM_HYDRO_BOUNDARY_PERIODIC, AERO_LBM_THERMAL_BOUNDARY_PERIODIC);
                c.z_max = make_face(AERO_LBM_HYDRO_BOUNDARY_PERIODIC, AERO_LBM_THERMAL_BOUNDARY_PERIODIC);
            }
            break;
        default:
            c.enabled = 0;
            c.preset = AERO_LBM_BENCHMARK_PRESET_NONE;
            break;
    }
    return c;
}

void ensure_bench() {
    if (!g_bench_ready) {
        g_bench = default_config();
        g_bench_ready = true;
    }
}

bool bench_active() { return g_bench.enabled != 0; }
bool bench_flag(uint32_t flag) { return bench_active() && (g_bench.flags & flag) != 0; }
bool heated_cavity() {
    return bench_active() && (g_bench.preset == AERO_LBM_BENCHMARK_PRESET_DIFFERENTIALLY_HEATED_CAVITY_2D ||
                              g_bench.preset == AERO_LBM_BENCHMARK_PRESET_DIFFERENTIALLY_HEATED_CAVITY_3D);
}
float norm3(const float* v) { return std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

const AeroLbmBoundaryFaceConfig& face_cfg(int i) {
    switch (i) {
        case 0: return g_bench.x_min;
        case 1: return g_bench.x_max;
        case 2: return g_bench.y_min;
        case 3: return g_bench.y_max;
        case 4: return g_bench.z_min;
        default: return g_bench.z_max;
    }
}

// benchmark_reference_speed (jni.cpp:831-871)
float reference_speed() {
    if (!bench_active()) return 0.0f;
    if (heated_cavity()) return clampf_h(finite_or(g_bench.mach_number, 0.05f), 1.0e-4f, 0.30f) * std::sqrt(kCs2);
    if (g_bench.preset == AERO_LBM_BENCHMARK_PRESET_CYLINDER_CROSSFLOW_2D) {
        const float s = norm3(g_bench.initial_velocity);
        if (s > 1.0e-8f) return s;
        return (2.0f / 3.0f) * norm3(g_bench.x_min.velocity);
    }
    float s = norm3(g_bench.initial_velocity);
    for (int i = 0; i < 6; ++i) s = std::max(s, norm3(face_cfg(i).velocity));
    return s;
}

float clamp_nu(float nu) { return clampf_h(nu, kNuMin, kNuMax); }

// effective_base_nu_shear (jni.cpp:947-961)
float base_nu_shear() {
    if (!bench_active()) return clamp_nu(kRuntimeMolecularNu0);
    if (heated_cavity()) {
        const float ra = std::max(1.0e-6f, finite_or(g_bench.rayleigh_number, 1.0e5f));
        const float pr = std::max(1.0e-6f, finite_or(g_bench.prandtl_number, 0.71f));
        const float len = std::max(1.0e-6f, finite_or(g_bench.reference_length, 1.0f));
        return clamp_nu(reference_speed() * len * std::sqrt(pr / ra));
    }
    const float re = finite_or(g_bench.reynolds_number, 0.0f);
    const float sp = reference_speed();
    const float len = std::max(1.0e-6f, finite_or(g_bench.reference_length, 1.0f));
    if (re <= 1.0e-6f || sp <= 1.0e-8f) return clamp_nu(kRuntimeMolecularNu0);
    return clamp_nu(sp * len / re);
}

float tau_shear_base() { return clampf_h(0.5f + 3.0f * clamp_nu(base_nu_shear()), kTauMinH, kTauMaxH); }
float tau_normal_base() {
    if (!bench_active()) return clampf_h(kTauNormalGame, kTauMinH, kTauMaxH);
    return clampf_h(0.5f + 3.0f * clamp_nu(clamp_nu(base_nu_shear())), kTauMinH, kTauMaxH);
}

// effective_boussinesq_beta (jni.cpp:1023-1031)
float boussinesq_beta() {
    if (g_buoyancy_beta_override >= 0.0f) return g_buoyancy_beta_override;
    if (!heated_cavity()) return kBoussinesqBeta;
    const float sp = reference_speed();
    const float len = std::max(1.0e-6f, finite_or(g_bench.reference_length, 1.0f));
    float tmin = 1.0e9f, tmax = -1.0e9f;
    bool any = false;
    for (int i = 0; i < 6; ++i) {
        const auto& f = face_cfg(i);
        if (f.thermal_kind != AERO_LBM_THERMAL_BOUNDARY_TEMPERATURE_DIRICHLET) continue;
        any = true;
        tmin = std::min(tmin, f.temperature);
        tmax = std::max(tmax, f.temperature);
    }
    const float span = any ? std::max(1.0e-6f, tmax - tmin) : 1.0f;
    return (sp * sp) / std::max(1.0e-6f, len * span);
}

}  // namespace

// ------------------------------------------------------------------ shared helpers
std::recursive_mutex& runtime_mutex() { return g_mutex; }

void set_error(const std::string& msg) { g_last_error = msg; }
void clear_error() { g_last_error.clear(); }
const std::string& last_error() { return g_last_error; }

cudaStream_t current_stream() {
    if (!g_stream) {
        if (cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking) == cudaSuccess) g_own_stream = true;
        else g_stream = nullptr;
    }
    return g_stream;
}

bool cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

CollideParams current_collide_params() {
    ensure_bench();
    CollideParams p{};
    p.tau_shear_base = tau_shear_base();
    p.tau_normal_base = tau_normal_base();
    p.nu0 = std::max(1e-6f, base_nu_shear());
    const float c = g_smagorinsky_c >= 0.0f ? g_smagorinsky_c : kSgsCDefault;
    p.sgs_c2 = c * c;
    p.sgs_nut_cap = kSgsNutToNu0Max * p.nu0;
    p.sgs_bulk = kSgsBulkCoupling;
    p.buoy_beta = boussinesq_beta();
    p.buoy_fmax = kBoussinesqForceMax;
    p.body_force[0] = p.body_force[1] = p.body_force[2] = 0.0f;
    if (bench_active()) {
        // The reference sanitises but never applies body_force; here it is a
        // uniform force density on every fluid cell.
        p.body_force[0] = g_bench.body_force[0];
        p.body_force[1] = g_bench.body_force[1];
        p.body_force[2] = g_bench.body_force[2];
    }
    p.max_speed = kMaxSpeed;
    p.enable_sgs = !bench_flag(AERO_LBM_BENCHMARK_FLAG_DISABLE_SGS);
    p.enable_buoyancy = !bench_flag(AERO_LBM_BENCHMARK_FLAG_DISABLE_BUOYANCY);
    p.gravity_axis = g_gravity_axis >= 0 ? g_gravity_axis : 1;
    // game-runtime terms (effective_enable_fan_forcing / _fan_noise_amp /
    // _sponge_alpha / _runtime_state_nudge, jni.cpp:676-822): on outside
    // benchmark mode, and in benchmark mode when their DISABLE flag is clear
    p.fan_beta = bench_flag(AERO_LBM_BENCHMARK_FLAG_DISABLE_FAN_FORCING) ? 0.0f : 0.07f;
    p.fan_noise_amp = bench_flag(AERO_LBM_BENCHMARK_FLAG_DISABLE_FAN_NOISE) ? 0.0f : 0.02f;
    p.fan_target_scale = 1.0f / (1.0f / (1.0f / 20.0f));
    p.sponge = bench_flag(AERO_LBM_BENCHMARK_FLAG_DISABLE_SPONGE) ? 0 : 1;
    p.state_nudge = bench_active() ? 0.0f : 0.08f;
    p.runtime_terms = (p.fan_beta > 0.0f || p.sponge || p.state_nudge > 0.0f) ? 1 : 0;
    return p;
}

FaceParams current_face_params() {
    ensure_bench();
    FaceParams f{};
    for (int i = 0; i < 6; ++i) {
        const auto& c = face_cfg(i);
        f.kind[i] = c.hydrodynamic_kind;
        f.velocity[i][0] = c.velocity[0];
        f.velocity[i][1] = c.velocity[1];
        f.velocity[i][2] = c.velocity[2];
        f.pressure[i] = c.pressure;
    }
    for (int a = 0; a < 3; ++a) {
        f.wrap_lo[a] = f.kind[2 * a] == kHydroPeriodic;
        f.wrap_hi[a] = f.kind[2 * a + 1] == kHydroPeriodic;
        if (f.wrap_lo[a] && f.wrap_hi[a]) f.periodic_mask |= 1 << a;
    }
    f.disable_convective = bench_flag(AERO_LBM_BENCHMARK_FLAG_DISABLE_CONVECTIVE_OUTFLOW) ? 1 : 0;
    f.max_speed = kMaxSpeed;
    f.cylinder_inlet = (bench_active() && g_bench.preset == AERO_LBM_BENCHMARK_PRESET_CYLINDER_CROSSFLOW_2D) ? 1 : 0;
    return f;
}

int streaming_mode_setting() { return g_stream_mode; }
int realtime_solver_mode() { return g_realtime_solver_mode; }

// ------------------------------------------------------------------ contexts
Context::~Context() { release_device(); }

void Context::release_device() {
    auto fr = [](void*& p) {
        if (p) cudaFree(p);
        p = nullptr;
    };
    for (int i = 0; i < 2; ++i) {
        fr(reinterpret_cast<void*&>(g[i]));
        fr(reinterpret_cast<void*&>(obstacle[i]));
        fr(reinterpret_cast<void*&>(ref_p[i]));
        fr(reinterpret_cast<void*&>(flags[i]));
        fr(reinterpret_cast<void*&>(d_face[i]));
    }
    fr(reinterpret_cast<void*&>(ref_ux));
    fr(reinterpret_cast<void*&>(ref_uy));
    fr(reinterpret_cast<void*&>(ref_uz));
    fr(reinterpret_cast<void*&>(temperature));
    fr(reinterpret_cast<void*&>(temperature_next));
    fr(reinterpret_cast<void*&>(temperature_scratch));
    fr(reinterpret_cast<void*&>(ref_temperature));
    fr(reinterpret_cast<void*&>(thermal_source));
    fr(reinterpret_cast<void*&>(u_last));
    thermal = false;
    fr(reinterpret_cast<void*&>(packet));
    fr(reinterpret_cast<void*&>(out));
    fr(reinterpret_cast<void*&>(force));
    fr(reinterpret_cast<void*&>(fault));
    fr(reinterpret_cast<void*&>(force3));
    fr(reinterpret_cast<void*&>(overlay_cells));
    fr(reinterpret_cast<void*&>(overlay_values));
    overlay_cap = 0;
    fr(reinterpret_cast<void*&>(patch_cells));
    fr(reinterpret_cast<void*&>(patch_solid));
    patch_cap = 0;
    pending_slot = -1;
    fr(shell);
    shell_count = 0;
    force_valid = false;
    f_ready = false;
    fr(ip);
    fr(reinterpret_cast<void*&>(solid_f));
    fr(reinterpret_cast<void*&>(fan_mask));
    if (copy_done) cudaEventDestroy(copy_done);
    copy_done = nullptr;
    drop_pending_fill(*this);
    fr(scratch);
    scratch_cap = 0;
    packet_cap = out_cap = 0;
    layout = 0;
    parity = 0;
    allocated = false;
    initialized = false;
}

bool Context::allocate(int nx_, int ny_, int nz_) {
    release_device();
    nx = nx_; ny = ny_; nz = nz_;
    cells = (long long)nx * ny * nz;
    if (cudaGetDevice(&device) != cudaSuccess) device = -1;
    const size_t c = (size_t)cells;
    auto al = [&](void** p, size_t bytes) { return cuda_ok(cudaMalloc(p, bytes + kCopySlack), "cudaMalloc"); };
    bool ok = true;
    for (int i = 0; i < 2 && ok; ++i) {
        ok = ok && al(reinterpret_cast<void**>(&obstacle[i]), c);
        ok = ok && al(reinterpret_cast<void**>(&ref_p[i]), c * sizeof(float));
        ok = ok && al(reinterpret_cast<void**>(&flags[i]), c * sizeof(uint32_t));
        ok = ok && al(reinterpret_cast<void**>(&d_face[i]), sizeof(FaceParams));
    }
    ok = ok && al(reinterpret_cast<void**>(&ref_ux), c * sizeof(float));
    ok = ok && al(reinterpret_cast<void**>(&ref_uy), c * sizeof(float));
    ok = ok && al(reinterpret_cast<void**>(&ref_uz), c * sizeof(float));
    ok = ok && al(reinterpret_cast<void**>(&temperature), c * sizeof(float));
    ok = ok && cuda_ok(cudaMemsetAsync(temperature, 0, c * sizeof(float), current_stream()), "cudaMemset(temperature)");
    ok = ok && al(reinterpret_cast<void**>(&fault), sizeof(int));
    ok = ok && cuda_ok(cudaMemsetAsync(fault, 0, sizeof(int), current_stream()), "cudaMemset(fault)");
    if (!ok) {
        release_device();
        return false;
    }
    allocated = true;
    initialized = false;
    f_ready = false;
    force_valid = false;
    slot = 0;
    cur = 0;
    step_counter = 0;
    return true;
}

CellFields Context::fields(int s) const {
    CellFields c{obstacle[s], ref_ux, ref_uy, ref_uz, ref_p[s], temperature};
    if (fan_mask) {
        c.fan_mask = fan_mask;
        c.fan_ux = fan_mask + cells;
        c.fan_uy = fan_mask + 2 * cells;
        c.fan_uz = fan_mask + 3 * cells;
    }
    if (thermal) {
        c.ref_temperature = ref_temperature;
        c.thermal_source = thermal_source;
        c.u_last = u_last;
        c.cells = cells;
    }
    return c;
}

ForceField Context::force_field() const {
    if (!force) return ForceField{nullptr, nullptr, nullptr};
    return ForceField{force, force + cells, force + 2 * cells};
}

Context* find_context(long long key) {
    auto it = g_contexts.find(key);
    return it == g_contexts.end() ? nullptr : it->second.get();
}

Context* get_or_create_context(long long key, int nx, int ny, int nz) {
    auto& slot = g_contexts[key];
    if (!slot) slot = std::make_unique<Context>();
    Context* c = slot.get();
    if (!c->allocated || c->nx != nx || c->ny != ny || c->nz != nz) {
        if (!c->allocate(nx, ny, nz)) {
            g_contexts.erase(key);
            return nullptr;
        }
    }
    return c;
}

void release_all_contexts() {
    g_contexts.clear();
}

const RuntimeView runtime_view() {
    return RuntimeView{g_cfg.initialized, g_cfg.nx, g_cfg.ny, g_cfg.nz, g_cfg.input_channels, g_cfg.output_channels};
}

// Faces the in-place layout takes: periodic on both sides of an axis,
// bounce-back, and the faces whose pulled values the end-of-call fill writes
// (equilibrium faces, symmetry, convective outflow: face_fill_ip_kernel). The
// cylinder preset stays on the two-buffer layout, whose state its
// momentum-exchange force reads.
static bool inplace_faces_ok(const FaceParams& f) {
    for (int a = 0; a < 3; ++a)
        if (f.wrap_lo[a] != f.wrap_hi[a]) return false;
    return !(bench_active() && g_bench.preset == AERO_LBM_BENCHMARK_PRESET_CYLINDER_CROSSFLOW_2D);
}

// Some face needs the end-of-call fill (a kind other than periodic and
// bounce-back, which the step kernel resolves itself).
// fill_face_mask: those faces (bit f), the set the fill visits.
static unsigned fill_face_mask(const FaceParams& f) {
    unsigned m = 0;
    for (int i = 0; i < 6; ++i) {
        const int k = f.kind[i];
        if (k == kHydroPeriodic || k == kHydroBounceBack) continue;
        if (k == kHydroInheritGame && f.disable_convective) continue;
        m |= 1u << i;
    }
    return m;
}
static bool faces_need_fill(const FaceParams& f) { return fill_face_mask(f) != 0; }

// Storage of an in-place context for the kernels that take it as a number:
// 0 FP32, 1 IEEE-half deviations, 2 16-bit fixed point.
static int ip_storage(const Context& ctx) {
    return ctx.ip_variant == kIpF16Fast ? 1 : (ctx.ip_variant == kIpI16Fast ? 2 : 0);
}

bool join_fill(Context& ctx, cudaStream_t s) {
    if (!ctx.fill_pending) return true;
    auto it = g_fill_args.find(&ctx);
    ctx.fill_pending = false;
    if (it == g_fill_args.end()) return true;
    const IpArgs a = it->second;
    g_fill_args.erase(it);
    return cuda_ok(ip_fill(ctx.ip_variant, ctx.ip, a, s), "face_fill_inplace");
}

static IpArgs ip_args(Context& ctx, int stream_slot, int cur_slot, const CollideParams& cp) {
    IpArgs a{};
    a.g = make_pad_geom(ctx.nx, ctx.ny, ctx.nz, ctx.periodic_mask);
    a.flags_prev = ctx.flags[stream_slot];
    a.obstacle_cur = ctx.obstacle[cur_slot];
    a.ref_p_prev = ctx.ref_p[stream_slot];
    a.face_prev = ctx.d_face[stream_slot];
    a.cur = ctx.fields(cur_slot);
    a.force = ctx.force_field();
    a.cp = cp;
    a.sc = Fp16Scale{ctx.fp16_scale, ctx.fp16_scale > 0.0f ? 1.0f / ctx.fp16_scale : 0.0f};
    a.cells_per_thread = g_cells_per_thread;
    a.streamed = g_streamed_step;
    a.fault = ctx.fault;
    a.solid_f = ctx.solid_f;
    return a;
}

// Per-brick FP16 scale: a power of two S such that the normalised deviation
// (f - w)/w of the largest expected state (reference speed u, |rho - 1| <= 0.03,
// a non-equilibrium margin of 0.5) times S stays below 2^14.
float fp16_scale_for_speed(float umax) {
    umax = std::min(std::max(umax, 0.0f), 0.57735026919f * 0.6f);
    const float dev = 0.03f + 3.0f * 1.7320508f * umax + 15.0f * umax * umax + 0.5f;
    float s = 1.0f;
    while (s * 2.0f * dev < 16384.0f && s < 65536.0f) s *= 2.0f;
    return s;
}

// Per-brick 16-bit fixed-point scale S = 32767 / d_max: d_max bounds the
// normalised deviation |f - w| / w for speeds up to twice the brick's
// reference speed (flows over obstacles accelerate), with |rho - 1| <= 0.03
// and a non-equilibrium margin of 0.5; values beyond it saturate.
float i16_scale_for_speed(float umax) {
    umax = std::min(std::max(2.0f * umax, 0.02f), 0.57735026919f * 0.6f);
    const float dev = 0.03f + 3.0f * 1.7320508f * umax + 4.5f * 3.0f * umax * umax + 0.5f;
    return 32767.0f / dev;
}

// First step of a context: pick the layout, the in-place variant and allocate.
static bool choose_layout(Context& ctx, const FaceParams& face, const float* packet, bool host_packet, int in_slot) {
    const bool local = inplace_faces_ok(face);
    const bool want_fp16 = g_realtime_solver_mode == AERO_LBM_REALTIME_SOLVER_D3Q27_FP16_INPLACE_EXPERIMENTAL;
    int layout = 0;
    if (g_stream_mode == 2) {
        if (!local) {
            set_error("in-place streaming requested but an axis is periodic on one side only, or the cylinder preset is set");
            return false;
        }
        layout = 1;
    } else if (g_stream_mode == 0) {
        layout = local ? 1 : 0;
    }
    if (want_fp16 && local) layout = 1;
    ctx.layout = layout;
    const size_t c = (size_t)ctx.cells;
    if (layout == 0) {
        for (int i = 0; i < 2; ++i)
            if (!ctx.g[i] && !cuda_ok(cudaMalloc(reinterpret_cast<void**>(&ctx.g[i]), c * 27 * sizeof(float)), "cudaMalloc(populations)"))
                return false;
        ctx.bytes_per_step = (uint64_t)c * (27ull * 4 * 2 + 1);
        return true;
    }
    ctx.periodic_mask = face.periodic_mask;
    ctx.ip_variant = want_fp16 ? (g_fp16_format == 1 ? kIpI16Fast : kIpF16Fast)
                               : (g_collision_mode == 0 ? kIpF32Exact : kIpF32Fast);
    const bool half = ctx.ip_variant == kIpF16Fast || ctx.ip_variant == kIpI16Fast;
    const PadGeom g = make_pad_geom(ctx.nx, ctx.ny, ctx.nz, ctx.periodic_mask);
    const size_t elem = half ? 2 : 4;
    const size_t bytes = (size_t)g.pcells * 27 * elem;
    if ((long long)g.pcells * 27 >= (1LL << 31)) {
        set_error("in-place layout: brick too large for 32-bit slot indexing");
        return false;
    }
    if (!cuda_ok(cudaMalloc(&ctx.ip, bytes + kCopySlack), "cudaMalloc(in-place populations)")) return false;
    if (!cuda_ok(cudaMemsetAsync(ctx.ip, 0, bytes, current_stream()), "cudaMemset(in-place)")) return false;
    ctx.bytes_per_step = (uint64_t)c * (27ull * elem * 2 + 1);
    if (half) {
        float umax = 0.0f;
        for (int i = 0; i < 6; ++i)
            umax = std::max(umax, std::sqrt(face.velocity[i][0] * face.velocity[i][0] + face.velocity[i][1] * face.velocity[i][1] +
                                            face.velocity[i][2] * face.velocity[i][2]));
        if (packet && host_packet) {
            const int in_ch = g_cfg.input_channels;
            for (size_t i = 0; i < c; ++i) {
                const float* p = packet + i * in_ch;
                if (p[0] > 0.5f) continue;
                const float s2 = p[5] * p[5] + p[6] * p[6] + p[7] * p[7];
                if (std::isfinite(s2)) umax = std::max(umax, std::sqrt(s2));
            }
        } else if (ctx.has_inputs) {
            // inputs that live on the device (a device packet or a device
            // build): the largest reference speed of the ingested fluid cells
            cudaStream_t s = current_stream();
            unsigned int* d_bits = nullptr;
            unsigned int bits = 0;
            const bool ok = cuda_ok(cudaMalloc(reinterpret_cast<void**>(&d_bits), sizeof(unsigned int)), "cudaMalloc(max speed)") &&
                            cuda_ok(cudaMemsetAsync(d_bits, 0, sizeof(unsigned int), s), "cudaMemset(max speed)") &&
                            cuda_ok(launch_max_fluid_speed(ctx.fields(in_slot), ctx.cells, d_bits, s), "max speed") &&
                            cuda_ok(cudaMemcpyAsync(&bits, d_bits, sizeof(unsigned int), cudaMemcpyDeviceToHost, s), "copy max speed") &&
                            cuda_ok(cudaStreamSynchronize(s), "sync max speed");
            if (d_bits) cudaFree(d_bits);
            if (!ok) return false;
            float dev_umax = 0.0f;
            std::memcpy(&dev_umax, &bits, sizeof(float));
            if (std::isfinite(dev_umax)) umax = std::max(umax, dev_umax);
        }
        ctx.fp16_scale = ctx.ip_variant == kIpI16Fast ? i16_scale_for_speed(umax) : fp16_scale_for_speed(umax);
    }
    return true;
}

// Build the pull classification of `slot` for faces `face` and keep a device
// copy of the faces for the kernels that stream with this slot.
static bool classify(Context& ctx, int slot, const FaceParams& face, const BrickDims& d, cudaStream_t s) {
    ctx.h_face[slot] = face;
    if (!cuda_ok(cudaMemcpyAsync(ctx.d_face[slot], &ctx.h_face[slot], sizeof(FaceParams), cudaMemcpyHostToDevice, s),
                 "upload faces")) return false;
    return cuda_ok(launch_build_flags(ctx.obstacle[slot], d, face, ctx.flags[slot], s), "build_flags");
}

// Temperature transport arrays of a context (allocated on first use).
static bool ensure_thermal(Context& ctx) {
    if (ctx.u_last) return true;
    const size_t c = (size_t)ctx.cells;
    auto al = [&](float** p, size_t n) {
        return cuda_ok(cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(float) + kCopySlack), "cudaMalloc(thermal)") &&
               cuda_ok(cudaMemsetAsync(*p, 0, n * sizeof(float), current_stream()), "cudaMemset(thermal)");
    };
    return al(&ctx.temperature_next, c) && al(&ctx.temperature_scratch, c) && al(&ctx.ref_temperature, c) &&
           al(&ctx.thermal_source, c) && al(&ctx.u_last, 3 * c);
}

// Thermal faces and diffusivity of the benchmark configuration
// (effective_thermal_diffusivity, jni.cpp:966-972).
static ThermalFaces current_thermal_faces() {
    ThermalFaces t{};
    for (int i = 0; i < 6; ++i) {
        const auto& c = face_cfg(i);
        t.kind[i] = c.thermal_kind;
        t.temperature[i] = c.temperature;
        t.heat_flux[i] = c.heat_flux;
    }
    return t;
}
static float thermal_diffusivity() {
    // runtime_molecular_alpha0 (jni.cpp:931-933): air's diffusivity nu / Pr in lattice units
    if (!bench_active()) return std::max(1.0e-8f, (1.50e-5f / 0.71f) * (1.0f / 20.0f) / (1.0f * 1.0f));
    if (!heated_cavity()) return kThermalDiffusivity;
    const float pr = std::max(1.0e-6f, finite_or(g_bench.prandtl_number, 0.71f));
    return base_nu_shear() / pr;
}

// One step of a context. packet may be null (cached step); out may be null.
static bool step_context_body(Context& ctx, const float* packet, float* out, float scale, bool host_packet,
                              const SparseOverlays* overlays, const DeviceFill* fill);

bool step_context(Context& ctx, const float* packet, float* out, float scale, bool host_packet,
                  const SparseOverlays* overlays, const DeviceFill* fill) {
    const bool ok = step_context_body(ctx, packet, out, scale, host_packet, overlays, fill);
    if (!ok && host_packet && !fill && (packet || (overlays && overlays->count > 0))) {
        // the caller owns its host buffers again when the call returns, also
        // after a failure: wait for the host-to-device copies queued before it
        // (a pinned buffer is read by DMA after cudaMemcpyAsync returns)
        cudaStreamSynchronize(current_stream());
    }
    return ok;
}

static bool step_context_body(Context& ctx, const float* packet, float* out, float scale, bool host_packet,
                              const SparseOverlays* overlays, const DeviceFill* fill) {
    cudaStream_t s = current_stream();
    const BrickDims d{ctx.nx, ctx.ny, ctx.nz, 0, ctx.cells};
    const FaceParams face_now = current_face_params();
    CollideParams cp = current_collide_params();
    cp.nx = ctx.nx;
    cp.ny = ctx.ny;
    cp.nz = ctx.nz;
    cp.step = ctx.step_counter;
    if (cp.fan_beta > 0.0f && !ctx.fan_mask) {
        // packet fan channels, kept from the ingest for the collision
        if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&ctx.fan_mask), (size_t)ctx.cells * 4 * sizeof(float)),
                     "cudaMalloc(fans)") ||
            !cuda_ok(cudaMemsetAsync(ctx.fan_mask, 0, (size_t)ctx.cells * 4 * sizeof(float), current_stream()),
                     "cudaMemset(fans)"))
            return false;
    }
    // The reference updates the temperature before every collision
    // (run_cpu_step, jni.cpp:8480-8507); it reaches the flow through the
    // buoyancy force.
    ctx.thermal = g_thermal_mode == 1 || (g_thermal_mode == -1 && cp.enable_buoyancy);
    if (ctx.thermal && !ensure_thermal(ctx)) return false;
    bool fused_transport = false;
    FusedTransport transport{};
    const int in_ch = g_cfg.input_channels;
    const bool have_packet = packet != nullptr || fill != nullptr;
    if (fill) host_packet = false;
    if (!have_packet && !ctx.has_inputs) {
        set_error("cached step requested before any packet was uploaded for this context");
        return false;
    }

    int new_slot = ctx.slot;
    const bool face_changed = std::memcmp(&face_now, &ctx.face_prev, sizeof(FaceParams)) != 0;
    // a device fill that rewrites the same mask keeps the classification
    const bool same_mask = fill && fill->mask_unchanged && ctx.initialized && !face_changed && ctx.pending_slot < 0;
    if (have_packet) {
        new_slot = ctx.initialized ? 1 - ctx.slot : ctx.slot;
        const size_t bytes = (size_t)ctx.cells * in_ch * sizeof(float);
        if (fill) {
            // the inputs are built on the device straight into the fields
            if (!cuda_ok(fill->launch(ctx.fields(new_slot), d, s, fill->user), "device input fill")) return false;
        } else {
            if (ctx.packet_cap < bytes) {
                if (ctx.packet) cudaFree(ctx.packet);
                ctx.packet = nullptr;
                ctx.packet_cap = 0;
                if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&ctx.packet), bytes), "cudaMalloc(packet)")) return false;
                ctx.packet_cap = bytes;
            }
            if (host_packet) {
                if (!cuda_ok(cudaMemcpyAsync(ctx.packet, packet, bytes, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync(packet)")) return false;
            } else {
                if (!cuda_ok(cudaMemcpyAsync(ctx.packet, packet, bytes, cudaMemcpyDeviceToDevice, s), "cudaMemcpyAsync(packet)")) return false;
            }
            if (!cuda_ok(launch_ingest_packet(ctx.packet, in_ch, d, ctx.fields(new_slot), s), "ingest_packet")) return false;
        }
        if (host_packet) {
            // the caller owns its packet again when the call returns: remember
            // when the copies from host memory (a pinned buffer is read by DMA
            // after cudaMemcpyAsync returns) have finished
            if (!ctx.copy_done && !cuda_ok(cudaEventCreateWithFlags(&ctx.copy_done, cudaEventDisableTiming), "copy event"))
                return false;
        }
        if (overlays && overlays->count > 0) {
            // apply_sparse_payload_overlays (jni.cpp:1696-1721), right after the ingest
            const int n = overlays->count;
            if (ctx.overlay_cap < n) {
                if (ctx.overlay_cells) cudaFree(ctx.overlay_cells);
                if (ctx.overlay_values) cudaFree(ctx.overlay_values);
                ctx.overlay_cells = nullptr;
                ctx.overlay_values = nullptr;
                ctx.overlay_cap = 0;
                if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&ctx.overlay_cells), (size_t)n * sizeof(int)), "cudaMalloc(overlays)") ||
                    !cuda_ok(cudaMalloc(reinterpret_cast<void**>(&ctx.overlay_values), (size_t)n * 6 * sizeof(float)), "cudaMalloc(overlays)"))
                    return false;
                ctx.overlay_cap = n;
            }
            if (!cuda_ok(cudaMemcpyAsync(ctx.overlay_cells, overlays->cells, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s), "copy overlays") ||
                !cuda_ok(cudaMemcpyAsync(ctx.overlay_values, overlays->values, (size_t)n * 6 * sizeof(float), cudaMemcpyHostToDevice, s), "copy overlays") ||
                !cuda_ok(launch_apply_overlays(ctx.overlay_cells, ctx.overlay_values, n, ctx.fields(new_slot), ctx.cells,
                                                  ctx.thermal ? (in_ch > kChThermalSource ? 1 : 2) : 0, s), "apply_overlays"))
                return false;
        }
        if (host_packet && !cuda_ok(cudaEventRecord(ctx.copy_done, s), "copy event")) return false;
        if (same_mask) {
            ctx.h_face[new_slot] = face_now;
            if (!cuda_ok(cudaMemcpyAsync(ctx.d_face[new_slot], ctx.d_face[ctx.slot], sizeof(FaceParams), cudaMemcpyDeviceToDevice, s),
                         "copy faces") ||
                !cuda_ok(cudaMemcpyAsync(ctx.flags[new_slot], ctx.flags[ctx.slot], (size_t)ctx.cells * sizeof(uint32_t),
                                         cudaMemcpyDeviceToDevice, s), "copy classification"))
                return false;
        } else if (!classify(ctx, new_slot, face_now, d, s)) {
            return false;
        }
        ctx.has_inputs = true;
    } else if (ctx.pending_slot >= 0) {
        // block edits staged the mask of this call (aero_lbm_patch_d3q27_f16_static_cells_rect)
        new_slot = ctx.pending_slot;
        if (face_changed && !classify(ctx, new_slot, face_now, d, s)) return false;
    } else if (face_changed && ctx.initialized) {
        // Same inputs, new faces: rebuild the classification into the other slot.
        new_slot = 1 - ctx.slot;
        if (!cuda_ok(cudaMemcpyAsync(ctx.obstacle[new_slot], ctx.obstacle[ctx.slot], (size_t)ctx.cells, cudaMemcpyDeviceToDevice, s), "copy obstacle")) return false;
        if (!cuda_ok(cudaMemcpyAsync(ctx.ref_p[new_slot], ctx.ref_p[ctx.slot], (size_t)ctx.cells * sizeof(float), cudaMemcpyDeviceToDevice, s), "copy ref_p")) return false;
        if (!classify(ctx, new_slot, face_now, d, s)) return false;
    } else if (face_changed) {
        if (!classify(ctx, new_slot, face_now, d, s)) return false;
    }

    if (!ctx.initialized && !choose_layout(ctx, face_now, packet, host_packet, new_slot)) return false;
    if (ctx.thermal) {
        if (!ctx.initialized) {
            const ThermalInitArgs ti{ctx.cells, ctx.temperature, ctx.u_last, ctx.obstacle[new_slot], ctx.ref_temperature,
                                     ctx.ref_ux, ctx.ref_uy, ctx.ref_uz, g_bench.initial_temperature, bench_active() ? 1 : 0};
            if (!cuda_ok(launch_thermal_init(ti, s), "thermal_init")) return false;
        } else if (!bench_active() && in_ch > 10) {
            const ThermalNudgeArgs tn{ctx.nx, ctx.ny, ctx.nz, ctx.temperature, ctx.obstacle[new_slot], ctx.ref_temperature,
                                      cp.state_nudge};
            if (!cuda_ok(launch_thermal_reference_nudge(tn, s), "thermal_reference")) return false;
        }
        // should_update_temperature (jni.cpp:2191-2196): every other call in runtime mode
        const bool update = bench_active() || ctx.step_counter % 2 == 0;
        ThermalArgs ta{};
        ta.nx = ctx.nx; ta.ny = ctx.ny; ta.nz = ctx.nz; ta.cells = ctx.cells;
        ta.t = ctx.temperature;
        ta.t_next = ctx.temperature_next;
        ta.u = ctx.u_last;
        ta.obstacle = ctx.obstacle[new_slot];
        ta.source = bench_flag(AERO_LBM_BENCHMARK_FLAG_DISABLE_INTERNAL_THERMAL_SOURCE) ? nullptr : ctx.thermal_source;
        ta.alpha = thermal_diffusivity();
        ta.faces = current_thermal_faces();
        // thermal_bfecc_active (jni.cpp:871-873); outside benchmark mode the
        // update also runs every other call with dt = 2 and a local eddy
        // diffusivity (effective_thermal_dt, effective_local_thermal_diffusivity)
        ta.bfecc = (!bench_active() || heated_cavity()) ? 1 : 0;
        ta.scratch = ctx.temperature_scratch;
        ta.dt = bench_active() ? 1.0f : 2.0f;
        ta.turbulent = (!bench_active() && cp.enable_sgs) ? 1 : 0;
        ta.sgs_c2 = cp.sgs_c2;
        ta.nu0 = clamp_nu(kRuntimeMolecularNu0);
        // The first-order branch runs inside the in-place step kernel
        // (thermal_fused.cuh) once the context has stepped: the state is
        // swapped here, the kernel reads the old one and writes the new one.
        fused_transport = update && ctx.initialized && ctx.layout == 1 && !ta.bfecc && ta.dt == 1.0f && !ta.turbulent &&
                          g_fused_transport;
        if (fused_transport) {
            transport.t = ctx.temperature;
            std::swap(ctx.temperature, ctx.temperature_next);
            transport.t_next = ctx.temperature;
            transport.u = ctx.u_last;
            transport.source = ta.source;
            transport.alpha = ta.alpha;
            transport.faces = ta.faces;
        } else if (update) {
            auto pf = g_fill_args.find(&ctx);
            if (ctx.fill_pending && ctx.layout == 1 && !ta.bfecc && pf != g_fill_args.end()) {
                // the last call's face pre-fill rides in the same grid
                const IpArgs fa = pf->second;
                g_fill_args.erase(pf);
                ctx.fill_pending = false;
                if (!cuda_ok(launch_thermal_update_fill(ta, ip_storage(ctx), ctx.ip, fa, s), "thermal_update + face_fill"))
                    return false;
            } else if (!cuda_ok(launch_thermal_update(ta, s), "thermal_update")) {
                return false;
            }
            std::swap(ctx.temperature, ta.bfecc ? ctx.temperature_scratch : ctx.temperature_next);
        }
    }
    if (ctx.layout == 0) {
        float* g_next = ctx.g[1 - ctx.cur];
        if (!ctx.initialized) {
            auto launch = g_collision_mode == 0 ? launch_init_collide_exact : launch_init_collide_fast;
            if (!cuda_ok(launch(d, ctx.fields(new_slot), ctx.force_field(), cp, g_next, s), "init_collide")) return false;
        } else if (ctx.f_ready) {
            // a halo exchange left the streamed state in g_next: collide it there
            auto launch = g_collision_mode == 0 ? launch_collide_ab_exact : launch_collide_ab_fast;
            if (!cuda_ok(launch(d, g_next, ctx.fields(new_slot), ctx.force_field(), cp, s), "collide_ab")) return false;
            ctx.f_ready = false;
        } else {
            auto launch = g_collision_mode == 0 ? launch_step_ab_exact : launch_step_ab_fast;
            if (!cuda_ok(launch(d, ctx.g[ctx.cur], g_next, ctx.flags[ctx.slot], ctx.obstacle[ctx.slot], ctx.ref_p[ctx.slot],
                                ctx.d_face[ctx.slot], ctx.fields(new_slot), ctx.force_field(), cp, s),
                         "step_ab")) return false;
        }
        ctx.cur = 1 - ctx.cur;
    } else {
        if (ctx.initialized && !inplace_faces_ok(face_now)) {
            set_error("in-place context: the faces changed to an axis periodic on one side only (or the cylinder "
                      "preset), which needs the two-buffer layout; release and re-create the context");
            return false;
        }
        if (!join_fill(ctx, s)) return false;
        IpArgs a = ip_args(ctx, ctx.slot, new_slot, cp);
        if (!ctx.initialized) {
            a.parity = 0;
            if (!cuda_ok(ip_init(ctx.ip_variant, ctx.ip, a, s), "init_inplace")) return false;
            ctx.parity = 1;
        } else {
            // a call with inputs can change the mask; one whose device fill
            // keeps it has no transitions to apply
            const bool inputs = have_packet || ctx.pending_slot >= 0;
            const bool transitions = inputs && !same_mask;
            if (inputs && !ctx.solid_f) {
                // the first call that can change the mask: solid cells so far
                // have been solid since initialisation and hold the rest state;
                // from now on they keep (and exchange) their own populations
                if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&ctx.solid_f), (size_t)ctx.cells * 27 * sizeof(float)),
                             "cudaMalloc(solid populations)") ||
                    !cuda_ok(launch_fill_rest(ctx.solid_f, ctx.cells, s), "fill solid populations"))
                    return false;
                a.solid_f = ctx.solid_f;
            }
            a.parity = ctx.parity;
            if (fused_transport) {
                a.transport = 1;
                a.tr = transport;
            }
            if (!cuda_ok(ip_step(ctx.ip_variant, ctx.ip, a, transitions, s), "step_inplace")) return false;
            ctx.parity ^= 1;
        }
    }
    ctx.slot = new_slot;
    ctx.pending_slot = -1;
    ctx.face_prev = face_now;
    ctx.initialized = true;
    ctx.step_counter += 1;
    // compute_benchmark_force (jni.cpp:2454-2492) after the collision: only the
    // cylinder preset reports a force; its outflow face keeps it on the
    // two-buffer layout, whose state is the post-collision populations
    ctx.force_valid = false;
    if (bench_active() && g_bench.preset == AERO_LBM_BENCHMARK_PRESET_CYLINDER_CROSSFLOW_2D && ctx.layout == 0) {
        if (!ctx.force3 && !cuda_ok(cudaMalloc(reinterpret_cast<void**>(&ctx.force3), 3 * sizeof(double)), "cudaMalloc(force)"))
            return false;
        if (!cuda_ok(launch_cylinder_force(ctx.g[ctx.cur], ctx.obstacle[new_slot], d, ctx.force3, s), "cylinder_force")) return false;
        ctx.force_valid = true;
    }
    if (ctx.layout == 1) {
        // Equilibrium-face sources of the next step, written now: between calls
        // every incoming slot then holds the cell's streamed population (the
        // reference's f), which the halo exchange reads and writes.
        if (faces_need_fill(face_now)) {
            // deferred: the next call's temperature update launches it in the
            // same grid; anything else that reads the populations first
            // launches it on its own (join_fill)
            IpArgs a = ip_args(ctx, new_slot, new_slot, cp);
            a.parity = ctx.parity;
            a.fill_faces = fill_face_mask(face_now);
            g_fill_args[&ctx] = a;
            ctx.fill_pending = true;
        }
        // the reference reads the shell in its FP16 in-place step only
        // (jni.cpp:6779-6790): a call in another solver mode keeps it unapplied
        if (ctx.shell_count > 0 &&
            g_realtime_solver_mode == AERO_LBM_REALTIME_SOLVER_D3Q27_FP16_INPLACE_EXPERIMENTAL) {
            if (!join_fill(ctx, s)) return false;
            IpArgs a = ip_args(ctx, new_slot, new_slot, cp);
            a.parity = ctx.parity;
            if (!cuda_ok(launch_shell_relax(ip_storage(ctx), ctx.ip, a, static_cast<const ShellCell*>(ctx.shell),
                                            ctx.shell_count, ctx.shell_layers, ctx.shell_relax, s),
                         "boundary_shell")) return false;
        }
    }

    if (out) return read_output(ctx, 1, g_cfg.output_channels, scale, out);
    if (have_packet && host_packet && !cuda_ok(cudaEventSynchronize(ctx.copy_done), "wait for the packet copy")) return false;
    return true;
}

bool output_device(Context& ctx, OutBox box, int out_ch, float scale, float* dev_out) {
    cudaStream_t s = current_stream();
    const BrickDims d{ctx.nx, ctx.ny, ctx.nz, 0, ctx.cells};
    if (ctx.layout == 0) {
        auto launch = g_collision_mode == 0 ? launch_output_ab_exact : launch_output_ab_fast;
        const float* g = ctx.f_ready ? ctx.g[1 - ctx.cur] : ctx.g[ctx.cur];
        return cuda_ok(launch(d, g, ctx.flags[ctx.slot], ctx.obstacle[ctx.slot], ctx.ref_p[ctx.slot], ctx.d_face[ctx.slot],
                              box, out_ch, scale, dev_out, s, ctx.f_ready ? 1 : 0),
                       "output");
    }
    if (!join_fill(ctx, s)) return false;
    IpArgs a = ip_args(ctx, ctx.slot, ctx.slot, current_collide_params());
    a.parity = ctx.parity;
    return cuda_ok(ip_output(ctx.ip_variant, ctx.ip, a, box, out_ch, scale, dev_out, s), "output_inplace");
}

bool read_output_box(Context& ctx, OutBox box, int out_ch, float scale, float* host_out, float* host_temperature);

bool read_output(Context& ctx, int stride, int out_ch, float scale, float* host_out) {
    return read_output_box(ctx, strided_box(ctx.nx, ctx.ny, ctx.nz, stride), out_ch, scale, host_out, nullptr);
}

// Output of a box; host_temperature (optional) receives the temperature of
// the same cells as aero_lbm_copy_flow_temperature_subrect reads it.
bool read_output_box(Context& ctx, OutBox box, int out_ch, float scale, float* host_out, float* host_temperature) {
    cudaStream_t s = current_stream();
    const size_t n = (size_t)box.count();
    const size_t bytes = n * (out_ch + (host_temperature ? 1 : 0)) * sizeof(float);
    if (ctx.out_cap < bytes) {
        if (ctx.out) cudaFree(ctx.out);
        ctx.out = nullptr;
        ctx.out_cap = 0;
        if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&ctx.out), bytes), "cudaMalloc(output)")) return false;
        ctx.out_cap = bytes;
    }
    if (!output_device(ctx, box, out_ch, scale, ctx.out)) return false;
    if (!cuda_ok(cudaMemcpyAsync(host_out, ctx.out, n * out_ch * sizeof(float), cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync(output)")) return false;
    if (host_temperature) {
        float* dev_t = ctx.out + n * out_ch;
        const BrickDims d{ctx.nx, ctx.ny, ctx.nz, 0, ctx.cells};
        if (!cuda_ok(launch_gather_temperature(ctx.temperature, ctx.obstacle[ctx.slot], d, box, dev_t, s), "gather_temperature") ||
            !cuda_ok(cudaMemcpyAsync(host_temperature, dev_t, n * sizeof(float), cudaMemcpyDeviceToHost, s),
                     "cudaMemcpyAsync(temperature)"))
            return false;
    }
    int fault = 0;
    if (!cuda_ok(cudaMemcpyAsync(&fault, ctx.fault, sizeof(int), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync(fault)")) return false;
    if (!cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize(output)")) return false;
    if (fault) {
        set_error("in-place step: a tile's bulk copies did not complete within the wait limit; the state is invalid");
        return false;
    }
    return true;
}

void record_timing(double copy_ms, double solver_ms, double readback_ms, double total_ms, bool cached) {
    g_timing.ticks += 1;
    g_timing.last_copy = copy_ms; g_timing.last_solver = solver_ms;
    g_timing.last_readback = readback_ms; g_timing.last_total = total_ms;
    g_timing.sum_copy += copy_ms; g_timing.sum_solver += solver_ms;
    g_timing.sum_readback += readback_ms; g_timing.sum_total += total_ms;
    if (cached) g_timing.cached_steps += 1;
    else g_timing.full_packet_steps += 1;
}

// Deferred halo exchanges (halo_batch_begin / halo_batch_flush): the slab
// copies of in-place contexts collect as jobs and go out as one launch per
// storage kind plus one for the temperature slabs.
struct HaloBatch {
    bool open = false;
    std::vector<HaloIpJob> ip[3];
    std::vector<HaloSoaJob> soa;
    int ip_max[3] = {0, 0, 0}, soa_max = 0;
    int device = -1;
    void* d_jobs = nullptr;       // device copy of the jobs of one flush
    void* h_jobs = nullptr;       // pinned staging
    size_t cap = 0;
    cudaEvent_t staged = nullptr; // the last upload from h_jobs has finished
};
static HaloBatch g_halo;

static int slab_cells(const HaloSlab& h) { return h.size[0] * h.size[1] * h.size[2]; }

void halo_batch_begin() {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    g_halo.open = true;
}

bool halo_batch_flush() {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    HaloBatch& B = g_halo;
    B.open = false;
    size_t bytes = B.soa.size() * sizeof(HaloSoaJob);
    for (auto& v : B.ip) bytes += v.size() * sizeof(HaloIpJob);
    if (bytes == 0) return true;
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "halo batch device")) return false;
    if (B.device != dev || B.cap < bytes) {
        if (B.staged) cudaEventSynchronize(B.staged);
        if (B.d_jobs && B.device == dev) cudaFree(B.d_jobs);
        if (B.h_jobs) cudaFreeHost(B.h_jobs);
        B.d_jobs = B.h_jobs = nullptr;
        const size_t cap = std::max<size_t>(bytes * 2, 16384);
        if (!cuda_ok(cudaMalloc(&B.d_jobs, cap), "halo batch jobs") || !cuda_ok(cudaMallocHost(&B.h_jobs, cap), "halo batch staging")) {
            B.cap = 0;
            return false;
        }
        B.cap = cap;
        B.device = dev;
        if (!B.staged && !cuda_ok(cudaEventCreateWithFlags(&B.staged, cudaEventDisableTiming), "halo batch event")) return false;
    } else if (!cuda_ok(cudaEventSynchronize(B.staged), "halo batch staging")) {
        return false;
    }
    cudaStream_t s = current_stream();
    char* h = static_cast<char*>(B.h_jobs);
    size_t off = 0;
    struct Part { int kind; size_t off; int n; int max; };
    std::vector<Part> parts;
    for (int k = 0; k < 3; ++k) {
        if (B.ip[k].empty()) continue;
        std::memcpy(h + off, B.ip[k].data(), B.ip[k].size() * sizeof(HaloIpJob));
        parts.push_back({k, off, (int)B.ip[k].size(), B.ip_max[k]});
        off += B.ip[k].size() * sizeof(HaloIpJob);
    }
    if (!B.soa.empty()) {
        std::memcpy(h + off, B.soa.data(), B.soa.size() * sizeof(HaloSoaJob));
        parts.push_back({3, off, (int)B.soa.size(), B.soa_max});
        off += B.soa.size() * sizeof(HaloSoaJob);
    }
    bool ok = cuda_ok(cudaMemcpyAsync(B.d_jobs, B.h_jobs, off, cudaMemcpyHostToDevice, s), "halo batch upload") &&
              cuda_ok(cudaEventRecord(B.staged, s), "halo batch event");
    for (const Part& p : parts) {
        if (!ok) break;
        const char* d = static_cast<const char*>(B.d_jobs) + p.off;
        ok = p.kind < 3 ? cuda_ok(launch_halo_ip_batch(p.kind, reinterpret_cast<const HaloIpJob*>(d), p.n, p.max, s), "halo_inplace")
                        : cuda_ok(launch_halo_soa_batch(reinterpret_cast<const HaloSoaJob*>(d), p.n, p.max, s), "halo_temperature");
    }
    for (auto& v : B.ip) v.clear();
    B.soa.clear();
    B.ip_max[0] = B.ip_max[1] = B.ip_max[2] = B.soa_max = 0;
    return ok;
}

}  // namespace aero

// ====================================================================== C ABI
using namespace aero;

namespace {

bool do_init(int nx, int ny, int nz, int in_ch, int out_ch) {
    release_all_contexts();
    g_timing = TimingStats{};
    if (nx <= 0 || ny <= 0 || nz <= 0 || in_ch < 9 || out_ch < 4) {
        g_cfg = RuntimeConfig{};
        set_error("aero_lbm_init_rect: invalid dimensions or channel counts");
        return false;
    }
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count <= 0) {
        g_cfg = RuntimeConfig{};
        set_error("aero_lbm_init_rect: no CUDA device available (this library has no CPU path)");
        return false;
    }
    if (!current_stream()) {
        g_cfg = RuntimeConfig{};
        set_error("aero_lbm_init_rect: cudaStreamCreate failed");
        return false;
    }
    g_cfg.initialized = true;
    g_cfg.nx = nx; g_cfg.ny = ny; g_cfg.nz = nz;
    g_cfg.input_channels = in_ch;
    g_cfg.output_channels = out_ch;
    cudaDeviceProp prop{};
    int dev = 0;
    cudaGetDevice(&dev);
    cudaGetDeviceProperties(&prop, dev);
    g_cfg.runtime_info = std::string("cuda|cumulant-d3q27+sgs+bouss:") + prop.name;
    return true;
}

bool step_impl(const float* packet, int nx, int ny, int nz, long long key, float* out, float scale, bool cached,
               const SparseOverlays* overlays = nullptr) {
    const auto t0 = Clock::now();
    clear_error();
    if (!g_cfg.initialized) {
        set_error("native_step_raw_dims: runtime not initialized");
        return false;
    }
    if (!cached && !packet) {
        set_error("native_step_raw_dims: missing packet");
        return false;
    }
    if (nx <= 0 || ny <= 0 || nz <= 0) {
        set_error("native_step_raw_dims: invalid dimensions");
        return false;
    }
    if (!std::isfinite(scale)) scale = 1.0f;
    Context* ctx = cached ? find_context(key) : get_or_create_context(key, nx, ny, nz);
    if (!ctx) {
        if (g_last_error.empty()) {
            set_error(cached ? "cached solver step requested before context initialization"
                             : "native_step_raw_dims: failed to allocate or acquire context");
        }
        return false;
    }
    if (cached && (ctx->nx != nx || ctx->ny != ny || ctx->nz != nz)) {
        set_error("cached solver step: dimensions differ from the resident context");
        return false;
    }
    const bool ok = step_context(*ctx, cached ? nullptr : packet, out, scale, true, overlays);
    if (!ok && g_last_error.empty()) set_error("native_step_raw_dims: step failed");
    record_timing(0.0, 0.0, 0.0, ms_since(t0), cached);
    return ok;
}

}  // namespace

bool aero::step_rect_device(long long key, int nx, int ny, int nz, const DeviceFill& fill) {
    const auto t0 = Clock::now();
    clear_error();
    if (!g_cfg.initialized) {
        set_error("native_step_raw_dims: runtime not initialized");
        return false;
    }
    if (nx <= 0 || ny <= 0 || nz <= 0) {
        set_error("native_step_raw_dims: invalid dimensions");
        return false;
    }
    Context* ctx = get_or_create_context(key, nx, ny, nz);
    if (!ctx) {
        if (g_last_error.empty()) set_error("native_step_raw_dims: failed to allocate or acquire context");
        return false;
    }
    const bool ok = step_context(*ctx, nullptr, nullptr, 1.0f, false, nullptr, &fill);
    if (!ok && g_last_error.empty()) set_error("native_step_raw_dims: step failed");
    record_timing(0.0, 0.0, 0.0, ms_since(t0), false);
    return ok;
}

extern "C" {

AERO_LBM_B200_EXPORT int aero_lbm_init_rect(int nx, int ny, int nz, int input_channels, int output_channels) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    ensure_bench();
    return do_init(nx, ny, nz, input_channels, output_channels) ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_init(int grid_size, int input_channels, int output_channels) {
    return aero_lbm_init_rect(grid_size, grid_size, grid_size, input_channels, output_channels);
}

AERO_LBM_B200_EXPORT int aero_lbm_step_rect(const float* packet, int nx, int ny, int nz, long long key, float* out) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    return step_impl(packet, nx, ny, nz, key, out, 1.0f, false) ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_step_rect_scaled(const float* packet, int nx, int ny, int nz, long long key, float scale,
                                                   float* out) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    return step_impl(packet, nx, ny, nz, key, out, scale, false) ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_step(const float* packet, int grid_size, long long key, float* out) {
    return aero_lbm_step_rect(packet, grid_size, grid_size, grid_size, key, out);
}

AERO_LBM_B200_EXPORT int aero_lbm_step_rect_cached(int nx, int ny, int nz, long long key, float* out) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    return step_impl(nullptr, nx, ny, nz, key, out, 1.0f, true) ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_step_rect_cached_scaled(int nx, int ny, int nz, long long key, float scale, float* out) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    return step_impl(nullptr, nx, ny, nz, key, out, scale, true) ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_has_context(long long key) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    return find_context(key) ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_context_realtime_cached_initialized(long long key) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    Context* c = find_context(key);
    return (c && c->initialized) ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_extract_flow_atlas_rect(int nx, int ny, int nz, long long key, int stride, float* out,
                                                          int value_count) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (!g_cfg.initialized || !out || stride <= 0 || nx <= 0 || ny <= 0 || nz <= 0) {
        set_error("extract_flow_atlas: invalid arguments or runtime not initialized");
        return 0;
    }
    const long long sx = (nx + stride - 1) / stride, sy = (ny + stride - 1) / stride, sz = (nz + stride - 1) / stride;
    if (sx * sy * sz <= 0 || (long long)value_count != sx * sy * sz * 4) {
        set_error("extract_flow_atlas: value_count does not match the atlas size");
        return 0;
    }
    Context* c = find_context(key);
    if (!c || !c->initialized || c->nx != nx || c->ny != ny || c->nz != nz) {
        set_error("extract_flow_atlas: no initialized context of these dimensions");
        return 0;
    }
    return read_output(*c, stride, 4, 1.0f, out) ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_get_flow_state_rect(int nx, int ny, int nz, long long key, float* out) {
    if (nx <= 0 || ny <= 0 || nz <= 0) return 0;
    const long long v = (long long)nx * ny * nz * 4;
    if (v > 0x7fffffffLL) return 0;
    return aero_lbm_extract_flow_atlas_rect(nx, ny, nz, key, 1, out, (int)v);
}

AERO_LBM_B200_EXPORT int aero_lbm_get_temperature_state_rect(int nx, int ny, int nz, long long key, float* out) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    Context* c = find_context(key);
    if (!g_cfg.initialized || !c || !out || c->nx != nx || c->ny != ny || c->nz != nz) {
        set_error("get_temperature_state: no context of these dimensions");
        return 0;
    }
    cudaStream_t s = current_stream();
    if (!cuda_ok(cudaMemcpyAsync(out, c->temperature, (size_t)c->cells * sizeof(float), cudaMemcpyDeviceToHost, s), "copy temperature")) return 0;
    return cuda_ok(cudaStreamSynchronize(s), "sync") ? 1 : 0;
}

// assign_temperature_state (jni.cpp:8028-8035): creates the context when it
// does not exist yet; values clamped with min(1, max(-1, v)).
AERO_LBM_B200_EXPORT int aero_lbm_set_temperature_state_rect(int nx, int ny, int nz, long long key, const float* t) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (!g_cfg.initialized || !t || nx <= 0 || ny <= 0 || nz <= 0) {
        set_error("set_temperature_state: runtime not initialised or bad arguments");
        return 0;
    }
    Context* c = get_or_create_context(key, nx, ny, nz);
    if (!c) return 0;
    std::unique_ptr<float[]> tmp(new float[(size_t)c->cells]);
    for (long long i = 0; i < c->cells; ++i) tmp[i] = clampf_h(t[i], -1.0f, 1.0f);
    cudaStream_t s = current_stream();
    if (!cuda_ok(cudaMemcpyAsync(c->temperature, tmp.get(), (size_t)c->cells * sizeof(float), cudaMemcpyHostToDevice, s), "copy temperature")) return 0;
    return cuda_ok(cudaStreamSynchronize(s), "sync") ? 1 : 0;
}

// exchange_context_halo_cpu_layers (jni.cpp:8266-8426) on device-resident
// contexts; the argument checks of native_exchange_halo_rect_layers_impl
// (jni.cpp:9693-9790). Both contexts must exist, be distinct, have the
// requested cubic shape and use the same storage; a context that has not
// stepped yet holds no populations and makes the call a no-op (the
// reference returns true for an empty context).
static bool exchange_halo(const char* who, int nx, int ny, int nz, int halo_layers, long long first_key,
                          long long second_key, int ox, int oy, int oz) {
    auto fail = [&](const std::string& m) {
        set_error(std::string(who) + ": " + m);
        return false;
    };
    if (!g_cfg.initialized) return fail("runtime not initialized");
    if (nx <= 0 || ny <= 0 || nz <= 0) return fail("invalid dimensions");
    if (halo_layers <= 0) return fail("halo_layers must be positive");
    if (ox < -1 || ox > 1 || oy < -1 || oy > 1 || oz < -1 || oz > 1) {
        std::ostringstream o;
        o << "invalid offset (" << ox << "," << oy << "," << oz << ")";
        return fail(o.str());
    }
    if (ox == 0 && oy == 0 && oz == 0) return fail("zero offset is invalid");
    if (nx != ny || ny != nz) {
        std::ostringstream o;
        o << "only cubic contexts are supported, got " << nx << "x" << ny << "x" << nz;
        return fail(o.str());
    }
    if (halo_layers * 2 >= nx) {
        std::ostringstream o;
        o << "invalid halo layout nx=" << nx << " halo=" << halo_layers;
        return fail(o.str());
    }
    Context* a = find_context(first_key);
    Context* b = find_context(second_key);
    if (!a || !b) {
        std::ostringstream o;
        o << "missing context(s) first=" << first_key << (a ? "" : " [missing]") << ", second=" << second_key
          << (b ? "" : " [missing]");
        return fail(o.str());
    }
    if (a == b) return fail("the two context keys are the same context");
    for (Context* c : {a, b})
        if (c->nx != nx || c->ny != ny || c->nz != nz) {
            std::ostringstream o;
            o << "context shape " << c->nx << "x" << c->ny << "x" << c->nz << " differs from the requested " << nx << "x"
              << ny << "x" << nz;
            return fail(o.str());
        }
    if (!a->initialized || !b->initialized) return true;
    if (a->layout != b->layout || (a->layout == 1 && a->ip_variant != b->ip_variant))
        return fail("the two contexts use different storage (layout or precision)");
    HaloSlab ab, ba;
    if (!halo_slabs(nx, halo_layers, ox, oy, oz, ab, ba)) return fail("halo slab bounds invalid");
    cudaStream_t s = current_stream();
    if (a->layout == 1) {
        auto side = [](Context& c) {
            return HaloIpSide{c.ip, make_pad_geom(c.nx, c.ny, c.nz, c.periodic_mask), c.flags[c.slot], c.parity,
                              Fp16Scale{c.fp16_scale, c.fp16_scale > 0.0f ? 1.0f / c.fp16_scale : 0.0f}, c.solid_f};
        };
        const int storage = a->ip_variant == kIpF16Fast ? 1 : (a->ip_variant == kIpI16Fast ? 2 : 0);
        if (!join_fill(*a, s) || !join_fill(*b, s)) return false;
        if (g_halo.open) {
            g_halo.ip[storage].push_back(HaloIpJob{side(*a), side(*b), ab});
            g_halo.ip[storage].push_back(HaloIpJob{side(*b), side(*a), ba});
            g_halo.ip_max[storage] = std::max({g_halo.ip_max[storage], slab_cells(ab), slab_cells(ba)});
        } else if (!cuda_ok(launch_halo_ip(storage, side(*a), side(*b), ab, ba, s), "halo_inplace")) {
            return false;
        }
    } else {
        for (Context* c : {a, b}) {
            if (c->f_ready) continue;
            const BrickDims d{c->nx, c->ny, c->nz, 0, c->cells};
            if (!cuda_ok(launch_materialise_ab(d, c->g[c->cur], c->flags[c->slot], c->obstacle[c->slot],
                                               c->ref_p[c->slot], c->d_face[c->slot], c->g[1 - c->cur], s),
                         "halo_materialise")) return false;
            c->f_ready = true;
        }
        if (!cuda_ok(launch_halo_soa(a->g[1 - a->cur], b->g[1 - b->cur], a->cells, ny, nz, 27, ab, s), "halo_f")) return false;
        if (!cuda_ok(launch_halo_soa(b->g[1 - b->cur], a->g[1 - a->cur], b->cells, ny, nz, 27, ba, s), "halo_f")) return false;
    }
    // should_exchange_temperature_halo (jni.cpp:2198-2207): in runtime mode the
    // temperature moves every other call; its slabs are exchanged only when
    // either context updated it in its last call
    auto updated_last = [](const Context* c) {
        return bench_active() || c->step_counter == 0 || (c->step_counter - 1) % 2 == 0;
    };
    if (updated_last(a) || updated_last(b)) {
        if (g_halo.open && a->layout == 1) {
            g_halo.soa.push_back(HaloSoaJob{a->temperature, b->temperature, a->cells, ny, nz, ab});
            g_halo.soa.push_back(HaloSoaJob{b->temperature, a->temperature, b->cells, ny, nz, ba});
            g_halo.soa_max = std::max({g_halo.soa_max, slab_cells(ab), slab_cells(ba)});
            return true;
        }
        if (!cuda_ok(launch_halo_soa(a->temperature, b->temperature, a->cells, ny, nz, 1, ab, s), "halo_temperature")) return false;
        if (!cuda_ok(launch_halo_soa(b->temperature, a->temperature, b->cells, ny, nz, 1, ba, s), "halo_temperature")) return false;
    }
    return true;
}

AERO_LBM_B200_EXPORT int aero_lbm_exchange_halo_layers_rect(int nx, int ny, int nz, int halo_layers, long long first_key,
                                                            long long second_key, int ox, int oy, int oz) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    return exchange_halo("exchange_halo_layers_rect", nx, ny, nz, halo_layers, first_key, second_key, ox, oy, oz) ? 1 : 0;
}

// native_exchange_halo_impl (jni.cpp:9623-9691): the configured cubic grid and
// max(1, n / 4) halo layers (exchange_context_halo_cpu, jni.cpp:8428-8430).
AERO_LBM_B200_EXPORT int aero_lbm_exchange_halo(int grid_size, long long first_key, long long second_key, int ox, int oy,
                                                int oz) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (!g_cfg.initialized) {
        set_error("exchange_halo: runtime not initialized");
        return 0;
    }
    if (g_cfg.nx != g_cfg.ny || g_cfg.ny != g_cfg.nz || grid_size != g_cfg.nx) {
        std::ostringstream o;
        o << "exchange_halo: grid size mismatch (requested=" << grid_size << ", configured=" << g_cfg.nx << "x"
          << g_cfg.ny << "x" << g_cfg.nz << ")";
        set_error(o.str());
        return 0;
    }
    return exchange_halo("exchange_halo", grid_size, grid_size, grid_size, std::max(1, grid_size / 4), first_key,
                         second_key, ox, oy, oz)
               ? 1
               : 0;
}

// native_step_raw_dims_with_sparse_overlays_impl (jni.cpp:8686-8745): a full
// step whose ingested reference fields are overridden at `overlay_count`
// cells (6 floats each: vx, vy, vz, p, T, source) before the collision.
AERO_LBM_B200_EXPORT int aero_lbm_step_rect_with_sparse_overlays(const float* packet, int nx, int ny, int nz, long long key,
                                                                 const int* overlay_cells, const float* overlay_values,
                                                                 int overlay_count, float* out) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (overlay_count < 0) {
        set_error("native_step_raw_dims_sparse: invalid overlay count");
        return 0;
    }
    if (overlay_count > 0 && (!overlay_cells || !overlay_values)) {
        set_error("native_step_raw_dims_sparse: missing overlay data");
        return 0;
    }
    const SparseOverlays ov{overlay_cells, overlay_values, overlay_count};
    return step_impl(packet, nx, ny, nz, key, out, 1.0f, false, &ov) ? 1 : 0;
}

// native_shift_context_impl + shift_context_cpu_state (jni.cpp:9603-9616,
// 8432-8478): the whole state moves by (dx, dy, dz) (new cell x holds old
// cell x + d); cells shifted in from outside get the rest equilibrium, fluid,
// zero reference fields and zero temperature. The classification is rebuilt
// from the shifted mask with the last call's faces; the next call collides
// the shifted streamed state.
AERO_LBM_B200_EXPORT int aero_lbm_shift_context(int grid_size, long long key, int dx, int dy, int dz) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (!g_cfg.initialized || g_cfg.nx != g_cfg.ny || g_cfg.ny != g_cfg.nz || grid_size != g_cfg.nx) {
        set_error("shift_context: runtime not initialized or grid size mismatch");
        return 0;
    }
    Context* c = find_context(key);
    if (!c) {
        set_error("shift_context: missing context");
        return 0;
    }
    if (c->nx != g_cfg.nx || c->ny != g_cfg.ny || c->nz != g_cfg.nz) {
        set_error("shift_context: context shape differs from the configured grid");
        return 0;
    }
    if (dx == 0 && dy == 0 && dz == 0) return 1;
    if (c->pending_slot >= 0) {
        set_error("shift_context: block edits are staged for the next call; step once before shifting");
        return 0;
    }
    if (std::abs(dx) >= c->nx || std::abs(dy) >= c->ny || std::abs(dz) >= c->nz) {
        set_error("shift_context: shift larger than the context");
        return 0;
    }
    cudaStream_t s = current_stream();
    const BrickDims d{c->nx, c->ny, c->nz, 0, c->cells};
    const size_t cells = (size_t)c->cells;
    float* tmp = nullptr;
    if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&tmp), cells * 27 * sizeof(float)), "cudaMalloc(shift)")) return 0;
    std::unique_ptr<float, decltype(&cudaFree)> tmp_guard(tmp, &cudaFree);
    // one component-major field of `comps` floats per cell, shifted in place through tmp
    auto shift_field = [&](float* p, int comps, float fill) {
        if (!p) return true;
        return cuda_ok(launch_shift_f32(p, tmp, d, comps, dx, dy, dz, fill, false, s), "shift") &&
               cuda_ok(cudaMemcpyAsync(p, tmp, cells * comps * sizeof(float), cudaMemcpyDeviceToDevice, s), "shift copy");
    };
    if (!shift_field(c->temperature, 1, 0.0f) || !shift_field(c->temperature_next, 1, 0.0f) ||
        !shift_field(c->temperature_scratch, 1, 0.0f) || !shift_field(c->u_last, 3, 0.0f))
        return 0;
    c->force_valid = false;
    if (!c->initialized) return cuda_ok(cudaStreamSynchronize(s), "sync") ? 1 : 0;
    const int slot = c->slot;
    IpView v{};
    int storage = 0;
    if (c->layout == 0) {
        // populations first, through the classification they were streamed with
        if (c->f_ready) {
            if (!cuda_ok(launch_shift_f32(c->g[1 - c->cur], c->g[c->cur], d, 27, dx, dy, dz, 0.0f, true, s), "shift f")) return 0;
            c->cur = 1 - c->cur;
        } else {
            if (!cuda_ok(launch_shift_materialise_ab(d, c->g[c->cur], c->flags[slot], c->obstacle[slot], c->ref_p[slot],
                                                     c->d_face[slot], dx, dy, dz, c->g[1 - c->cur], s),
                         "shift materialise")) return 0;
            c->f_ready = true;
        }
    } else {
        storage = c->ip_variant == kIpF16Fast ? 1 : (c->ip_variant == kIpI16Fast ? 2 : 0);
        if (c->solid_f) {
            if (!cuda_ok(launch_shift_f32(c->solid_f, tmp, d, 27, dx, dy, dz, 0.0f, true, s), "shift solid") ||
                !cuda_ok(cudaMemcpyAsync(c->solid_f, tmp, cells * 27 * sizeof(float), cudaMemcpyDeviceToDevice, s),
                         "shift solid copy"))
                return 0;
        }
        if (!join_fill(*c, s)) return 0;
        v = IpView{c->ip, make_pad_geom(c->nx, c->ny, c->nz, c->periodic_mask), c->flags[slot], c->parity,
                   Fp16Scale{c->fp16_scale, c->fp16_scale > 0.0f ? 1.0f / c->fp16_scale : 0.0f}};
        if (!cuda_ok(launch_ip_gather_shifted(storage, v, dx, dy, dz, tmp, s), "shift gather")) return 0;
    }
    // the reference fields (the in-place populations wait in tmp; scalar
    // shifts then go through the obstacle's spare slot and the spare buffer)
    uint8_t* ob_tmp = c->obstacle[1 - slot];
    if (!cuda_ok(launch_shift_u8(c->obstacle[slot], ob_tmp, d, dx, dy, dz, s), "shift obstacle") ||
        !cuda_ok(cudaMemcpyAsync(c->obstacle[slot], ob_tmp, cells, cudaMemcpyDeviceToDevice, s), "shift obstacle copy"))
        return 0;
    float* f_tmp = c->ref_p[1 - slot];
    auto shift_scalar = [&](float* p) {
        if (!p) return true;
        return cuda_ok(launch_shift_f32(p, f_tmp, d, 1, dx, dy, dz, 0.0f, false, s), "shift") &&
               cuda_ok(cudaMemcpyAsync(p, f_tmp, cells * sizeof(float), cudaMemcpyDeviceToDevice, s), "shift copy");
    };
    if (!shift_scalar(c->ref_p[slot]) || !shift_scalar(c->ref_ux) || !shift_scalar(c->ref_uy) || !shift_scalar(c->ref_uz) ||
        !shift_scalar(c->ref_temperature) || !shift_scalar(c->thermal_source))
        return 0;
    if (!cuda_ok(launch_build_flags(c->obstacle[slot], d, c->h_face[slot], c->flags[slot], s), "shift flags")) return 0;
    if (c->layout == 1) {
        v.flags = c->flags[slot];
        if (!cuda_ok(launch_ip_scatter(storage, v, tmp, s), "shift scatter")) return 0;
    }
    return cuda_ok(cudaStreamSynchronize(s), "sync") ? 1 : 0;
}

// Block edits (patch_d3q27_f16_static_cells, jni.cpp:6156-6260, 4725-4778,
// 9905-9960) on an in-place context that has stepped: the mask of the next
// call is the current one with the patched cells set solid / fluid, and every
// patched cell restarts at rest (its incoming populations, or its stored
// populations while it is solid). The next call, cached or not, steps with
// mask transitions; a call with a packet replaces the staged mask. Fan
// directions are accepted and ignored (fans are not modelled).
AERO_LBM_B200_EXPORT int aero_lbm_patch_d3q27_f16_static_cells_rect(int nx, int ny, int nz, long long key, int count,
                                                                    const int* cells, const uint8_t* solid,
                                                                    const uint8_t* fan_dir) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (!g_cfg.initialized) {
        set_error("patch_d3q27_f16_static_cells: runtime is not initialized");
        return 0;
    }
    if (count <= 0) return 1;
    if (!cells || !solid || !fan_dir) {
        set_error("patch_d3q27_f16_static_cells: missing patch arrays");
        return 0;
    }
    if (nx <= 0 || ny <= 0 || nz <= 0 || nx != g_cfg.nx || ny != g_cfg.ny || nz != g_cfg.nz) {
        set_error("patch_d3q27_f16_static_cells: invalid dimensions");
        return 0;
    }
    Context* c = find_context(key);
    if (!c) {
        set_error("patch_d3q27_f16_static_cells: context not found");
        return 0;
    }
    if (c->nx != nx || c->ny != ny || c->nz != nz) {
        set_error("patch_d3q27_f16_static_cells: context shape mismatch");
        return 0;
    }
    if (!c->initialized || c->layout != 1) {
        set_error("patch_d3q27_f16_static_cells: needs an in-place context that has stepped");
        return 0;
    }
    cudaStream_t s = current_stream();
    if (c->patch_cap < count) {
        if (c->patch_cells) cudaFree(c->patch_cells);
        if (c->patch_solid) cudaFree(c->patch_solid);
        c->patch_cells = nullptr;
        c->patch_solid = nullptr;
        c->patch_cap = 0;
        if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&c->patch_cells), (size_t)count * sizeof(int)), "cudaMalloc(patch)") ||
            !cuda_ok(cudaMalloc(reinterpret_cast<void**>(&c->patch_solid), (size_t)count), "cudaMalloc(patch)"))
            return 0;
        c->patch_cap = count;
    }
    if (!cuda_ok(cudaMemcpyAsync(c->patch_cells, cells, (size_t)count * sizeof(int), cudaMemcpyHostToDevice, s), "copy patch") ||
        !cuda_ok(cudaMemcpyAsync(c->patch_solid, solid, (size_t)count, cudaMemcpyHostToDevice, s), "copy patch"))
        return 0;
    const int target = 1 - c->slot;
    const BrickDims d{c->nx, c->ny, c->nz, 0, c->cells};
    const uint8_t* base = c->obstacle[c->pending_slot >= 0 ? c->pending_slot : c->slot];
    if (c->pending_slot < 0 &&
        !cuda_ok(cudaMemcpyAsync(c->ref_p[target], c->ref_p[c->slot], (size_t)c->cells * sizeof(float),
                                 cudaMemcpyDeviceToDevice, s), "copy pressure proxy"))
        return 0;
    if (!cuda_ok(launch_patch_mask(base, c->obstacle[target], c->cells, c->patch_cells, c->patch_solid, count, s),
                 "patch mask") ||
        !classify(*c, target, c->face_prev, d, s))
        return 0;
    IpArgs a = ip_args(*c, c->slot, c->slot, current_collide_params());
    a.parity = c->parity;
    if (!join_fill(*c, s) ||
        !cuda_ok(launch_patch_reset(ip_storage(*c), c->ip, a, c->patch_cells, count, s), "patch reset")) return 0;
    c->pending_slot = target;
    return cuda_ok(cudaStreamSynchronize(s), "sync") ? 1 : 0;
}

// upload_d3q27_f16_boundary_shell (jni.cpp:6449-6540): fluid cells within
// shell_layers of a face in face_mask (bit i: x-, x+, y-, y+, z-, z+) get a
// layer (1 outermost) and a target (the flow state's velocity, speed-clamped,
// and pressure, rounded to half precision); after every later call made in
// the FP16 in-place solver mode their state is relaxed toward it (edits.cuh). Needs an in-place context that has
// stepped. A zero mask, layer count or relaxation clears the shell.
AERO_LBM_B200_EXPORT int aero_lbm_set_d3q27_f16_boundary_shell_rect(int nx, int ny, int nz, long long key,
                                                                    const float* flow, int channels, int face_mask,
                                                                    int shell_layers, float relaxation) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (!g_cfg.initialized) {
        set_error("set_d3q27_f16_boundary_shell: runtime is not initialized");
        return 0;
    }
    if (nx <= 0 || ny <= 0 || nz <= 0 || nx != g_cfg.nx || ny != g_cfg.ny || nz != g_cfg.nz) {
        set_error("set_d3q27_f16_boundary_shell: invalid dimensions");
        return 0;
    }
    if (!flow || channels < 4) {
        set_error("set_d3q27_f16_boundary_shell: missing flow state");
        return 0;
    }
    Context* c = find_context(key);
    if (!c) {
        set_error("set_d3q27_f16_boundary_shell: context not found");
        return 0;
    }
    if (c->nx != nx || c->ny != ny || c->nz != nz) {
        set_error("set_d3q27_f16_boundary_shell: context shape mismatch");
        return 0;
    }
    auto clear = [&]() {
        if (c->shell) cudaFree(c->shell);
        c->shell = nullptr;
        c->shell_count = 0;
        c->shell_layers = 0;
        c->shell_relax = 0.0f;
        return 1;
    };
    if (face_mask == 0 || shell_layers <= 0 || !(relaxation > 0.0f)) return clear();
    if (!c->initialized || c->layout != 1) {
        set_error("set_d3q27_f16_boundary_shell: needs an in-place context that has stepped");
        return 0;
    }
    const int layers = std::max(1, std::min({shell_layers, nx, ny, nz}));
    const float relax = clampf_h(finite_or(relaxation, 0.0f), 0.0f, 0.5f);
    if (relax <= 0.0f) return clear();
    cudaStream_t s = current_stream();
    std::vector<uint8_t> solid((size_t)c->cells);
    const uint8_t* mask = c->obstacle[c->pending_slot >= 0 ? c->pending_slot : c->slot];
    if (!cuda_ok(cudaMemcpyAsync(solid.data(), mask, solid.size(), cudaMemcpyDeviceToHost, s), "copy mask") ||
        !cuda_ok(cudaStreamSynchronize(s), "sync"))
        return 0;
    auto half_round = [](float v) { return __half2float(__float2half_rn(v)); };
    std::vector<ShellCell> list;
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                const long long cell = ((long long)x * ny + y) * nz + z;
                if (solid[(size_t)cell]) continue;
                int best = layers + 1;
                if ((face_mask & 1) && x < layers) best = std::min(best, x + 1);
                if ((face_mask & 2) && x >= nx - layers) best = std::min(best, nx - x);
                if ((face_mask & 4) && y < layers) best = std::min(best, y + 1);
                if ((face_mask & 8) && y >= ny - layers) best = std::min(best, ny - y);
                if ((face_mask & 16) && z < layers) best = std::min(best, z + 1);
                if ((face_mask & 32) && z >= nz - layers) best = std::min(best, nz - z);
                if (best > layers) continue;
                const float* v = flow + (size_t)cell * (size_t)channels;
                float vx = finite_or(v[0], 0.0f), vy = finite_or(v[1], 0.0f), vz = finite_or(v[2], 0.0f);
                const float p = clampf_h(finite_or(v[3], 0.0f), -0.03f, 0.03f);
                const float s2 = vx * vx + vy * vy + vz * vz;
                if (!std::isfinite(s2) || s2 > kMaxSpeed * kMaxSpeed) {
                    if (!std::isfinite(s2) || s2 <= 0.0f) {
                        vx = vy = vz = 0.0f;
                    } else {
                        const float k = kMaxSpeed / std::sqrt(s2);
                        vx *= k; vy *= k; vz *= k;
                    }
                }
                list.push_back(ShellCell{(int)cell, best, half_round(vx), half_round(vy), half_round(vz), half_round(p)});
            }
    clear();
    if (list.empty()) return 1;
    if (!cuda_ok(cudaMalloc(&c->shell, list.size() * sizeof(ShellCell)), "cudaMalloc(shell)")) return 0;
    if (!cuda_ok(cudaMemcpyAsync(c->shell, list.data(), list.size() * sizeof(ShellCell), cudaMemcpyHostToDevice, s),
                 "copy shell") ||
        !cuda_ok(cudaStreamSynchronize(s), "sync"))
        return 0;
    c->shell_count = (int)list.size();
    c->shell_layers = layers;
    c->shell_relax = relax;
    return 1;
}

// clear_d3q27_f16_boundary_shell (jni.cpp:6443-6447, 10024-10037): 1 also
// when the context does not exist.
AERO_LBM_B200_EXPORT int aero_lbm_clear_d3q27_f16_boundary_shell_rect(long long key) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    Context* c = find_context(key);
    if (c) {
        if (c->shell) cudaFree(c->shell);
        c->shell = nullptr;
        c->shell_count = 0;
        c->shell_layers = 0;
        c->shell_relax = 0.0f;
    }
    return 1;
}

// The compact (heuristic) solver is not part of this library: no context is
// ever compact-initialised (jni.cpp:10071-10078 answers 0 without it too).
AERO_LBM_B200_EXPORT int aero_lbm_context_compact_initialized(long long) { return 0; }

// native_sample_temperature_point_raw_dims_impl (jni.cpp:8899-8947, CPU
// branch): the raw temperature state of one cell.
AERO_LBM_B200_EXPORT int aero_lbm_sample_temperature_point_rect(int nx, int ny, int nz, long long key, int x, int y, int z,
                                                                float* out) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (!g_cfg.initialized || !out || nx <= 0 || ny <= 0 || nz <= 0 || x < 0 || y < 0 || z < 0 || x >= nx || y >= ny ||
        z >= nz) {
        set_error("sample_temperature_point: invalid arguments");
        return 0;
    }
    Context* c = find_context(key);
    if (!c || c->nx != nx || c->ny != ny || c->nz != nz) {
        set_error("sample_temperature_point: no context of these dimensions");
        return 0;
    }
    cudaStream_t s = current_stream();
    const long long cell = ((long long)x * ny + y) * nz + z;
    return cuda_ok(cudaMemcpyAsync(out, c->temperature + cell, sizeof(float), cudaMemcpyDeviceToHost, s), "copy temperature") &&
                   cuda_ok(cudaStreamSynchronize(s), "sync")
               ? 1
               : 0;
}

// native_sample_flow_point_raw_dims_impl (jni.cpp:8949-9244, CPU branch):
// write_output of one cell (velocity unscaled, clamp(rho - 1)); 0 on solids.
AERO_LBM_B200_EXPORT int aero_lbm_sample_flow_point_rect(int nx, int ny, int nz, long long key, int x, int y, int z,
                                                         float* out) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (!g_cfg.initialized || !out || nx <= 0 || ny <= 0 || nz <= 0 || x < 0 || y < 0 || z < 0 || x >= nx || y >= ny ||
        z >= nz) {
        set_error("sample_flow_point: invalid arguments");
        return 0;
    }
    Context* c = find_context(key);
    if (!c || !c->initialized || c->nx != nx || c->ny != ny || c->nz != nz) {
        set_error("sample_flow_point: no initialized context of these dimensions");
        return 0;
    }
    return read_output_box(*c, OutBox{x, y, z, 1, 1, 1, 1}, 4, 1.0f, out, nullptr) ? 1 : 0;
}

// native_copy_flow_temperature_subrect_raw_dims_impl (jni.cpp:9451-9526): the
// flow (4 floats per cell) and the temperature (0 on solids, clamped) of the
// box [offset, offset + copy) in cell order, x outermost.
AERO_LBM_B200_EXPORT int aero_lbm_copy_flow_temperature_subrect(int nx, int ny, int nz, long long key, int ox, int oy, int oz,
                                                                int cnx, int cny, int cnz, float* out_flow,
                                                                float* out_temperature) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (!g_cfg.initialized || !out_flow || !out_temperature || nx <= 0 || ny <= 0 || nz <= 0 || cnx <= 0 || cny <= 0 ||
        cnz <= 0 || ox < 0 || oy < 0 || oz < 0 || ox + cnx > nx || oy + cny > ny || oz + cnz > nz) {
        set_error("copy_flow_temperature_subrect: invalid arguments");
        return 0;
    }
    Context* c = find_context(key);
    if (!c || !c->initialized || c->nx != nx || c->ny != ny || c->nz != nz) {
        set_error("copy_flow_temperature_subrect: no initialized context of these dimensions");
        return 0;
    }
    return read_output_box(*c, OutBox{ox, oy, oz, cnx, cny, cnz, 1}, 4, 1.0f, out_flow, out_temperature) ? 1 : 0;
}

// aero_lbm_get_last_force (jni.cpp:10259-10267): the momentum-exchange force
// of the last call (cylinder preset: sum / nz; otherwise 0).
AERO_LBM_B200_EXPORT int aero_lbm_get_last_force(long long key, float* fx, float* fy, float* fz) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    Context* c = find_context(key);
    if (!c) {
        set_error("get_last_force: missing context");
        return 0;
    }
    float f[3] = {0.0f, 0.0f, 0.0f};
    if (c->force_valid) {
        double h[3];
        cudaStream_t s = current_stream();
        if (!cuda_ok(cudaMemcpyAsync(h, c->force3, sizeof(h), cudaMemcpyDeviceToHost, s), "copy force") ||
            !cuda_ok(cudaStreamSynchronize(s), "sync"))
            return 0;
        const double inv_depth = c->nz > 0 ? 1.0 / (double)c->nz : 1.0;
        for (int k = 0; k < 3; ++k) f[k] = (float)(h[k] * inv_depth);
    }
    if (fx) *fx = f[0];
    if (fy) *fy = f[1];
    if (fz) *fz = f[2];
    return 1;
}

// memory_info_string (jni.cpp:5436-5457): device bytes per category. The
// categories follow the reference's names: d3q27_* for in-place contexts,
// classic_* for two-buffer ones.
AERO_LBM_B200_EXPORT const char* aero_lbm_memory_info(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    static std::string text;
    unsigned long long ip_dist = 0, ip_solid = 0, ip_class = 0, ip_out = 0, ab_dist = 0, ab_payload = 0, ab_out = 0,
                       temp = 0, contexts = 0, cells = 0;
    for (const auto& kv : g_contexts) {
        const Context& c = *kv.second;
        if (!c.allocated) continue;
        const unsigned long long n = (unsigned long long)c.cells;
        contexts += 1;
        cells += n;
        const unsigned long long t = n * 4ull * (1 + (c.temperature_next ? 2 : 0) + (c.ref_temperature ? 2 : 0)) +
                                     (c.u_last ? n * 12ull : 0);
        temp += t;
        if (c.layout == 1 && c.ip) {
            const unsigned long long pc = (unsigned long long)(c.nx + 2) * (c.ny + 2) * pad_row(c.nz);
            ip_dist += pc * 27ull * (c.ip_variant == kIpF32Exact || c.ip_variant == kIpF32Fast ? 4ull : 2ull);
            ip_solid += 2ull * n;
            ip_class += 2ull * n * 4ull;
            ip_out += c.out_cap;
        } else {
            ab_dist += 2ull * n * 27ull * 4ull;
            ab_out += c.out_cap;
        }
        ab_payload += c.packet_cap;
    }
    const unsigned long long total = ip_dist + ip_solid + ip_class + ip_out + ab_dist + ab_payload + ab_out + temp;
    text = "gpu_bytes(total=" + std::to_string(total) + ",d3q27_dist=" + std::to_string(ip_dist) +
           ",d3q27_solid=" + std::to_string(ip_solid) + ",d3q27_class=" + std::to_string(ip_class) +
           ",d3q27_fan=0,d3q27_active=0,d3q27_boundary=0,d3q27_output=" + std::to_string(ip_out) +
           ",compact_state=0,compact_solid=0,compact_output=0,classic_payload=" + std::to_string(ab_payload) +
           ",classic_dist=" + std::to_string(ab_dist) + ",classic_output=" + std::to_string(ab_out) +
           ",classic_temperature=" + std::to_string(temp) + ",classic_thermal_dist=0,contexts=" +
           std::to_string(contexts) + ",cells=" + std::to_string(cells) + ")";
    return text.c_str();
}

AERO_LBM_B200_EXPORT void aero_lbm_release_context(long long key) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    g_contexts.erase(key);
}

AERO_LBM_B200_EXPORT void aero_lbm_shutdown(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    release_all_contexts();
    g_cfg = RuntimeConfig{};
    g_timing = TimingStats{};
}

AERO_LBM_B200_EXPORT const char* aero_lbm_runtime_info(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    return g_cfg.runtime_info.c_str();
}

AERO_LBM_B200_EXPORT const char* aero_lbm_last_error(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    return g_last_error.c_str();
}

AERO_LBM_B200_EXPORT const char* aero_lbm_timing_info(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (g_timing.ticks == 0) {
        g_timing_text = "ticks=0";
        return g_timing_text.c_str();
    }
    const double inv = 1.0 / double(g_timing.ticks);
    std::ostringstream o;
    o.setf(std::ios::fixed);
    o.precision(3);
    o << "ticks=" << g_timing.ticks << " path=cuda last_ms(total=" << g_timing.last_total << ")"
      << " avg_ms(total=" << g_timing.sum_total * inv << ")"
      << " steps(full_packet=" << g_timing.full_packet_steps << ",cached=" << g_timing.cached_steps << ")"
      << " launches=" << kernel_launch_count();
    g_timing_text = o.str();
    return g_timing_text.c_str();
}

AERO_LBM_B200_EXPORT void aero_lbm_reset_timing(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    g_timing = TimingStats{};
}

AERO_LBM_B200_EXPORT void aero_lbm_set_realtime_solver_mode(int mode) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    g_realtime_solver_mode = (mode >= 0 && mode <= 3) ? mode : AERO_LBM_REALTIME_SOLVER_AUTO;
}

AERO_LBM_B200_EXPORT int aero_lbm_finish(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (!g_stream) return 1;
    return cuda_ok(cudaStreamSynchronize(g_stream), "aero_lbm_finish") ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_get_timing_snapshot(AeroLbmTimingSnapshot* out) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (!out) return 0;
    AeroLbmTimingSnapshot s{};
    s.ticks = g_timing.ticks;
    s.last_payload_copy_ms = g_timing.last_copy;
    s.last_solver_ms = g_timing.last_solver;
    s.last_readback_ms = g_timing.last_readback;
    s.last_total_ms = g_timing.last_total;
    if (g_timing.ticks) {
        const double inv = 1.0 / double(g_timing.ticks);
        s.avg_payload_copy_ms = g_timing.sum_copy * inv;
        s.avg_solver_ms = g_timing.sum_solver * inv;
        s.avg_readback_ms = g_timing.sum_readback * inv;
        s.avg_total_ms = g_timing.sum_total * inv;
    }
    *out = s;
    return 1;
}

AERO_LBM_B200_EXPORT void aero_lbm_benchmark_default_config(AeroLbmBenchmarkConfig* out) {
    if (out) *out = default_config();
}

AERO_LBM_B200_EXPORT int aero_lbm_benchmark_default_preset_config(int preset, AeroLbmBenchmarkConfig* out) {
    if (!out || !valid_preset(preset)) return 0;
    *out = preset_config(preset);
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_benchmark_set_config(const AeroLbmBenchmarkConfig* config) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (!config) return 0;
    AeroLbmBenchmarkConfig c = *config;
    sanitize(c);
    g_bench = c;
    g_bench_ready = true;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_benchmark_get_config(AeroLbmBenchmarkConfig* out) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (!out) return 0;
    ensure_bench();
    *out = g_bench;
    return 1;
}

AERO_LBM_B200_EXPORT void aero_lbm_benchmark_reset_config(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    g_bench = default_config();
    g_bench_ready = true;
}

AERO_LBM_B200_EXPORT const char* aero_lbm_benchmark_info(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    ensure_bench();
    std::ostringstream o;
    o << "enabled=" << g_bench.enabled << " preset=" << g_bench.preset << " flags=0x" << std::hex << g_bench.flags << std::dec
      << " Re=" << g_bench.reynolds_number << " tau_shear=" << tau_shear_base() << " tau_normal=" << tau_normal_base();
    g_bench_text = o.str();
    return g_bench_text.c_str();
}

AERO_LBM_B200_EXPORT void aero_lbm_b200_set_stream(void* stream) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (g_own_stream && g_stream) cudaStreamDestroy(g_stream);
    g_own_stream = false;
    g_stream = static_cast<cudaStream_t>(stream);
    if (!g_stream) current_stream();
}

AERO_LBM_B200_EXPORT unsigned long long aero_lbm_b200_launch_count(void) { return kernel_launch_count(); }

AERO_LBM_B200_EXPORT int aero_lbm_b200_kernel_timer(int on) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    step_timer_reset(on != 0);
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_kernel_time(double* total_ms, int* launches) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (!total_ms || !launches) return 0;
    return step_timer_read(total_ms, launches) ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_advance_rect(long long key, int steps) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    if (steps < 0) {
        set_error("advance_rect: negative step count");
        return 0;
    }
    Context* c = find_context(key);
    if (!c || !c->has_inputs) {
        set_error("advance_rect: context has no resident inputs");
        return 0;
    }
    for (int i = 0; i < steps; ++i)
        if (!step_context(*c, nullptr, nullptr, 1.0f, true)) return 0;
    return 1;
}

AERO_LBM_B200_EXPORT void aero_lbm_b200_reset_tuning(void) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    g_thermal_mode = -1;
    g_streamed_step = 0;
    g_fused_transport = 0;
    g_cells_per_thread = 2;
    g_fp16_format = 1;
    g_stream_mode = 0;
    g_collision_mode = 0;
    g_smagorinsky_c = -1.0f;
    g_buoyancy_beta_override = -1.0f;
    g_gravity_axis = -1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_set_streaming_mode(int mode) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (mode < 0 || mode > 2) return 0;
    g_stream_mode = mode;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_conservation_sums(long long key, double* out4) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    Context* c = find_context(key);
    if (!c || !c->initialized || !out4) {
        set_error("conservation_sums: no initialized context or null output");
        return 0;
    }
    cudaStream_t s = current_stream();
    const int blocks = conservation_blocks(c->cells);
    const size_t need = (size_t)blocks * 4 * sizeof(double) + 4 * sizeof(double);
    if (c->scratch_cap < need) {
        if (c->scratch) cudaFree(c->scratch);
        c->scratch = nullptr;
        c->scratch_cap = 0;
        if (!cuda_ok(cudaMalloc(&c->scratch, need), "cudaMalloc(conservation scratch)")) return 0;
        c->scratch_cap = need;
    }
    double* partials = static_cast<double*>(c->scratch);
    double* dev_out = partials + (size_t)blocks * 4;
    cudaError_t e;
    if (c->layout == 0) {
        const float* g = c->f_ready ? c->g[1 - c->cur] : c->g[c->cur];
        e = launch_conservation_ab(c->nx, c->ny, c->nz, g, c->flags[c->slot], c->obstacle[c->slot], c->ref_p[c->slot],
                                   c->d_face[c->slot], partials, dev_out, s, c->f_ready ? 1 : 0);
    } else {
        IpArgs a = ip_args(*c, c->slot, c->slot, current_collide_params());
        a.parity = c->parity;
        e = join_fill(*c, s) ? launch_conservation_ip(c->ip_variant, c->ip, a, partials, dev_out, s)
                             : cudaErrorUnknown;
    }
    if (!cuda_ok(e, "conservation kernels")) return 0;
    if (!cuda_ok(cudaMemcpyAsync(out4, dev_out, 4 * sizeof(double), cudaMemcpyDeviceToHost, s), "copy sums")) return 0;
    return cuda_ok(cudaStreamSynchronize(s), "sync") ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_set_collision_mode(int mode) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (mode < 0 || mode > 1) return 0;
    g_collision_mode = mode;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_set_cells_per_thread(int n) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (n != 1 && n != 2) {
        set_error("set_cells_per_thread: 1 or 2");
        return 0;
    }
    g_cells_per_thread = n;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_set_thermal_transport(int mode) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (mode < -1 || mode > 1) {
        set_error("set_thermal_transport: -1, 0 or 1");
        return 0;
    }
    g_thermal_mode = mode;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_set_fused_transport(int on) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (on != 0 && on != 1) {
        set_error("set_fused_transport: 0 (separate pass) or 1 (inside the in-place step)");
        return 0;
    }
    g_fused_transport = on;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_set_streamed_step(int on) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (on != 0 && on != 1) {
        set_error("set_streamed_step: 0 or 1");
        return 0;
    }
    g_streamed_step = on;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_set_fp16_format(int format) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    if (format != 0 && format != 1) {
        set_error("set_fp16_format: 0 (IEEE half) or 1 (16-bit fixed point)");
        return 0;
    }
    g_fp16_format = format;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_set_force_field(long long key, const float* force_soa, int value_count) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    clear_error();
    Context* c = find_context(key);
    if (!c) {
        set_error("set_force_field: unknown context");
        return 0;
    }
    if (!force_soa) {
        if (c->force) cudaFree(c->force);
        c->force = nullptr;
        return 1;
    }
    if ((long long)value_count != 3 * c->cells) {
        set_error("set_force_field: value_count must be 3 * cells");
        return 0;
    }
    if (!c->force && !cuda_ok(cudaMalloc(reinterpret_cast<void**>(&c->force), (size_t)c->cells * 3 * sizeof(float) + kCopySlack), "cudaMalloc(force)")) return 0;
    cudaStream_t s = current_stream();
    if (!cuda_ok(cudaMemcpyAsync(c->force, force_soa, (size_t)c->cells * 3 * sizeof(float), cudaMemcpyHostToDevice, s), "copy force")) return 0;
    return cuda_ok(cudaStreamSynchronize(s), "sync") ? 1 : 0;
}

AERO_LBM_B200_EXPORT void aero_lbm_b200_set_physics_overrides(float smagorinsky_c, float buoyancy_beta, int gravity_axis) {
    std::lock_guard<std::recursive_mutex> lk(g_mutex);
    g_smagorinsky_c = std::isfinite(smagorinsky_c) ? smagorinsky_c : -1.0f;
    g_buoyancy_beta_override = std::isfinite(buoyancy_beta) ? buoyancy_beta : -1.0f;
    g_gravity_axis = (gravity_axis >= 0 && gravity_axis <= 2) ? gravity_axis : -1;
}

}  // extern "C"
