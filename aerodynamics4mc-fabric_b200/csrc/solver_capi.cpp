// Wind-tunnel C ABI (handle based), layered on the per-context LBM ABI.
//
// Same observable behaviour as the reference's aero_solver_* layer
// (native/src/aero_solver_capi.cpp): an 11-channel packet per handle, the
// boundary mode mapped onto the boundary configuration (inlet velocity
// Dirichlet at x-, convective outflow or pressure outlet at x+, symmetry
// elsewhere; closed and periodic modes), SGS and buoyancy off, velocities
// converted between m/s and lattice units with dx/dt. Creating a solver
// re-initialises the LBM runtime and drops other handles, as the reference
// does (aero_solver_capi.cpp:356-414).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/aero_lbm_b200.h"

namespace {

constexpr int kInputChannels = 11;
constexpr int kOutputChannels = AERO_SOLVER_FLOW_CHANNELS;
constexpr float kDefaultDx = 1.0f;
constexpr float kDefaultDt = 0.05f;
constexpr float kDefaultDensity = 1.225f;
constexpr float kDefaultViscosity = 1.5e-5f;
constexpr float kMinLatticeNu = 1.0e-7f;
constexpr float kMaxLatticeNu = 0.12f;

struct Tunnel {
    long long handle = 0;
    long long context_key = 0;
    AeroGridDesc grid{};
    int cells = 0;
    bool custom_flow = false;
    bool packet_dirty = true;
    bool uploaded = false;
    AeroBoundaryDesc packet_boundary{};
    std::vector<uint8_t> solid;
    std::vector<float> packet;
};

std::mutex g_mu;
std::unordered_map<long long, std::unique_ptr<Tunnel>> g_tunnels;
long long g_next = 1;
std::string g_err;

void set_err(const std::string& m) { g_err = m; }
float finite_or(float v, float fb) { return std::isfinite(v) ? v : fb; }
float to_lattice(const AeroGridDesc& g, float v) { return finite_or(v, 0.0f) / (g.dx / g.dt); }

bool grid_ok(const AeroGridDesc& g, int* cells) {
    if (g.nx <= 0 || g.ny <= 0 || g.nz <= 0) {
        set_err("invalid grid dimensions");
        return false;
    }
    if (!std::isfinite(g.dx) || g.dx <= 0.0f || !std::isfinite(g.dt) || g.dt <= 0.0f) {
        set_err("invalid grid dx/dt");
        return false;
    }
    const long long c = (long long)g.nx * g.ny * g.nz;
    if (c <= 0 || c > (long long)std::numeric_limits<int>::max()) {
        set_err("grid cell count overflows int");
        return false;
    }
    *cells = (int)c;
    return true;
}

Tunnel* lookup(long long h) {
    auto it = g_tunnels.find(h);
    if (it == g_tunnels.end() || !it->second) {
        set_err("invalid solver handle");
        return nullptr;
    }
    return it->second.get();
}

void write_flow(Tunnel& t, size_t cell, float vx, float vy, float vz, float p) {
    float* rec = t.packet.data() + cell * kInputChannels;
    rec[5] = to_lattice(t.grid, vx);
    rec[6] = to_lattice(t.grid, vy);
    rec[7] = to_lattice(t.grid, vz);
    rec[8] = finite_or(p, 0.0f);
}

void fill_packet(Tunnel& t, const AeroBoundaryDesc& b, bool overwrite_flow) {
    for (int c = 0; c < t.cells; ++c) {
        float* rec = t.packet.data() + (size_t)c * kInputChannels;
        const bool solid = t.solid[(size_t)c] != 0;
        rec[0] = solid ? 1.0f : 0.0f;
        rec[1] = rec[2] = rec[3] = rec[4] = 0.0f;
        rec[9] = rec[10] = 0.0f;
        if (solid) write_flow(t, (size_t)c, 0.0f, 0.0f, 0.0f, 0.0f);
        else if (overwrite_flow) write_flow(t, (size_t)c, finite_or(b.inlet_vx, 0.0f), finite_or(b.inlet_vy, 0.0f),
                                            finite_or(b.inlet_vz, 0.0f), b.outlet_pressure);
    }
}

bool same_packet_boundary(const AeroBoundaryDesc& a, const AeroBoundaryDesc& b) {
    return a.mode == b.mode && a.inlet_vx == b.inlet_vx && a.inlet_vy == b.inlet_vy && a.inlet_vz == b.inlet_vz &&
           a.outlet_pressure == b.outlet_pressure;
}

float lattice_nu(const Tunnel& t, const AeroBoundaryDesc& b) {
    const float visc = finite_or(b.viscosity, kDefaultViscosity);
    const float nu = visc > 0.0f ? visc * t.grid.dt / (t.grid.dx * t.grid.dx) : kDefaultViscosity;
    return std::clamp(nu, kMinLatticeNu, kMaxLatticeNu);
}

AeroLbmBoundaryFaceConfig face(int hydro) {
    AeroLbmBoundaryFaceConfig f{};
    f.hydrodynamic_kind = hydro;
    f.thermal_kind = AERO_LBM_THERMAL_BOUNDARY_DISABLED;
    return f;
}

// configure_benchmark_boundary (aero_solver_capi.cpp:209-261)
bool configure(const Tunnel& t, const AeroBoundaryDesc& b) {
    AeroLbmBenchmarkConfig c{};
    aero_lbm_benchmark_default_config(&c);
    c.enabled = 1;
    c.preset = AERO_LBM_BENCHMARK_PRESET_NONE;
    c.flags |= AERO_LBM_BENCHMARK_FLAG_DISABLE_FAN_FORCING | AERO_LBM_BENCHMARK_FLAG_DISABLE_FAN_NOISE |
               AERO_LBM_BENCHMARK_FLAG_DISABLE_SPONGE | AERO_LBM_BENCHMARK_FLAG_DISABLE_OBSTACLE_BOUNCE_BLEND |
               AERO_LBM_BENCHMARK_FLAG_DISABLE_SGS | AERO_LBM_BENCHMARK_FLAG_DISABLE_INTERNAL_THERMAL_SOURCE |
               AERO_LBM_BENCHMARK_FLAG_DISABLE_BUOYANCY;
    c.flags &= ~(uint32_t)AERO_LBM_BENCHMARK_FLAG_DISABLE_CONVECTIVE_OUTFLOW;
    c.reference_density = std::max(1.0e-6f, finite_or(b.density, kDefaultDensity));
    c.reference_temperature = 0.0f;
    c.reference_length = 1.0f;
    c.initial_velocity[0] = to_lattice(t.grid, b.inlet_vx);
    c.initial_velocity[1] = to_lattice(t.grid, b.inlet_vy);
    c.initial_velocity[2] = to_lattice(t.grid, b.inlet_vz);
    c.initial_pressure = finite_or(b.outlet_pressure, 0.0f);
    const float speed = std::max(
        std::sqrt(c.initial_velocity[0] * c.initial_velocity[0] + c.initial_velocity[1] * c.initial_velocity[1] +
                  c.initial_velocity[2] * c.initial_velocity[2]),
        1.0e-6f);
    c.reynolds_number = std::max(1.0e-6f, speed / lattice_nu(t, b));
    c.mach_number = std::clamp(speed / std::sqrt(1.0f / 3.0f), 1.0e-4f, 0.30f);
    const int mode = b.mode == 0 ? AERO_SOLVER_BOUNDARY_WIND_TUNNEL : b.mode;
    auto all = [&](int k) { c.x_min = c.x_max = c.y_min = c.y_max = c.z_min = c.z_max = face(k); };
    switch (mode) {
        case AERO_SOLVER_BOUNDARY_CLOSED:
            all(AERO_LBM_HYDRO_BOUNDARY_BOUNCE_BACK);
            break;
        case AERO_SOLVER_BOUNDARY_PERIODIC:
            all(AERO_LBM_HYDRO_BOUNDARY_PERIODIC);
            break;
        case AERO_SOLVER_BOUNDARY_WIND_TUNNEL_PRESSURE_OUTLET:
            all(AERO_LBM_HYDRO_BOUNDARY_SYMMETRY);
            c.x_min = face(AERO_LBM_HYDRO_BOUNDARY_VELOCITY_DIRICHLET);
            c.x_max = face(AERO_LBM_HYDRO_BOUNDARY_PRESSURE_DIRICHLET);
            c.x_max.pressure = finite_or(b.outlet_pressure, 0.0f);
            break;
        case AERO_SOLVER_BOUNDARY_WIND_TUNNEL:
            all(AERO_LBM_HYDRO_BOUNDARY_SYMMETRY);
            c.x_min = face(AERO_LBM_HYDRO_BOUNDARY_VELOCITY_DIRICHLET);
            c.x_max = face(AERO_LBM_HYDRO_BOUNDARY_CONVECTIVE_OUTFLOW);
            break;
        default:
            set_err("invalid wind-tunnel boundary mode");
            return false;
    }
    c.x_min.velocity[0] = c.initial_velocity[0];
    c.x_min.velocity[1] = c.initial_velocity[1];
    c.x_min.velocity[2] = c.initial_velocity[2];
    return aero_lbm_benchmark_set_config(&c) != 0;
}

// step_solver_locked (aero_solver_capi.cpp:268-330); the resident-packet
// (cached) path is always available on this runtime.
bool step_locked(Tunnel& t, const AeroBoundaryDesc& b, int steps, float* out, int out_count) {
    if (steps <= 0) {
        set_err("steps must be positive");
        return false;
    }
    if (out && out_count != t.cells * kOutputChannels) {
        set_err("invalid output flow buffer");
        return false;
    }
    if (!configure(t, b)) {
        if (g_err.empty()) set_err(std::string("failed to configure boundary: ") + aero_lbm_last_error());
        return false;
    }
    const bool overwrite = !t.custom_flow;
    const bool changed = overwrite && !same_packet_boundary(t.packet_boundary, b);
    if (t.packet_dirty || changed) {
        fill_packet(t, b, overwrite);
        t.packet_boundary = b;
        t.packet_dirty = false;
        t.uploaded = false;
    }
    const float scale = t.grid.dx / t.grid.dt;
    for (int s = 0; s < steps; ++s) {
        float* step_out = (out && s + 1 == steps) ? out : nullptr;
        int ok = 0;
        if (t.uploaded) {
            ok = aero_lbm_step_rect_cached_scaled(t.grid.nx, t.grid.ny, t.grid.nz, t.context_key, scale, step_out);
        } else {
            ok = aero_lbm_step_rect_scaled(t.packet.data(), t.grid.nx, t.grid.ny, t.grid.nz, t.context_key, scale, step_out);
            t.uploaded = ok != 0;
        }
        if (!ok) {
            set_err(std::string("aero_lbm_step_rect failed: ") + aero_lbm_last_error());
            return false;
        }
    }
    return true;
}

}  // namespace

extern "C" {

AERO_LBM_B200_EXPORT void aero_solver_default_grid(AeroGridDesc* g) {
    if (!g) return;
    g->nx = g->ny = g->nz = 64;
    g->dx = kDefaultDx;
    g->dt = kDefaultDt;
}

AERO_LBM_B200_EXPORT void aero_solver_default_boundary(AeroBoundaryDesc* b) {
    if (!b) return;
    b->mode = AERO_SOLVER_BOUNDARY_WIND_TUNNEL;
    b->inlet_vx = 5.0f;
    b->inlet_vy = 0.0f;
    b->inlet_vz = 0.0f;
    b->outlet_pressure = 0.0f;
    b->density = kDefaultDensity;
    b->viscosity = kDefaultViscosity;
}

AERO_LBM_B200_EXPORT int aero_solver_create_with_grid(const AeroGridDesc* grid, long long* out_handle) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_err.clear();
    if (!grid || !out_handle) {
        set_err("missing grid or output handle");
        return AERO_SOLVER_STATUS_ERROR;
    }
    int cells = 0;
    if (!grid_ok(*grid, &cells)) return AERO_SOLVER_STATUS_ERROR;
    if (!aero_lbm_init_rect(grid->nx, grid->ny, grid->nz, kInputChannels, kOutputChannels)) {
        set_err(std::string("aero_lbm_init_rect failed: ") + aero_lbm_last_error());
        return AERO_SOLVER_STATUS_ERROR;
    }
    g_tunnels.clear();
    auto t = std::make_unique<Tunnel>();
    t->handle = g_next++;
    if (g_next <= 0) g_next = 1;
    t->context_key = t->handle;
    t->grid = *grid;
    t->cells = cells;
    t->solid.assign((size_t)cells, 0u);
    t->packet.assign((size_t)cells * kInputChannels, 0.0f);
    AeroBoundaryDesc b{};
    aero_solver_default_boundary(&b);
    fill_packet(*t, b, true);
    t->packet_boundary = b;
    t->packet_dirty = false;
    const long long h = t->handle;
    g_tunnels.emplace(h, std::move(t));
    *out_handle = h;
    return AERO_SOLVER_STATUS_OK;
}

AERO_LBM_B200_EXPORT int aero_solver_create(int nx, int ny, int nz, float dx, float dt, long long* out_handle) {
    AeroGridDesc g{nx, ny, nz, dx, dt};
    return aero_solver_create_with_grid(&g, out_handle);
}

AERO_LBM_B200_EXPORT int aero_solver_set_solid_mask(long long handle, const uint8_t* mask, int cell_count) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_err.clear();
    Tunnel* t = lookup(handle);
    if (!t) return AERO_SOLVER_STATUS_ERROR;
    if (!mask || cell_count != t->cells) {
        set_err("invalid solid mask buffer");
        return AERO_SOLVER_STATUS_ERROR;
    }
    t->solid.assign(mask, mask + cell_count);
    t->custom_flow = false;
    t->packet_dirty = true;
    t->uploaded = false;
    aero_lbm_release_context(t->context_key);
    return AERO_SOLVER_STATUS_OK;
}

AERO_LBM_B200_EXPORT int aero_solver_set_flow_state(long long handle, const float* flow, int value_count) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_err.clear();
    Tunnel* t = lookup(handle);
    if (!t) return AERO_SOLVER_STATUS_ERROR;
    if (!flow || value_count != t->cells * kOutputChannels) {
        set_err("invalid flow state buffer");
        return AERO_SOLVER_STATUS_ERROR;
    }
    for (int c = 0; c < t->cells; ++c) {
        if (t->solid[(size_t)c]) {
            write_flow(*t, (size_t)c, 0.0f, 0.0f, 0.0f, 0.0f);
            continue;
        }
        const float* f = flow + (size_t)c * kOutputChannels;
        write_flow(*t, (size_t)c, f[0], f[1], f[2], f[3]);
    }
    t->custom_flow = true;
    t->packet_dirty = false;
    t->uploaded = false;
    aero_lbm_release_context(t->context_key);
    return AERO_SOLVER_STATUS_OK;
}

AERO_LBM_B200_EXPORT int aero_solver_step_wind_tunnel(long long handle, const AeroBoundaryDesc* boundary, int steps,
                                                      float* out_flow, int out_value_count) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_err.clear();
    Tunnel* t = lookup(handle);
    if (!t) return AERO_SOLVER_STATUS_ERROR;
    AeroBoundaryDesc b{};
    aero_solver_default_boundary(&b);
    if (boundary) b = *boundary;
    return step_locked(*t, b, steps, out_flow, out_value_count) ? AERO_SOLVER_STATUS_OK : AERO_SOLVER_STATUS_ERROR;
}

AERO_LBM_B200_EXPORT int aero_solver_advance_wind_tunnel(long long handle, const AeroBoundaryDesc* boundary, int steps) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_err.clear();
    Tunnel* t = lookup(handle);
    if (!t) return AERO_SOLVER_STATUS_ERROR;
    AeroBoundaryDesc b{};
    aero_solver_default_boundary(&b);
    if (boundary) b = *boundary;
    return step_locked(*t, b, steps, nullptr, 0) ? AERO_SOLVER_STATUS_OK : AERO_SOLVER_STATUS_ERROR;
}

AERO_LBM_B200_EXPORT int aero_solver_run_wind_tunnel(const AeroStepInput* in, AeroStepOutput* out) {
    if (!in || !out || !out->flow_out) {
        std::lock_guard<std::mutex> lk(g_mu);
        set_err("missing step input or output");
        return AERO_SOLVER_STATUS_ERROR;
    }
    long long h = 0;
    if (!aero_solver_create_with_grid(&in->grid, &h)) {
        out->status = AERO_SOLVER_STATUS_ERROR;
        return AERO_SOLVER_STATUS_ERROR;
    }
    const int cells = in->grid.nx * in->grid.ny * in->grid.nz;
    if (in->solid_mask && !aero_solver_set_solid_mask(h, in->solid_mask, cells)) {
        aero_solver_destroy(h);
        out->status = AERO_SOLVER_STATUS_ERROR;
        return AERO_SOLVER_STATUS_ERROR;
    }
    if (in->prev_flow && !aero_solver_set_flow_state(h, in->prev_flow, cells * kOutputChannels)) {
        aero_solver_destroy(h);
        out->status = AERO_SOLVER_STATUS_ERROR;
        return AERO_SOLVER_STATUS_ERROR;
    }
    const int ok = aero_solver_step_wind_tunnel(h, &in->boundary, in->steps, out->flow_out, cells * kOutputChannels);
    float vmax = 0.0f;
    if (ok) {
        for (int c = 0; c < cells; ++c) {
            const float* f = out->flow_out + (size_t)c * kOutputChannels;
            const float s = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
            if (std::isfinite(s)) vmax = std::max(vmax, s);
        }
    }
    out->max_velocity = vmax;
    out->status = ok;
    aero_solver_destroy(h);
    return ok;
}

AERO_LBM_B200_EXPORT void aero_solver_destroy(long long handle) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_tunnels.find(handle);
    if (it == g_tunnels.end()) return;
    aero_lbm_release_context(it->second->context_key);
    g_tunnels.erase(it);
}

AERO_LBM_B200_EXPORT const char* aero_solver_last_error(void) {
    return g_err.empty() ? aero_lbm_last_error() : g_err.c_str();
}

AERO_LBM_B200_EXPORT const char* aero_solver_runtime_info(void) { return aero_lbm_runtime_info(); }

AERO_LBM_B200_EXPORT int aero_solver_finish(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_err.clear();
    if (!aero_lbm_finish()) {
        set_err(std::string("aero_lbm_finish failed: ") + aero_lbm_last_error());
        return AERO_SOLVER_STATUS_ERROR;
    }
    return AERO_SOLVER_STATUS_OK;
}

}  // extern "C"
