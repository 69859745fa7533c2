// Host side of the D3Q19 mesoscale ABI: contexts keyed like the reference's
// (native/src/aero_lbm_mesoscale.cpp:215-240, 1397-1510), per-call transport
// derivation, seeding, and the two step paths: the reference model (two
// launches per call, hydrodynamic + thermal distributions) and the
// hydrodynamic-only fused step (one launch per call, FP32 or FP16 storage).
#include <algorithm>
#include <cmath>
#include <map>
#include <string>

#include "../../include/aero_lbm_b200.h"
#include "meso.cuh"
#include "runtime_internal.h"

namespace aero {
namespace {

struct Transport {
    float velocity_scale, nu_lattice, alpha_lattice, tau_shear, tau_thermal;
};

// valid_transport_spec (native/src/aero_lbm_hydro_core.cpp:7-21)
bool config_valid(const AeroLbmMesoscaleConfig* c) {
    return c && c->abi_version == AERO_LBM_MESOSCALE_ABI_VERSION && c->struct_size >= sizeof(AeroLbmMesoscaleConfig) &&
           c->nx > 0 && c->ny > 0 && c->nz > 0 && std::isfinite(c->dx_m) && std::isfinite(c->dt_s) &&
           std::isfinite(c->molecular_nu_m2_s) && std::isfinite(c->prandtl_air) && std::isfinite(c->turbulent_prandtl) &&
           c->dx_m > 0.0f && c->dt_s > 0.0f && c->molecular_nu_m2_s > 0.0f && c->prandtl_air > 0.0f &&
           c->turbulent_prandtl > 0.0f;
}

// derive_hydro_transport / derive_thermal_transport
// (native/src/aero_lbm_hydro_core.cpp:22-31, native/src/aero_lbm_thermal_core.cpp:5-15,
//  native/include/aero_lbm_hydro_core.h:109-115, native/include/aero_lbm_thermal_core.h:22-28)
Transport derive(const AeroLbmMesoscaleConfig& c) {
    Transport t{};
    t.velocity_scale = c.dx_m / c.dt_s;
    t.nu_lattice = c.molecular_nu_m2_s * c.dt_s / (c.dx_m * c.dx_m);
    t.tau_shear = 0.5f + 3.0f * t.nu_lattice;
    const float alpha = c.molecular_nu_m2_s / c.prandtl_air;
    t.alpha_lattice = alpha * c.dt_s / (c.dx_m * c.dx_m);
    t.tau_thermal = 0.5f + t.alpha_lattice / 0.25f;
    return t;
}

// trt_odd_tau (native/src/aero_lbm_mesoscale.cpp:269-272)
float trt_odd_tau(float even_tau) {
    const float d = std::max(0.03f, even_tau - 0.5f);
    return std::clamp(0.5f + 0.25f / d, 0.55f, 2.5f);
}

AeroLbmB200MesoscaleOptions default_options() {
    AeroLbmB200MesoscaleOptions o{};
    o.tau_hydro = 0.58;
    o.smagorinsky_c = 0.1;
    return o;
}

struct MesoContext {
    AeroLbmMesoscaleConfig config{};
    AeroLbmB200MesoscaleOptions opt = default_options();
    int nx = 0, ny = 0, nz = 0;
    long long cells = 0;
    bool initialized = false;
    bool hydro = false;     // layout of the allocated state
    int storage = 0;        // kMesoStore* of the allocated state (hydro only)
    float fp16_scale = 1.0f;
    float* forcing[2] = {nullptr, nullptr};
    uint8_t* solid[2] = {nullptr, nullptr};
    uint32_t* flags[2] = {nullptr, nullptr};  // hydro: pull classification of solid[k]
    int fslot = 0;          // forcing / mask of the last step call
    // reference model
    float *f = nullptr, *g = nullptr, *pf = nullptr, *pg = nullptr;
    float *ambient = nullptr, *deep = nullptr, *surface = nullptr, *ndeep = nullptr, *nsurf = nullptr;
    // hydrodynamic only
    void* pop[2] = {nullptr, nullptr};
    int cur = 0;
    float* out = nullptr;   // device output state, cells x 6
    bool out_valid = false; // reference model: out holds the last step's state

    ~MesoContext() { release(); }
    void release() {
        for (void* p : {(void*)forcing[0], (void*)forcing[1], (void*)solid[0], (void*)solid[1], (void*)flags[0],
                        (void*)flags[1], (void*)f, (void*)g,
                        (void*)pf, (void*)pg, (void*)ambient, (void*)deep, (void*)surface, (void*)ndeep, (void*)nsurf,
                        pop[0], pop[1], (void*)out})
            if (p) cudaFree(p);
        forcing[0] = forcing[1] = nullptr;
        solid[0] = solid[1] = nullptr;
        flags[0] = flags[1] = nullptr;
        f = g = pf = pg = ambient = deep = surface = ndeep = nsurf = out = nullptr;
        pop[0] = pop[1] = nullptr;
        cells = 0;
        initialized = false;
        out_valid = false;
    }
    double bytes_per_step() const {
        if (hydro) return (double)cells * (19.0 * 2.0 * (storage ? 2.0 : 4.0) + 1.0);
        // collide: f, g read + written; stream: post f, g read, f, g written; forcing 2 x 100 B; fields; output
        return (double)cells * (19.0 * 4.0 * 8.0 + 2.0 * 100.0 + 10.0 * 4.0 + 24.0);
    }
};

std::map<long long, MesoContext*> g_meso;
long long g_next_meso_key = 1;

template <class T>
bool dev_alloc(T** p, size_t count, const char* what) {
    return cuda_ok(cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T)), what);
}

bool allocate(MesoContext& c) {
    c.release();
    c.nx = c.config.nx;
    c.ny = c.config.ny;
    c.nz = c.config.nz;
    c.cells = (long long)c.nx * c.ny * c.nz;
    c.hydro = c.opt.hydro_only != 0;
    c.storage = c.hydro ? c.opt.storage : 0;
    const size_t n = (size_t)c.cells;
    bool ok = dev_alloc(&c.forcing[0], n * kMesoForcingChannels, "meso forcing") &&
              dev_alloc(&c.forcing[1], n * kMesoForcingChannels, "meso forcing") &&
              dev_alloc(&c.solid[0], n, "meso mask") && dev_alloc(&c.solid[1], n, "meso mask") &&
              dev_alloc(&c.out, n * kMesoStateChannels, "meso output");
    if (!ok) return false;
    if (c.hydro) {
        const size_t bytes = n * 19 * (c.storage ? 2 : 4);
        ok = cuda_ok(cudaMalloc(&c.pop[0], bytes), "meso populations") && cuda_ok(cudaMalloc(&c.pop[1], bytes), "meso populations") &&
             dev_alloc(&c.flags[0], n, "meso flags") && dev_alloc(&c.flags[1], n, "meso flags");
    } else {
        ok = dev_alloc(&c.f, n * 19, "meso f") && dev_alloc(&c.g, n * 19, "meso g") && dev_alloc(&c.pf, n * 19, "meso post f") &&
             dev_alloc(&c.pg, n * 19, "meso post g") && dev_alloc(&c.ambient, n, "meso ambient") &&
             dev_alloc(&c.deep, n, "meso deep") && dev_alloc(&c.surface, n, "meso surface") &&
             dev_alloc(&c.ndeep, n, "meso deep") && dev_alloc(&c.nsurf, n, "meso surface");
    }
    return ok;
}

meso::HydroRates rates(const MesoContext& c, const Transport& t) {
    meso::HydroRates h{};
    const float tau_h = c.opt.fixed_tau ? (float)c.opt.tau_hydro : std::clamp(t.tau_shear, 0.58f, 2.5f);
    h.tau_h = tau_h;
    h.omega_even = 1.0f / tau_h;
    h.omega_odd = 1.0f / trt_odd_tau(tau_h);
    h.enable_sgs = c.opt.enable_sgs ? 1 : 0;
    h.smagorinsky_c = (float)c.opt.smagorinsky_c;
    h.fx = (float)c.opt.body_force[0];
    h.fy = (float)c.opt.body_force[1];
    h.fz = (float)c.opt.body_force[2];
    h.forced = (h.fx != 0.0f || h.fy != 0.0f || h.fz != 0.0f) ? 1 : 0;
    return h;
}

meso::MesoArgs model_args(MesoContext& c, const Transport& t, int slot, float* out_state) {
    meso::MesoArgs a{};
    a.nx = c.nx;
    a.ny = c.ny;
    a.nz = c.nz;
    a.periodic_sides = c.opt.periodic_sides ? 1 : 0;
    a.free_slip_top = c.opt.free_slip_top ? 1 : 0;
    a.edge_blend = c.opt.disable_edge_blend ? 0 : 1;
    a.dt_s = c.config.dt_s;
    a.velocity_scale = t.velocity_scale;
    a.max_speed = 0.35f * t.velocity_scale;
    a.h = rates(c, t);
    const float tau_t = std::clamp(t.tau_thermal, 0.58f, 2.5f);
    a.omega_t_even = 1.0f / tau_t;
    a.omega_t_odd = 1.0f / trt_odd_tau(tau_t);
    a.forcing = c.forcing[slot];
    a.f = c.f;
    a.g = c.g;
    a.post_f = c.pf;
    a.post_g = c.pg;
    a.ambient = c.ambient;
    a.deep = c.deep;
    a.surface = c.surface;
    a.next_deep = c.ndeep;
    a.next_surface = c.nsurf;
    a.out_state = out_state;
    return a;
}

meso::HydroArgs hydro_args(const MesoContext& c, const Transport& t, int prev_slot, int cur_slot) {
    meso::HydroArgs a{};
    a.nx = c.nx;
    a.ny = c.ny;
    a.nz = c.nz;
    a.periodic_sides = c.opt.periodic_sides ? 1 : 0;
    a.free_slip_top = c.opt.free_slip_top ? 1 : 0;
    a.edge_blend = c.opt.disable_edge_blend ? 0 : 1;
    a.velocity_scale = t.velocity_scale;
    a.max_speed = 0.35f * t.velocity_scale;
    a.scale = c.storage ? c.fp16_scale : 1.0f;
    a.inv_scale = c.storage ? 1.0f / c.fp16_scale : 1.0f;
    a.h = rates(c, t);
    a.solid_prev = c.solid[prev_slot];
    a.flags_prev = c.flags[prev_slot];
    a.solid_cur = c.solid[cur_slot];
    a.forcing_prev = c.forcing[prev_slot];
    a.src = c.pop[c.cur];
    a.dst = c.pop[c.cur ^ 1];
    a.out_state = c.out;
    return a;
}

int hydro_threads(const MesoContext& c) { return c.opt.threads > 0 ? c.opt.threads : 256; }

// One step of the reference model on forcing slot `slot` (two launches).
bool model_step(MesoContext& c, const Transport& t, int slot, cudaStream_t s) {
    if (!cuda_ok(meso_launch_step(model_args(c, t, slot, c.out), s), "mesoscale step")) return false;
    std::swap(c.deep, c.ndeep);
    std::swap(c.surface, c.nsurf);
    c.out_valid = true;
    return true;
}

// One hydrodynamic-only call: fused pull (prev_slot) + collision (cur_slot).
bool hydro_step(MesoContext& c, const Transport& t, int prev_slot, int cur_slot, cudaStream_t s) {
    const meso::HydroArgs a = hydro_args(c, t, prev_slot, cur_slot);
    const bool packed = c.opt.collision == 1 && c.nz % 2 == 0;
    if (!cuda_ok(packed ? meso_hydro_fast_step(a, c.storage, s) : meso_hydro_launch(a, kHydroStep, c.storage, hydro_threads(c), s),
                 "mesoscale hydro step"))
        return false;
    c.cur ^= 1;
    return true;
}

bool hydro_output(MesoContext& c, const Transport& t, cudaStream_t s) {
    const meso::HydroArgs a = hydro_args(c, t, c.fslot, c.fslot);
    return cuda_ok(meso_hydro_launch(a, kHydroOutput, c.storage, hydro_threads(c), s), "mesoscale hydro output");
}

// Largest |lattice wind| of the seeding forcing (host copy), for the FP16 scale.
float seed_speed(const float* forcing, long long cells, float velocity_scale) {
    const float den = std::max(1.0e-6f, velocity_scale);
    float m = 0.0f;
    for (long long i = 0; i < cells; ++i) {
        const float* F = forcing + i * kMesoForcingChannels;
        if (F[kChSolidMask] > 0.5f) continue;
        const float bx = (F[kChBackgroundWindX] + F[kChNestedWindXDelta] + F[kChConvectiveInflowX] + F[kChTornadoWindX]) / den;
        const float bz = (F[kChBackgroundWindZ] + F[kChNestedWindZDelta] + F[kChConvectiveInflowZ] + F[kChTornadoWindZ]) / den;
        const float by = (F[kChNestedUpdraft] + F[kChTornadoUpdraft]) / den;
        m = std::max(m, std::sqrt(bx * bx + by * by + bz * bz));
    }
    return std::min(m, 0.35f * 1.7320508f);
}

MesoContext* find_meso(long long key) {
    auto it = g_meso.find(key);
    return it == g_meso.end() ? nullptr : it->second;
}

}  // namespace
}  // namespace aero

using namespace aero;

extern "C" {

AERO_LBM_B200_EXPORT void aero_lbm_mesoscale_default_config(AeroLbmMesoscaleConfig* c) {
    if (!c) return;
    *c = AeroLbmMesoscaleConfig{};
    c->abi_version = AERO_LBM_MESOSCALE_ABI_VERSION;
    c->struct_size = sizeof(AeroLbmMesoscaleConfig);
    c->nx = 32;
    c->ny = 4;
    c->nz = 32;
    c->dx_m = 64.0f;
    c->dt_s = 5.0f;
    c->molecular_nu_m2_s = 1.5e-5f;
    c->prandtl_air = 0.71f;
    c->turbulent_prandtl = 0.85f;
    c->reference_density_kg_m3 = 1.225f;
    c->ambient_air_temperature_k = 288.15f;
    c->deep_ground_temperature_k = 289.65f;
}

AERO_LBM_B200_EXPORT int aero_lbm_mesoscale_derive_transport(const AeroLbmMesoscaleConfig* config,
                                                             AeroLbmMesoscaleTransport* out) {
    if (!config_valid(config) || !out) return 0;
    const Transport t = derive(*config);
    out->velocity_scale_m_s_per_lattice = t.velocity_scale;
    out->nu_molecular_lattice = t.nu_lattice;
    out->alpha_molecular_lattice = t.alpha_lattice;
    out->tau_shear_molecular = t.tau_shear;
    out->tau_thermal_molecular = t.tau_thermal;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_mesoscale_create_context(const AeroLbmMesoscaleConfig* config, long long* out_key) {
    std::lock_guard<std::recursive_mutex> lk(runtime_mutex());
    if (!config_valid(config) || !out_key) return 0;
    auto* c = new MesoContext();
    c->config = *config;
    const long long key = g_next_meso_key++;
    g_meso[key] = c;
    *out_key = key;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_mesoscale_step_context(long long key, const AeroLbmMesoscaleConfig* config,
                                                         const float* forcing, float* out_state) {
    std::lock_guard<std::recursive_mutex> lk(runtime_mutex());
    clear_error();
    if (!config_valid(config) || !forcing || !out_state) {
        set_error("mesoscale_step_context: invalid config or null forcing / output");
        return 0;
    }
    MesoContext* c = find_meso(key);
    if (!c) {
        set_error("mesoscale_step_context: unknown context");
        return 0;
    }
    const bool shape_changed = c->nx != config->nx || c->ny != config->ny || c->nz != config->nz;
    c->config = *config;
    if (shape_changed || !c->cells || c->hydro != (c->opt.hydro_only != 0) ||
        c->storage != (c->opt.hydro_only != 0 ? c->opt.storage : 0)) {
        if (!allocate(*c)) return 0;
    }
    const Transport t = derive(*config);
    cudaStream_t s = current_stream();
    const size_t fbytes = (size_t)c->cells * kMesoForcingChannels * sizeof(float);
    const int slot = c->initialized ? (c->fslot ^ 1) : 0;
    if (!cuda_ok(cudaMemcpyAsync(c->forcing[slot], forcing, fbytes, cudaMemcpyHostToDevice, s), "mesoscale forcing upload"))
        return 0;
    if (c->hydro) {
        if (!c->initialized) {
            const float us = seed_speed(forcing, c->cells, t.velocity_scale);
            c->fp16_scale = c->storage == kMesoStoreF16 ? fp16_scale_for_speed(us)
                          : c->storage == kMesoStoreI16 ? i16_scale_for_speed(us) : 1.0f;
            c->cur = 0;
            if (!cuda_ok(meso_hydro_seed(c->forcing[slot], c->nx, c->ny, c->nz, t.velocity_scale, c->storage, c->fp16_scale,
                                         c->pop[0], c->solid[slot], s), "mesoscale hydro seed") ||
                !cuda_ok(meso_hydro_flags(hydro_args(*c, t, slot, slot), c->solid[slot], c->flags[slot], s), "mesoscale flags"))
                return 0;
            const meso::HydroArgs a = hydro_args(*c, t, slot, slot);
            if (!cuda_ok(meso_hydro_launch(a, kHydroInit, c->storage, hydro_threads(*c), s), "mesoscale hydro init")) return 0;
            c->cur = 1;
            c->initialized = true;
        } else {
            if (!cuda_ok(meso_hydro_mask(c->forcing[slot], c->cells, c->solid[slot], s), "mesoscale mask") ||
                !cuda_ok(meso_hydro_flags(hydro_args(*c, t, slot, slot), c->solid[slot], c->flags[slot], s), "mesoscale flags"))
                return 0;
            if (!hydro_step(*c, t, c->fslot, slot, s)) return 0;
        }
        c->fslot = slot;
        if (!hydro_output(*c, t, s)) return 0;
    } else {
        if (!c->initialized) {
            if (!cuda_ok(meso_launch_seed(model_args(*c, t, slot, nullptr), s), "mesoscale seed")) return 0;
            c->initialized = true;
        }
        c->fslot = slot;
        if (!model_step(*c, t, slot, s)) return 0;
    }
    const size_t obytes = (size_t)c->cells * kMesoStateChannels * sizeof(float);
    if (!cuda_ok(cudaMemcpyAsync(out_state, c->out, obytes, cudaMemcpyDeviceToHost, s), "mesoscale output copy")) return 0;
    return cuda_ok(cudaStreamSynchronize(s), "mesoscale step sync") ? 1 : 0;
}

AERO_LBM_B200_EXPORT void aero_lbm_mesoscale_release_context(long long key) {
    std::lock_guard<std::recursive_mutex> lk(runtime_mutex());
    auto it = g_meso.find(key);
    if (it == g_meso.end()) return;
    cudaStreamSynchronize(current_stream());
    delete it->second;
    g_meso.erase(it);
}

AERO_LBM_B200_EXPORT void aero_lbm_b200_mesoscale_default_options(AeroLbmB200MesoscaleOptions* out) {
    if (out) *out = default_options();
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_mesoscale_set_options(long long key, const AeroLbmB200MesoscaleOptions* o) {
    std::lock_guard<std::recursive_mutex> lk(runtime_mutex());
    clear_error();
    MesoContext* c = find_meso(key);
    if (!c || !o) {
        set_error("mesoscale_set_options: unknown context or null options");
        return 0;
    }
    if (o->storage < 0 || o->storage > 2 || (o->storage != 0 && !o->hydro_only)) {
        set_error("mesoscale_set_options: storage 0 (FP32), 1 (FP16) or 2 (16-bit fixed point); 16-bit storage needs hydro_only");
        return 0;
    }
    if (o->collision != 0 && o->collision != 1) {
        set_error("mesoscale_set_options: collision 0 (reference order) or 1 (packed two-cell)");
        return 0;
    }
    if (o->threads != 0 && o->threads != 64 && o->threads != 128 && o->threads != 256) {
        set_error("mesoscale_set_options: threads must be 0, 64, 128 or 256");
        return 0;
    }
    if (o->fixed_tau && !(o->tau_hydro > 0.5)) {
        set_error("mesoscale_set_options: tau_hydro must exceed 0.5");
        return 0;
    }
    const bool relayout = (o->hydro_only != 0) != (c->opt.hydro_only != 0) || o->storage != c->opt.storage;
    c->opt = *o;
    c->initialized = false;
    if (relayout) c->release();
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_mesoscale_advance(long long key, int steps) {
    std::lock_guard<std::recursive_mutex> lk(runtime_mutex());
    clear_error();
    MesoContext* c = find_meso(key);
    if (!c || !c->initialized || steps < 0) {
        set_error("mesoscale_advance: no initialised context (step it once first) or negative steps");
        return 0;
    }
    const Transport t = derive(c->config);
    cudaStream_t s = current_stream();
    for (int k = 0; k < steps; ++k) {
        const bool ok = c->hydro ? hydro_step(*c, t, c->fslot, c->fslot, s) : model_step(*c, t, c->fslot, s);
        if (!ok) return 0;
    }
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_mesoscale_read_state(long long key, float* out_state) {
    std::lock_guard<std::recursive_mutex> lk(runtime_mutex());
    clear_error();
    MesoContext* c = find_meso(key);
    if (!c || !c->initialized || !out_state) {
        set_error("mesoscale_read_state: no initialised context or null output");
        return 0;
    }
    cudaStream_t s = current_stream();
    if (c->hydro && !hydro_output(*c, derive(c->config), s)) return 0;
    const size_t obytes = (size_t)c->cells * kMesoStateChannels * sizeof(float);
    if (!cuda_ok(cudaMemcpyAsync(out_state, c->out, obytes, cudaMemcpyDeviceToHost, s), "mesoscale output copy")) return 0;
    return cuda_ok(cudaStreamSynchronize(s), "mesoscale read sync") ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_mesoscale_info(long long key, long long* out_cells, double* out_bytes) {
    std::lock_guard<std::recursive_mutex> lk(runtime_mutex());
    MesoContext* c = find_meso(key);
    if (!c || !c->cells) return 0;
    if (out_cells) *out_cells = c->cells;
    if (out_bytes) *out_bytes = c->bytes_per_step();
    return 1;
}

}  // extern "C"
