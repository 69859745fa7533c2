// The brick-world service: aero_lbm_simulation_* (the reference's
// native/src/aero_lbm_simulation_bridge.cpp, C ABI at :4562-5535, declared in
// native/include/aero_lbm_capi.h:303-456), the entry points the mod's
// ClientL2Solver reaches through JNI.
//
// Bookkeeping (active sets, dirty flags, seeding, face bootstrap, compact-mode
// counters, world deltas) follows the reference statement for statement in
// effect; the data plane does not: brick state stays on the device between
// ticks, each brick's inputs are built by one kernel straight into its
// context (no host packet, no copy), the dynamic state is refreshed by one
// kernel after the step (no readback), and the packed int16 atlas is
// quantised on the device into page-locked host memory.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <mutex>
#include <set>
#include <string>

#include "brick_world.h"
#include "runtime_internal.h"

namespace aero {
namespace bw {

namespace {

constexpr int kGhostLayers = 1;                     // k_brick_face_ghost_layers (simulation_bridge.cpp:481)
constexpr uint64_t kInactiveRetentionEpochs = 16;   // k_brick_inactive_retention_epochs (:482)
constexpr int kFaceOffsets[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
constexpr int kFlagCapacity = 1 << 16;              // bricks with a flag word at once, per service

// rho_air * c_p * V_cell * T_scale of temperature_source_from_power_watts
// (simulation_bridge.cpp:3152-3158), folded in float as the reference's
// constant expression is.
constexpr float kSourceDenominator = 1.225f * 1005.0f * 1.0f * 20.0f;

struct Service {
    bool l2_initialized = false;
    int l2_n = 0;
    int focus[4] = {0, 0, 0, 0};
    std::map<long long, World> worlds;
    long long next_context_key = -1;  // internal context keys count down (simulation_bridge.cpp:905-907)
    int next_upload_id = 1;
    std::map<int, std::shared_ptr<PendingStaticUpload>> pending_uploads;
    // flag words: one per brick with a dynamic state on the device
    int* d_flags = nullptr;
    int* h_flags = nullptr;
    std::vector<int> free_slots;
    int slot_high = 0;
    std::vector<Brick*> flag_waiters;
    // publish staging: floats of the strided output, int16 atlas in mapped host memory
    float* d_atlas = nullptr;
    size_t atlas_cap = 0;  // samples
    int16_t* h_atlas = nullptr;
    int16_t* h_atlas_dev = nullptr;
    size_t h_atlas_cap = 0;
    ~Service();
};

std::mutex g_mutex;  // the reference's g_simulation_mutex: one lock around every entry point
std::unique_ptr<Service> g_service;
long long g_service_key = 0;
std::string g_last_error;
uint64_t g_static_version = 0;

void set_sim_error(const std::string& m) { g_last_error = m; }

std::string coord_text(const Coord& c) {
    return "(" + std::to_string(c.x) + "," + std::to_string(c.y) + "," + std::to_string(c.z) + ")";
}

bool cells_of(int n, int* out) {
    if (n <= 0) return false;
    const long long c = (long long)n * n * n;
    if (c <= 0 || c > std::numeric_limits<int>::max()) return false;
    *out = (int)c;
    return true;
}

int normalize_mode(int m) { return (m >= AERO_LBM_REALTIME_SOLVER_AUTO && m <= 3) ? m : AERO_LBM_REALTIME_SOLVER_CLASSIC_D3Q27; }

bool env_flag(const char* name, bool fallback) {
    const char* v = std::getenv(name);
    if (!v) return fallback;
    return std::strcmp(v, "0") != 0 && std::strcmp(v, "false") != 0 && std::strcmp(v, "FALSE") != 0 &&
           std::strcmp(v, "off") != 0 && std::strcmp(v, "OFF") != 0;
}
bool simulation_compact_env() { return env_flag("AERO_LBM_SIMULATION_COMPACT", false); }
// brick_world_compact_enabled (simulation_bridge.cpp:377-385)
bool brick_world_compact_env() {
    if (std::getenv("AERO_LBM_BRICK_WORLD_COMPACT")) return env_flag("AERO_LBM_BRICK_WORLD_COMPACT", true);
    if (std::getenv("AERO_LBM_SIMULATION_COMPACT")) return simulation_compact_env();
    return false;
}
bool experimental(const World& w) {
    switch (normalize_mode(w.solver_mode)) {
        case AERO_LBM_REALTIME_SOLVER_COMPACT_EXPERIMENTAL:
        case AERO_LBM_REALTIME_SOLVER_D3Q27_FP16_INPLACE_EXPERIMENTAL: return true;
        case AERO_LBM_REALTIME_SOLVER_AUTO: return brick_world_compact_env();
        default: return false;
    }
}
const char* mode_name(int m) {
    switch (normalize_mode(m)) {
        case AERO_LBM_REALTIME_SOLVER_AUTO: return "auto";
        case AERO_LBM_REALTIME_SOLVER_COMPACT_EXPERIMENTAL: return "compact-experimental";
        case AERO_LBM_REALTIME_SOLVER_D3Q27_FP16_INPLACE_EXPERIMENTAL: return "d3q27-fp16-inplace-experimental";
        default: return "classic-d3q27";
    }
}

// The realtime solver mode of one brick step (RealtimeSolverModeScope,
// simulation_bridge.cpp:426-434): process-global in the per-context runtime.
struct ModeScope {
    explicit ModeScope(int m) { aero_lbm_set_realtime_solver_mode(normalize_mode(m)); }
    ~ModeScope() { aero_lbm_set_realtime_solver_mode(AERO_LBM_REALTIME_SOLVER_AUTO); }
};

// configure_simulation_compact_boundary (simulation_bridge.cpp:449-469)
bool configure_compact(const float v[3], int n) {
    AeroLbmBenchmarkConfig cfg{};
    aero_lbm_benchmark_default_config(&cfg);
    cfg.enabled = 1;
    cfg.preset = AERO_LBM_BENCHMARK_PRESET_NONE;
    cfg.reference_length = (float)std::max(1, n);
    for (int a = 0; a < 3; ++a) cfg.initial_velocity[a] = v[a];
    auto face = [](int hydro) {
        AeroLbmBoundaryFaceConfig f{};
        f.hydrodynamic_kind = hydro;
        f.thermal_kind = AERO_LBM_THERMAL_BOUNDARY_DISABLED;
        return f;
    };
    cfg.x_min = face(AERO_LBM_HYDRO_BOUNDARY_VELOCITY_DIRICHLET);
    for (int a = 0; a < 3; ++a) cfg.x_min.velocity[a] = v[a];
    cfg.x_max = face(AERO_LBM_HYDRO_BOUNDARY_CONVECTIVE_OUTFLOW);
    cfg.y_min = cfg.y_max = cfg.z_min = cfg.z_max = face(AERO_LBM_HYDRO_BOUNDARY_SYMMETRY);
    return aero_lbm_benchmark_set_config(&cfg) != 0;
}

bool has_static(const World& w, const Brick& b) { return b.stat && !b.stat->obstacle.empty() && w.brick_size > 0; }
bool solver_active(const World& w, const Brick& b) { return b.active && has_static(w, b); }
bool compact_ready(const World& w, const Brick& b) {
    return experimental(w) && b.compact_active && b.context != 0 && !b.forcing_dirty && !b.geometry_dirty &&
           !b.pending_reinit && b.has_dynamic;
}
bool resident(const Brick& b) {
    return b.active_hint || b.active || b.geometry_dirty || b.forcing_dirty || b.pending_reinit;
}

// ------------------------------------------------------------ host helpers
bool host_nonzero(const HostDynamic& d) {
    for (size_t i = 0; i + 2 < d.flow.size(); i += kFlowChannels)
        if (std::fabs(d.flow[i]) > 1.0e-8f || std::fabs(d.flow[i + 1]) > 1.0e-8f || std::fabs(d.flow[i + 2]) > 1.0e-8f)
            return true;
    return false;
}

// apply_brick_static_constraints (simulation_bridge.cpp:1202-1236) on a host copy
void host_constrain(const StaticFields& s, HostDynamic& d) {
    const size_t cells = d.air.size();
    if (s.obstacle.size() != cells) return;
    for (size_t c = 0; c < cells; ++c) {
        if (s.obstacle[c] != 0) {
            std::fill_n(d.flow.begin() + (std::ptrdiff_t)(c * kFlowChannels), kFlowChannels, 0.0f);
            d.air[c] = 0.0f;
            d.surface[c] = 0.0f;
        } else if (s.open_face_mask[c] == 0 && s.surface_kind[c] == 0 && !(s.emitter_power[c] > 0.0f)) {
            d.surface[c] = 0.0f;
        }
    }
}

// quantize_signed (simulation_bridge.cpp:3122-3128)
int16_t host_quantize(float v, float range) {
    if (!(range > 0.0f) || !std::isfinite(v)) return 0;
    const float r = std::clamp(v / range, -1.0f, 1.0f);
    return (int16_t)std::lround(r * 32767.0f);
}

int exposed_mask(const World& w, const Coord& c) {
    int m = 0;
    for (int f = 0; f < 6; ++f) {
        const Coord nc{c.x + kFaceOffsets[f][0], c.y + kFaceOffsets[f][1], c.z + kFaceOffsets[f][2]};
        auto it = w.bricks.find(nc);
        if (it == w.bricks.end() || !solver_active(w, it->second)) m |= 1 << f;
    }
    return m;
}

// ------------------------------------------------------------ device memory
size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

Service::~Service() {
    if (d_flags) cudaFree(d_flags);
    if (h_flags) cudaFreeHost(h_flags);
    if (d_atlas) cudaFree(d_atlas);
    if (h_atlas) cudaFreeHost(h_atlas);
}

void free_brick_memory(Service& svc, Brick& b) {
    if (b.mem.block) cudaFree(b.mem.block);
    b.mem = BrickMemory{};
    b.static_on_device = 0;
    b.reference_on_device = false;
    if (b.flag_slot >= 0) svc.free_slots.push_back(b.flag_slot);
    b.flag_slot = -1;
    b.flag_pending = false;
    svc.flag_waiters.erase(std::remove(svc.flag_waiters.begin(), svc.flag_waiters.end(), &b), svc.flag_waiters.end());
}

bool alloc_brick_memory(Service& svc, const World& w, Brick& b) {
    if (b.mem.block) return true;
    const size_t c = (size_t)w.brick_size * w.brick_size * w.brick_size;
    const size_t parts[] = {c, c, c * 2, c * 4,                                  // static
                            c * 16, c * 4, c * 4, c * 16, c * 4, c * 4,          // dynamic x 2
                            c * 16, c * 4};                                      // reference
    size_t total = 0;
    for (size_t p : parts) total += align256(p);
    char* base = nullptr;
    if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&base), total), "cudaMalloc(brick)")) return false;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base + off;
        off += align256(bytes);
        return p;
    };
    b.mem.block = base;
    b.mem.obstacle = reinterpret_cast<uint8_t*>(take(parts[0]));
    b.mem.surface_kind = reinterpret_cast<uint8_t*>(take(parts[1]));
    b.mem.open_face_mask = reinterpret_cast<uint16_t*>(take(parts[2]));
    b.mem.emitter_power = reinterpret_cast<float*>(take(parts[3]));
    for (int i = 0; i < 2; ++i) {
        b.mem.flow[i] = reinterpret_cast<float*>(take(c * 16));
        b.mem.air[i] = reinterpret_cast<float*>(take(c * 4));
        b.mem.surface[i] = reinterpret_cast<float*>(take(c * 4));
    }
    b.mem.ref_flow = reinterpret_cast<float*>(take(parts[10]));
    b.mem.ref_air = reinterpret_cast<float*>(take(parts[11]));
    if (b.flag_slot < 0) {
        if (!svc.d_flags) {
            if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&svc.d_flags), kFlagCapacity * sizeof(int)), "cudaMalloc(flags)") ||
                !cuda_ok(cudaMallocHost(reinterpret_cast<void**>(&svc.h_flags), kFlagCapacity * sizeof(int)), "cudaMallocHost(flags)"))
                return false;
        }
        if (!svc.free_slots.empty()) {
            b.flag_slot = svc.free_slots.back();
            svc.free_slots.pop_back();
        } else if (svc.slot_high < kFlagCapacity) {
            b.flag_slot = svc.slot_high++;
        } else {
            set_sim_error("brick world: more than 65536 bricks hold a dynamic state");
            return false;
        }
    }
    return true;
}

StaticDev static_dev(const Brick& b) {
    return StaticDev{b.mem.obstacle, b.mem.surface_kind, b.mem.open_face_mask, b.mem.emitter_power};
}

bool upload_dynamic(const World& w, Brick& b, int idx, const HostDynamic& d) {
    cudaStream_t s = current_stream();
    const size_t c = (size_t)w.brick_size * w.brick_size * w.brick_size;
    return cuda_ok(cudaMemcpyAsync(b.mem.flow[idx], d.flow.data(), c * 16, cudaMemcpyHostToDevice, s), "upload dynamic") &&
           cuda_ok(cudaMemcpyAsync(b.mem.air[idx], d.air.data(), c * 4, cudaMemcpyHostToDevice, s), "upload dynamic") &&
           cuda_ok(cudaMemcpyAsync(b.mem.surface[idx], d.surface.data(), c * 4, cudaMemcpyHostToDevice, s), "upload dynamic") &&
           cuda_ok(cudaStreamSynchronize(s), "upload dynamic");
}

// Device copies of everything the brick's kernels read: static fields, a
// dynamic state uploaded by the caller, the boundary reference.
bool device_ready(Service& svc, const World& w, Brick& b) {
    if (!alloc_brick_memory(svc, w, b)) return false;
    cudaStream_t s = current_stream();
    const size_t c = (size_t)w.brick_size * w.brick_size * w.brick_size;
    if (b.stat && b.static_on_device != b.static_version) {
        const StaticFields& st = *b.stat;
        if (!cuda_ok(cudaMemcpyAsync(b.mem.obstacle, st.obstacle.data(), c, cudaMemcpyHostToDevice, s), "upload static") ||
            !cuda_ok(cudaMemcpyAsync(b.mem.surface_kind, st.surface_kind.data(), c, cudaMemcpyHostToDevice, s), "upload static") ||
            !cuda_ok(cudaMemcpyAsync(b.mem.open_face_mask, st.open_face_mask.data(), c * 2, cudaMemcpyHostToDevice, s), "upload static") ||
            !cuda_ok(cudaMemcpyAsync(b.mem.emitter_power, st.emitter_power.data(), c * 4, cudaMemcpyHostToDevice, s), "upload static") ||
            !cuda_ok(cudaStreamSynchronize(s), "upload static"))
            return false;
        b.static_on_device = b.static_version;
    }
    if (b.pending_upload) {
        if (!upload_dynamic(w, b, b.cur, *b.pending_upload)) return false;
        b.pending_upload.reset();
    }
    if (b.reference && !b.reference_on_device) {
        if (!cuda_ok(cudaMemcpyAsync(b.mem.ref_flow, b.reference->flow.data(), c * 16, cudaMemcpyHostToDevice, s), "upload reference") ||
            !cuda_ok(cudaMemcpyAsync(b.mem.ref_air, b.reference->air.data(), c * 4, cudaMemcpyHostToDevice, s), "upload reference") ||
            !cuda_ok(cudaStreamSynchronize(s), "upload reference"))
            return false;
        b.reference_on_device = true;
    }
    return true;
}

// Host copy of dynamic buffer idx.
bool pull(const World& w, Brick& b, int idx, HostDynamic& out) {
    const size_t c = (size_t)w.brick_size * w.brick_size * w.brick_size;
    if (b.pending_upload && idx == b.cur) {
        out = *b.pending_upload;
        return true;
    }
    out.flow.resize(c * kFlowChannels);
    out.air.resize(c);
    out.surface.resize(c);
    cudaStream_t s = current_stream();
    return cuda_ok(cudaMemcpyAsync(out.flow.data(), b.mem.flow[idx], c * 16, cudaMemcpyDeviceToHost, s), "read dynamic") &&
           cuda_ok(cudaMemcpyAsync(out.air.data(), b.mem.air[idx], c * 4, cudaMemcpyDeviceToHost, s), "read dynamic") &&
           cuda_ok(cudaMemcpyAsync(out.surface.data(), b.mem.surface[idx], c * 4, cudaMemcpyDeviceToHost, s), "read dynamic") &&
           cuda_ok(cudaStreamSynchronize(s), "read dynamic");
}

void expect_flag(Service& svc, Brick& b) {
    if (!b.flag_pending) svc.flag_waiters.push_back(&b);
    b.flag_pending = true;
}

// Read the flag words of every brick whose dynamic state changed on the device.
bool resolve_flags(Service& svc) {
    if (svc.flag_waiters.empty()) return true;
    cudaStream_t s = current_stream();
    if (!cuda_ok(cudaMemcpyAsync(svc.h_flags, svc.d_flags, (size_t)svc.slot_high * sizeof(int), cudaMemcpyDeviceToHost, s),
                 "read flags") ||
        !cuda_ok(cudaStreamSynchronize(s), "read flags"))
        return false;
    for (Brick* b : svc.flag_waiters) {
        b->nonzero = (svc.h_flags[b->flag_slot] & kFlagAfter) != 0;
        b->flag_pending = false;
    }
    svc.flag_waiters.clear();
    return true;
}

// Static constraints on the dynamic state (apply_brick_static_constraints);
// a no-op when the state was already constrained with these static fields.
bool constrain(Service& svc, World& w, Brick& b) {
    if (!b.stat || !b.has_dynamic || b.constrained_version == b.static_version) return true;
    if (b.pending_upload && !b.mem.block) {
        host_constrain(*b.stat, *b.pending_upload);
        b.nonzero = host_nonzero(*b.pending_upload);
        b.constrained_version = b.static_version;
        return true;
    }
    if (!device_ready(svc, w, b)) return false;
    cudaStream_t s = current_stream();
    SyncArgs a{};
    a.cells = (long long)w.brick_size * w.brick_size * w.brick_size;
    a.flow = b.mem.flow[b.cur];
    a.air = b.mem.air[b.cur];
    a.surface = b.mem.surface[b.cur];
    a.st = static_dev(b);
    a.flag = svc.d_flags + b.flag_slot;
    if (!cuda_ok(cudaMemsetAsync(a.flag, 0, sizeof(int), s), "clear flag") || !cuda_ok(launch_sync(a, s), "constrain"))
        return false;
    expect_flag(svc, b);
    b.constrained_version = b.static_version;
    return true;
}

// sync_brick_dynamic_from_context (simulation_bridge.cpp:1598-1615): the
// context's flow output and temperature state into dynamic buffer dst (the
// surface temperature taken from buffer surface_from); with `constrain`, the
// static constraints the reference applies right after.
bool sync_from_context(Service& svc, World& w, Brick& b, int dst, int surface_from, bool with_constraints) {
    Context* ctx = find_context(b.context);
    const int n = w.brick_size;
    if (!ctx || !ctx->initialized || ctx->nx != n || ctx->ny != n || ctx->nz != n) {
        set_error("extract_flow_atlas: no initialized context of these dimensions");
        return false;
    }
    if (!device_ready(svc, w, b)) return false;
    cudaStream_t s = current_stream();
    if (!output_device(*ctx, strided_box(n, n, n, 1), kFlowChannels, 1.0f, b.mem.flow[dst])) return false;
    SyncArgs a{};
    a.cells = (long long)n * n * n;
    a.flow = b.mem.flow[dst];
    a.air = b.mem.air[dst];
    a.surface = b.mem.surface[dst];
    a.temperature = ctx->temperature;
    a.surface_src = b.mem.surface[surface_from];
    if (with_constraints && b.stat) a.st = static_dev(b);
    a.flag = svc.d_flags + b.flag_slot;
    if (!cuda_ok(cudaMemsetAsync(a.flag, 0, sizeof(int), s), "clear flag") || !cuda_ok(launch_sync(a, s), "sync dynamic"))
        return false;
    expect_flag(svc, b);
    b.constrained_version = (with_constraints && b.stat) ? b.static_version : 0;
    b.stale = false;
    return true;
}

void release_context(Service& svc, Brick& b) {
    (void)svc;
    if (b.context != 0) {
        aero_lbm_release_context(b.context);
        b.context = 0;
    }
    b.stepped_context = 0;
    b.compact_active = false;
    b.stale = false;
    b.pending_patch_cells.clear();
}

void drop_dynamic(Service& svc, Brick& b) {
    b.has_dynamic = false;
    b.pending_upload.reset();
    b.nonzero = false;
    if (b.flag_pending) {
        b.flag_pending = false;
        svc.flag_waiters.erase(std::remove(svc.flag_waiters.begin(), svc.flag_waiters.end(), &b), svc.flag_waiters.end());
    }
}

// ensure_brick_dynamic_region_storage (simulation_bridge.cpp:1189-1200): a zero state.
bool ensure_dynamic(Service& svc, World& w, Brick& b) {
    if (b.has_dynamic) return true;
    if (!device_ready(svc, w, b)) return false;
    const size_t c = (size_t)w.brick_size * w.brick_size * w.brick_size;
    cudaStream_t s = current_stream();
    if (!cuda_ok(cudaMemsetAsync(b.mem.flow[b.cur], 0, c * 16, s), "zero dynamic") ||
        !cuda_ok(cudaMemsetAsync(b.mem.air[b.cur], 0, c * 4, s), "zero dynamic") ||
        !cuda_ok(cudaMemsetAsync(b.mem.surface[b.cur], 0, c * 4, s), "zero dynamic"))
        return false;
    b.has_dynamic = true;
    b.nonzero = false;
    b.constrained_version = b.static_version;  // zeros satisfy every constraint
    return true;
}

void erase_brick(Service& svc, Brick& b) {
    release_context(svc, b);
    drop_dynamic(svc, b);
    free_brick_memory(svc, b);
}

// ------------------------------------------------------------ active sets
void recompute_active(World& w) {
    for (auto& [c, b] : w.bricks) {
        const bool hinted = w.hint_closure.count(c) != 0;
        b.active = w.exact_hints ? (hinted && has_static(w, b))
                                 : ((hinted && has_static(w, b)) || b.geometry_dirty || b.forcing_dirty || b.pending_reinit);
        if (b.active) b.last_active_epoch = w.epoch;
    }
}

void prune(Service& svc, World& w) {
    for (auto it = w.bricks.begin(); it != w.bricks.end();) {
        Brick& b = it->second;
        if (w.exact_hints && !w.hint_closure.count(it->first)) {
            erase_brick(svc, b);
            it = w.bricks.erase(it);
            continue;
        }
        const bool stale = !b.active && !b.geometry_dirty && !b.forcing_dirty && !b.pending_reinit &&
                           w.epoch > b.last_active_epoch && (w.epoch - b.last_active_epoch) > kInactiveRetentionEpochs;
        if (!stale) {
            ++it;
            continue;
        }
        erase_brick(svc, b);
        w.hint_closure.erase(it->first);
        it = w.bricks.erase(it);
    }
}

// clear_unbacked_placeholder_bricks (simulation_bridge.cpp:1865-1883)
void clear_unbacked(Service& svc, World& w) {
    for (auto& [c, b] : w.bricks) {
        if (b.active_hint || has_static(w, b)) continue;
        release_context(svc, b);
        b.geometry_dirty = b.forcing_dirty = b.pending_reinit = false;
        b.active = false;
        b.pending_patch_cells.clear();
        drop_dynamic(svc, b);
        b.reference.reset();
        b.reference_on_device = false;
    }
}

void reset_world(Service& svc, World& w) {
    for (auto& [c, b] : w.bricks) erase_brick(svc, b);
    w = World{};
}

bool ensure_l2(Service& svc, int n) {
    if (svc.l2_initialized && svc.l2_n == n) return true;
    if (!aero_lbm_init_rect(n, n, n, kPacketChannels, kFlowChannels)) {
        set_sim_error(std::string("simulation_l2_runtime_init failed: ") + aero_lbm_last_error());
        return false;
    }
    svc.l2_initialized = true;
    svc.l2_n = n;
    return true;
}

// ------------------------------------------------------------ seeding and face bootstrap (host paths)
struct Snapshot {
    int buffer;
    bool nonzero;
};
using Snapshots = std::map<Coord, Snapshot>;

struct SnapshotCache {
    std::map<Coord, std::unique_ptr<HostDynamic>> data;
    const HostDynamic* get(World& w, const Coord& c, const Snapshot& s) {
        auto it = data.find(c);
        if (it != data.end()) return it->second.get();
        auto h = std::make_unique<HostDynamic>();
        if (!pull(w, w.bricks.at(c), s.buffer, *h)) return nullptr;
        return (data[c] = std::move(h)).get();
    }
};

// compute_brick_mean_state (simulation_bridge.cpp:1261-1283): float sums in cell order
void brick_mean(const HostDynamic& d, float flow[4], float& air, float& surface) {
    flow[0] = flow[1] = flow[2] = flow[3] = 0.0f;
    air = surface = 0.0f;
    const size_t cells = d.air.size();
    for (size_t c = 0; c < cells; ++c) {
        for (int k = 0; k < kFlowChannels; ++k) flow[k] += d.flow[c * kFlowChannels + k];
        air += d.air[c];
        surface += d.surface[c];
    }
    const float inv = 1.0f / (float)cells;
    for (int k = 0; k < kFlowChannels; ++k) flow[k] *= inv;
    air *= inv;
    surface *= inv;
}

// seed_brick_from_neighbor_means (simulation_bridge.cpp:1285-1331)
bool seed_from_neighbors(World& w, const Coord& c, const Snapshots& snaps, SnapshotCache& cache, HostDynamic& d) {
    float acc[4] = {0, 0, 0, 0}, acc_air = 0.0f, acc_surface = 0.0f;
    int count = 0;
    for (const auto& o : kFaceOffsets) {
        const Coord nc{c.x + o[0], c.y + o[1], c.z + o[2]};
        auto it = snaps.find(nc);
        if (it == snaps.end() || !it->second.nonzero) continue;
        const HostDynamic* nd = cache.get(w, nc, it->second);
        if (!nd) continue;
        float m[4], ma, ms;
        brick_mean(*nd, m, ma, ms);
        for (int k = 0; k < 4; ++k) acc[k] += m[k];
        acc_air += ma;
        acc_surface += ms;
        ++count;
    }
    if (count <= 0) return false;
    const float inv = 1.0f / (float)count;
    for (int k = 0; k < 4; ++k) acc[k] *= inv;
    acc_air *= inv;
    acc_surface *= inv;
    for (size_t cell = 0; cell < d.air.size(); ++cell) {
        for (int k = 0; k < 4; ++k) d.flow[cell * 4 + k] = acc[k];
        d.air[cell] = acc_air;
        d.surface[cell] = acc_surface;
    }
    return true;
}

// copy_brick_face_ghost_from_neighbor (simulation_bridge.cpp:1350-1409)
void copy_face_ghost(int n, const HostDynamic& nb, int axis, bool positive, HostDynamic& d) {
    const int layers = std::max(1, std::min(kGhostLayers, n));
    auto copy = [&](int dx, int dy, int dz, int sx, int sy, int sz) {
        const size_t dst = ((size_t)dx * n + dy) * n + dz, src = ((size_t)sx * n + sy) * n + sz;
        for (int k = 0; k < 4; ++k) d.flow[dst * 4 + k] = nb.flow[src * 4 + k];
        d.air[dst] = nb.air[src];
        d.surface[dst] = nb.surface[src];
    };
    for (int l = 0; l < layers; ++l) {
        const int df = positive ? n - 1 - l : l, sf = positive ? l : n - 1 - l;
        for (int u = 0; u < n; ++u)
            for (int v = 0; v < n; ++v) {
                if (axis == 0) copy(df, u, v, sf, u, v);
                else if (axis == 1) copy(u, df, v, u, sf, v);
                else copy(u, v, df, u, v, sf);
            }
    }
}

// One cell of build_brick_step_packet (simulation_bridge.cpp:1497-1596) on the
// host, for the compact-mode packet summary.
struct CompactSummary {
    bool supported = false;
    float v[3] = {0, 0, 0};
    int fluid = 0, obstacle = 0, fan = 0, thermal = 0, nonfinite = 0;
};

// summarize_compact_brick_packet (simulation_bridge.cpp:330-370) over the
// packet the brick's step builds from `d`.
CompactSummary summarize(const World& w, const Coord& c, const Brick& b, const HostDynamic& d) {
    CompactSummary s;
    const int n = w.brick_size;
    const StaticFields& st = *b.stat;
    const HostDynamic* ref = b.reference.get();
    const int e = ref ? exposed_mask(w, c) : 0;
    const int L = std::max(1, std::min(kBoundaryReferenceLayers, n));
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int x = 0; x < n; ++x)
        for (int y = 0; y < n; ++y)
            for (int z = 0; z < n; ++z) {
                const size_t cell = ((size_t)x * n + y) * n + z;
                if (st.obstacle[cell] != 0) {
                    s.obstacle++;
                    continue;
                }
                const uint8_t k = st.surface_kind[cell];
                if (k >= 32 && k <= 37) s.fan++;
                if (st.emitter_power[cell] > 0.0f) {
                    const float src = std::clamp(st.emitter_power[cell] * 0.05f / kSourceDenominator, -0.006f, 0.006f);
                    if (std::fabs(src) > 1.0e-8f) s.thermal++;
                }
                const bool use_ref = ((e & 1) && x < L) || ((e & 2) && x >= n - L) || ((e & 4) && y < L) ||
                                     ((e & 8) && y >= n - L) || ((e & 16) && z < L) || ((e & 32) && z >= n - L);
                const float* f = (use_ref ? ref->flow.data() : d.flow.data()) + cell * 4;
                if (!std::isfinite(f[0]) || !std::isfinite(f[1]) || !std::isfinite(f[2])) {
                    s.nonfinite++;
                    continue;
                }
                sx += f[0];
                sy += f[1];
                sz += f[2];
                s.fluid++;
            }
    if (s.fluid > 0) {
        s.v[0] = (float)(sx / s.fluid);
        s.v[1] = (float)(sy / s.fluid);
        s.v[2] = (float)(sz / s.fluid);
    }
    s.supported = s.fluid > 0 && s.fan == 0;
    return s;
}

// ------------------------------------------------------------ one brick step
struct Next {
    int buffer;                          // dynamic buffer the step reads
    std::unique_ptr<HostDynamic> host;   // host copy when the tick rebuilt it (seeding, bootstrap)
    bool nonzero;
};

struct Fallback {
    Brick* brick;
    int buffer;
    std::unique_ptr<HostDynamic> host;
};

cudaError_t fill_launch(const CellFields& out, const BrickDims& d, cudaStream_t s, void* user) {
    (void)d;
    return launch_fill(*static_cast<const FillArgs*>(user), out, s);
}

// apply_pending_static_patches_to_d3q27 (simulation_bridge.cpp:1617-1676)
bool apply_pending_patches(World& w, Brick& b) {
    const int n = w.brick_size;
    if (b.pending_patch_cells.empty() || b.context == 0 || !b.stat) return false;
    w.d3q27_patch_attempts++;
    const int total = n * n * n;
    std::vector<int> cells;
    std::vector<uint8_t> solid, fan;
    std::set<int> seen;
    for (int cell : b.pending_patch_cells) {
        if (cell < 0 || cell >= total || !seen.insert(cell).second) continue;
        const uint8_t s = b.stat->obstacle[cell] != 0 ? 1u : 0u;
        cells.push_back(cell);
        solid.push_back(s);
        const uint8_t k = b.stat->surface_kind[cell];
        fan.push_back(s ? 0u : (k >= 32 && k <= 37 ? (uint8_t)(k - 31) : 0u));
    }
    if (cells.empty()) {
        b.pending_patch_cells.clear();
        b.forcing_dirty = false;
        return true;
    }
    if (!aero_lbm_patch_d3q27_f16_static_cells_rect(n, n, n, b.context, (int)cells.size(), cells.data(), solid.data(),
                                                    fan.data())) {
        w.d3q27_patch_failures++;
        return false;
    }
    w.d3q27_patch_steps++;
    w.d3q27_patch_cells += cells.size();
    w.d3q27_patch_upload_bytes_est += (uint64_t)cells.size() * (sizeof(int) + 2u + 27u * (sizeof(int) + 1u) + sizeof(int));
    b.pending_patch_cells.clear();
    b.forcing_dirty = b.geometry_dirty = b.pending_reinit = false;
    b.stale = true;
    return true;
}

// step_brick_compact_cached (simulation_bridge.cpp:1678-1704)
bool step_compact_cached(World& w, Brick& b) {
    const int n = w.brick_size;
    w.compact_cached_attempts++;
    if (!experimental(w) || !b.compact_active || b.context == 0 || b.geometry_dirty || b.pending_reinit) {
        w.compact_cached_failures++;
        return false;
    }
    if (b.forcing_dirty && !apply_pending_patches(w, b)) {
        w.compact_cached_failures++;
        return false;
    }
    bool ok = false;
    if (configure_compact(b.compact_v, n)) ok = aero_lbm_step_rect_cached(n, n, n, b.context, nullptr) != 0;
    aero_lbm_benchmark_reset_config();
    if (ok) {
        b.stale = true;
        w.compact_cached_steps++;
    } else {
        w.compact_cached_failures++;
    }
    return ok;
}

// update_brick_d3q27_boundary_shell (simulation_bridge.cpp:1470-1495)
void update_shell(World& w, const Coord& c, Brick& b) {
    if (b.context == 0) return;
    const int mask = exposed_mask(w, c);
    if (mask == 0 || !b.reference) {
        aero_lbm_clear_d3q27_f16_boundary_shell_rect(b.context);
        return;
    }
    const int n = w.brick_size;
    (void)aero_lbm_set_d3q27_f16_boundary_shell_rect(n, n, n, b.context, b.reference->flow.data(), kFlowChannels, mask,
                                                     kBoundaryReferenceLayers, kBoundaryReferenceRelaxation);
}

// The state a failed step leaves: the reference keeps the state the step started from.
void adopt_next(Brick& b, Next& next) {
    if (next.buffer != b.cur) {
        b.cur = next.buffer;
        b.nonzero = next.nonzero;
        b.constrained_version = b.static_version;
    }
}

// step_brick_actual (simulation_bridge.cpp:1706-1832)
bool step_brick(Service& svc, World& w, const Coord& c, Brick& b, Next& next, std::vector<Fallback>& fallbacks) {
    ModeScope scope(w.solver_mode);
    const int n = w.brick_size;
    if (step_compact_cached(w, b)) return true;
    const bool arm_fallback = b.forcing_dirty && next.nonzero;
    w.packet_build_steps++;
    if (!b.stat || !b.has_dynamic) {
        set_sim_error("brick_step_packet: missing or invalid brick state at " + coord_text(c));
        return false;
    }
    if (!device_ready(svc, w, b)) {
        set_sim_error("brick_step_packet: device upload failed at " + coord_text(c) + ": " + last_error());
        return false;
    }
    const bool had_context = b.context != 0;
    if (b.context == 0) b.context = svc.next_context_key--;

    FillArgs fa{};
    fa.n = n;
    fa.st = static_dev(b);
    fa.flow = b.mem.flow[next.buffer];
    fa.air = b.mem.air[next.buffer];
    if (b.reference) {
        fa.ref_flow = b.mem.ref_flow;
        fa.ref_air = b.mem.ref_air;
        fa.exposed = exposed_mask(w, c);
    }
    fa.ref_layers = std::max(1, std::min(kBoundaryReferenceLayers, n));
    fa.source_denominator = kSourceDenominator;
    // the mask comes from the static fields alone: unchanged since this
    // context's last step, the step keeps its pull classification
    const DeviceFill fill{fill_launch, &fa,
                          had_context && b.stepped_context == b.context && b.stepped_version == b.static_version};

    bool step_ok = false, compact_ok = false, have_summary = false, fill_stepped = false;
    CompactSummary sum;
    if (experimental(w)) {
        HostDynamic tmp;
        const HostDynamic* src = next.host.get();
        if (!src) {
            if (!pull(w, b, next.buffer, tmp)) return false;
            src = &tmp;
        }
        sum = summarize(w, c, b, *src);
        have_summary = true;
        w.compact_last_fluid_cells = (uint64_t)std::max(0, sum.fluid);
        w.compact_last_obstacle_cells = (uint64_t)std::max(0, sum.obstacle);
        w.compact_last_fan_cells = (uint64_t)std::max(0, sum.fan);
        w.compact_last_thermal_cells = (uint64_t)std::max(0, sum.thermal);
        w.compact_last_nonfinite_cells = (uint64_t)std::max(0, sum.nonfinite);
        if (sum.supported && configure_compact(sum.v, n)) {
            if (had_context && b.compact_active) step_ok = aero_lbm_step_rect_cached(n, n, n, b.context, nullptr) != 0;
            if (!step_ok) step_ok = fill_stepped = step_rect_device(b.context, n, n, n, fill);
            if (step_ok && aero_lbm_context_realtime_cached_initialized(b.context)) {
                compact_ok = true;
                w.compact_initial_steps++;
                if (sum.thermal > 0) w.compact_thermal_ignored_steps++;
                b.compact_active = true;
                std::copy(sum.v, sum.v + 3, b.compact_v);
                b.stale = true;
            } else if (step_ok) {
                w.compact_initial_failures++;
                w.d3q27_steps++;
                b.compact_active = false;
            }
        } else if (!sum.supported) {
            if (sum.fan > 0) w.compact_reject_fan_steps++;
            else w.compact_reject_empty_steps++;
        } else {
            w.compact_initial_failures++;
        }
        aero_lbm_benchmark_reset_config();
    }
    if (!step_ok) {
        b.compact_active = false;
        w.d3q27_steps++;
        const bool fallback_faces = have_summary && configure_compact(sum.v, n);
        step_ok = fill_stepped = step_rect_device(b.context, n, n, n, fill);
        aero_lbm_benchmark_reset_config();
        if (step_ok && fallback_faces && aero_lbm_context_realtime_cached_initialized(b.context)) {
            compact_ok = true;
            b.compact_active = true;
            std::copy(sum.v, sum.v + 3, b.compact_v);
            b.stale = true;
        }
    }
    if (!step_ok) {
        set_sim_error("brick_step_actual: aero_lbm_step_rect failed at " + coord_text(c) + ": " + last_error());
        release_context(svc, b);
        adopt_next(b, next);
        return false;
    }
    if (fill_stepped) {
        b.stepped_version = b.static_version;
        b.stepped_context = b.context;
    }
    if (compact_ok) {
        adopt_next(b, next);
        update_shell(w, c, b);
        b.pending_patch_cells.clear();
        return true;
    }
    const int out = 1 - b.cur;
    if (!sync_from_context(svc, w, b, out, next.buffer, true)) {
        set_sim_error("brick_step_actual: sync from context failed at " + coord_text(c) + ": " + last_error());
        release_context(svc, b);
        adopt_next(b, next);
        return false;
    }
    if (arm_fallback) fallbacks.push_back(Fallback{&b, next.buffer, std::move(next.host)});
    b.cur = out;
    update_shell(w, c, b);
    b.pending_patch_cells.clear();
    return true;
}

// ------------------------------------------------------------ one world tick
bool step_world(Service& svc, long long wkey, World& w, int steps);

void apply_pending_deltas(Service& svc, long long wkey, World& w) {
    if (w.pending_deltas.empty()) return;
    std::vector<AeroLbmWorldDelta> pending;
    pending.swap(w.pending_deltas);
    std::vector<int> consumed;
    for (const AeroLbmWorldDelta& d : pending) {
        if (d.type == 9) {  // k_world_delta_brick_static_brick_upload
            auto it = svc.pending_uploads.find(d.data1);
            if (it == svc.pending_uploads.end()) continue;
            const PendingStaticUpload& up = *it->second;
            consumed.push_back(d.data1);
            if (up.world != wkey || !up.fields) continue;
            install_static(w, w.bricks[up.coord], std::make_unique<StaticFields>(*up.fields));
            continue;
        }
        apply_world_delta(w, d);
    }
    for (int id : consumed) svc.pending_uploads.erase(id);
    recompute_active(w);
    prune(svc, w);
}

// step_brick_world_runtime (simulation_bridge.cpp:1004-1171)
bool step_world(Service& svc, long long wkey, World& w, int steps) {
    if (steps <= 0) return false;
    const int n = w.brick_size;
    if (!ensure_l2(svc, n)) {
        set_sim_error("brick_step_runtime_init failed for world=" + std::to_string(wkey) + " brickSize=" + std::to_string(n) +
                      ": " + aero_lbm_last_error());
        return false;
    }
    bool all_ok = true;
    apply_pending_deltas(svc, wkey, w);
    clear_unbacked(svc, w);
    for (int step = 0; step < steps; ++step) {
        w.epoch++;
        recompute_active(w);
        // bricks whose static fields changed under a live context re-read it first
        for (auto& [c, b] : w.bricks)
            if (solver_active(w, b) && b.context != 0 && b.forcing_dirty && b.has_dynamic)
                (void)sync_from_context(svc, w, b, b.cur, b.cur, false);
        if (!resolve_flags(svc)) return false;
        std::set<Coord> needs_seed;
        for (auto& [c, b] : w.bricks) {
            if (!solver_active(w, b)) continue;
            const bool compact_fast = compact_ready(w, b);
            const bool had_nonzero = compact_fast || (b.has_dynamic && b.nonzero);
            if ((b.pending_reinit || b.geometry_dirty || !had_nonzero) && b.context != 0) release_context(svc, b);
            if (!ensure_dynamic(svc, w, b)) return false;
            if (!compact_fast && !constrain(svc, w, b)) return false;
            if (!had_nonzero) needs_seed.insert(c);
        }
        if (!resolve_flags(svc)) return false;
        Snapshots snaps;
        for (auto& [c, b] : w.bricks)
            if (solver_active(w, b) && b.has_dynamic) snaps[c] = Snapshot{b.cur, b.nonzero};
        // face halos between neighbouring bricks (positive faces; the exchange
        // copies both ways); the slabs of all pairs are disjoint, so their
        // copies go out together
        halo_batch_begin();
        for (auto& [c, b] : w.bricks) {
            if (!solver_active(w, b) || b.context == 0) continue;
            for (int f = 1; f < 6; f += 2) {
                const Coord nc{c.x + kFaceOffsets[f][0], c.y + kFaceOffsets[f][1], c.z + kFaceOffsets[f][2]};
                auto it = w.bricks.find(nc);
                if (it == w.bricks.end()) continue;
                Brick& nb = it->second;
                if (!solver_active(w, nb) || nb.context == 0) continue;
                if (n <= 2 * kGhostLayers || !b.has_dynamic || !nb.has_dynamic || !b.nonzero || !nb.nonzero) continue;
                (void)aero_lbm_exchange_halo_layers_rect(n, n, n, kGhostLayers, b.context, nb.context, kFaceOffsets[f][0],
                                                         kFaceOffsets[f][1], kFaceOffsets[f][2]);
            }
        }
        if (!halo_batch_flush()) {
            set_sim_error("step_brick_world_runtime: halo exchange failed: " + last_error());
            return false;
        }
        std::vector<Fallback> fallbacks;
        SnapshotCache cache;
        for (auto& [c, b] : w.bricks) {
            if (!solver_active(w, b) || !b.has_dynamic) continue;
            const bool seed = needs_seed.count(c) != 0;
            if (compact_ready(w, b) && !seed) {
                Next next{b.cur, nullptr, b.nonzero};
                if (!step_brick(svc, w, c, b, next, fallbacks)) all_ok = false;
                continue;
            }
            if (!ensure_dynamic(svc, w, b) || !device_ready(svc, w, b)) return false;
            const bool bootstrap = seed || b.context == 0;
            Next next{b.cur, nullptr, b.nonzero};
            if (seed || bootstrap) {
                auto host = std::make_unique<HostDynamic>();
                if (!pull(w, b, b.cur, *host)) return false;
                bool seeded = !seed;
                if (seed) {
                    // seed_brick_from_boundary_reference (simulation_bridge.cpp:1333-1348), then the neighbours' means
                    if (b.reference && host_nonzero(*b.reference)) {
                        *host = *b.reference;
                        seeded = true;
                    } else {
                        seeded = seed_from_neighbors(w, c, snaps, cache, *host);
                    }
                }
                for (int f = 0; f < 6; ++f) {
                    const Coord nc{c.x + kFaceOffsets[f][0], c.y + kFaceOffsets[f][1], c.z + kFaceOffsets[f][2]};
                    auto it = snaps.find(nc);
                    if (it == snaps.end() || !it->second.nonzero) continue;
                    const HostDynamic* nd = cache.get(w, nc, it->second);
                    if (nd) copy_face_ghost(n, *nd, f / 2, (f & 1) != 0, *host);
                }
                const bool nz = host_nonzero(*host);
                if (seed && !seeded && !nz) continue;
                host_constrain(*b.stat, *host);
                if (!upload_dynamic(w, b, 1 - b.cur, *host)) return false;
                next.buffer = 1 - b.cur;
                next.nonzero = host_nonzero(*host);
                next.host = std::move(host);
            }
            if (!step_brick(svc, w, c, b, next, fallbacks)) all_ok = false;
            b.pending_reinit = b.geometry_dirty = b.forcing_dirty = false;
        }
        if (!resolve_flags(svc)) return false;
        // a step whose output came back all zero after its static fields
        // changed keeps the state it started from (zero_output_fallback)
        for (Fallback& fb : fallbacks) {
            Brick& b = *fb.brick;
            if (svc.h_flags[b.flag_slot] & kFlagBefore) continue;
            if (fb.host) {
                if (!upload_dynamic(w, b, b.cur, *fb.host)) return false;
            } else {
                b.cur = fb.buffer;
            }
            b.nonzero = true;
            b.constrained_version = b.static_version;
            release_context(svc, b);
        }
        recompute_active(w);
        prune(svc, w);
    }
    return all_ok;
}

Service* lookup(long long key) { return (g_service && g_service_key != 0 && key == g_service_key) ? g_service.get() : nullptr; }

World* find_world(Service& svc, long long wkey, const char* who) {
    auto it = svc.worlds.find(wkey);
    if (it == svc.worlds.end()) {
        set_sim_error(std::string(who) + ": missing brick runtime");
        return nullptr;
    }
    return &it->second;
}

// set_brick_world_active_hints_locked (simulation_bridge.cpp:4670-4738)
int set_hints(long long skey, long long wkey, int n, const int* coords, int count, bool closure, const char* who) {
    Service* svc = lookup(skey);
    if (!svc) {
        set_sim_error(std::string(who) + ": missing service");
        return 0;
    }
    if (count < 0 || (count > 0 && !coords)) {
        set_sim_error(std::string(who) + ": invalid hint payload");
        return 0;
    }
    World* w = find_world(*svc, wkey, who);
    if (!w) return 0;
    if (w->brick_size != n) {
        set_sim_error(std::string(who) + ": brick size mismatch");
        return 0;
    }
    w->exact_hints = !closure;
    for (auto& [c, b] : w->bricks) b.active_hint = false;
    w->hint_closure.clear();
    w->epoch++;
    for (int i = 0; i < count; ++i) {
        const Coord c{coords[3 * i], coords[3 * i + 1], coords[3 * i + 2]};
        Brick& b = w->bricks[c];
        b.active_hint = true;
        b.last_hint_epoch = b.last_active_epoch = w->epoch;
        w->hint_closure[c] = true;
        if (closure)
            for (const auto& o : kFaceOffsets) w->hint_closure[Coord{c.x + o[0], c.y + o[1], c.z + o[2]}] = true;
    }
    for (const auto& [c, v] : w->hint_closure) w->bricks.try_emplace(c);
    recompute_active(*w);
    prune(*svc, *w);
    return 1;
}

template <typename F>
int count_bricks(const World& w, F pred) {
    int n = 0;
    for (const auto& [c, b] : w.bricks) n += pred(b) ? 1 : 0;
    return n;
}

int copy_coords(const World& w, bool resident_set, int* out, int cap) {
    if (cap > 0 && !out) return -1;
    int k = 0;
    for (const auto& [c, b] : w.bricks) {
        if (resident_set ? !resident(b) : !b.active) continue;
        if (k >= cap) return -1;
        out[3 * k] = c.x;
        out[3 * k + 1] = c.y;
        out[3 * k + 2] = c.z;
        ++k;
    }
    return k;
}

std::unique_ptr<HostDynamic> host_dynamic_from(int cells, const float* flow, const float* air, const float* surface) {
    auto d = std::make_unique<HostDynamic>();
    d->flow.assign(flow, flow + (size_t)cells * kFlowChannels);
    d->air.assign(air, air + cells);
    d->surface.assign(surface, surface + cells);
    return d;
}

}  // namespace

// ------------------------------------------------------------ shared with the delta module
void static_changed(World& w, Brick& b, bool constrain_dynamic) {
    const bool was_constrained = b.constrained_version == b.static_version;
    b.static_version = ++g_static_version;
    if (constrain_dynamic) {
        if (b.has_dynamic && g_service) (void)constrain(*g_service, w, b);
    } else if (was_constrained) {
        b.constrained_version = b.static_version;
    }
}

// install_static_brick_region (simulation_bridge.cpp:2660-2685)
void install_static(World& w, Brick& b, std::unique_ptr<StaticFields> fields) {
    const bool live = b.context != 0 || b.has_dynamic;
    const size_t cells = (size_t)w.brick_size * w.brick_size * w.brick_size;
    if (fields) ensure_source_fields(*fields, cells);
    b.stat = std::move(fields);
    b.pending_patch_cells.clear();
    if (live) {
        b.forcing_dirty = true;
        b.geometry_dirty = b.pending_reinit = false;
        static_changed(w, b, true);
    } else {
        b.static_version = ++g_static_version;
        b.geometry_dirty = b.pending_reinit = true;
    }
    b.active = true;
    b.last_active_epoch = w.epoch;
}

void mark_brick(World& w, const Coord& c, bool geometry, bool forcing, bool reinit) {
    Brick& b = w.bricks[c];
    b.geometry_dirty = b.geometry_dirty || geometry;
    b.forcing_dirty = b.forcing_dirty || forcing;
    b.pending_reinit = b.pending_reinit || reinit;
    b.active = true;
    b.last_active_epoch = w.epoch;
}

}  // namespace bw
}  // namespace aero

// ====================================================================== C ABI
using namespace aero;
using namespace aero::bw;

namespace {
struct Locks {
    std::lock_guard<std::mutex> service{bw_lock()};
    std::lock_guard<std::recursive_mutex> runtime{runtime_mutex()};
    static std::mutex& bw_lock() { return aero::bw::g_mutex; }
};
}  // namespace

extern "C" {

// aero_lbm_simulation_create_service (simulation_bridge.cpp:4562-4573)
AERO_LBM_B200_EXPORT int aero_lbm_simulation_create_service(long long* out_service_key) {
    Locks lk;
    if (!out_service_key) {
        set_sim_error("simulation_create_service: out_service_key is null");
        return 0;
    }
    if (!g_service) {
        g_service = std::make_unique<Service>();
        g_service_key = 1;
    }
    *out_service_key = g_service_key;
    return 1;
}

// aero_lbm_simulation_release_service (simulation_bridge.cpp:4575-4583). The
// service's worlds and device memory are released with it.
AERO_LBM_B200_EXPORT void aero_lbm_simulation_release_service(long long service_key) {
    {
        Locks lk;
        if (g_service && service_key == g_service_key) {
            for (auto& [k, w] : g_service->worlds) reset_world(*g_service, w);
            g_service.reset();
            g_service_key = 0;
        }
        if (g_service) return;
    }
    aero_lbm_shutdown();
}

// aero_lbm_simulation_set_focus (simulation_bridge.cpp:4585-4603)
AERO_LBM_B200_EXPORT int aero_lbm_simulation_set_focus(long long service_key, int block_x, int block_y, int block_z,
                                                       int radius_blocks) {
    Locks lk;
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_set_focus: missing service");
        return 0;
    }
    svc->focus[0] = block_x;
    svc->focus[1] = block_y;
    svc->focus[2] = block_z;
    svc->focus[3] = radius_blocks;
    return 1;
}

// aero_lbm_simulation_submit_world_deltas (simulation_bridge.cpp:4605-4629,
// apply_world_delta_to_brick_runtimes :2811-2825): brick deltas queue on
// their world (data0, 0 meaning 1) and apply at its next step; type 6 drops
// the world.
AERO_LBM_B200_EXPORT int aero_lbm_simulation_submit_world_deltas(long long service_key, const AeroLbmWorldDelta* deltas,
                                                                 int delta_count) {
    Locks lk;
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_submit_world_deltas: missing service");
        return 0;
    }
    if (delta_count < 0) {
        set_sim_error("simulation_submit_world_deltas: negative delta_count");
        return 0;
    }
    if (delta_count > 0 && !deltas) {
        set_sim_error("simulation_submit_world_deltas: deltas is null");
        return 0;
    }
    for (int i = 0; i < delta_count; ++i) {
        const AeroLbmWorldDelta& d = deltas[i];
        long long wkey = d.data0 == 0 ? 1 : (long long)d.data0;
        auto it = svc->worlds.find(wkey);
        if (d.type == 6) {
            if (it != svc->worlds.end()) {
                reset_world(*svc, it->second);
                svc->worlds.erase(it);
            }
            continue;
        }
        if (it != svc->worlds.end()) it->second.pending_deltas.push_back(d);
    }
    return 1;
}

// aero_lbm_simulation_ensure_brick_world_runtime (simulation_bridge.cpp:4631-4645, 638-665)
AERO_LBM_B200_EXPORT int aero_lbm_simulation_ensure_brick_world_runtime(long long service_key, long long world_key,
                                                                        int brick_size, float dx_meters, float dt_seconds) {
    Locks lk;
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_ensure_brick_world_runtime: missing service");
        return 0;
    }
    if (world_key == 0) {
        set_sim_error("simulation_brick_world_runtime: invalid world key");
        return 0;
    }
    if (brick_size <= 0 || !std::isfinite(dx_meters) || dx_meters <= 0.0f || !std::isfinite(dt_seconds) || dt_seconds <= 0.0f) {
        set_sim_error("simulation_brick_world_runtime: invalid runtime config");
        return 0;
    }
    auto [it, inserted] = svc->worlds.try_emplace(world_key);
    World& w = it->second;
    if (inserted || w.brick_size != brick_size || w.dx != dx_meters || w.dt != dt_seconds) {
        reset_world(*svc, w);
        w.brick_size = brick_size;
        w.dx = dx_meters;
        w.dt = dt_seconds;
    }
    return 1;
}

// aero_lbm_simulation_set_brick_world_solver_mode (simulation_bridge.cpp:4647-4672)
AERO_LBM_B200_EXPORT int aero_lbm_simulation_set_brick_world_solver_mode(long long service_key, long long world_key,
                                                                         int solver_mode) {
    Locks lk;
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_set_brick_world_solver_mode: missing service");
        return 0;
    }
    World* w = find_world(*svc, world_key, "simulation_set_brick_world_solver_mode");
    if (!w) return 0;
    const int m = normalize_mode(solver_mode);
    if (w->solver_mode != m) {
        w->solver_mode = m;
        for (auto& [c, b] : w->bricks) {
            release_context(*svc, b);
            b.pending_reinit = true;
            b.stale = true;
        }
        w->epoch++;
    }
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_simulation_set_brick_world_active_hints(long long service_key, long long world_key,
                                                                          int brick_size, const int* brick_coords,
                                                                          int brick_count) {
    Locks lk;
    return set_hints(service_key, world_key, brick_size, brick_coords, brick_count, true,
                     "simulation_set_brick_world_active_hints");
}

AERO_LBM_B200_EXPORT int aero_lbm_simulation_set_brick_world_exact_active_hints(long long service_key, long long world_key,
                                                                                int brick_size, const int* brick_coords,
                                                                                int brick_count) {
    Locks lk;
    return set_hints(service_key, world_key, brick_size, brick_coords, brick_count, false,
                     "simulation_set_brick_world_exact_active_hints");
}

// aero_lbm_simulation_get_brick_world_runtime_status (simulation_bridge.cpp:4778-4812)
AERO_LBM_B200_EXPORT int aero_lbm_simulation_get_brick_world_runtime_status(long long service_key, long long world_key,
                                                                            int* out_status, int status_count) {
    Locks lk;
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_get_brick_world_runtime_status: missing service");
        return 0;
    }
    if (!out_status || status_count < AERO_LBM_SIMULATION_BRICK_RUNTIME_STATUS_FIELDS) {
        set_sim_error("simulation_get_brick_world_runtime_status: invalid output buffer");
        return 0;
    }
    World* w = find_world(*svc, world_key, "simulation_get_brick_world_runtime_status");
    if (!w) return 0;
    out_status[0] = w->brick_size;
    out_status[1] = (int)w->bricks.size();
    out_status[2] = count_bricks(*w, [](const Brick& b) { return b.active_hint; });
    out_status[3] = count_bricks(*w, [](const Brick& b) { return b.active; });
    out_status[4] = count_bricks(*w, [](const Brick& b) { return b.geometry_dirty; });
    out_status[5] = count_bricks(*w, [](const Brick& b) { return b.forcing_dirty; });
    out_status[6] = count_bricks(*w, [](const Brick& b) { return b.pending_reinit; });
    out_status[7] = (int)std::min<uint64_t>(w->epoch, (uint64_t)std::numeric_limits<int>::max());
    return 1;
}

// aero_lbm_simulation_step_brick_world_runtime (simulation_bridge.cpp:4814-4835)
AERO_LBM_B200_EXPORT int aero_lbm_simulation_step_brick_world_runtime(long long service_key, long long world_key,
                                                                      int step_count) {
    Locks lk;
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_step_brick_world_runtime: missing service");
        return 0;
    }
    if (step_count <= 0) {
        set_sim_error("simulation_step_brick_world_runtime: invalid step count");
        return 0;
    }
    World* w = find_world(*svc, world_key, "simulation_step_brick_world_runtime");
    if (!w) return 0;
    return step_world(*svc, world_key, *w, step_count) ? 1 : 0;
}

AERO_LBM_B200_EXPORT int aero_lbm_simulation_get_brick_world_resident_brick_count(long long service_key, long long world_key) {
    Locks lk;
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_get_brick_world_resident_brick_count: missing service");
        return -1;
    }
    auto it = svc->worlds.find(world_key);
    return it == svc->worlds.end() ? 0 : count_bricks(it->second, [](const Brick& b) { return resident(b); });
}

AERO_LBM_B200_EXPORT int aero_lbm_simulation_copy_brick_world_resident_bricks(long long service_key, long long world_key,
                                                                              int* out_coords, int brick_capacity) {
    Locks lk;
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_copy_brick_world_resident_bricks: missing service");
        return -1;
    }
    if (brick_capacity < 0) {
        set_sim_error("simulation_copy_brick_world_resident_bricks: invalid brick capacity");
        return -1;
    }
    auto it = svc->worlds.find(world_key);
    if (it == svc->worlds.end()) return 0;
    const int k = copy_coords(it->second, true, out_coords, brick_capacity);
    if (k < 0) set_sim_error("simulation_copy_brick_world_resident_bricks: output buffer too small");
    return k;
}

AERO_LBM_B200_EXPORT int aero_lbm_simulation_get_brick_world_active_brick_count(long long service_key, long long world_key) {
    Locks lk;
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_get_brick_world_active_brick_count: missing service");
        return -1;
    }
    auto it = svc->worlds.find(world_key);
    return it == svc->worlds.end() ? 0 : count_bricks(it->second, [](const Brick& b) { return b.active; });
}

AERO_LBM_B200_EXPORT int aero_lbm_simulation_copy_brick_world_active_bricks(long long service_key, long long world_key,
                                                                            int* out_coords, int brick_capacity) {
    Locks lk;
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_copy_brick_world_active_bricks: missing service");
        return -1;
    }
    if (brick_capacity < 0) {
        set_sim_error("simulation_copy_brick_world_active_bricks: invalid brick capacity");
        return -1;
    }
    auto it = svc->worlds.find(world_key);
    if (it == svc->worlds.end()) return 0;
    const int k = copy_coords(it->second, false, out_coords, brick_capacity);
    if (k < 0) set_sim_error("simulation_copy_brick_world_active_bricks: output buffer too small");
    return k;
}

// aero_lbm_simulation_upload_brick_world_static_brick_with_sources (simulation_bridge.cpp:4957-5031)
AERO_LBM_B200_EXPORT int aero_lbm_simulation_upload_brick_world_static_brick_with_sources(
    long long service_key, long long world_key, int brick_size, int brick_x, int brick_y, int brick_z,
    const uint8_t* obstacle, const uint8_t* surface_kind, const uint16_t* open_face_mask, const float* emitter_power_watts,
    const uint8_t* source_fan_dir, const float* source_emitter_power_watts, const uint8_t* face_sky_exposure,
    const uint8_t* face_direct_exposure) {
    Locks lk;
    int cells = 0;
    if (!cells_of(brick_size, &cells)) {
        set_sim_error("simulation_upload_brick_world_static_brick: invalid brick size");
        return 0;
    }
    if (!obstacle || !surface_kind || !open_face_mask || !emitter_power_watts || !face_sky_exposure || !face_direct_exposure) {
        set_sim_error("simulation_upload_brick_world_static_brick: null brick buffers");
        return 0;
    }
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_upload_brick_world_static_brick: missing service");
        return 0;
    }
    World* w = find_world(*svc, world_key, "simulation_upload_brick_world_static_brick");
    if (!w) return 0;
    if (w->brick_size != brick_size) {
        set_sim_error("simulation_upload_brick_world_static_brick: brick size mismatch");
        return 0;
    }
    auto f = std::make_unique<StaticFields>();
    f->obstacle.assign(obstacle, obstacle + cells);
    f->surface_kind.assign(surface_kind, surface_kind + cells);
    f->open_face_mask.assign(open_face_mask, open_face_mask + cells);
    f->emitter_power.assign(emitter_power_watts, emitter_power_watts + cells);
    if (source_fan_dir) f->source_fan_dir.assign(source_fan_dir, source_fan_dir + cells);
    else f->source_fan_dir.assign(cells, 0u);
    if (source_emitter_power_watts) f->source_emitter_power.assign(source_emitter_power_watts, source_emitter_power_watts + cells);
    else f->source_emitter_power.assign(cells, 0.0f);
    if (source_fan_dir || source_emitter_power_watts) rebuild_static_from_sources(*f, brick_size);
    f->face_sky.assign(face_sky_exposure, face_sky_exposure + (size_t)cells * 6);
    f->face_direct.assign(face_direct_exposure, face_direct_exposure + (size_t)cells * 6);
    install_static(*w, w->bricks[Coord{brick_x, brick_y, brick_z}], std::move(f));
    return 1;
}

// aero_lbm_simulation_upload_brick_world_static_brick (simulation_bridge.cpp:4925-4955)
AERO_LBM_B200_EXPORT int aero_lbm_simulation_upload_brick_world_static_brick(
    long long service_key, long long world_key, int brick_size, int brick_x, int brick_y, int brick_z,
    const uint8_t* obstacle, const uint8_t* surface_kind, const uint16_t* open_face_mask, const float* emitter_power_watts,
    const uint8_t* face_sky_exposure, const uint8_t* face_direct_exposure) {
    return aero_lbm_simulation_upload_brick_world_static_brick_with_sources(
        service_key, world_key, brick_size, brick_x, brick_y, brick_z, obstacle, surface_kind, open_face_mask,
        emitter_power_watts, nullptr, nullptr, face_sky_exposure, face_direct_exposure);
}

// aero_lbm_simulation_queue_brick_world_static_brick_upload (simulation_bridge.cpp:5033-5112):
// installed at the world's next step, in submission order with the world deltas.
AERO_LBM_B200_EXPORT int aero_lbm_simulation_queue_brick_world_static_brick_upload(
    long long service_key, long long world_key, int brick_size, int brick_x, int brick_y, int brick_z,
    const uint8_t* obstacle, const uint8_t* surface_kind, const uint16_t* open_face_mask, const float* emitter_power_watts,
    const uint8_t* face_sky_exposure, const uint8_t* face_direct_exposure) {
    Locks lk;
    int cells = 0;
    if (!cells_of(brick_size, &cells)) {
        set_sim_error("simulation_queue_brick_world_static_brick_upload: invalid brick size");
        return 0;
    }
    if (!obstacle || !surface_kind || !open_face_mask || !emitter_power_watts || !face_sky_exposure || !face_direct_exposure) {
        set_sim_error("simulation_queue_brick_world_static_brick_upload: null brick buffers");
        return 0;
    }
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_queue_brick_world_static_brick_upload: missing service");
        return 0;
    }
    World* w = find_world(*svc, world_key, "simulation_queue_brick_world_static_brick_upload");
    if (!w) return 0;
    if (w->brick_size != brick_size) {
        set_sim_error("simulation_queue_brick_world_static_brick_upload: brick size mismatch");
        return 0;
    }
    auto up = std::make_shared<PendingStaticUpload>();
    up->world = world_key;
    up->coord = Coord{brick_x, brick_y, brick_z};
    up->fields = std::make_unique<StaticFields>();
    StaticFields& f = *up->fields;
    f.obstacle.assign(obstacle, obstacle + cells);
    f.surface_kind.assign(surface_kind, surface_kind + cells);
    f.open_face_mask.assign(open_face_mask, open_face_mask + cells);
    f.emitter_power.assign(emitter_power_watts, emitter_power_watts + cells);
    f.face_sky.assign(face_sky_exposure, face_sky_exposure + (size_t)cells * 6);
    f.face_direct.assign(face_direct_exposure, face_direct_exposure + (size_t)cells * 6);
    int id = svc->next_upload_id++;
    if (id <= 0) id = svc->next_upload_id = 1;
    svc->pending_uploads[id] = up;
    AeroLbmWorldDelta d{};
    d.type = 9;
    d.x = brick_x;
    d.y = brick_y;
    d.z = brick_z;
    d.data0 = (int)world_key;
    d.data1 = id;
    w->pending_deltas.push_back(d);
    return 1;
}

// aero_lbm_simulation_copy_brick_world_dynamic_brick (simulation_bridge.cpp:5240-5299)
AERO_LBM_B200_EXPORT int aero_lbm_simulation_copy_brick_world_dynamic_brick(long long service_key, long long world_key,
                                                                            int brick_size, int brick_x, int brick_y,
                                                                            int brick_z, float* out_flow_state,
                                                                            float* out_air_temperature,
                                                                            float* out_surface_temperature) {
    Locks lk;
    int cells = 0;
    if (!cells_of(brick_size, &cells) || !out_flow_state || !out_air_temperature || !out_surface_temperature) {
        set_sim_error("simulation_copy_brick_world_dynamic_brick: invalid arguments");
        return 0;
    }
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_copy_brick_world_dynamic_brick: missing service");
        return 0;
    }
    World* w = find_world(*svc, world_key, "simulation_copy_brick_world_dynamic_brick");
    if (!w) return 0;
    if (w->brick_size != brick_size) {
        set_sim_error("simulation_copy_brick_world_dynamic_brick: brick size mismatch");
        return 0;
    }
    auto it = w->bricks.find(Coord{brick_x, brick_y, brick_z});
    if (it == w->bricks.end() || !it->second.has_dynamic) return 0;
    Brick& b = it->second;
    if (b.stale && b.context != 0) {
        if (!sync_from_context(*svc, *w, b, b.cur, b.cur, false)) {
            set_sim_error(std::string("simulation_copy_brick_world_dynamic_brick sync failed: ") + last_error());
            return 0;
        }
    }
    HostDynamic d;
    if (!pull(*w, b, b.cur, d)) {
        set_sim_error(std::string("simulation_copy_brick_world_dynamic_brick: ") + last_error());
        return 0;
    }
    std::copy(d.flow.begin(), d.flow.end(), out_flow_state);
    std::copy(d.air.begin(), d.air.end(), out_air_temperature);
    std::copy(d.surface.begin(), d.surface.end(), out_surface_temperature);
    return 1;
}

// aero_lbm_simulation_copy_brick_world_packed_flow_atlas (simulation_bridge.cpp:5301-5410).
// The strided output and its quantisation run on the device; the int16
// atlas is written into page-locked host memory by the kernel itself.
AERO_LBM_B200_EXPORT int aero_lbm_simulation_copy_brick_world_packed_flow_atlas(long long service_key, long long world_key,
                                                                                int brick_size, int brick_x, int brick_y,
                                                                                int brick_z, int sample_stride,
                                                                                int16_t* out_packed_flow,
                                                                                int packed_value_count) {
    Locks lk;
    int cells = 0;
    if (!cells_of(brick_size, &cells) || sample_stride <= 0 || !out_packed_flow) {
        set_sim_error("simulation_copy_brick_world_packed_flow_atlas: invalid arguments");
        return 0;
    }
    const int res = (brick_size + sample_stride - 1) / sample_stride;
    int samples = 0;
    if (!cells_of(res, &samples) || (long long)packed_value_count != (long long)samples * kAtlasChannels) {
        set_sim_error("simulation_copy_brick_world_packed_flow_atlas: output size mismatch");
        return 0;
    }
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_copy_brick_world_packed_flow_atlas: missing service");
        return 0;
    }
    World* w = find_world(*svc, world_key, "simulation_copy_brick_world_packed_flow_atlas");
    if (!w) return 0;
    if (w->brick_size != brick_size) {
        set_sim_error("simulation_copy_brick_world_packed_flow_atlas: brick size mismatch");
        return 0;
    }
    auto it = w->bricks.find(Coord{brick_x, brick_y, brick_z});
    if (it == w->bricks.end() || !it->second.has_dynamic) return 0;
    Brick& b = it->second;
    const float vscale = w->dt > 0.0f ? w->dx / w->dt : 1.0f;
    if (b.pending_upload && b.context == 0) {
        // a dynamic state the caller uploaded that no step has read yet
        const HostDynamic& d = *b.pending_upload;
        size_t k = 0;
        for (int x = 0; x < res; ++x)
            for (int y = 0; y < res; ++y)
                for (int z = 0; z < res; ++z, k += 4) {
                    const size_t src = (((size_t)std::min(brick_size - 1, x * sample_stride) * brick_size +
                                         std::min(brick_size - 1, y * sample_stride)) * brick_size +
                                        std::min(brick_size - 1, z * sample_stride)) * 4;
                    out_packed_flow[k] = host_quantize(d.flow[src] * vscale, kAtlasVelocityRange);
                    out_packed_flow[k + 1] = host_quantize(d.flow[src + 1] * vscale, kAtlasVelocityRange);
                    out_packed_flow[k + 2] = host_quantize(d.flow[src + 2] * vscale, kAtlasVelocityRange);
                    out_packed_flow[k + 3] = host_quantize(d.flow[src + 3], kAtlasPressureRange);
                }
        return 1;
    }
    cudaStream_t s = current_stream();
    if ((size_t)samples > svc->h_atlas_cap) {
        if (svc->h_atlas) cudaFreeHost(svc->h_atlas);
        svc->h_atlas = nullptr;
        svc->h_atlas_cap = 0;
        if (!cuda_ok(cudaHostAlloc(reinterpret_cast<void**>(&svc->h_atlas), (size_t)samples * 8, cudaHostAllocMapped),
                     "cudaHostAlloc(atlas)") ||
            !cuda_ok(cudaHostGetDevicePointer(reinterpret_cast<void**>(&svc->h_atlas_dev), svc->h_atlas, 0), "atlas pointer")) {
            set_sim_error(std::string("simulation_copy_brick_world_packed_flow_atlas: ") + last_error());
            return 0;
        }
        svc->h_atlas_cap = samples;
    }
    PublishArgs pa{};
    pa.stride = sample_stride;
    pa.res = res;
    pa.velocity_scale = vscale;
    pa.out = svc->h_atlas_dev;
    if (b.context != 0) {
        Context* ctx = find_context(b.context);
        if (!ctx || !ctx->initialized || ctx->nx != brick_size || ctx->ny != brick_size || ctx->nz != brick_size) {
            set_sim_error("simulation_copy_brick_world_packed_flow_atlas extract failed: "
                          "extract_flow_atlas: no initialized context of these dimensions");
            return 0;
        }
        if ((size_t)samples > svc->atlas_cap) {
            if (svc->d_atlas) cudaFree(svc->d_atlas);
            svc->d_atlas = nullptr;
            svc->atlas_cap = 0;
            if (!cuda_ok(cudaMalloc(reinterpret_cast<void**>(&svc->d_atlas), (size_t)samples * 16), "cudaMalloc(atlas)")) {
                set_sim_error(std::string("simulation_copy_brick_world_packed_flow_atlas: ") + last_error());
                return 0;
            }
            svc->atlas_cap = samples;
        }
        if (!output_device(*ctx, strided_box(brick_size, brick_size, brick_size, sample_stride), kFlowChannels, 1.0f,
                           svc->d_atlas)) {
            set_sim_error(std::string("simulation_copy_brick_world_packed_flow_atlas extract failed: ") + last_error());
            return 0;
        }
        pa.src = svc->d_atlas;
        pa.dense_n = 0;
    } else {
        if (!device_ready(*svc, *w, b)) {
            set_sim_error(std::string("simulation_copy_brick_world_packed_flow_atlas: ") + last_error());
            return 0;
        }
        pa.src = b.mem.flow[b.cur];
        pa.dense_n = brick_size;
    }
    if (!cuda_ok(launch_publish(pa, s), "publish atlas") || !cuda_ok(cudaStreamSynchronize(s), "publish atlas")) {
        set_sim_error(std::string("simulation_copy_brick_world_packed_flow_atlas: ") + last_error());
        return 0;
    }
    std::memcpy(out_packed_flow, svc->h_atlas, (size_t)samples * 8);
    return 1;
}

// aero_lbm_simulation_upload_brick_world_dynamic_brick (simulation_bridge.cpp:5412-5477)
AERO_LBM_B200_EXPORT int aero_lbm_simulation_upload_brick_world_dynamic_brick(long long service_key, long long world_key,
                                                                              int brick_size, int brick_x, int brick_y,
                                                                              int brick_z, const float* flow_state,
                                                                              const float* air_temperature,
                                                                              const float* surface_temperature) {
    Locks lk;
    int cells = 0;
    if (!cells_of(brick_size, &cells) || !flow_state || !air_temperature || !surface_temperature) {
        set_sim_error("simulation_upload_brick_world_dynamic_brick: invalid arguments");
        return 0;
    }
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_upload_brick_world_dynamic_brick: missing service");
        return 0;
    }
    World* w = find_world(*svc, world_key, "simulation_upload_brick_world_dynamic_brick");
    if (!w) return 0;
    if (w->brick_size != brick_size) {
        set_sim_error("simulation_upload_brick_world_dynamic_brick: brick size mismatch");
        return 0;
    }
    Brick& b = w->bricks[Coord{brick_x, brick_y, brick_z}];
    if (b.context != 0) {
        release_context(*svc, b);
        w->dynamic_upload_resets++;
    }
    drop_dynamic(*svc, b);
    auto d = host_dynamic_from(cells, flow_state, air_temperature, surface_temperature);
    if (b.stat) host_constrain(*b.stat, *d);
    b.nonzero = host_nonzero(*d);
    b.constrained_version = b.stat ? b.static_version : 0;
    b.has_dynamic = true;
    b.pending_upload = std::move(d);
    b.compact_active = false;
    b.stale = false;
    b.active = true;
    b.last_active_epoch = w->epoch;
    b.pending_reinit = false;
    b.forcing_dirty = false;
    return 1;
}

// aero_lbm_simulation_upload_brick_world_boundary_reference_brick (simulation_bridge.cpp:5479-5535)
AERO_LBM_B200_EXPORT int aero_lbm_simulation_upload_brick_world_boundary_reference_brick(
    long long service_key, long long world_key, int brick_size, int brick_x, int brick_y, int brick_z,
    const float* flow_state, const float* air_temperature, const float* surface_temperature) {
    Locks lk;
    int cells = 0;
    if (!cells_of(brick_size, &cells) || !flow_state || !air_temperature || !surface_temperature) {
        set_sim_error("simulation_upload_brick_world_boundary_reference_brick: invalid arguments");
        return 0;
    }
    Service* svc = lookup(service_key);
    if (!svc) {
        set_sim_error("simulation_upload_brick_world_boundary_reference_brick: missing service");
        return 0;
    }
    World* w = find_world(*svc, world_key, "simulation_upload_brick_world_boundary_reference_brick");
    if (!w) return 0;
    if (w->brick_size != brick_size) {
        set_sim_error("simulation_upload_brick_world_boundary_reference_brick: brick size mismatch");
        return 0;
    }
    const Coord c{brick_x, brick_y, brick_z};
    Brick& b = w->bricks[c];
    b.reference = host_dynamic_from(cells, flow_state, air_temperature, surface_temperature);
    b.reference_on_device = false;
    b.active = true;
    b.last_active_epoch = w->epoch;
    update_shell(*w, c, b);
    return 1;
}

// aero_lbm_simulation_runtime_info (simulation_bridge.cpp:6866-7017): the
// reference's key set; regions, atlases and the compact model do not exist here.
AERO_LBM_B200_EXPORT const char* aero_lbm_simulation_runtime_info(void) {
    static std::string text;
    Locks lk;
    size_t worlds = 0, bricks = 0, active = 0, solver = 0, statics = 0, dynamics = 0, contexts = 0, compact_ctx = 0,
           compact_ready_n = 0, stale = 0, exact = 0;
    uint64_t c[18] = {0};
    uint64_t last[5] = {0, 0, 0, 0, 0};
    uint64_t epoch = 0;
    bool any_exp = false, mixed = false;
    int mode = -1;
    if (g_service) {
        worlds = g_service->worlds.size();
        for (const auto& [k, w] : g_service->worlds) {
            const int m = normalize_mode(w.solver_mode);
            any_exp = any_exp || experimental(w);
            if (mode < 0) mode = m;
            else if (mode != m) mixed = true;
            bricks += w.bricks.size();
            for (const auto& [cc, b] : w.bricks) {
                active += b.active;
                solver += solver_active(w, b);
                statics += has_static(w, b);
                dynamics += b.has_dynamic;
                contexts += b.context != 0;
                compact_ctx += b.compact_active && b.context != 0;
                compact_ready_n += compact_ready(w, b);
                stale += b.stale;
            }
            exact += w.exact_hints;
            const uint64_t v[18] = {w.compact_cached_attempts, w.compact_cached_steps, w.compact_cached_failures,
                                    w.compact_initial_steps, w.compact_initial_failures, w.compact_reject_empty_steps,
                                    w.compact_reject_fan_steps, w.compact_thermal_ignored_steps, w.d3q27_steps,
                                    w.d3q27_patch_attempts, w.d3q27_patch_steps, w.d3q27_patch_failures,
                                    w.d3q27_patch_cells, w.d3q27_patch_upload_bytes_est, w.packet_build_steps,
                                    w.dynamic_upload_resets, 0, 0};
            for (int i = 0; i < 16; ++i) c[i] += v[i];
            const uint64_t l[5] = {w.compact_last_fluid_cells, w.compact_last_obstacle_cells, w.compact_last_fan_cells,
                                   w.compact_last_thermal_cells, w.compact_last_nonfinite_cells};
            for (int i = 0; i < 5; ++i) last[i] = std::max(last[i], l[i]);
            epoch = std::max(epoch, w.epoch);
        }
    }
    auto clean = [](std::string s, bool spaces) {
        std::replace(s.begin(), s.end(), '|', '/');
        if (spaces) std::replace(s.begin(), s.end(), ' ', '_');
        return s;
    };
    const std::string solver_rt = clean(aero_lbm_runtime_info(), false);
    const std::string memory = clean(aero_lbm_memory_info(), true);
    const std::string timing = clean(aero_lbm_timing_info(), true);
    const std::string bw_mode = mixed ? "mixed" : (mode < 0 ? "none" : mode_name(mode));
    auto kv = [](const char* k, uint64_t v) { return std::string("|") + k + "=" + std::to_string(v); };
    text = "simulation_bridge|services=" + std::to_string(g_service ? 1 : 0) + "|solver_runtime=" + solver_rt +
           "|compact_experimental=" + (simulation_compact_env() ? "on" : "off") + "|brick_world_solver=" + bw_mode +
           "|brick_world_compact=" + (any_exp ? "on" : "off") + kv("active_regions", 0) + kv("static_regions", 0) +
           kv("dynamic_regions", 0) + kv("atlases", 0) + kv("brick_worlds", worlds) + kv("bricks", bricks) +
           kv("active_bricks", active) + kv("solver_active_bricks", solver) + kv("static_bricks", statics) +
           kv("dynamic_bricks", dynamics) + kv("context_bricks", contexts) + kv("compact_context_bricks", compact_ctx) +
           kv("compact_ready_bricks", compact_ready_n) + kv("stale_dynamic_bricks", stale) + kv("exact_hint_worlds", exact) +
           kv("compact_cached_attempts", c[0]) + kv("compact_cached_steps", c[1]) + kv("compact_cached_failures", c[2]) +
           kv("compact_initial_steps", c[3]) + kv("compact_initial_failures", c[4]) +
           kv("compact_reject_empty_steps", c[5]) + kv("compact_reject_fan_steps", c[6]) +
           kv("compact_thermal_ignored_steps", c[7]) + kv("d3q27_steps", c[8]) + kv("d3q27_patch_attempts", c[9]) +
           kv("d3q27_patch_steps", c[10]) + kv("d3q27_patch_failures", c[11]) + kv("d3q27_patch_cells", c[12]) +
           kv("d3q27_patch_upload_bytes_est", c[13]) + kv("packet_build_steps", c[14]) +
           kv("dynamic_upload_resets", c[15]) + kv("compact_last_fluid_cells", last[0]) +
           kv("compact_last_obstacle_cells", last[1]) + kv("compact_last_fan_cells", last[2]) +
           kv("compact_last_thermal_cells", last[3]) + kv("compact_last_nonfinite_cells", last[4]) +
           "|native_memory=" + memory + "|native_timing=" + timing + kv("brick_epoch_max", epoch);
    return text.c_str();
}

AERO_LBM_B200_EXPORT const char* aero_lbm_simulation_last_error(void) {
    static std::string text;
    Locks lk;
    text = g_last_error;
    return text.c_str();
}

}  // extern "C"
