// Host side of the brick-world service (aero_lbm_simulation_*): bricks of one
// world, their static and dynamic fields and their solver contexts.
//
// The reference service (native/src/aero_lbm_simulation_bridge.cpp) keeps
// every brick's dynamic state in host vectors, rebuilds an 11-channel packet
// per brick per tick on the host, steps it through aero_lbm_step_rect and reads
// the whole flow and temperature back. Here a brick's static fields and its
// dynamic state live on the device (two buffers per brick, so that the state
// a tick started from stays readable while the brick steps); a tick builds
// each brick's inputs with one kernel straight into its context, refreshes the
// dynamic state with one kernel after the step, and reads back nothing but one
// flag word per brick. Host copies are made only on the rare paths that the
// reference decides on whole-brick contents (seeding a brick from its
// neighbours, face bootstrap, the compact-mode packet summary) and when the
// caller asks for a brick.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "aero_lbm_b200.h"
#include "brick_world.cuh"

namespace aero {
namespace bw {

struct Coord {
    int x = 0, y = 0, z = 0;
    bool operator<(const Coord& o) const { return x != o.x ? x < o.x : (y != o.y ? y < o.y : z < o.z); }
    bool operator==(const Coord& o) const { return x == o.x && y == o.y && z == o.z; }
};

// Static fields as the caller uploads them (StaticRegionData,
// simulation_bridge.cpp:22-33), kept on the host for the world-delta patches.
struct StaticFields {
    std::vector<uint8_t> obstacle, surface_kind, source_fan_dir, face_sky, face_direct;
    std::vector<uint16_t> open_face_mask;
    std::vector<float> emitter_power, source_emitter_power;
};

// A host copy of a dynamic brick (DynamicRegionData's three arrays).
struct HostDynamic {
    std::vector<float> flow, air, surface;
};

// Device memory of one brick: static fields, two dynamic buffers, the
// boundary reference.
struct BrickMemory {
    void* block = nullptr;
    uint8_t* obstacle = nullptr;
    uint8_t* surface_kind = nullptr;
    uint16_t* open_face_mask = nullptr;
    float* emitter_power = nullptr;
    float* flow[2] = {nullptr, nullptr};
    float* air[2] = {nullptr, nullptr};
    float* surface[2] = {nullptr, nullptr};
    float* ref_flow = nullptr;
    float* ref_air = nullptr;
};

struct Brick {
    // bookkeeping flags of BrickData (simulation_bridge.cpp:128-148)
    bool active_hint = false, active = false;
    bool geometry_dirty = false, forcing_dirty = false, pending_reinit = false;
    uint64_t last_hint_epoch = 0, last_active_epoch = 0;
    long long context = 0;
    bool compact_active = false;
    bool stale = false;  // the context is ahead of the dynamic state
    float compact_v[3] = {0.0f, 0.0f, 0.0f};
    std::vector<int> pending_patch_cells;

    std::unique_ptr<StaticFields> stat;
    uint64_t static_version = 0;  // bumped on every change of stat
    uint64_t static_on_device = 0;  // version of the device copy (0: none)
    // static version and context of the last step built from the static fields
    // (its mask is the context's current one)
    uint64_t stepped_version = 0;
    long long stepped_context = 0;

    // dynamic state: buffer `cur` on the device, or a host copy not yet uploaded
    bool has_dynamic = false;
    int cur = 0;
    std::unique_ptr<HostDynamic> pending_upload;
    bool nonzero = false;        // some cell of the dynamic flow has |u_i| > 1e-8
    bool flag_pending = false;   // nonzero is being recomputed on the device (flag slot)
    uint64_t constrained_version = 0;  // static version the dynamic buffer was last constrained with (0: not since a sync)

    std::shared_ptr<const HostDynamic> reference;  // boundary reference
    bool reference_on_device = false;

    BrickMemory mem;
    int flag_slot = -1;
};

struct World {
    int brick_size = 0;
    float dx = 1.0f, dt = 0.05f;
    int solver_mode = AERO_LBM_REALTIME_SOLVER_CLASSIC_D3Q27;
    bool exact_hints = false;
    uint64_t epoch = 0;
    std::map<Coord, Brick> bricks;
    std::map<Coord, bool> hint_closure;
    std::vector<AeroLbmWorldDelta> pending_deltas;
    // counters of FluidWorldRuntime (simulation_bridge.cpp:150-181), reported by runtime_info
    uint64_t compact_cached_attempts = 0, compact_cached_steps = 0, compact_cached_failures = 0;
    uint64_t compact_initial_steps = 0, compact_initial_failures = 0;
    uint64_t compact_reject_empty_steps = 0, compact_reject_fan_steps = 0, compact_thermal_ignored_steps = 0;
    uint64_t d3q27_steps = 0, d3q27_patch_attempts = 0, d3q27_patch_steps = 0, d3q27_patch_failures = 0;
    uint64_t d3q27_patch_cells = 0, d3q27_patch_upload_bytes_est = 0;
    uint64_t packet_build_steps = 0, dynamic_upload_resets = 0;
    uint64_t compact_last_fluid_cells = 0, compact_last_obstacle_cells = 0, compact_last_fan_cells = 0;
    uint64_t compact_last_thermal_cells = 0, compact_last_nonfinite_cells = 0;
};

struct PendingStaticUpload {
    long long world = 0;
    Coord coord;
    std::unique_ptr<StaticFields> fields;
};

// World-delta handling (brick_world_deltas.cpp): static patches applied on
// the host copy of the static fields.
void apply_world_delta(World& w, const AeroLbmWorldDelta& d);
void rebuild_static_from_sources(StaticFields& s, int n);
void ensure_source_fields(StaticFields& s, size_t cells);
// The host copy of a brick's static fields changed: the device copy is
// refreshed at the next device use; with constrain_dynamic the dynamic state
// takes the static constraints at once (apply_brick_static_constraints),
// otherwise it keeps whatever constraint state it had (the constraint fields
// themselves did not change). Implemented by the service.
void static_changed(World& w, Brick& b, bool constrain_dynamic);
void install_static(World& w, Brick& b, std::unique_ptr<StaticFields> fields);
void mark_brick(World& w, const Coord& c, bool geometry, bool forcing, bool reinit);

}  // namespace bw
}  // namespace aero
