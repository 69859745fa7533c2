// Device side of the brick-world service (brick_world.cu): the kernels that
// replace the reference service's per-brick host loops
// (native/src/aero_lbm_simulation_bridge.cpp) with passes over device-resident
// brick state.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "d3q27_kernels.cuh"

namespace aero {
namespace bw {

// Flow channels of a dynamic brick (ux, uy, uz, pressure proxy) and of the
// packed atlas (AERO_LBM_SIMULATION_FLOW_STATE_CHANNELS / _PACKED_ATLAS_CHANNELS).
constexpr int kFlowChannels = 4;
constexpr int kAtlasChannels = 4;
constexpr int kPacketChannels = 11;
// Quantisation ranges of the packed atlas (simulation_bridge.cpp:234-235).
constexpr float kAtlasVelocityRange = 5.6f;
constexpr float kAtlasPressureRange = 0.03f;
// Boundary-reference layers blended into exposed faces (simulation_bridge.cpp:261-262).
constexpr int kBoundaryReferenceLayers = 8;
constexpr float kBoundaryReferenceRelaxation = 0.10f;

// Static fields of one brick on the device.
struct StaticDev {
    const uint8_t* obstacle;
    const uint8_t* surface_kind;
    const uint16_t* open_face_mask;
    const float* emitter_power;
};

// Inputs of one brick's call, built on the device straight into the context's
// per-cell fields (build_brick_step_packet, simulation_bridge.cpp:1497-1596,
// followed by the runtime's ingest_payload).
struct FillArgs {
    int n;
    StaticDev st;
    const float* flow;       // dynamic brick the packet reads (4 x cells, AoS)
    const float* air;        // its air temperature
    const float* ref_flow;   // boundary reference (null: none)
    const float* ref_air;
    int exposed;             // bit f: face f (x-, x+, y-, y+, z-, z+) reads the reference in its outer layers
    int ref_layers;
    float source_denominator;  // rho_air * c_p * V_cell * T_scale, folded in float like the reference's constant
};

// Dynamic-brick refresh after a call (sync_brick_dynamic_from_context +
// apply_brick_static_constraints, simulation_bridge.cpp:1598-1615, 1202-1236).
// The flow channels have been written by the runtime's output pass.
struct SyncArgs {
    long long cells;
    float* flow;
    float* air;
    float* surface;
    const float* temperature;  // context temperature state copied into air (null: keep air)
    const float* surface_src;  // surface temperature copied into surface (null: keep)
    StaticDev st;              // obstacle null: no constraints
    int* flag;                 // kFlagBefore / kFlagAfter bits or-ed in (null: none)
};
// Flag bits: some cell has a velocity component above 1e-8 in magnitude
// (dynamic_has_nonzero_flow, simulation_bridge.cpp:1245-1259), after the
// static constraints, and in the flow before them.
constexpr int kFlagAfter = 1;
constexpr int kFlagBefore = 2;

// Packed int16 atlas (copy_brick_world_packed_flow_atlas, simulation_bridge.cpp:5301-5410).
struct PublishArgs {
    const float* src;   // 4 floats per sample
    int dense_n;        // > 0: src is the dense n^3 brick, sampled at min(n-1, a*stride); 0: src is the atlas
    int stride;
    int res;            // atlas resolution per axis
    float velocity_scale;
    int16_t* out;
};

cudaError_t launch_fill(const FillArgs& a, const CellFields& out, cudaStream_t s);
cudaError_t launch_sync(const SyncArgs& a, cudaStream_t s);
cudaError_t launch_publish(const PublishArgs& a, cudaStream_t s);

}  // namespace bw
}  // namespace aero
