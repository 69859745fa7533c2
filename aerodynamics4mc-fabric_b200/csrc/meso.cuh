// D3Q19 mesoscale step: shared definitions (forcing channels, kernel
// arguments, launchers).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace aero {

// forcing channels of aero_lbm_mesoscale_step_context
// (native/src/aero_lbm_mesoscale.cpp:115-139), cells x 25 floats, AoS
constexpr int kMesoForcingChannels = 25;
constexpr int kMesoStateChannels = 6;  // ambient, deep ground, surface, wind x, y, z
enum MesoChannel : int {
    kChTerrainHeight = 0,
    kChAmbientTarget = 2,
    kChDeepGroundTarget = 3,
    kChSurfaceTarget = 4,
    kChRoughness = 5,
    kChBackgroundWindX = 6,
    kChBackgroundWindZ = 7,
    kChHumidity = 9,
    kChConvectiveHeating = 10,
    kChConvectiveMoistening = 11,
    kChConvectiveInflowX = 12,
    kChConvectiveInflowZ = 13,
    kChTornadoWindX = 14,
    kChTornadoWindZ = 15,
    kChTornadoHeating = 16,
    kChTornadoMoistening = 17,
    kChTornadoUpdraft = 18,
    kChNestedUpdraft = 19,
    kChNestedWindXDelta = 20,
    kChNestedWindZDelta = 21,
    kChNestedAmbientDelta = 22,
    kChNestedSurfaceDelta = 23,
    kChSolidMask = 24,
};

namespace meso {

// Hydrodynamic TRT rates and the optional Guo body force / Smagorinsky model.
struct HydroRates {
    int forced, enable_sgs;
    float tau_h, omega_even, omega_odd, smagorinsky_c, fx, fy, fz;
};

// One step of the reference model (hydrodynamic + thermal distributions).
// Populations are SoA: f[q*cells+cell].
struct MesoArgs {
    int nx, ny, nz;
    int periodic_sides, free_slip_top, edge_blend;
    float dt_s, velocity_scale, max_speed;
    HydroRates h;
    float omega_t_even, omega_t_odd;
    const float* forcing;  // cells x 25 (AoS, as passed by the caller)
    float* f;              // current hydrodynamic populations (19 x cells)
    float* g;              // current thermal populations (19 x cells)
    float* post_f;         // post-collision scratch (19 x cells)
    float* post_g;
    float* ambient;        // macro temperature of the previous step (read), this step (written)
    float* deep;           // deep-ground / surface temperatures of the previous step
    float* surface;
    float* next_deep;      // ... of this step
    float* next_surface;
    float* out_state;      // cells x 6 (AoS) or null
};

// One launch of the hydrodynamic-only step (fused pull + collision on two
// population buffers; the buffers hold post-collision values).
struct HydroArgs {
    int nx, ny, nz;
    int periodic_sides, free_slip_top, edge_blend;
    float velocity_scale, max_speed;
    float scale, inv_scale;        // FP16 deviation scale (FP16 storage only)
    HydroRates h;
    const uint8_t* solid_prev;     // mask the pull streams with (the previous call's)
    const uint32_t* flags_prev;    // pull classification of solid_prev (meso_hydro_flags)
    const uint8_t* solid_cur;      // mask of this call's collision
    const float* forcing_prev;     // previous call's forcing (open-boundary winds)
    const void* src;               // 19 x cells, float or __half
    void* dst;
    float* out_state;              // output launch: cells x 6
};

}  // namespace meso

cudaError_t meso_launch_seed(const meso::MesoArgs& a, cudaStream_t s);
cudaError_t meso_launch_step(const meso::MesoArgs& a, cudaStream_t s);

// Hydrodynamic-only step. `fp16` selects __half deviation storage.
enum MesoHydroMode { kHydroInit = 0, kHydroStep = 1, kHydroOutput = 2 };
// Population storage of the hydrodynamic-only step.
enum MesoStorage { kMesoStoreF32 = 0, kMesoStoreF16 = 1, kMesoStoreI16 = 2 };
cudaError_t meso_hydro_seed(const float* forcing, int nx, int ny, int nz, float velocity_scale, int storage, float scale,
                            void* dst, uint8_t* solid, cudaStream_t s);
cudaError_t meso_hydro_mask(const float* forcing, long long cells, uint8_t* solid, cudaStream_t s);
// Pull classification word per cell: bit q (0..18) = direction q bounces back,
// kHydroSlow = the cell pulls through an open side or the lid, or is blended,
// kHydroSelfSolid = the cell is solid.
constexpr uint32_t kHydroSelfSolid = 1u << 31;
constexpr uint32_t kHydroSlow = 1u << 30;
cudaError_t meso_hydro_flags(const meso::HydroArgs& a, const uint8_t* solid, uint32_t* flags, cudaStream_t s);
cudaError_t meso_hydro_launch(const meso::HydroArgs& a, int mode, int storage, int threads, cudaStream_t s);
// Fused step with two z-adjacent cells per thread and the TRT collision in
// packed FP32 (meso_fast.cu); nz must be even.
cudaError_t meso_hydro_fast_step(const meso::HydroArgs& a, int storage, cudaStream_t s);

}  // namespace aero
