// Temperature transport of the brick step: the reference's benchmark-mode
// scalar update (update_temperature_field, native/src/aero_lbm_jni.cpp:2049-2143,
// first-order branch; helpers 738-769 and 1783-1950), run before every
// collision so that the Boussinesq force sees the transported field:
//
//   T'(x) = clamp(A + dt (alpha lap T(x) + s(x)), -1, 1),   dt = 1,
//   A     = trilinear sample of T at x - dt u(x), u = the previous collision's
//           velocity (post-clamp midpoint velocity; 0 on solid cells),
//   lap   = sum of the six face neighbours - 6 T(x),
//
// where a neighbour or sample corner that is solid, or outside a face that is
// not thermally periodic, takes the face rule (Dirichlet: the face temperature,
// Neumann: T(x) + heat flux, otherwise T(x); for the sample the centre's T(x)
// stands in). Solid cells hold 0. Built with --fmad=false and the reference's
// operation order: bit-identical to the reference CPU step.
//
// The heated-cavity presets (and the reference outside benchmark mode) take
// the BFECC branch instead (jni.cpp:2050-2135): S = A_-(T), N = clamp(T +
// (T - A_+(S)) / 2), T' = clamp(clamp(A_-(N), local min/max of T) + dt (alpha
// lap T + s)), with A_-/A_+ the trilinear samples at x -/+ dt u (their
// fallback the sampled field's own value at x), three launches.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "d3q27_kernels.cuh"

namespace aero {

// Thermal face kinds (native/include/aero_lbm_capi.h:57-62).
enum ThermalKind { kThermalInherit = 0, kThermalDisabled = 1, kThermalPeriodic = 2, kThermalAdiabatic = 3,
                   kThermalDirichlet = 4, kThermalNeumann = 5 };

struct ThermalFaces {
    int kind[6];            // x-, x+, y-, y+, z-, z+
    float temperature[6];   // Dirichlet value (clamped to +-1 when used)
    float heat_flux[6];     // Neumann increment
};

// Tagged staging of the transport's neighbourhood (bricks without a Neumann
// face): an entry that stands for the querying cell's own value (a solid cell
// or a face that returns the cell's value) holds this NaN payload, which no
// float operation produces, instead of a separate code.
constexpr unsigned kOwnTag = 0x7fbadbadu;

__host__ __device__ __forceinline__ bool no_neumann(const ThermalFaces& F) {
    bool none = true;
#pragma unroll
    for (int f = 0; f < 6; ++f) none = none && F.kind[f] != kThermalNeumann;
    return none;
}

struct ThermalArgs {
    int nx, ny, nz;
    long long cells;
    const float* t;             // state before the update
    float* t_next;              // state after the update
    const float* u;             // previous collision velocity, SoA (ux, uy, uz), 3 x cells
    const uint8_t* obstacle;    // mask of this call
    const float* source;        // per-cell source (clamped to +-0.006) or null
    float alpha;                // thermal diffusivity
    ThermalFaces faces;
    int bfecc;                  // 1: the BFECC branch (heated-cavity presets); the result lands in scratch
    float* scratch;             // BFECC: third state buffer
    // Runtime mode (benchmark off): the BFECC update runs every other call
    // with dt = 2 and adds a local eddy diffusivity nu_t / 0.85 from the last
    // collision's velocity gradients (runtime_local_turbulent_nu and
    // effective_local_thermal_diffusivity, jni.cpp:1972-2047).
    float dt;                   // effective_thermal_dt: 1, or 2 in runtime mode
    int turbulent;              // add the local eddy diffusivity
    float sgs_c2;               // Smagorinsky C^2 of the eddy viscosity
    float nu0;                  // runtime molecular viscosity (its cap is 5 nu0)
    int pairs;                  // set by the launch: z-pair vector access allowed (even nz, aligned fields)
    int xchunk;                 // set by the launch: x-planes per transport block
    int zero_bits;              // set by the launch: 0, a run-time zero for the packed products
};

// Runtime mode, every call after the first (apply_runtime_temperature_reference,
// jni.cpp:8037-8064): solid cells hold 0; fluid cells in the 8 outer layers
// move toward the packet temperature by the state nudge factor.
struct ThermalNudgeArgs {
    int nx, ny, nz;
    float* t;
    const uint8_t* obstacle;
    const float* ref_t;
    float nudge;                // 0.08
};
cudaError_t launch_thermal_reference_nudge(const ThermalNudgeArgs& a, cudaStream_t s);

// First call of a context: the state and the velocity the first update
// advects with (initialize_distributions, jni.cpp:1752-1781). benchmark: a
// state of magnitude < 1e-8 takes initial_temperature, any other fluid cell
// the packet's reference temperature; otherwise fluid cells take the
// reference temperature. u = the packet velocity on fluid cells, 0 on solids.
struct ThermalInitArgs {
    long long cells;
    float* t;
    float* u;                   // SoA 3 x cells
    const uint8_t* obstacle;
    const float* ref_t;
    const float* ref_ux;
    const float* ref_uy;
    const float* ref_uz;
    float initial_temperature;
    int benchmark;
};

cudaError_t launch_thermal_init(const ThermalInitArgs& a, cudaStream_t s);
struct IpArgs;
// The first-order transport (not BFECC) and, in the same launch, the face
// pre-fill of an in-place context (storage: 0 FP32, 1 IEEE half, 2 16-bit
// fixed point; f its populations, fill the fill's arguments).
cudaError_t launch_thermal_update_fill(const ThermalArgs& a, int storage, void* f, const IpArgs& fill, cudaStream_t s);
cudaError_t launch_thermal_update(const ThermalArgs& a, cudaStream_t s);

}  // namespace aero
