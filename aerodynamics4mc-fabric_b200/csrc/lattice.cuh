// D3Q27 lattice for the brick step.
//
// Direction numbering follows the reference so that population arrays, cell
// masks and the C ABI stay interchangeable with it:
//   q = (ix * 3 + iy) * 3 + iz,  c = (ix - 1, iy - 1, iz - 1),  rest q = 13,
//   opposite(q) = 26 - q,        w = w1(ix) w1(iy) w1(iz), w1 = {1/6, 2/3, 1/6}
// (native/include/aero_lbm_hydro_core.h:7-90).
//
// Cell index: cell = (x * ny + y) * nz + z (z fastest), populations are
// structure-of-arrays f[q * cells + cell] (native/src/aero_lbm_jni.cpp:1180-1191).
#pragma once

#include <cstdint>

namespace aero {

constexpr int kQ27 = 27;
constexpr int kRest27 = 13;

__host__ __device__ constexpr int q_cx(int q) { return q / 9 - 1; }
__host__ __device__ constexpr int q_cy(int q) { return (q / 3) % 3 - 1; }
__host__ __device__ constexpr int q_cz(int q) { return q % 3 - 1; }
__host__ __device__ constexpr int q_opp(int q) { return 26 - q; }

// Product weights in float, evaluated as (w1[ix] * w1[iy]) * w1[iz] like the
// reference's constexpr table.
__host__ __device__ constexpr float w1f(int i) { return i == 1 ? 2.0f / 3.0f : 1.0f / 6.0f; }
__host__ __device__ constexpr float q_w(int q) { return w1f(q / 9) * w1f((q / 3) % 3) * w1f(q % 3); }

// Face ids, in the reference's order: x-, x+, y-, y+, z-, z+.
enum FaceId { kFaceXMin = 0, kFaceXMax, kFaceYMin, kFaceYMax, kFaceZMin, kFaceZMax };

// Hydrodynamic face kinds (values are the C ABI's AeroLbmHydrodynamicBoundaryKind).
enum HydroKind {
    kHydroInheritGame = 0,
    kHydroPeriodic = 1,
    kHydroBounceBack = 2,
    kHydroMovingWall = 3,
    kHydroVelocity = 4,
    kHydroPressure = 5,
    kHydroConvective = 6,
    kHydroSymmetry = 7,
};

// Per-cell pull classification word (built once per call from the mask and
// the face configuration; see build_flags_kernel):
//   bits 0..26 : the source cell of direction q is a bounce-back source
//                (a solid cell, or outside a bounce-back face)
//   bit 27     : this cell is solid
//   bit 28     : some source of this cell lies outside a non-periodic face
//                whose value is not plain bounce-back (equilibrium, symmetry,
//                convective outflow): the cell takes the boundary path
constexpr uint32_t kFlagSelfSolid = 1u << 27;
constexpr uint32_t kFlagFaceSpecial = 1u << 28;
constexpr uint32_t kFlagBounceMask = (1u << 27) - 1u;

// Coordinates of cell (x*ny + y)*nz + z. Grids hold fewer than 2^31 cells, so
// 32-bit unsigned division suffices (a 64-bit division costs several times the
// instructions).
__host__ __device__ __forceinline__ void cell_xyz32(long long cell, int ny, int nz, int& x, int& y, int& z) {
    const unsigned c = (unsigned)cell, unz = (unsigned)nz, uny = (unsigned)ny;
    const unsigned line = c / unz;
    z = (int)(c - line * unz);
    const unsigned xx = line / uny;
    y = (int)(line - xx * uny);
    x = (int)xx;
}

}  // namespace aero
