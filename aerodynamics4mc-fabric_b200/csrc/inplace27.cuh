// In-place ("esoteric pull") D3Q27 storage: one population array updated in
// place, alternating between two slot maps on even and odd steps
// (Lehmann et al., "Esoteric Pull and Esoteric Push", Computation 10(6) 2022).
//
// Directions are paired (q, 26 - q); q > 13 is the "positive" member. Every
// link x -> x + c (c positive) keeps its two in-transit populations in the
// memory of the cell at the link's positive end. With parity p of the step:
//   incoming f_q, q positive : own cell,        slot (p == 0 ? opp(q) : q)
//   incoming f_q, q negative : cell x - c_q,    slot (p == 0 ? opp(q) : q)
//   outgoing f*_q, q positive: cell x + c_q,    slot (p == 0 ? q : opp(q))
//   outgoing f*_q, q negative: own cell,        slot (p == 0 ? q : opp(q))
//   rest q = 13              : own cell, slot 13
// Every slot is read and then overwritten by exactly one cell per step, so the
// update is race-free with a single array. Half-way bounce-back of direction q
// (its source is solid, or outside a bounce-back face) reads the same cell's
// slot with the parity flipped: that slot holds the cell's own outgoing
// opp(q) population of the previous step, which no other cell touches.
//
// Storage is padded by one ghost cell on every side: ghost cells are never
// updated and hold the in-transit populations of links that cross a
// non-periodic face (bounce-back faces read them back; equilibrium faces
// ignore them). Periodic axes wrap instead. Padded index:
//   p(x, y, z) = ((x + 1) * (ny + 2) + (y + 1)) * pz + (z + 2),
// with a row length pz = nz + 3 rounded up to even (one unused element
// before the z = -1 ghost): every row starts at an even element, so the
// slots of an even z and of z + 1 form one aligned 2-element vector.
#pragma once

#include <cuda_fp16.h>

#include "lattice.cuh"

namespace aero {

__host__ __device__ constexpr bool q_positive(int q) { return q > 13; }

// Per-brick FP16 storage scale (deviation from the rest weights).
struct Fp16Scale {
    float scale;      // S: stored half = (f - w_q) * S / w_q
    float inv_scale;  // 1 / S
};

// Population storage policies.
struct StoreF32 {
    using T = float;
    __device__ __forceinline__ static float load(const float* __restrict__ a, int q, const Fp16Scale&) {
        (void)q;
        return __ldg(a);
    }
    __device__ __forceinline__ static void store(float* __restrict__ a, int q, float v, const Fp16Scale&) {
        (void)q;
        *a = v;
    }
};

// FP16 deviation storage: h = (f - w_q) * (S / w_q) = f * (S / w_q) - S,
// f = w_q + h * (w_q / S). The per-brick scale S keeps |h| far below the FP16
// range for any admissible state (|u| <= the speed clamp); a state that
// overflows anyway stores inf, and the next collision reseeds that cell (the
// reference's rule for non-finite populations).
struct StoreF16Dev {
    using T = __half;
    __device__ __forceinline__ static float load(const __half* __restrict__ a, int q, const Fp16Scale& s) {
        const float h = __half2float(__ldg(a));
        return fmaf(h, q_w(q) * s.inv_scale, q_w(q));
    }
    __device__ __forceinline__ static void store(__half* __restrict__ a, int q, float v, const Fp16Scale& s) {
        *a = __float2half_rn(fmaf(v, s.scale * (1.0f / q_w(q)), -s.scale));
    }
};

// 16-bit fixed-point deviation storage: h = round((f - w_q) * S / w_q),
// saturated to [-32767, 32767], f = w_q + h * w_q / S, with a per-brick
// scale S = 32767 / d_max (d_max bounds |f - w_q| / w_q for the brick's
// speeds). Same bytes as IEEE half, but a uniform resolution d_max / 32767
// over the whole range instead of 11 significant bits: the deviations that
// carry the flow (|f - w| / w ~ 0.1-1) are stored 5-10x more precisely. A
// non-finite value stores 0 (the rest weight).
// max.NaN keeps a NaN (which the conversion stores as 0) and lifts everything
// below -32767 to it before the saturating conversion: the same result as
// saturating to [-32768, 32767] and then raising -32768 to -32767.
__device__ __forceinline__ short sat_round_s16(float x) {
    float y;
    asm("max.NaN.f32 %0, %1, 0fC6FFFE00;" : "=f"(y) : "f"(x));  // -32767.0
    short r;
    asm("cvt.rni.sat.s16.f32 %0, %1;" : "=h"(r) : "f"(y));
    return r;
}
// Exact int16 -> float of both halves of a 32-bit word (low half first):
// 2^23 + 2^22 + h has h in its low mantissa bits for |h| < 2^22, so one
// integer add and one packed float subtract replace two conversions.
__device__ __forceinline__ float2 s16x2_to_float2(unsigned w) {
    const int lo = (int)(short)(w & 0xFFFFu), hi = (int)w >> 16;
    const float2 b = make_float2(__int_as_float(0x4B400000 + lo), __int_as_float(0x4B400000 + hi));
    return __fadd2_rn(b, make_float2(-12582912.0f, -12582912.0f));
}
struct StoreI16Dev {
    using T = short;
    __device__ __forceinline__ static float load(const short* __restrict__ a, int q, const Fp16Scale& s) {
        return fmaf((float)__ldg(a), q_w(q) * s.inv_scale, q_w(q));
    }
    __device__ __forceinline__ static void store(short* __restrict__ a, int q, float v, const Fp16Scale& s) {
        *a = sat_round_s16(fmaf(v, s.scale * (1.0f / q_w(q)), -s.scale));
    }
};

// Populations of solid cells are kept beside the lattice at a canonical
// parity: entry solid_slot(q, p) holds population q entering a step of
// parity p (a solid cell's populations flip every call, as the parity does).
__host__ __device__ __forceinline__ int solid_slot(int q, int parity) { return parity ? q_opp(q) : q; }

// Geometry of one padded brick and the per-axis wrap rule.
struct PadGeom {
    int nx, ny, nz;
    int py, pz;            // padded ny + 2; row length nz + 3 rounded up to even
    int pcells;            // (nx + 2) (ny + 2) pz
    int wrap[3];           // axis wraps (periodic on both faces)
};

__host__ __device__ constexpr int pad_row(int nz) { return (nz + 4) & ~1; }

__host__ __device__ inline PadGeom make_pad_geom(int nx, int ny, int nz, int periodic_mask) {
    PadGeom g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.py = ny + 2; g.pz = pad_row(nz);
    g.pcells = (nx + 2) * (ny + 2) * g.pz;
    g.wrap[0] = (periodic_mask >> 0) & 1;
    g.wrap[1] = (periodic_mask >> 1) & 1;
    g.wrap[2] = (periodic_mask >> 2) & 1;
    return g;
}

__device__ __forceinline__ int pad_index(const PadGeom& g, int x, int y, int z) {
    return ((x + 1) * g.py + (y + 1)) * g.pz + (z + 2);
}

// Neighbour coordinate along one axis: wrapped on periodic axes, else may be
// -1 or n (a ghost cell).
__device__ __forceinline__ int axis_neighbour(int c, int d, int n, int wrap) {
    int v = c + d;
    if (wrap) v = v < 0 ? v + n : (v >= n ? v - n : v);
    return v;
}

// Offsets of the three neighbour positions (-1, 0, +1) per axis in padded
// index units, so that the padded index of x + c is X[cx+1] + Y[cy+1] + Z[cz+1].
struct NeighbourOffsets {
    int X[3], Y[3], Z[3];
};

__device__ __forceinline__ NeighbourOffsets neighbour_offsets(const PadGeom& g, int x, int y, int z) {
    NeighbourOffsets o;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        o.X[k] = (axis_neighbour(x, k - 1, g.nx, g.wrap[0]) + 1) * g.py * g.pz;
        o.Y[k] = (axis_neighbour(y, k - 1, g.ny, g.wrap[1]) + 1) * g.pz;
        o.Z[k] = axis_neighbour(z, k - 1, g.nz, g.wrap[2]) + 2;
    }
    return o;
}

// Padded index of x + d*c_q (d = +1 destination, -1 source).
__device__ __forceinline__ int link_cell(const NeighbourOffsets& o, int q, int d) {
    const int ix = 1 + d * q_cx(q), iy = 1 + d * q_cy(q), iz = 1 + d * q_cz(q);
    return o.X[ix] + o.Y[iy] + o.Z[iz];
}

// Memory cell and slot direction of incoming population q at parity p
// (bounce = read the flipped slot).
__device__ __forceinline__ void incoming_slot(const NeighbourOffsets& o, int own, int q, int p, bool bounce,
                                              int& cell, int& dir) {
    const bool even = (p == 0) != bounce;
    dir = q == kRest27 ? kRest27 : (even ? q_opp(q) : q);
    cell = (q == kRest27 || q_positive(q)) ? own : link_cell(o, q, -1);
}

// Slot offsets relative to a cell's own padded index, for a cell none of
// whose neighbours wraps around a periodic axis (the neighbour along c is
// then own + link_offset(c)); launch-uniform apart from the bounce choice.
__host__ __device__ __forceinline__ int link_offset(const PadGeom& g, int q) { return (q_cx(q) * g.py + q_cy(q)) * g.pz + q_cz(q); }
// bounce: the parity-flipped slot of the same memory cell
__host__ __device__ __forceinline__ int in_offset(const PadGeom& g, int q, int p, bool bounce = false) {
    const bool even = (p == 0) != bounce;
    const int dir = q == kRest27 ? kRest27 : (even ? q_opp(q) : q);
    const int cell = (q == kRest27 || q_positive(q)) ? 0 : -link_offset(g, q);
    return dir * g.pcells + cell;
}
__host__ __device__ __forceinline__ int out_offset(const PadGeom& g, int q, int p) {
    const int dir = q == kRest27 ? kRest27 : (p == 0 ? q : q_opp(q));
    const int cell = (q == kRest27 || !q_positive(q)) ? 0 : link_offset(g, q);
    return dir * g.pcells + cell;
}
// True when no neighbour of (x, y, z) wraps around a periodic axis.
__device__ __forceinline__ bool no_wrap(const PadGeom& g, int x, int y, int z) {
    return !((g.wrap[0] && (x == 0 || x == g.nx - 1)) || (g.wrap[1] && (y == 0 || y == g.ny - 1)) ||
             (g.wrap[2] && (z == 0 || z == g.nz - 1)));
}

// Memory cell and slot direction of outgoing population q at parity p.
__device__ __forceinline__ void outgoing_slot(const NeighbourOffsets& o, int own, int q, int p, int& cell, int& dir) {
    dir = q == kRest27 ? kRest27 : (p == 0 ? q : q_opp(q));
    cell = (q == kRest27 || !q_positive(q)) ? own : link_cell(o, q, +1);
}

}  // namespace aero
