// In-place (esoteric pull) D3Q27 brick step kernels, templated on the
// population storage (FP32 or FP16 deviation) and the collision arithmetic
// (reference order or factorised). See inplace27.cuh for the slot maps.
//
// The step kernels resolve periodic and bounce-back faces themselves; every
// other face kind (equilibrium faces, symmetry, convective outflow) has its
// pulled values written into the ghost layer by face_fill_ip_kernel after the
// previous call's step, from the post-collision populations that step left
// (ip_face_source). An axis that is periodic on one side only has no in-place
// form.
#pragma once

#include "pdl.cuh"
#include "d3q27_step.cuh"
#include "collide27_x2.cuh"
#include "collide27_exact_x2.cuh"
#include "inplace27.cuh"
#include "thermal_fused.cuh"

namespace aero {

struct IpArgs {
    PadGeom g;
    int parity;                      // parity of this step's slot maps
    const uint32_t* flags_prev;      // pull classification of the streaming call
    const uint8_t* obstacle_cur;     // mask of this call (collide / skip)
    const float* ref_p_prev;         // pressure proxy of the streaming call (equilibrium faces)
    const FaceParams* face_prev;     // faces of the streaming call (device memory)
    CellFields cur;
    ForceField force;
    CollideParams cp;
    Fp16Scale sc;
    int cells_per_thread;            // 1 one cell per thread, 2 two cells per thread (packed collision)
    int streamed;                    // factorised two-cell step: populations streamed by bulk async copies
    int* fault;                      // device word set to 1 by a streamed step whose copies never landed
    // Temperature transport computed by the step kernel itself (1) before each
    // collision (thermal_fused.cuh), or by a separate pass (0); the launch
    // then provides fused_smem_bytes(block span) of dynamic shared memory.
    int transport;
    FusedTransport tr;
    // Populations of solid cells (27 x cells FP32, null = all at rest): the
    // reference keeps a solid cell's streamed populations and flips them
    // every call (jni.cpp:2209-2452: f_post = f, f'[q] = f_post[opp q]); they
    // come back when the cell opens again. Stored at a canonical parity:
    // entry (p ? opp(q) : q) holds population q at a step of parity p.
    float* solid_f;
    // Slot offsets of the launch's parity relative to a cell's own padded
    // index, for cells none of whose neighbours wraps (in_offset / out_offset
    // of inplace27.cuh, filled by the launcher): incoming [q][bounce],
    // outgoing [q]. Launch-uniform, read from the parameter space.
    int off_in[27][2];
    int off_out[27];
    // Faces the face pre-fill visits (bit f, faces x-, x+, y-, y+, z-, z+);
    // 0 = all six. A face whose links are all bounce-back or periodic needs no
    // visit: the deciding face of every link the fill writes is in the set.
    unsigned fill_faces;
};


// Equilibrium value of a face (velocity / pressure / moving wall), the only
// non-bounce-back faces the in-place layout accepts
// (boundary_equilibrium_value, jni.cpp:1519-1561).
__device__ __forceinline__ float ip_face_equilibrium(const FaceParams& F, int q, float ref_p, int y, int sx, int sy, int sz,
                                                     int nx, int ny, int nz) {
    const int face = oob_face(sx, sy, sz, nx, ny, nz);
    const int kind = F.kind[face];
    float rho = 1.0f + clampf_dev(ref_p, -0.03f, 0.03f);
    float ux = 0.0f, uy = 0.0f, uz = 0.0f;
    if (kind == kHydroPressure) {
        rho = 1.0f + clampf_dev(F.pressure[face], -0.03f, 0.03f);
    } else {
        ux = F.velocity[face][0]; uy = F.velocity[face][1]; uz = F.velocity[face][2];
        if (F.cylinder_inlet && sx < 0) {
            ux = cylinder_inlet_ux(ny, y, F.velocity[face][0]);
            uy = 0.0f; uz = 0.0f;
        }
    }
    rho = clampf_dev(rho, 0.97f, 1.03f);
    const float s2 = ux * ux + uy * uy + uz * uz;
    if (s2 > F.max_speed * F.max_speed && s2 > 0.0f) {
        const float sc = F.max_speed / sqrtf(s2);
        ux *= sc; uy *= sc; uz *= sc;
    }
    return feq27(q, rho, ux, uy, uz);
}

// Incoming populations of a fluid cell at parity p, read between calls: the
// face pre-fill a call leaves runs before any such read, so each incoming
// slot (the face sources included) holds the cell's streamed population.
template <class S>
__device__ __forceinline__ void ip_pull(const typename S::T* __restrict__ f, const IpArgs& a, const PadGeom& G,
                                        const NeighbourOffsets& o, int own, uint32_t w, int p, float (&fl)[27]) {
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        int c, d;
        incoming_slot(o, own, q, p, (w >> q) & 1u, c, d);
        fl[q] = S::load(f + (long long)d * G.pcells + c, q, a.sc);
    }
}

template <class S>
__device__ __forceinline__ void ip_push(typename S::T* __restrict__ f, const IpArgs& a, const PadGeom& G,
                                        const NeighbourOffsets& o, int own, int p, const float (&fl)[27]) {
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        int c, d;
        outgoing_slot(o, own, q, p, c, d);
        S::store(f + (long long)d * G.pcells + c, q, fl[q], a.sc);
    }
}

__device__ __forceinline__ void cell_coords(const PadGeom& G, long long cell, int& x, int& y, int& z) {
    cell_xyz32(cell, G.ny, G.nz, x, y, z);
}

// Reseed a cell into the in-place state (out of line: rare path; scalar
// arguments only so the hot kernel keeps its populations in registers).
template <class S>
static __device__ __noinline__ void reseed_push_ip(typename S::T* __restrict__ f, const float* ref_p, const float* ref_ux,
                                                    const float* ref_uy, const float* ref_uz, float max_speed,
                                                    float fp16_scale, long long cell, int x, int y, int z, int nx,
                                                    int ny, int nz, int wrap_mask, int parity, float* u_last) {
    float rho, ux, uy, uz;
    reseed_state(ReseedSource{ref_p, ref_ux, ref_uy, ref_uz, cell}, max_speed, rho, ux, uy, uz);
    if (u_last) {
        const long long cells = (long long)nx * ny * nz;
        u_last[cell] = ux;
        u_last[cells + cell] = uy;
        u_last[2 * cells + cell] = uz;
    }
    const PadGeom g = make_pad_geom(nx, ny, nz, wrap_mask);
    const NeighbourOffsets o = neighbour_offsets(g, x, y, z);
    const int own = pad_index(g, x, y, z);
    const Fp16Scale sc{fp16_scale, 1.0f / fp16_scale};
#pragma unroll 1
    for (int q = 0; q < 27; ++q) {
        int c, d;
        outgoing_slot(o, own, q, parity, c, d);
        S::store(f + (long long)d * g.pcells + c, q, feq27(q, rho, ux, uy, uz), sc);
    }
}

template <class S>
__device__ __forceinline__ void reseed_push(typename S::T* f, const IpArgs& a, long long cell, int x, int y, int z,
                                            int parity) {
    const int wrap_mask = a.g.wrap[0] | (a.g.wrap[1] << 1) | (a.g.wrap[2] << 2);
    reseed_push_ip<S>(f, a.cur.ref_p, a.cur.ref_ux, a.cur.ref_uy, a.cur.ref_uz, a.cp.max_speed, a.sc.scale, cell, x, y,
                      z, a.g.nx, a.g.ny, a.g.nz, wrap_mask, parity, a.cur.u_last);
}

// Velocities a two-cell step leaves for the temperature transport: the
// collision's on collided lanes, 0 on lanes that are solid now or were at
// the streaming call (a reseeded lane records its own in reseed_push; a
// cell that opened up is recorded by the transition kernel).
__device__ __forceinline__ void record_u2(const CellFields& c, long long cell0, bool has1, bool col0, bool col1,
                                          bool reseed0, bool reseed1, const F2 (&u)[3]) {
    if (!c.u_last) return;
    if (!reseed0) record_u(c, cell0, col0 ? u[0].v.x : 0.0f, col0 ? u[1].v.x : 0.0f, col0 ? u[2].v.x : 0.0f);
    if (has1 && !reseed1)
        record_u(c, cell0 + 1, col1 ? u[0].v.y : 0.0f, col1 ? u[1].v.y : 0.0f, col1 ? u[2].v.y : 0.0f);
}

// Fused pull-stream + collide + push of one step. Sources outside
// equilibrium faces were pre-filled into their slots by face_fill_ip_kernel,
// so every incoming population is a plain (or bounce-back) slot read.
// Launch geometry of the step: one block row per (x, y) line, z along the
// block (grid = (ceil(nz / block), ny, nx)), so the cell coordinates need no
// division.
__device__ __forceinline__ bool line_cell(const PadGeom& G, int& x, int& y, int& z, long long& cell) {
    z = blockIdx.x * blockDim.x + threadIdx.x;
    y = blockIdx.y;
    x = blockIdx.z;
    cell = ((long long)x * G.ny + y) * G.nz + z;
    return z < G.nz;
}

inline dim3 line_grid(const PadGeom& g, int block, int cells_per_thread = 1) {
    const int n = (g.nz + cells_per_thread - 1) / cells_per_thread;
    return dim3((unsigned)((n + block - 1) / block), (unsigned)g.ny, (unsigned)g.nx);
}

// Threads per block of the line launch: a multiple of 32 covering n, at most 128.
inline int line_block(int n) { return n >= 128 ? 128 : ((n + 31) / 32) * 32; }

// Shared memory of the fused temperature transport for a block covering
// `span` cells of a line: nine staged rows of span + 2 values and codes.
inline size_t fused_smem_bytes(int span) { return (size_t)9 * (span + 2) * (sizeof(float) + 1); }

template <int kCells>
__device__ __forceinline__ void fused_transport(const IpArgs& a, int x, int y, int z_begin, int span,
                                                const int (&zs)[kCells], float (&tn)[kCells]) {
    extern __shared__ float fused_sv[];
    const int W = span + 2;
    thermal_fused::update_cells<kCells>(a.tr, a.obstacle_cur, a.g.nx, a.g.ny, a.g.nz, x, y, z_begin, span, zs, tn,
                                        fused_sv, reinterpret_cast<unsigned char*>(fused_sv + 9 * W));
}

template <class S, bool kExact, int kParity, bool kTransport>
__global__ void __launch_bounds__(128) step_ip_kernel(typename S::T* __restrict__ f, IpArgs a) {
    const PadGeom G = a.g;
    int x, y, z;
    long long cell;
    const bool in_line = line_cell(G, x, y, z, cell);
    float tn[1] = {0.0f};
    if (kTransport) {
        const int z_begin = blockIdx.x * blockDim.x;
        const int zs[1] = {z};
        fused_transport<1>(a, x, y, z_begin, min((int)blockDim.x, G.nz - z_begin), zs, tn);
    }
    if (!in_line) return;
    const uint32_t w = a.flags_prev[cell];
    if (w & kFlagSelfSolid) {  // memory of a solid cell is link storage; transitions run separately
        record_u(a.cur, cell, 0.0f, 0.0f, 0.0f);
        return;
    }
    const int own = pad_index(G, x, y, z);
    const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
    float fl[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        int c, d;
        incoming_slot(o, own, q, kParity, (w >> q) & 1u, c, d);
        fl[q] = S::load(f + (d * G.pcells + c), q, a.sc);
    }
    if (a.obstacle_cur[cell]) record_u(a.cur, cell, 0.0f, 0.0f, 0.0f);
    if (!a.obstacle_cur[cell] && !collide_cell<kExact>(fl, a.cp, a.cur, a.force, cell, x, y, z, kTransport ? tn : nullptr)) {
        reseed_push<S>(f, a, cell, x, y, z, kParity);
        return;
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        int c, d;
        outgoing_slot(o, own, q, kParity, c, d);
        S::store(f + (d * G.pcells + c), q, fl[q], a.sc);
    }
}

// Loads and stores of two cells' populations of one direction: at two
// addresses, or (load2 / store2) as one aligned 2-element vector at p (the
// first cell's slot; the second cell's is the next element).
template <class S>
struct PairIO;
template <>
struct PairIO<StoreF32> {
    __device__ __forceinline__ static F2 load(const float* p0, const float* p1, int, const Fp16Scale&) {
        return f2(__ldg(p0), __ldg(p1));
    }
    __device__ __forceinline__ static F2 load2(const float* p, int, const Fp16Scale&) {
        return F2{__ldg(reinterpret_cast<const float2*>(p))};
    }
    __device__ __forceinline__ static F2 load2p(const float* p, const float* p1, bool fix, int, const Fp16Scale&) {
        float2 r = __ldg(reinterpret_cast<const float2*>(p));
        if (fix) r.y = __ldg(p1);
        return F2{r};
    }
    __device__ __forceinline__ static void store(float* p0, float* p1, bool s0, bool s1, int, F2 v, const Fp16Scale&) {
        if (s0) *p0 = v.v.x;
        if (s1) *p1 = v.v.y;
    }
    __device__ __forceinline__ static void store2(float* p, int, F2 v, const Fp16Scale&) {
        *reinterpret_cast<float2*>(p) = v.v;
    }
};
template <>
struct PairIO<StoreF16Dev> {
    __device__ __forceinline__ static F2 decode(float2 h, int q, const Fp16Scale& s) {
        const float w = q_w(q), k = w * s.inv_scale;
        return F2{__ffma2_rn(h, make_float2(k, k), make_float2(w, w))};
    }
    __device__ __forceinline__ static float2 encode(F2 v, int q, const Fp16Scale& s) {
        const float k = s.scale * (1.0f / q_w(q));
        return __ffma2_rn(v.v, make_float2(k, k), make_float2(-s.scale, -s.scale));
    }
    __device__ __forceinline__ static F2 load(const __half* p0, const __half* p1, int q, const Fp16Scale& s) {
        return decode(make_float2(__half2float(__ldg(p0)), __half2float(__ldg(p1))), q, s);
    }
    __device__ __forceinline__ static F2 load2(const __half* p, int q, const Fp16Scale& s) {
        return decode(__half22float2(__ldg(reinterpret_cast<const __half2*>(p))), q, s);
    }
    __device__ __forceinline__ static F2 load2p(const __half* p, const __half* p1, bool fix, int q, const Fp16Scale& s) {
        const __half2 r = __ldg(reinterpret_cast<const __half2*>(p));
        __half y = __high2half(r);
        if (fix) y = __ldg(p1);
        return decode(make_float2(__low2float(r), __half2float(y)), q, s);
    }
    __device__ __forceinline__ static void store(__half* p0, __half* p1, bool s0, bool s1, int q, F2 v, const Fp16Scale& s) {
        const float2 h = encode(v, q, s);
        if (s0) *p0 = __float2half_rn(h.x);
        if (s1) *p1 = __float2half_rn(h.y);
    }
    __device__ __forceinline__ static void store2(__half* p, int q, F2 v, const Fp16Scale& s) {
        const float2 h = encode(v, q, s);
        *reinterpret_cast<__half2*>(p) = __floats2half2_rn(h.x, h.y);
    }
};

template <>
struct PairIO<StoreI16Dev> {
    __device__ __forceinline__ static F2 decode(float2 h, int q, const Fp16Scale& s) {
        const float w = q_w(q), k = w * s.inv_scale;
        return F2{__ffma2_rn(h, make_float2(k, k), make_float2(w, w))};
    }
    __device__ __forceinline__ static float2 encode(F2 v, int q, const Fp16Scale& s) {
        const float k = s.scale * (1.0f / q_w(q));
        return __ffma2_rn(v.v, make_float2(k, k), make_float2(-s.scale, -s.scale));
    }
    __device__ __forceinline__ static F2 load(const short* p0, const short* p1, int q, const Fp16Scale& s) {
        const unsigned r = (unsigned)(unsigned short)__ldg(p0) | ((unsigned)(unsigned short)__ldg(p1) << 16);
        return decode(s16x2_to_float2(r), q, s);
    }
    __device__ __forceinline__ static F2 load2(const short* p, int q, const Fp16Scale& s) {
        return decode(s16x2_to_float2(__ldg(reinterpret_cast<const unsigned*>(p))), q, s);
    }
    __device__ __forceinline__ static F2 load2p(const short* p, const short* p1, bool fix, int q, const Fp16Scale& s) {
        unsigned r = __ldg(reinterpret_cast<const unsigned*>(p));
        if (fix) r = (r & 0xFFFFu) | ((unsigned)(unsigned short)__ldg(p1) << 16);
        return decode(s16x2_to_float2(r), q, s);
    }
    __device__ __forceinline__ static void store(short* p0, short* p1, bool s0, bool s1, int q, F2 v, const Fp16Scale& s) {
        const float2 h = encode(v, q, s);
        if (s0) *p0 = sat_round_s16(h.x);
        if (s1) *p1 = sat_round_s16(h.y);
    }
    __device__ __forceinline__ static void store2(short* p, int q, F2 v, const Fp16Scale& s) {
        const float2 h = encode(v, q, s);
        *reinterpret_cast<short2*>(p) = make_short2(sat_round_s16(h.x), sat_round_s16(h.y));
    }
};

// Whether the slot pair of direction q at a launch-uniform offset from an
// even padded index is 2-element aligned (slot planes are pcells apart, an
// even count): incoming slots sit in the cell's own memory (positive q and
// the rest slot) or in the memory of the cell at -c_q, whose padded offset is
// odd exactly when c_z != 0 (a bounce-back read takes the other slot of the
// same memory cell, so the same rule holds); outgoing slots sit in the own
// memory (negative q and rest) or at +c_q.
// AERO_PAIR_VECTOR_LOADS / _STORES select the vector form per build. Measured
// on the 128^3 terrain brick (B200): vector stores shorten the step, vector
// loads lengthen it (more load latency exposed: 136 us against 104 us for the
// 16-bit step), so loads stay scalar by default.
#ifndef AERO_PAIR_VECTOR_LOADS
#define AERO_PAIR_VECTOR_LOADS 0
#endif
#ifndef AERO_PAIR_VECTOR_STORES
#define AERO_PAIR_VECTOR_STORES 1
#endif
__host__ __device__ constexpr bool in_pair_aligned(int q) {
    return AERO_PAIR_VECTOR_LOADS && (q == kRest27 || q_positive(q) || q_cz(q) == 0);
}
__host__ __device__ constexpr bool out_pair_aligned(int q) {
    return AERO_PAIR_VECTOR_STORES && (q == kRest27 || !q_positive(q) || q_cz(q) == 0);
}

// Step with two z-adjacent cells per thread and the collision in packed FP32:
// the factorised collision (collide27_x2.cuh), or with kExact the
// reference-order one (collide27_exact_x2.cuh, bit-identical per lane to the
// one-cell kernel); line grid over cell pairs.
// Pairs without periodic wraps address every slot at a launch-uniform offset
// (one of two per direction, by the bounce-back bit; the second cell's slots
// one element after the first's).
// A cell that is fluid at the streaming call and solid now is not collided:
// its streamed populations pass through (reloaded from its incoming slots,
// which only this cell writes, before any store). A lane whose input is not
// finite is reseeded.
#ifndef AERO_IP2_MIN_BLOCKS
#define AERO_IP2_MIN_BLOCKS 5
#endif
#ifndef AERO_IP2X_MIN_BLOCKS
#define AERO_IP2X_MIN_BLOCKS 4
#endif
template <class S, bool kExact, int kParity, bool kTransport>
__global__ void __launch_bounds__(128, kExact ? AERO_IP2X_MIN_BLOCKS : AERO_IP2_MIN_BLOCKS) step_ip2_kernel(typename S::T* __restrict__ f, IpArgs a) {
    // launched after the transport (and the face pre-fill) with launch_pdl
    pdl_trigger();
    pdl_wait();
    const PadGeom& G = a.g;
    const int z0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int y = blockIdx.y, x = blockIdx.z;
    float tn[2] = {0.0f, 0.0f};
    if (kTransport) {
        const int z_begin = 2 * blockIdx.x * blockDim.x;
        const int zs[2] = {z0, z0 + 1};
        fused_transport<2>(a, x, y, z_begin, min(2 * (int)blockDim.x, G.nz - z_begin), zs, tn);
    }
    if (z0 >= G.nz) return;
    const long long cell0 = ((long long)x * G.ny + y) * G.nz + z0;
    const bool has1 = z0 + 1 < G.nz;
    const uint32_t w0 = a.flags_prev[cell0];
    const uint32_t w1 = has1 ? a.flags_prev[cell0 + 1] : kFlagSelfSolid;
    const bool live0 = !(w0 & kFlagSelfSolid), live1 = !(w1 & kFlagSelfSolid);
    if (!live0 && !live1) {
        if (a.cur.u_last) {
            record_u(a.cur, cell0, 0.0f, 0.0f, 0.0f);
            if (has1) record_u(a.cur, cell0 + 1, 0.0f, 0.0f, 0.0f);
        }
        return;
    }
    const bool pass0 = live0 && a.obstacle_cur[cell0] != 0;
    const bool pass1 = live1 && a.obstacle_cur[cell0 + 1] != 0;
    const int own0 = pad_index(G, x, y, z0);
    const int own1 = own0 + 1;  // z0 + 1 (the ghost cell when z0 + 1 == nz: inside the padded array)
    const bool flat = no_wrap(G, x, y, z0) && (!has1 || no_wrap(G, x, y, z0 + 1));
    typename S::T* __restrict__ base0 = f + own0;
    F2 fl[27];
    if (flat) {
        // own0 is even (even z0, even row starts): with vector loads built in,
        // an aligned direction reads both cells' slots as one vector at the
        // first cell's offset; when the bounce-back bits differ the second
        // lane is replaced by a scalar load from its own slot (a predicated
        // load, no branch)
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            const bool b0 = (w0 >> q) & 1u, b1 = (w1 >> q) & 1u;
            const int o0 = b0 ? a.off_in[q][1] : a.off_in[q][0];
            const int o1 = b1 ? a.off_in[q][1] : a.off_in[q][0];
            if (in_pair_aligned(q)) fl[q] = PairIO<S>::load2p(base0 + o0, base0 + 1 + o1, b0 != b1, q, a.sc);
            else fl[q] = PairIO<S>::load(base0 + o0, base0 + 1 + o1, q, a.sc);
        }
    } else {
        const NeighbourOffsets o0 = neighbour_offsets(G, x, y, z0);
        const NeighbourOffsets o1 = neighbour_offsets(G, x, y, has1 ? z0 + 1 : z0);
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            int c0, d0, c1, d1;
            incoming_slot(o0, own0, q, kParity, (w0 >> q) & 1u, c0, d0);
            incoming_slot(o1, own1, q, kParity, (w1 >> q) & 1u, c1, d1);
            fl[q] = PairIO<S>::load(f + (d0 * G.pcells + c0), f + (d1 * G.pcells + c1), q, a.sc);
        }
    }
    const float* temp = a.cur.temperature;
    const F2 t = !a.cp.enable_buoyancy ? f2(0.0f)
                 : kTransport          ? f2(tn[0], tn[1])
                                       : f2(temp[cell0], has1 ? temp[cell0 + 1] : 0.0f);
    F2 cfx = f2(0.0f), cfy = f2(0.0f), cfz = f2(0.0f);
    if (a.force.fx) {
        cfx = f2(a.force.fx[cell0], has1 ? a.force.fx[cell0 + 1] : 0.0f);
        cfy = f2(a.force.fy[cell0], has1 ? a.force.fy[cell0 + 1] : 0.0f);
        cfz = f2(a.force.fz[cell0], has1 ? a.force.fz[cell0 + 1] : 0.0f);
    }
    bool ok[2];
    F2 uc[3];
    if (kExact) exact::collide27_exact_x2(fl, a.cp, t, cfx, cfy, cfz, ok, uc);
    else collide27_x2(fl, a.cp, t, cfx, cfy, cfz, ok, uc);
    record_u2(a.cur, cell0, has1, live0 && !pass0 && ok[0], live1 && !pass1 && ok[1], live0 && !ok[0] && !pass0,
              live1 && !ok[1] && !pass1, uc);
    if (pass0 || pass1) {
        const NeighbourOffsets o0 = neighbour_offsets(G, x, y, z0);
        const NeighbourOffsets o1 = neighbour_offsets(G, x, y, has1 ? z0 + 1 : z0);
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            int c, d;
            if (pass0) {
                incoming_slot(o0, own0, q, kParity, (w0 >> q) & 1u, c, d);
                fl[q].v.x = S::load(f + (d * G.pcells + c), q, a.sc);
            }
            if (pass1) {
                incoming_slot(o1, own1, q, kParity, (w1 >> q) & 1u, c, d);
                fl[q].v.y = S::load(f + (d * G.pcells + c), q, a.sc);
            }
        }
    }
    const bool st0 = live0 && (ok[0] || pass0), st1 = live1 && (ok[1] || pass1);
    if (live0 && !ok[0] && !pass0) reseed_push<S>(f, a, cell0, x, y, z0, kParity);
    if (live1 && !ok[1] && !pass1) reseed_push<S>(f, a, cell0 + 1, x, y, z0 + 1, kParity);
    if (flat) {
        if (st0 && st1) {
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                const int off = a.off_out[q];
                if (out_pair_aligned(q)) PairIO<S>::store2(base0 + off, q, fl[q], a.sc);
                else PairIO<S>::store(base0 + off, base0 + off + 1, true, true, q, fl[q], a.sc);
            }
        } else {
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                const int off = a.off_out[q];
                PairIO<S>::store(base0 + off, base0 + off + 1, st0, st1, q, fl[q], a.sc);
            }
        }
        return;
    }
    const NeighbourOffsets o0 = neighbour_offsets(G, x, y, z0);
    const NeighbourOffsets o1 = neighbour_offsets(G, x, y, has1 ? z0 + 1 : z0);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        int c0, d0, c1, d1;
        outgoing_slot(o0, own0, q, kParity, c0, d0);
        outgoing_slot(o1, own1, q, kParity, c1, d1);
        PairIO<S>::store(f + (d0 * G.pcells + c0), f + (d1 * G.pcells + c1), st0, st1, q, fl[q], a.sc);
    }
}

// Source of incoming population q of boundary cell (x, y, z) whose pull
// source (sx, sy, sz) lies outside a face that is neither periodic nor
// bounce-back, for the step of parity p (benchmark_hydrodynamic_boundary_value,
// jni.cpp:1494-1602). Equilibrium faces need only the face's state. Symmetry
// copies the post-collision population q of the clamped source cell;
// convective outflow extrapolates it from the two cells inward along the
// face normal, f1 + 0.15 (f1 - f2) (f1 alone when the second cell is solid);
// a solid source cell (f1's) gives the half-way bounce-back value. The
// post-collision populations are those the last step left: when the fill
// runs they still sit in their outgoing slots of parity p ^ 1, and the
// bounce-back value in the cell's flipped slot of parity p. Products and sums
// round separately (the reference's order).
template <class S>
__device__ __forceinline__ float ip_face_source(const typename S::T* __restrict__ f, const IpArgs& a, const PadGeom& G,
                                                const NeighbourOffsets& o, int own, long long cell, int x, int y, int z,
                                                int q, int sx, int sy, int sz, int p) {
    const FaceParams& F = *a.face_prev;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const int face = oob_face(sx, sy, sz, nx, ny, nz);
    const int kind = F.kind[face];
    if (kind == kHydroVelocity || kind == kHydroPressure || kind == kHydroMovingWall)
        return ip_face_equilibrium(F, q, a.ref_p_prev[cell], y, sx, sy, sz, nx, ny, nz);
    int c, d;
    incoming_slot(o, own, q, p, true, c, d);
    const float bounced = S::load(f + (long long)d * G.pcells + c, q, a.sc);
    // post-collision population q of cell (ix, iy, iz) after the last step:
    // outgoing_slot at parity p ^ 1 (the cell's own memory, or for positive q
    // the memory of its neighbour at +c_q), without the full offset table
    auto post = [&](int ix, int iy, int iz) {
        const int pd = q == kRest27 ? kRest27 : ((p ^ 1) == 0 ? q : q_opp(q));
        int pc;
        if (q != kRest27 && q_positive(q))
            pc = pad_index(G, axis_neighbour(ix, q_cx(q), nx, G.wrap[0]), axis_neighbour(iy, q_cy(q), ny, G.wrap[1]),
                           axis_neighbour(iz, q_cz(q), nz, G.wrap[2]));
        else
            pc = pad_index(G, ix, iy, iz);
        return S::load(f + (long long)pd * G.pcells + pc, q, a.sc);
    };
    auto solid = [&](int ix, int iy, int iz) { return a.obstacle_cur[((long long)ix * ny + iy) * nz + iz] != 0; };
    // the mask bytes and the populations are loaded before any test (all
    // inside the brick), so the loads of a cell's directions are in flight
    // together instead of one dependent round trip after another
    if (kind == kHydroSymmetry) {
        const int ix = min(max(sx, 0), nx - 1), iy = min(max(sy, 0), ny - 1), iz = min(max(sz, 0), nz - 1);
        const bool si = solid(ix, iy, iz);
        const float fi = post(ix, iy, iz);
        return si ? bounced : fi;
    }
    if (kind == kHydroInheritGame && F.disable_convective) return bounced;
    const int dx = (sx < 0 || sx >= nx) ? q_cx(q) : 0;
    const int dy = (sy < 0 || sy >= ny) ? q_cy(q) : 0;
    const int dz = (sz < 0 || sz >= nz) ? q_cz(q) : 0;
    const int x1 = min(max(x + dx, 0), nx - 1), y1 = min(max(y + dy, 0), ny - 1), z1 = min(max(z + dz, 0), nz - 1);
    const int x2 = min(max(x + 2 * dx, 0), nx - 1), y2 = min(max(y + 2 * dy, 0), ny - 1), z2 = min(max(z + 2 * dz, 0), nz - 1);
    const bool s1 = solid(x1, y1, z1), s2 = solid(x2, y2, z2);
    const float f1 = post(x1, y1, z1), f2 = post(x2, y2, z2);
    if (s1) return bounced;
    if (s2) return f1;
    return __fadd_rn(f1, __fmul_rn(0.15f, __fsub_rn(f1, f2)));
}

// Before a step of parity p: write the source of every incoming population
// whose pull source lies outside a face that is neither periodic nor
// bounce-back (ip_face_source) into the slot the pulling cell reads at parity
// p (a ghost-cell slot, or for positive directions the cell's own slot that
// only the never-updated ghost would write). These slots are written by no
// step and read by no other fill thread, so the fill runs right after the
// step that produced the post-collision populations it reads. One thread per
// link: a cell of one of the six boundary layers and one of the nine
// directions that pull across that face (c along the face's axis pointing
// into the brick), consecutive threads along the face's cells, so that each
// thread makes one round of independent loads. A link that crosses two or
// three faces (edge and corner cells) is visited once per face; every visit
// writes the same value.
// face_fill_count: threads of the fill.
__host__ __device__ __forceinline__ unsigned fill_face_set(unsigned fill_faces) { return fill_faces ? fill_faces & 0x3Fu : 0x3Fu; }
__host__ __device__ __forceinline__ long long face_area(const PadGeom& g, int face) {
    const int axis = face >> 1;
    return axis == 0 ? (long long)g.ny * g.nz : (axis == 1 ? (long long)g.nx * g.nz : (long long)g.nx * g.ny);
}
inline long long face_fill_count(const PadGeom& g, unsigned fill_faces) {
    long long n = 0;
    for (int f = 0; f < 6; ++f)
        if ((fill_face_set(fill_faces) >> f) & 1u) n += 9 * face_area(g, f);
    return n;
}

template <class S>
__device__ __forceinline__ void face_fill_cell(typename S::T* __restrict__ f, const IpArgs& a, unsigned i) {
    const PadGeom& G = a.g;
    const int nx = G.nx, ny = G.ny, nz = G.nz;
    const unsigned set = fill_face_set(a.fill_faces);
    // the face of thread i (launch-uniform set; 32-bit indices: 9 x the
    // boundary layers of a brick stay far below 2^32)
    int face = -1;
    unsigned area = 0;
#pragma unroll
    for (int fc = 0; fc < 6; ++fc) {
        if (face >= 0 || !((set >> fc) & 1u)) continue;
        const unsigned n = (unsigned)face_area(G, fc);
        if (i < 9 * n) {
            face = fc;
            area = n;
        } else {
            i -= 9 * n;
        }
    }
    if (face < 0) return;
    // slot s of the nine inward directions: the two other axes' components
    // (s / 3 - 1, s % 3 - 1) in (x, y, z) order; consecutive threads along the
    // face's cells
    const unsigned s = i / area, r = i - s * area;
    const bool hi = face & 1;
    const int in = hi ? 0 : 2;  // component + 1 along the face's axis, pointing into the brick
    int x, y, z, q;
    if (face < 2) {
        x = hi ? nx - 1 : 0;
        y = (int)(r / (unsigned)nz);
        z = (int)(r - (unsigned)y * nz);
        q = in * 9 + (int)s;
    } else if (face < 4) {
        y = hi ? ny - 1 : 0;
        x = (int)(r / (unsigned)nz);
        z = (int)(r - (unsigned)x * nz);
        q = (int)(s / 3) * 9 + in * 3 + (int)(s % 3);
    } else {
        z = hi ? nz - 1 : 0;
        x = (int)(r / (unsigned)ny);
        y = (int)(r - (unsigned)x * ny);
        q = (int)(s / 3) * 9 + (int)(s % 3) * 3 + in;
    }
    const long long cell = ((long long)x * ny + y) * nz + z;
    const uint32_t w = a.flags_prev[cell];
    if ((w & kFlagSelfSolid) || !(w & kFlagFaceSpecial) || ((w >> q) & 1u)) return;
    const int sx = axis_neighbour(x, -q_cx(q), nx, G.wrap[0]);
    const int sy = axis_neighbour(y, -q_cy(q), ny, G.wrap[1]);
    const int sz = axis_neighbour(z, -q_cz(q), nz, G.wrap[2]);
    if (sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz) return;
    const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
    const int own = pad_index(G, x, y, z);
    const float v = ip_face_source<S>(f, a, G, o, own, cell, x, y, z, q, sx, sy, sz, a.parity);
    int c, d;
    incoming_slot(o, own, q, a.parity, false, c, d);
    S::store(f + (long long)d * G.pcells + c, q, v, a.sc);
}

template <class S>
__global__ void face_fill_ip_kernel(typename S::T* __restrict__ f, IpArgs a) {
    face_fill_cell<S>(f, a, blockIdx.x * blockDim.x + threadIdx.x);
}

// Cells that were solid at the streaming call and are fluid now: start from
// the populations the cell held while solid (a.solid_f; the rest
// equilibrium for a cell solid since initialisation), collide and push. Cells
// that turn solid in this call keep their streamed populations in a.solid_f:
// the step kernel pushed them uncollided, so they sit in the cell's outgoing
// slots. Runs after step_ip_kernel of the same parity; the slots it writes
// were only read (as bounce-back) by that launch.
template <class S, bool kExact>
__global__ void __launch_bounds__(128) transition_ip_kernel(typename S::T* __restrict__ f, IpArgs a) {
    const PadGeom G = a.g;
    const long long cells = (long long)G.nx * G.ny * G.nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    const bool was_solid = (a.flags_prev[cell] & kFlagSelfSolid) != 0, solid = a.obstacle_cur[cell] != 0;
    if (was_solid == solid) return;
    int x, y, z;
    cell_coords(G, cell, x, y, z);
    const int own = pad_index(G, x, y, z);
    const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
    if (solid) {
        if (!a.solid_f) return;
#pragma unroll 1
        for (int q = 0; q < 27; ++q) {
            int c, d;
            outgoing_slot(o, own, q, a.parity, c, d);
            a.solid_f[(long long)solid_slot(q, a.parity) * cells + cell] = S::load(f + (long long)d * G.pcells + c, q, a.sc);
        }
        return;
    }
    float fl[27];
#pragma unroll
    for (int q = 0; q < 27; ++q)
        fl[q] = a.solid_f ? a.solid_f[(long long)solid_slot(q, a.parity) * cells + cell] : q_w(q);
    if (!collide_cell<kExact>(fl, a.cp, a.cur, a.force, cell, x, y, z)) {
        reseed_push<S>(f, a, cell, x, y, z, a.parity);
        return;
    }
    ip_push<S>(f, a, G, o, own, a.parity, fl);
}

// First call: populations from the reference state (initialize_distributions,
// jni.cpp:1752-1781), collide, push with parity 0. Solid cells hold nothing.
template <class S, bool kExact>
__global__ void __launch_bounds__(128) init_ip_kernel(typename S::T* __restrict__ f, IpArgs a) {
    const PadGeom G = a.g;
    const long long cells = (long long)G.nx * G.ny * G.nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    if (a.cur.obstacle[cell]) {
        record_u(a.cur, cell, 0.0f, 0.0f, 0.0f);
        return;
    }
    int x, y, z;
    cell_coords(G, cell, x, y, z);
    const int own = pad_index(G, x, y, z);
    const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
    const float rho = clampf_dev(1.0f + a.cur.ref_p[cell], 0.97f, 1.03f);
    const float ux = a.cur.ref_ux[cell], uy = a.cur.ref_uy[cell], uz = a.cur.ref_uz[cell];
    float fl[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) fl[q] = feq27(q, rho, ux, uy, uz);
    if (!collide_cell<kExact>(fl, a.cp, a.cur, a.force, cell, x, y, z)) {
        reseed_push<S>(f, a, cell, x, y, z, 0);
        return;
    }
    ip_push<S>(f, a, G, o, own, 0, fl);
}

// Macro output of the streamed state (what the next step would pull), with
// write_output / strided-extract semantics. Read-only.
template <class S, bool kExact>
__global__ void output_ip_kernel(const typename S::T* __restrict__ f, IpArgs a, OutBox b, int out_ch, float scale,
                                 float* __restrict__ out) {
    const PadGeom G = a.g;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.count()) return;
    const int az = (int)(i % b.sz);
    const int ay = (int)((i / b.sz) % b.sy);
    const int ax = (int)(i / ((long long)b.sy * b.sz));
    const int x = min(G.nx - 1, b.ox + ax * b.stride), y = min(G.ny - 1, b.oy + ay * b.stride),
              z = min(G.nz - 1, b.oz + az * b.stride);
    const long long cell = ((long long)x * G.ny + y) * G.nz + z;
    const uint32_t w = a.flags_prev[cell];
    float o4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (!(w & kFlagSelfSolid)) {
        const int own = pad_index(G, x, y, z);
        const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
        float fl[27];
        ip_pull<S>(f, a, G, o, own, w, a.parity, fl);
        if (kExact) exact::macro_out_exact(fl, false, scale, o4);
        else macro_out(fl, false, scale, o4);
    }
    float* dst = out + i * out_ch;
    dst[0] = o4[0]; dst[1] = o4[1]; dst[2] = o4[2]; dst[3] = o4[3];
    for (int c = 4; c < out_ch; ++c) dst[c] = 0.0f;
}

}  // namespace aero
