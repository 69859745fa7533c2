// Batched brick engine: many independent bricks of uneven sizes, each with
// its own mask, relaxation time, body force and storage precision (FP32 or
// FP16 deviation), advanced by ONE persistent launch per tick over a work list
// of (brick, tile) units, followed by a stride-s velocity publish that writes
// the reference's packed int16 atlas for every brick
// (aero_lbm_simulation_copy_brick_world_packed_flow_atlas,
// native/src/aero_lbm_simulation_bridge.cpp:5301-5410, quantize_signed 3122-3128).
//
// The reference steps bricks one after another from the host, one
// aero_lbm_step_rect call each (sim.cpp:1092-1166). Here all bricks share one
// in-place (esoteric pull) update with a global parity; the tick (step +
// publish) can be captured once as a CUDA graph (two ticks per graph, one of
// each parity) and replayed, and the launch shape (threads per tile, resident
// tiles) is chosen by timing candidates on the live bricks.
//
// Faces: each brick's faces are periodic or bounce-back (the local kinds that
// need no per-step boundary fill).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/aero_lbm_b200.h"
#include "d3q27_inplace.cuh"
#include "runtime_internal.h"

namespace aero {

struct BrickDesc {
    void* f;                  // padded in-place populations (float or __half)
    const uint32_t* flags;    // pull classification (mask + faces)
    const uint8_t* obstacle;
    const float* temperature; // unused (buoyancy off in batches); kept for the collision interface
    const float* ref;         // 4 x cells: ref_p, ux, uy, uz (reseed state)
    CollideParams cp;
    PadGeom g;
    Fp16Scale sc;
    int precision;            // 0 fp32, 1 fp16
    int unit_begin;           // first work unit of this brick
    int atlas_offset;         // first atlas record (4 x int16) of this brick
    int pairs;                // 1: two z-adjacent cells per thread (nz even), packed FP32 collision
};

namespace {

template <class S, int kParity>
__device__ __forceinline__ void batch_cell(const BrickDesc& b, int cell) {
    const PadGeom& G = b.g;
    typename S::T* f = static_cast<typename S::T*>(b.f);
    const uint32_t w = b.flags[cell];
    if (w & kFlagSelfSolid) return;
    int x, y, z;
    cell_coords(G, cell, x, y, z);
    const int own = pad_index(G, x, y, z);
    const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
    float fl[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        int c, d;
        incoming_slot(o, own, q, kParity, (w >> q) & 1u, c, d);
        fl[q] = S::load(f + (d * G.pcells + c), q, b.sc);
    }
    if (!b.obstacle[cell]) {
        CollideOut co;
        if (!collide27(fl, b.cp, b.temperature, 0.0f, 0.0f, 0.0f, co)) {
            const long long cells = (long long)G.nx * G.ny * G.nz;
            const int wrap_mask = G.wrap[0] | (G.wrap[1] << 1) | (G.wrap[2] << 2);
            reseed_push_ip<S>(f, b.ref, b.ref + cells, b.ref + 2 * cells, b.ref + 3 * cells, b.cp.max_speed,
                              b.sc.scale, cell, x, y, z, G.nx, G.ny, G.nz, wrap_mask, kParity, nullptr);
            return;
        }
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        int c, d;
        outgoing_slot(o, own, q, kParity, c, d);
        S::store(f + (d * G.pcells + c), q, fl[q], b.sc);
    }
}

// Two z-adjacent cells (cell0 even, nz even) with the collision in packed FP32
// (collide27_x2.cuh): the batch form of step_ip2_kernel. Cells without
// periodic wraps address their slots at offsets uniform over the brick.
template <class S, int kParity>
__device__ __forceinline__ void batch_pair(const BrickDesc& b, int cell0) {
    const PadGeom& G = b.g;
    typename S::T* f = static_cast<typename S::T*>(b.f);
    const uint32_t w0 = b.flags[cell0], w1 = b.flags[cell0 + 1];
    const bool live0 = !(w0 & kFlagSelfSolid), live1 = !(w1 & kFlagSelfSolid);
    if (!live0 && !live1) return;
    if ((live0 && b.obstacle[cell0]) || (live1 && b.obstacle[cell0 + 1])) {
        // fluid at streaming, solid now: the one-cell path passes it through
        batch_cell<S, kParity>(b, cell0);
        batch_cell<S, kParity>(b, cell0 + 1);
        return;
    }
    int x, y, z0;
    cell_coords(G, cell0, x, y, z0);
    const int own0 = pad_index(G, x, y, z0);
    const bool flat = no_wrap(G, x, y, z0) && no_wrap(G, x, y, z0 + 1);
    typename S::T* __restrict__ base0 = f + own0;
    F2 fl[27];
    if (flat) {
#pragma unroll
        for (int q = 0; q < 27; ++q)
            fl[q] = PairIO<S>::load(base0 + in_offset(G, q, kParity, (w0 >> q) & 1u),
                                    base0 + 1 + in_offset(G, q, kParity, (w1 >> q) & 1u), q, b.sc);
    } else {
        const NeighbourOffsets o0 = neighbour_offsets(G, x, y, z0);
        const NeighbourOffsets o1 = neighbour_offsets(G, x, y, z0 + 1);
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            int c0, d0, c1, d1;
            incoming_slot(o0, own0, q, kParity, (w0 >> q) & 1u, c0, d0);
            incoming_slot(o1, own0 + 1, q, kParity, (w1 >> q) & 1u, c1, d1);
            fl[q] = PairIO<S>::load(f + (d0 * G.pcells + c0), f + (d1 * G.pcells + c1), q, b.sc);
        }
    }
    bool ok[2];
    F2 uc[3];
    collide27_x2(fl, b.cp, f2(0.0f), f2(0.0f), f2(0.0f), f2(0.0f), ok, uc);
    const bool st0 = live0 && ok[0], st1 = live1 && ok[1];
    if (live0 && !ok[0] || live1 && !ok[1]) {
        const long long cells = (long long)G.nx * G.ny * G.nz;
        const int wrap_mask = G.wrap[0] | (G.wrap[1] << 1) | (G.wrap[2] << 2);
        for (int k = 0; k < 2; ++k)
            if ((k == 0 ? live0 && !ok[0] : live1 && !ok[1]))
                reseed_push_ip<S>(f, b.ref, b.ref + cells, b.ref + 2 * cells, b.ref + 3 * cells, b.cp.max_speed, b.sc.scale,
                                  cell0 + k, x, y, z0 + k, G.nx, G.ny, G.nz, wrap_mask, kParity, nullptr);
    }
    if (flat) {
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            const int off = out_offset(G, q, kParity);
            PairIO<S>::store(base0 + off, base0 + off + 1, st0, st1, q, fl[q], b.sc);
        }
        return;
    }
    const NeighbourOffsets o0 = neighbour_offsets(G, x, y, z0);
    const NeighbourOffsets o1 = neighbour_offsets(G, x, y, z0 + 1);
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        int c0, d0, c1, d1;
        outgoing_slot(o0, own0, q, kParity, c0, d0);
        outgoing_slot(o1, own0 + 1, q, kParity, c1, d1);
        PairIO<S>::store(f + (d0 * G.pcells + c0), f + (d1 * G.pcells + c1), st0, st1, q, fl[q], b.sc);
    }
}

// Cells per thread of a brick's work units.
__device__ __forceinline__ int unit_span(const BrickDesc& b) { return b.pairs ? 2 : 1; }

// Copy one brick descriptor into shared memory (one 32-bit word per thread).
__device__ __forceinline__ void stage_desc(BrickDesc& dst, const BrickDesc* src) {
    constexpr int kWords = (int)(sizeof(BrickDesc) / 4);
    static_assert(sizeof(BrickDesc) % 4 == 0, "descriptor must be word-sized");
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
    for (int i = threadIdx.x; i < kWords; i += blockDim.x) d[i] = s[i];
}

// One persistent launch per tick: each resident tile walks the work list with
// a fixed stride; a unit is `blockDim.x` consecutive cells of one brick, or
// `2 * blockDim.x` (two z-adjacent cells per thread) for bricks with even nz.
// The unit's brick descriptor is staged in shared memory, so its fields are
// read where they are used instead of occupying registers.
template <int kParity>
__global__ void batch_step_kernel(const BrickDesc* __restrict__ descs, const int* __restrict__ unit_brick, int units) {
    __shared__ BrickDesc sd;
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        __syncthreads();
        stage_desc(sd, descs + unit_brick[u]);
        __syncthreads();
        const int cells = sd.g.nx * sd.g.ny * sd.g.nz;
        const int span = unit_span(sd);
        const int cell = ((u - sd.unit_begin) * blockDim.x + threadIdx.x) * span;
        if (cell >= cells) continue;
        if (span == 2) {
            if (sd.precision == 1) batch_pair<StoreF16Dev, kParity>(sd, cell);
            else batch_pair<StoreF32, kParity>(sd, cell);
        } else {
            if (sd.precision == 1) batch_cell<StoreF16Dev, kParity>(sd, cell);
            else batch_cell<StoreF32, kParity>(sd, cell);
        }
    }
}

template <class S>
__device__ __forceinline__ void publish_cell(const BrickDesc& b, int x, int y, int z, int parity, float vscale,
                                             short* rec) {
    const PadGeom& G = b.g;
    const int cell = (x * G.ny + y) * G.nz + z;
    const uint32_t w = b.flags[cell];
    float o4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (!(w & kFlagSelfSolid)) {
        const typename S::T* f = static_cast<const typename S::T*>(b.f);
        const int own = pad_index(G, x, y, z);
        const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
        float fl[27];
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            int c, d;
            incoming_slot(o, own, q, parity, (w >> q) & 1u, c, d);
            fl[q] = S::load(f + (d * G.pcells + c), q, b.sc);
        }
        macro_out(fl, false, 1.0f, o4);
    }
    // quantize_signed: lround(clamp(v / range, -1, 1) * 32767)
    const float ranges[4] = {5.6f, 5.6f, 5.6f, 0.03f};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float v = k < 3 ? o4[k] * vscale : o4[k];
        short q = 0;
        if (isfinite(v)) q = (short)lroundf(fminf(1.0f, fmaxf(-1.0f, v / ranges[k])) * 32767.0f);
        rec[k] = q;
    }
}

// Stride-s publish of every brick: block b handles brick b's atlas records.
__global__ void batch_publish_kernel(const BrickDesc* __restrict__ descs, int parity, int stride, float vscale,
                                     short* __restrict__ atlas) {
    const BrickDesc& b = descs[blockIdx.x];
    const int sx = (b.g.nx + stride - 1) / stride, sy = (b.g.ny + stride - 1) / stride, sz = (b.g.nz + stride - 1) / stride;
    const int n = sx * sy * sz;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int az = i % sz, ay = (i / sz) % sy, ax = i / (sy * sz);
        const int x = min(b.g.nx - 1, ax * stride), y = min(b.g.ny - 1, ay * stride), z = min(b.g.nz - 1, az * stride);
        short* rec = atlas + 4LL * (b.atlas_offset + i);
        if (b.precision == 1) publish_cell<StoreF16Dev>(b, x, y, z, parity, vscale, rec);
        else publish_cell<StoreF32>(b, x, y, z, parity, vscale, rec);
    }
}

// First tick: populations from the reference state, collide, push parity 0.
__global__ void batch_init_kernel(const BrickDesc* __restrict__ descs, const int* __restrict__ unit_brick, int units) {
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        const BrickDesc& b = descs[unit_brick[u]];
        const int cells = b.g.nx * b.g.ny * b.g.nz;
        const int span = unit_span(b);
        for (int k = 0; k < span; ++k) {
        const int cell = ((u - b.unit_begin) * blockDim.x + threadIdx.x) * span + k;
        if (cell >= cells || b.obstacle[cell]) continue;
        const PadGeom& G = b.g;
        int x, y, z;
        cell_coords(G, cell, x, y, z);
        const int own = pad_index(G, x, y, z);
        const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
        const float rho = clampf_dev(1.0f + b.ref[cell], 0.97f, 1.03f);
        const float ux = b.ref[cells + cell], uy = b.ref[2 * cells + cell], uz = b.ref[3 * cells + cell];
        float fl[27];
#pragma unroll
        for (int q = 0; q < 27; ++q) fl[q] = feq27(q, rho, ux, uy, uz);
        CollideOut co;
        collide27(fl, b.cp, b.temperature, 0.0f, 0.0f, 0.0f, co);
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            int c, d;
            outgoing_slot(o, own, q, 0, c, d);
            if (b.precision == 1) StoreF16Dev::store(static_cast<__half*>(b.f) + (d * G.pcells + c), q, fl[q], b.sc);
            else StoreF32::store(static_cast<float*>(b.f) + (d * G.pcells + c), q, fl[q], b.sc);
        }
        }
    }
}

// Flow state (write_output semantics, scale 1) of one brick, for readback.
__global__ void batch_flow_kernel(const BrickDesc* __restrict__ descs, int brick, int parity, float* __restrict__ out) {
    const BrickDesc& b = descs[brick];
    const int cells = b.g.nx * b.g.ny * b.g.nz;
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    const PadGeom& G = b.g;
    int x, y, z;
    cell_coords(G, cell, x, y, z);
    const uint32_t w = b.flags[cell];
    float o4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (!(w & kFlagSelfSolid)) {
        const int own = pad_index(G, x, y, z);
        const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
        float fl[27];
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            int c, d;
            incoming_slot(o, own, q, parity, (w >> q) & 1u, c, d);
            fl[q] = b.precision == 1 ? StoreF16Dev::load(static_cast<const __half*>(b.f) + (d * G.pcells + c), q, b.sc)
                                     : StoreF32::load(static_cast<const float*>(b.f) + (d * G.pcells + c), q, b.sc);
        }
        macro_out(fl, false, 1.0f, o4);
    }
    out[4LL * cell + 0] = o4[0];
    out[4LL * cell + 1] = o4[1];
    out[4LL * cell + 2] = o4[2];
    out[4LL * cell + 3] = o4[3];
}

// ------------------------------------------------------------------ host side
struct HostBrick {
    int nx, ny, nz, precision;
    float fp16_scale = 1.0f;
    float tau, force[3];
    int faces[6];
    std::vector<uint8_t> obstacle;
    std::vector<float> ref;  // 4 x cells
    // device
    void* f = nullptr;
    uint32_t* flags = nullptr;
    uint8_t* d_obstacle = nullptr;
    float* d_ref = nullptr;
    float* d_temperature = nullptr;
    int atlas_cells = 0;
};

struct LaunchShape {
    int threads = 128;
    int blocks_per_sm = 8;
};

struct Batch {
    std::vector<HostBrick> bricks;
    BrickDesc* d_descs = nullptr;
    int* d_unit_brick = nullptr;
    int units = 0;
    short* d_atlas = nullptr;
    int atlas_records = 0;
    int stride = 4;
    float velocity_scale = 20.0f;  // dx/dt of the publish (m/s per lattice unit)
    bool finalized = false;
    bool initialized = false;
    int parity = 0;
    uint64_t ticks = 0;
    LaunchShape shape;
    bool tuned = false;
    bool use_graph = true;
    bool publish = true;
    cudaGraphExec_t graph = nullptr;
    LaunchShape graph_shape;
    bool graph_publish = false;
    cudaStream_t graph_stream = nullptr;
    int sms = 148;
    long long cells_total = 0;
    double bytes_per_tick = 0.0;

    ~Batch() { release(); }
    void release() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        for (auto& b : bricks) {
            if (b.f) cudaFree(b.f);
            if (b.flags) cudaFree(b.flags);
            if (b.d_obstacle) cudaFree(b.d_obstacle);
            if (b.d_ref) cudaFree(b.d_ref);
            if (b.d_temperature) cudaFree(b.d_temperature);
            b.f = nullptr; b.flags = nullptr; b.d_obstacle = nullptr; b.d_ref = nullptr; b.d_temperature = nullptr;
        }
        if (d_descs) cudaFree(d_descs);
        if (d_unit_brick) cudaFree(d_unit_brick);
        if (d_atlas) cudaFree(d_atlas);
        d_descs = nullptr; d_unit_brick = nullptr; d_atlas = nullptr;
    }
};

std::mutex g_batch_mutex;
std::unordered_map<long long, std::unique_ptr<Batch>> g_batches;
long long g_next_batch = 1;
std::string g_batch_error;

void berr(const std::string& m) { g_batch_error = m; }
bool bok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    berr(std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

Batch* lookup_batch(long long h) {
    auto it = g_batches.find(h);
    if (it == g_batches.end()) {
        berr("unknown batch handle");
        return nullptr;
    }
    return it->second.get();
}

constexpr float kMaxSpeedB = 0.57735026919f * 0.60f;

CollideParams brick_collide_params(const HostBrick& b) {
    CollideParams p{};
    const float nu = (b.tau - 0.5f) / 3.0f;
    p.tau_shear_base = b.tau;
    p.tau_normal_base = b.tau;
    p.nu0 = std::max(1e-6f, nu);
    p.sgs_c2 = 0.025f * 0.025f;
    p.sgs_nut_cap = 5.0f * p.nu0;
    p.sgs_bulk = 0.30f;
    p.buoy_beta = 0.0f;
    p.buoy_fmax = 0.02f;
    p.body_force[0] = b.force[0];
    p.body_force[1] = b.force[1];
    p.body_force[2] = b.force[2];
    p.max_speed = kMaxSpeedB;
    p.enable_sgs = 1;
    p.enable_buoyancy = 0;
    p.gravity_axis = 2;
    return p;
}

// Build the unit list for `threads`-cell units and upload descriptors.
bool build_units(Batch& B, int threads) {
    std::vector<BrickDesc> descs(B.bricks.size());
    std::vector<int> unit_brick;
    int atlas = 0;
    for (size_t i = 0; i < B.bricks.size(); ++i) {
        HostBrick& hb = B.bricks[i];
        BrickDesc d{};
        d.f = hb.f;
        d.flags = hb.flags;
        d.obstacle = hb.d_obstacle;
        d.temperature = hb.d_temperature;
        d.ref = hb.d_ref;
        d.cp = brick_collide_params(hb);
        int mask = 0;
        for (int a = 0; a < 3; ++a)
            if (hb.faces[2 * a] == kHydroPeriodic && hb.faces[2 * a + 1] == kHydroPeriodic) mask |= 1 << a;
        d.g = make_pad_geom(hb.nx, hb.ny, hb.nz, mask);
        d.precision = hb.precision;
        d.sc = Fp16Scale{hb.fp16_scale, 1.0f / hb.fp16_scale};
        d.unit_begin = (int)unit_brick.size();
        d.pairs = (hb.nz % 2 == 0) ? 1 : 0;
        const int cells = hb.nx * hb.ny * hb.nz;
        const int span = threads * (d.pairs ? 2 : 1);
        const int nunits = (cells + span - 1) / span;
        for (int u = 0; u < nunits; ++u) unit_brick.push_back((int)i);
        d.atlas_offset = atlas;
        atlas += hb.atlas_cells;
        descs[i] = d;
    }
    if (B.d_descs) cudaFree(B.d_descs);
    if (B.d_unit_brick) cudaFree(B.d_unit_brick);
    B.d_descs = nullptr;
    B.d_unit_brick = nullptr;
    if (!bok(cudaMalloc(&B.d_descs, descs.size() * sizeof(BrickDesc)), "cudaMalloc(descs)")) return false;
    if (!bok(cudaMalloc(&B.d_unit_brick, unit_brick.size() * sizeof(int)), "cudaMalloc(units)")) return false;
    if (!bok(cudaMemcpy(B.d_descs, descs.data(), descs.size() * sizeof(BrickDesc), cudaMemcpyHostToDevice), "upload descs")) return false;
    if (!bok(cudaMemcpy(B.d_unit_brick, unit_brick.data(), unit_brick.size() * sizeof(int), cudaMemcpyHostToDevice), "upload units")) return false;
    B.units = (int)unit_brick.size();
    B.atlas_records = atlas;
    B.shape.threads = threads;
    return true;
}

bool launch_tick(Batch& B, int parity, bool publish, const LaunchShape& sh, cudaStream_t s) {
    const int grid = std::max(1, std::min(B.units, sh.blocks_per_sm * B.sms));
    if (parity == 0) batch_step_kernel<0><<<grid, sh.threads, 0, s>>>(B.d_descs, B.d_unit_brick, B.units);
    else batch_step_kernel<1><<<grid, sh.threads, 0, s>>>(B.d_descs, B.d_unit_brick, B.units);
    count_launch();
    if (!bok(cudaGetLastError(), "batch_step_kernel")) return false;
    if (publish) {
        batch_publish_kernel<<<(int)B.bricks.size(), 256, 0, s>>>(B.d_descs, parity ^ 1, B.stride, B.velocity_scale, B.d_atlas);
        count_launch();
        if (!bok(cudaGetLastError(), "batch_publish_kernel")) return false;
    }
    return true;
}

bool ensure_graph(Batch& B, cudaStream_t s) {
    if (B.graph && B.graph_shape.threads == B.shape.threads && B.graph_shape.blocks_per_sm == B.shape.blocks_per_sm &&
        B.graph_publish == B.publish && B.graph_stream == s)
        return true;
    if (B.graph) cudaGraphExecDestroy(B.graph);
    B.graph = nullptr;
    cudaGraph_t g = nullptr;
    if (!bok(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture")) return false;
    const bool ok = launch_tick(B, 0, B.publish, B.shape, s) && launch_tick(B, 1, B.publish, B.shape, s);
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (!ok) {
        if (g) cudaGraphDestroy(g);
        return false;
    }
    if (!bok(e, "cudaStreamEndCapture")) return false;
    e = cudaGraphInstantiate(&B.graph, g, 0);
    cudaGraphDestroy(g);
    if (!bok(e, "cudaGraphInstantiate")) return false;
    B.graph_shape = B.shape;
    B.graph_publish = B.publish;
    B.graph_stream = s;
    return true;
}

bool run_ticks(Batch& B, int n, cudaStream_t s) {
    int left = n;
    if (!B.initialized && left > 0) {
        // The first tick collides the initial equilibrium (no streaming), like
        // the first aero_lbm_step_rect call of a context.
        const int grid = std::max(1, std::min(B.units, 8 * B.sms));
        batch_init_kernel<<<grid, B.shape.threads, 0, s>>>(B.d_descs, B.d_unit_brick, B.units);
        count_launch();
        if (!bok(cudaGetLastError(), "batch_init_kernel")) return false;
        if (B.publish) {
            batch_publish_kernel<<<(int)B.bricks.size(), 256, 0, s>>>(B.d_descs, 1, B.stride, B.velocity_scale, B.d_atlas);
            count_launch();
            if (!bok(cudaGetLastError(), "batch_publish_kernel")) return false;
        }
        B.initialized = true;
        B.parity = 1;
        --left;
        ++B.ticks;
    }
    // Graph replays cover pairs of ticks starting at parity 0.
    if (B.use_graph && left >= 2) {
        if (B.parity == 1) {
            if (!launch_tick(B, 1, B.publish, B.shape, s)) return false;
            B.parity = 0;
            --left;
            ++B.ticks;
        }
        if (left >= 2) {
            if (!ensure_graph(B, s)) return false;
            while (left >= 2) {
                if (!bok(cudaGraphLaunch(B.graph, s), "cudaGraphLaunch")) return false;
                left -= 2;
                B.ticks += 2;
                // counts the two kernels per tick inside the replay
                for (int k = 0; k < (B.publish ? 4 : 2); ++k) count_launch();
            }
        }
    }
    while (left > 0) {
        if (!launch_tick(B, B.parity, B.publish, B.shape, s)) return false;
        B.parity ^= 1;
        --left;
        ++B.ticks;
    }
    return true;
}

}  // namespace
}  // namespace aero

using namespace aero;

extern "C" {

AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_create(long long* out_handle) {
    std::lock_guard<std::mutex> lk(g_batch_mutex);
    g_batch_error.clear();
    if (!out_handle) {
        berr("batch_create: null handle");
        return 0;
    }
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count <= 0) {
        berr("batch_create: no CUDA device available (this library has no CPU path)");
        return 0;
    }
    auto b = std::make_unique<Batch>();
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    const long long h = g_next_batch++;
    g_batches[h] = std::move(b);
    *out_handle = h;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_add_brick(long long handle, int nx, int ny, int nz, int precision,
                                                       const uint8_t* obstacle, const float* init_velocity_soa,
                                                       float tau, const float* body_force, const int* face_kinds,
                                                       int* out_index) {
    std::lock_guard<std::mutex> lk(g_batch_mutex);
    g_batch_error.clear();
    Batch* B = lookup_batch(handle);
    if (!B) return 0;
    if (B->finalized) {
        berr("batch_add_brick: batch already finalized");
        return 0;
    }
    if (nx <= 0 || ny <= 0 || nz <= 0 || (long long)(nx + 2) * (ny + 2) * pad_row(nz) * 27 >= (1LL << 31)) {
        berr("batch_add_brick: invalid or too large brick dimensions");
        return 0;
    }
    if (precision != 0 && precision != 1) {
        berr("batch_add_brick: precision must be 0 (fp32) or 1 (fp16)");
        return 0;
    }
    if (!(tau > 0.5f && tau <= 0.95f)) {
        berr("batch_add_brick: tau must lie in (0.5, 0.95]");
        return 0;
    }
    HostBrick hb{};
    hb.nx = nx; hb.ny = ny; hb.nz = nz; hb.precision = precision;
    hb.tau = tau;
    for (int a = 0; a < 3; ++a) hb.force[a] = body_force ? body_force[a] : 0.0f;
    for (int i = 0; i < 6; ++i) {
        const int k = face_kinds ? face_kinds[i] : kHydroPeriodic;
        if (k != kHydroPeriodic && k != kHydroBounceBack) {
            berr("batch_add_brick: batch bricks take periodic or bounce-back faces");
            return 0;
        }
        hb.faces[i] = k;
    }
    const size_t cells = (size_t)nx * ny * nz;
    hb.obstacle.assign(cells, 0);
    if (obstacle) for (size_t c = 0; c < cells; ++c) hb.obstacle[c] = obstacle[c] ? 1 : 0;
    hb.ref.assign(4 * cells, 0.0f);
    if (init_velocity_soa)
        for (size_t c = 0; c < cells; ++c)
            for (int a = 0; a < 3; ++a) {
                const float v = init_velocity_soa[a * cells + c];
                hb.ref[(a + 1) * cells + c] = (std::isfinite(v) && !hb.obstacle[c]) ? v : 0.0f;
            }
    float umax = 0.0f;
    for (size_t c = 0; c < cells; ++c) {
        const float a = hb.ref[cells + c], bb = hb.ref[2 * cells + c], cc = hb.ref[3 * cells + c];
        umax = std::max(umax, std::sqrt(a * a + bb * bb + cc * cc));
    }
    hb.fp16_scale = precision == 1 ? fp16_scale_for_speed(umax + 0.05f) : 1.0f;
    hb.atlas_cells = ((nx + B->stride - 1) / B->stride) * ((ny + B->stride - 1) / B->stride) * ((nz + B->stride - 1) / B->stride);
    B->bricks.push_back(std::move(hb));
    if (out_index) *out_index = (int)B->bricks.size() - 1;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_finalize(long long handle, int publish_stride, float velocity_scale) {
    std::lock_guard<std::mutex> lk(g_batch_mutex);
    g_batch_error.clear();
    Batch* B = lookup_batch(handle);
    if (!B) return 0;
    if (B->finalized || B->bricks.empty()) {
        berr("batch_finalize: already finalized or no bricks");
        return 0;
    }
    if (publish_stride <= 0) {
        berr("batch_finalize: publish stride must be positive");
        return 0;
    }
    B->stride = publish_stride;
    B->velocity_scale = std::isfinite(velocity_scale) && velocity_scale > 0.0f ? velocity_scale : 1.0f;
    cudaStream_t s = current_stream();
    int atlas = 0;
    double bytes = 0.0;
    for (auto& hb : B->bricks) {
        const size_t cells = (size_t)hb.nx * hb.ny * hb.nz;
        hb.atlas_cells = ((hb.nx + B->stride - 1) / B->stride) * ((hb.ny + B->stride - 1) / B->stride) *
                         ((hb.nz + B->stride - 1) / B->stride);
        atlas += hb.atlas_cells;
        const PadGeom g = make_pad_geom(hb.nx, hb.ny, hb.nz, 0);
        const size_t elem = hb.precision == 1 ? 2 : 4;
        if (!bok(cudaMalloc(&hb.f, (size_t)g.pcells * 27 * elem), "cudaMalloc(brick populations)")) return 0;
        if (!bok(cudaMemsetAsync(hb.f, 0, (size_t)g.pcells * 27 * elem, s), "memset")) return 0;
        if (!bok(cudaMalloc(&hb.flags, cells * sizeof(uint32_t)), "cudaMalloc(flags)")) return 0;
        if (!bok(cudaMalloc(&hb.d_obstacle, cells), "cudaMalloc(obstacle)")) return 0;
        if (!bok(cudaMalloc(&hb.d_ref, 4 * cells * sizeof(float)), "cudaMalloc(ref)")) return 0;
        if (!bok(cudaMalloc(&hb.d_temperature, cells * sizeof(float)), "cudaMalloc(temperature)")) return 0;
        if (!bok(cudaMemsetAsync(hb.d_temperature, 0, cells * sizeof(float), s), "memset")) return 0;
        if (!bok(cudaMemcpyAsync(hb.d_obstacle, hb.obstacle.data(), cells, cudaMemcpyHostToDevice, s), "upload obstacle")) return 0;
        if (!bok(cudaMemcpyAsync(hb.d_ref, hb.ref.data(), 4 * cells * sizeof(float), cudaMemcpyHostToDevice, s), "upload ref")) return 0;
        FaceParams fp{};
        for (int i = 0; i < 6; ++i) fp.kind[i] = hb.faces[i];
        for (int a = 0; a < 3; ++a) {
            fp.wrap_lo[a] = hb.faces[2 * a] == kHydroPeriodic;
            fp.wrap_hi[a] = hb.faces[2 * a + 1] == kHydroPeriodic;
        }
        fp.max_speed = kMaxSpeedB;
        const BrickDims d{hb.nx, hb.ny, hb.nz, 0, (long long)cells};
        if (!bok(launch_build_flags(hb.d_obstacle, d, fp, hb.flags, s), "build_flags")) return 0;
        bytes += (double)cells * (27.0 * 2.0 * elem + 1.0);
        B->cells_total += (long long)cells;
    }
    if (!bok(cudaMalloc(&B->d_atlas, (size_t)atlas * 4 * sizeof(short)), "cudaMalloc(atlas)")) return 0;
    if (!bok(cudaMemsetAsync(B->d_atlas, 0, (size_t)atlas * 4 * sizeof(short), s), "memset(atlas)")) return 0;
    if (!bok(cudaStreamSynchronize(s), "sync")) return 0;
    if (!build_units(*B, B->shape.threads)) return 0;
    B->bytes_per_tick = bytes;
    B->finalized = true;
    // host copies are not needed any more
    for (auto& hb : B->bricks) {
        std::vector<uint8_t>().swap(hb.obstacle);
        std::vector<float>().swap(hb.ref);
    }
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_set_options(long long handle, int use_graph, int publish) {
    std::lock_guard<std::mutex> lk(g_batch_mutex);
    g_batch_error.clear();
    Batch* B = lookup_batch(handle);
    if (!B) return 0;
    B->use_graph = use_graph != 0;
    B->publish = publish != 0;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_tick(long long handle, int ticks) {
    std::lock_guard<std::mutex> lk(g_batch_mutex);
    g_batch_error.clear();
    Batch* B = lookup_batch(handle);
    if (!B) return 0;
    if (!B->finalized) {
        berr("batch_tick: finalize the batch first");
        return 0;
    }
    if (ticks < 0) {
        berr("batch_tick: negative tick count");
        return 0;
    }
    return run_ticks(*B, ticks, current_stream()) ? 1 : 0;
}

// Time candidate launch shapes on the live bricks (trial ticks are real ticks)
// and keep the fastest. Candidates: threads per tile {64, 128, 256} x resident
// tiles per SM {2, 4, 8, 16}.
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_autotune(long long handle, int trial_ticks, int* out_threads,
                                                      int* out_blocks_per_sm, float* out_ms_per_tick) {
    std::lock_guard<std::mutex> lk(g_batch_mutex);
    g_batch_error.clear();
    Batch* B = lookup_batch(handle);
    if (!B) return 0;
    if (!B->finalized) {
        berr("batch_autotune: finalize the batch first");
        return 0;
    }
    cudaStream_t s = current_stream();
    trial_ticks = std::max(2, trial_ticks + (trial_ticks & 1));
    if (!B->initialized && !run_ticks(*B, 1, s)) return 0;  // the first (initialising) tick
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best_ms = 1e30f;
    LaunchShape best = B->shape;
    const int threads_c[3] = {64, 128, 256};
    const int bps_c[4] = {2, 4, 8, 16};
    for (int t : threads_c) {
        if (!build_units(*B, t)) return 0;
        for (int bps : bps_c) {
            if (t * bps > 2048) continue;
            LaunchShape sh{t, bps};
            // one untimed tick, then the timed trial
            if (!launch_tick(*B, B->parity, B->publish, sh, s)) return 0;
            B->parity ^= 1;
            ++B->ticks;
            cudaEventRecord(e0, s);
            for (int k = 0; k < trial_ticks; ++k) {
                if (!launch_tick(*B, B->parity, B->publish, sh, s)) return 0;
                B->parity ^= 1;
                ++B->ticks;
            }
            cudaEventRecord(e1, s);
            if (!bok(cudaEventSynchronize(e1), "autotune sync")) return 0;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= trial_ticks;
            if (ms < best_ms) {
                best_ms = ms;
                best = sh;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!build_units(*B, best.threads)) return 0;
    B->shape = best;
    B->tuned = true;
    if (out_threads) *out_threads = best.threads;
    if (out_blocks_per_sm) *out_blocks_per_sm = best.blocks_per_sm;
    if (out_ms_per_tick) *out_ms_per_tick = best_ms;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_info(long long handle, long long* out_cells, double* out_bytes_per_tick,
                                                  int* out_atlas_records, int* out_units, long long* out_ticks) {
    std::lock_guard<std::mutex> lk(g_batch_mutex);
    Batch* B = lookup_batch(handle);
    if (!B) return 0;
    if (out_ticks) *out_ticks = (long long)B->ticks;
    if (out_cells) *out_cells = B->cells_total;
    if (out_bytes_per_tick) *out_bytes_per_tick = B->bytes_per_tick;
    if (out_atlas_records) *out_atlas_records = B->atlas_records;
    if (out_units) *out_units = B->units;
    return 1;
}

// Published int16 atlas of one brick (4 int16 per atlas cell: vx, vy, vz in
// units of 5.6 m/s / 32767, rho - 1 in units of 0.03 / 32767), as written by
// the last published tick.
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_copy_atlas(long long handle, int brick, int16_t* out, int value_count) {
    std::lock_guard<std::mutex> lk(g_batch_mutex);
    g_batch_error.clear();
    Batch* B = lookup_batch(handle);
    if (!B) return 0;
    if (!B->finalized || brick < 0 || brick >= (int)B->bricks.size() || !out) {
        berr("batch_copy_atlas: invalid brick or batch not finalized");
        return 0;
    }
    int offset = 0;
    for (int i = 0; i < brick; ++i) offset += B->bricks[i].atlas_cells;
    const HostBrick& hb = B->bricks[brick];
    if (value_count != hb.atlas_cells * 4) {
        berr("batch_copy_atlas: value_count must be 4 x atlas cells");
        return 0;
    }
    cudaStream_t s = current_stream();
    if (!bok(cudaMemcpyAsync(out, B->d_atlas + 4LL * offset, (size_t)value_count * sizeof(short), cudaMemcpyDeviceToHost, s), "copy atlas")) return 0;
    return bok(cudaStreamSynchronize(s), "sync") ? 1 : 0;
}

// Full flow state of one brick (cells x 4 floats: ux, uy, uz, clamped rho-1).
AERO_LBM_B200_EXPORT int aero_lbm_b200_batch_copy_flow(long long handle, int brick, float* out, int value_count) {
    std::lock_guard<std::mutex> lk(g_batch_mutex);
    g_batch_error.clear();
    Batch* B = lookup_batch(handle);
    if (!B) return 0;
    if (!B->finalized || !B->initialized || brick < 0 || brick >= (int)B->bricks.size() || !out) {
        berr("batch_copy_flow: invalid brick or batch not yet stepped");
        return 0;
    }
    const HostBrick& hb = B->bricks[brick];
    const int cells = hb.nx * hb.ny * hb.nz;
    if (value_count != cells * 4) {
        berr("batch_copy_flow: value_count must be 4 x cells");
        return 0;
    }
    cudaStream_t s = current_stream();
    float* d = nullptr;
    if (!bok(cudaMalloc(&d, (size_t)cells * 4 * sizeof(float)), "cudaMalloc(flow)")) return 0;
    batch_flow_kernel<<<(cells + 127) / 128, 128, 0, s>>>(B->d_descs, brick, B->parity, d);
    count_launch();
    bool ok = bok(cudaGetLastError(), "batch_flow_kernel") &&
              bok(cudaMemcpyAsync(out, d, (size_t)cells * 4 * sizeof(float), cudaMemcpyDeviceToHost, s), "copy flow") &&
              bok(cudaStreamSynchronize(s), "sync");
    cudaFree(d);
    return ok ? 1 : 0;
}

AERO_LBM_B200_EXPORT void aero_lbm_b200_batch_destroy(long long handle) {
    std::lock_guard<std::mutex> lk(g_batch_mutex);
    g_batches.erase(handle);
}

AERO_LBM_B200_EXPORT const char* aero_lbm_b200_batch_last_error(void) { return g_batch_error.c_str(); }

}  // extern "C"
