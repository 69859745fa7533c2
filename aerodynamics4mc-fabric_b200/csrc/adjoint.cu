// Discrete adjoint of the D3Q27 brick step with checkpointed recomputation.
//
// Forward model (per call n = 1..N, two population buffers, pull layout):
//   s_1 = C(feq(1, u_in))                     fluid cells, initial equilibrium
//   s_n = C(P(s_{n-1}))                       n >= 2
//   u_probe = j / clamp(rho) of P(s_N)        the brick step's velocity output
// where P pulls each direction from its source cell (periodic faces wrap;
// solid sources and bounce-back faces return the cell's own opposite
// population; velocity faces supply feq(1, u_in)), and C is the factorised
// cumulant collision with Smagorinsky SGS, Boussinesq buoyancy along +z from a
// static temperature field, and a per-cell body-force field (adjoint27.cuh).
// Loss L = sum over probes of |u_probe - target|^2.
//
// Reverse sweep: lambda_N is seeded at the probe cells; for n = N..1 one
// launch per call recomputes the cell's collision from s_{n-1} (or the initial
// equilibrium), applies its transposed Jacobian to lambda_n, accumulates the
// body-force gradient of the cell in FP64, and scatters the pre-collision
// adjoint along the transposed pull (every population slot is read by exactly
// one fluid cell, so the scatter needs no atomics); velocity-face pulls and
// the initial equilibrium accumulate the inflow gradient in FP64. States are
// checkpointed every K calls during the forward run and recomputed segment by
// segment (K = 1 stores every state and recomputes nothing).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/aero_lbm_b200.h"
#include "adjoint27.cuh"
#include "d3q27_kernels.cuh"
#include "runtime_internal.h"

namespace aero {
namespace adj {
namespace {

struct Geo {
    int nx, ny, nz;
    long long cells;
    int kind[6];  // per face: 1 periodic, 2 bounce-back, 4 velocity
    const uint8_t* solid;
};

enum PullKind { kPullSlot = 0, kPullBounce = 1, kPullFace = 2 };

// Source of direction q for cell (x, y, z) (the brick step's pull rules:
// periodic axes wrap; then the first out-of-range axis in the order x-, x+,
// y-, y+, z-, z+ names the face).
__host__ __device__ __forceinline__ int pull_source(const Geo& G, int x, int y, int z, int q, long long& src) {
    int s[3] = {x - q_cx(q), y - q_cy(q), z - q_cz(q)};
    const int n[3] = {G.nx, G.ny, G.nz};
    int face = -1;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (s[a] < 0 || s[a] >= n[a]) {
            const int fid = 2 * a + (s[a] < 0 ? 0 : 1);
            if (G.kind[fid] == kHydroPeriodic) {
                s[a] = s[a] < 0 ? s[a] + n[a] : s[a] - n[a];
            } else if (face < 0) {
                face = fid;
            }
        }
    }
    if (face >= 0) return G.kind[face] == kHydroVelocity ? kPullFace : kPullBounce;
    src = ((long long)s[0] * G.ny + s[1]) * G.nz + s[2];
    return G.solid[src] ? kPullBounce : kPullSlot;
}

__device__ __forceinline__ void cell_xyz(const Geo& G, long long i, int& x, int& y, int& z) {
    cell_xyz32(i, G.ny, G.nz, x, y, z);
}

template <class T>
__device__ __forceinline__ void pull_cell(const Geo& G, const T* __restrict__ s, long long i, int x, int y, int z,
                                          const T (&uin)[3], T (&p)[27]) {
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        long long src = 0;
        const int k = pull_source(G, x, y, z, q, src);
        p[q] = k == kPullSlot ? s[(long long)q * G.cells + src]
             : k == kPullBounce ? s[(long long)q_opp(q) * G.cells + i]
                                : feq_t<T>(q, T(1), uin[0], uin[1], uin[2]);
    }
}

template <class T>
struct StepArgs {
    Geo G;
    CollideParams cp;
    const float* temperature;  // cells or null
    const float* force;        // 3 x cells (SoA) or null
    T uin[3];
    const T* src;
    T* dst;
};

template <class T>
__device__ __forceinline__ void cell_force(const StepArgs<T>& A, long long i, T& t, T& fx, T& fy, T& fz) {
    t = A.temperature ? T(A.temperature[i]) : T(0);
    fx = fy = fz = T(0);
    if (A.force) {
        fx = T(A.force[i]);
        fy = T(A.force[A.G.cells + i]);
        fz = T(A.force[2 * A.G.cells + i]);
    }
}

// One forward call: init (kInit, collide the equilibrium) or pull + collide.
template <class T, bool kInit>
__global__ void __launch_bounds__(128) adj_step_kernel(StepArgs<T> A) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.G.cells) return;
    T* __restrict__ dst = A.dst;
    if (A.G.solid[i]) {
#pragma unroll
        for (int q = 0; q < 27; ++q) dst[(long long)q * A.G.cells + i] = wq<T>(q);
        return;
    }
    T p[27];
    if (kInit) {
#pragma unroll
        for (int q = 0; q < 27; ++q) p[q] = feq_t<T>(q, T(1), A.uin[0], A.uin[1], A.uin[2]);
    } else {
        int x, y, z;
        cell_xyz(A.G, i, x, y, z);
        pull_cell<T>(A.G, A.src, i, x, y, z, A.uin, p);
    }
    T t, fx, fy, fz;
    cell_force(A, i, t, fx, fy, fz);
    T fo[27];
    CollideTape<T> tape;
    collide_fwd<T>(p, A.cp, t, fx, fy, fz, fo, tape);
#pragma unroll
    for (int q = 0; q < 27; ++q) dst[(long long)q * A.G.cells + i] = fo[q];
}

// Probe velocities of P(s) and the loss sum (FP64).
template <class T>
__global__ void adj_probe_kernel(Geo G, const T* __restrict__ s, T ux_in, T uy_in, T uz_in, int nprobe,
                                 const long long* __restrict__ cells, const float* __restrict__ target,
                                 float* __restrict__ out_u, double* __restrict__ probe_loss) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nprobe) return;
    const long long i = cells[k];
    int x, y, z;
    cell_xyz(G, i, x, y, z);
    const T uin[3] = {ux_in, uy_in, uz_in};
    T p[27], u[3], rc;
    bool rf;
    pull_cell<T>(G, s, i, x, y, z, uin, p);
    probe_velocity<T>(p, u, rc, rf);
    double l = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double d = (double)u[a] - (double)target[3 * k + a];
        l += d * d;
        out_u[3 * k + a] = (float)u[a];
    }
    probe_loss[k] = l;
}

// Scatter of a pre-collision adjoint along the transposed pull; velocity-face
// pulls add to the inflow gradient. Every fluid cell's slot of the output is
// the source of exactly one pull of the forward step (a neighbour's slot
// pull, or the cell's own bounce-back), except the slot (opp q, cell) of a
// direction q that the cell pulls from a velocity face: nothing reads that
// population, so its adjoint is zero, written here. With kAccumulate false
// the launch therefore writes every fluid slot of lam_prev exactly once and
// needs no clearing pass (solid cells' slots are never read).
template <bool kAccumulate>
__device__ __forceinline__ void scatter(const Geo& G, long long i, int x, int y, int z, const float (&lam)[27],
                                        const float (&uin)[3], float* __restrict__ lam_prev, double (&du)[3]) {
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        long long src = 0;
        const int k = pull_source(G, x, y, z, q, src);
        if (k == kPullFace) {
            float d[3];
            dfeq_du<float>(q, 1.0f, uin[0], uin[1], uin[2], d);
            du[0] += (double)lam[q] * d[0];
            du[1] += (double)lam[q] * d[1];
            du[2] += (double)lam[q] * d[2];
            if (!kAccumulate) lam_prev[(long long)q_opp(q) * G.cells + i] = 0.0f;
            continue;
        }
        float* slot = k == kPullSlot ? lam_prev + (long long)q * G.cells + src : lam_prev + (long long)q_opp(q) * G.cells + i;
        if (kAccumulate) *slot += lam[q];
        else *slot = lam[q];
    }
}

// Block sum of the per-thread inflow-gradient parts, added to this block's
// own slot (launches are serial on the stream, so the sum over blocks and
// calls is formed in a fixed order: the result is deterministic).
__device__ __forceinline__ void add_du(double (&du)[3], double* __restrict__ du_part) {
    __shared__ double sh[3][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double v = du[a];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[a][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double t = 0.0;
            for (int w = 0; w < nw; ++w) t += sh[a][w];
            du_part[3 * blockIdx.x + a] += t;
        }
    }
}

// lambda_N at the probe cells: dL/du through the probe observable, scattered
// (one thread, probes in order: probes may share slots).
__global__ void adj_seed_kernel(Geo G, const float* __restrict__ s, float ux_in, float uy_in, float uz_in, int nprobe,
                                const long long* __restrict__ cells, const float* __restrict__ target,
                                float* __restrict__ lam, double* __restrict__ du_slot) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double du[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < nprobe; ++k) {
        const long long i = cells[k];
        int x, y, z;
        cell_xyz(G, i, x, y, z);
        const float uin[3] = {ux_in, uy_in, uz_in};
        float p[27], u[3], rc;
        bool rf;
        pull_cell<float>(G, s, i, x, y, z, uin, p);
        probe_velocity<float>(p, u, rc, rf);
        const float lu[3] = {2.0f * (u[0] - target[3 * k]), 2.0f * (u[1] - target[3 * k + 1]), 2.0f * (u[2] - target[3 * k + 2])};
        float lp[27];
        probe_velocity_vjp<float>(u, rc, rf, lu, lp);
        scatter<true>(G, i, x, y, z, lp, uin, lam, du);
    }
    du_slot[0] = du[0];
    du_slot[1] = du[1];
    du_slot[2] = du[2];
}

// One reverse call: lambda_n (cell-local read) -> lambda_{n-1} (scatter),
// body-force gradient of the cell, inflow gradient.
#ifndef AERO_ADJ_REV_MIN_BLOCKS
#define AERO_ADJ_REV_MIN_BLOCKS 5
#endif
template <bool kInit>
__global__ void __launch_bounds__(128, AERO_ADJ_REV_MIN_BLOCKS) adj_reverse_kernel(StepArgs<float> A, const float* __restrict__ lam_n,
                                                          float* __restrict__ lam_prev, double* __restrict__ grad_f,
                                                          double* __restrict__ du_part) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double du[3] = {0.0, 0.0, 0.0};
    if (i < A.G.cells && !A.G.solid[i]) {
        int x, y, z;
        cell_xyz(A.G, i, x, y, z);
        float p[27];
        if (kInit) {
#pragma unroll
            for (int q = 0; q < 27; ++q) p[q] = feq_t<float>(q, 1.0f, A.uin[0], A.uin[1], A.uin[2]);
        } else {
            pull_cell<float>(A.G, A.src, i, x, y, z, A.uin, p);
        }
        float t, fx, fy, fz;
        cell_force(A, i, t, fx, fy, fz);
        float fo[27];
        CollideTape<float> tape;
        collide_fwd<float, false>(p, A.cp, t, fx, fy, fz, fo, tape);
        float lo[27], li[27], lf[3];
#pragma unroll
        for (int q = 0; q < 27; ++q) lo[q] = lam_n[(long long)q * A.G.cells + i];
        collide_vjp<float>(tape, A.cp, lo, li, lf);
        grad_f[i] += (double)lf[0];
        grad_f[A.G.cells + i] += (double)lf[1];
        grad_f[2 * A.G.cells + i] += (double)lf[2];
        if (kInit) {
#pragma unroll
            for (int q = 0; q < 27; ++q) {
                float d[3];
                dfeq_du<float>(q, 1.0f, A.uin[0], A.uin[1], A.uin[2], d);
                du[0] += (double)li[q] * d[0];
                du[1] += (double)li[q] * d[1];
                du[2] += (double)li[q] * d[2];
            }
        } else {
            scatter<false>(A.G, i, x, y, z, li, A.uin, lam_prev, du);
        }
    }
    add_du(du, du_part);
}

// ------------------------------------------------------------------ host side
struct Brick {
    AeroLbmB200AdjointConfig cfg{};
    Geo geo{};
    CollideParams cp{};
    long long cells = 0;
    size_t state_elems = 0;
    uint8_t* solid = nullptr;
    float* temperature = nullptr;
    float* force = nullptr;
    float* st[2] = {nullptr, nullptr};
    double* st64[2] = {nullptr, nullptr};
    std::vector<float*> ckpt;  // ckpt[j] = s_{jK} for j >= 1 (index 0 unused)
    std::vector<float*> seg;   // two sets of K - 1 recomputed segment states
    cudaStream_t side = nullptr;  // recomputation stream (overlaps the reverse launches)
    float* lam[2] = {nullptr, nullptr};
    double* grad_f = nullptr;
    double* probe_loss = nullptr;  // per probe
    double* du_part = nullptr;     // 3 x (reverse blocks + 1): inflow-gradient parts, the last slot from the seed
    int rev_blocks = 0;
    int nprobe = 0;
    long long* probe_cells = nullptr;
    float* probe_target = nullptr;
    float* probe_u = nullptr;
    double fwd_ms = 0.0, rev_ms = 0.0, recompute_ms = 0.0, total_ms = 0.0;
    int fwd_steps = 0, rev_steps = 0;

    ~Brick() {
        for (void* p : {(void*)solid, (void*)temperature, (void*)force, (void*)st[0], (void*)st[1], (void*)st64[0],
                        (void*)st64[1], (void*)lam[0], (void*)lam[1], (void*)grad_f, (void*)probe_loss, (void*)du_part, (void*)probe_cells,
                        (void*)probe_target, (void*)probe_u})
            if (p) cudaFree(p);
        for (float* p : ckpt)
            if (p) cudaFree(p);
        for (float* p : seg)
            if (p) cudaFree(p);
        if (side) cudaStreamDestroy(side);
    }
};

std::mutex g_adj_mutex;
std::map<long long, Brick*> g_adj;
long long g_next_adj = 1;
std::string g_adj_error;

bool adj_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    g_adj_error = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

CollideParams params_of(const AeroLbmB200AdjointConfig& c) {
    CollideParams p{};
    const float nu = std::min(std::max((c.tau - 0.5f) / 3.0f, 1.0e-8f), (0.95f - 0.5f) / 3.0f);
    p.tau_shear_base = std::min(std::max(0.5f + 3.0f * nu, kTauMin), kTauMax);
    p.tau_normal_base = p.tau_shear_base;
    p.nu0 = std::max(1e-6f, nu);
    p.sgs_c2 = c.smagorinsky_c * c.smagorinsky_c;
    p.sgs_nut_cap = 5.0f * p.nu0;
    p.sgs_bulk = 0.30f;
    p.buoy_beta = c.buoyancy_beta;
    p.buoy_fmax = 0.02f;
    p.max_speed = 0.57735026919f * 0.60f;
    p.enable_sgs = c.smagorinsky_c > 0.0f ? 1 : 0;
    p.enable_buoyancy = c.buoyancy_beta != 0.0f ? 1 : 0;
    p.gravity_axis = 2;
    return p;
}

template <class T>
StepArgs<T> step_args(const Brick& b, const float* inflow, const T* src, T* dst) {
    StepArgs<T> a{};
    a.G = b.geo;
    a.cp = b.cp;
    a.temperature = b.temperature;
    a.force = b.force;
    a.uin[0] = T(inflow[0]);
    a.uin[1] = T(inflow[1]);
    a.uin[2] = T(inflow[2]);
    a.src = src;
    a.dst = dst;
    return a;
}

unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

template <class T>
bool launch_step(const Brick& b, const float* inflow, bool init, const T* src, T* dst, cudaStream_t s) {
    const StepArgs<T> a = step_args<T>(b, inflow, src, dst);
    if (init) adj_step_kernel<T, true><<<blocks_for(b.cells, 128), 128, 0, s>>>(a);
    else adj_step_kernel<T, false><<<blocks_for(b.cells, 128), 128, 0, s>>>(a);
    count_launch();
    return adj_ok(cudaGetLastError(), "adjoint forward step");
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

bool upload_force(Brick& b, const float* force_soa, cudaStream_t s) {
    if (!force_soa) return adj_ok(cudaMemsetAsync(b.force, 0, 3 * b.cells * sizeof(float), s), "force clear");
    return adj_ok(cudaMemcpyAsync(b.force, force_soa, 3 * b.cells * sizeof(float), cudaMemcpyHostToDevice, s), "force upload");
}

Brick* find_brick(long long h) {
    auto it = g_adj.find(h);
    return it == g_adj.end() ? nullptr : it->second;
}

}  // namespace
}  // namespace adj
}  // namespace aero

using namespace aero;
using namespace aero::adj;

extern "C" {

AERO_LBM_B200_EXPORT void aero_lbm_b200_adjoint_default_config(AeroLbmB200AdjointConfig* c) {
    if (!c) return;
    *c = AeroLbmB200AdjointConfig{};
    c->nx = c->ny = c->nz = 64;
    c->face_kind[0] = c->face_kind[1] = AERO_LBM_HYDRO_BOUNDARY_VELOCITY_DIRICHLET;
    c->face_kind[2] = c->face_kind[3] = AERO_LBM_HYDRO_BOUNDARY_PERIODIC;
    c->face_kind[4] = AERO_LBM_HYDRO_BOUNDARY_BOUNCE_BACK;
    c->face_kind[5] = AERO_LBM_HYDRO_BOUNDARY_VELOCITY_DIRICHLET;
    c->tau = 0.55f;
    c->smagorinsky_c = 0.1f;
    c->buoyancy_beta = 1e-4f;
    c->steps = 200;
    c->checkpoint_every = 20;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_create(const AeroLbmB200AdjointConfig* cfg, const uint8_t* obstacle,
                                                      const float* temperature, long long* out_handle) {
    std::lock_guard<std::mutex> lk(g_adj_mutex);
    g_adj_error.clear();
    if (!cfg || !obstacle || !out_handle || cfg->nx <= 0 || cfg->ny <= 0 || cfg->nz <= 0 || cfg->steps < 1 ||
        cfg->checkpoint_every < 1 || !(cfg->tau > 0.5f) || cfg->smagorinsky_c < 0.0f) {
        g_adj_error = "adjoint_create: invalid config (dims > 0, steps >= 1, checkpoint_every >= 1, tau > 0.5)";
        return 0;
    }
    for (int f = 0; f < 6; ++f) {
        const int k = cfg->face_kind[f];
        if (k != AERO_LBM_HYDRO_BOUNDARY_PERIODIC && k != AERO_LBM_HYDRO_BOUNDARY_BOUNCE_BACK &&
            k != AERO_LBM_HYDRO_BOUNDARY_VELOCITY_DIRICHLET) {
            g_adj_error = "adjoint_create: face kinds must be periodic, bounce-back or velocity";
            return 0;
        }
        if ((k == AERO_LBM_HYDRO_BOUNDARY_PERIODIC) != (cfg->face_kind[f ^ 1] == AERO_LBM_HYDRO_BOUNDARY_PERIODIC)) {
            g_adj_error = "adjoint_create: a periodic face needs a periodic opposite face";
            return 0;
        }
    }
    auto* b = new Brick();
    b->cfg = *cfg;
    b->cells = (long long)cfg->nx * cfg->ny * cfg->nz;
    b->state_elems = (size_t)b->cells * 27;
    b->cp = params_of(*cfg);
    const size_t n = (size_t)b->cells;
    bool ok = adj_ok(cudaMalloc(&b->solid, n), "adjoint alloc") &&
              adj_ok(cudaMalloc(&b->force, 3 * n * sizeof(float)), "adjoint alloc") &&
              adj_ok(cudaMalloc(&b->st[0], b->state_elems * sizeof(float)), "adjoint alloc") &&
              adj_ok(cudaMalloc(&b->st[1], b->state_elems * sizeof(float)), "adjoint alloc") &&
              adj_ok(cudaMalloc(&b->lam[0], b->state_elems * sizeof(float)), "adjoint alloc") &&
              adj_ok(cudaMalloc(&b->lam[1], b->state_elems * sizeof(float)), "adjoint alloc") &&
              adj_ok(cudaMalloc(&b->grad_f, 3 * n * sizeof(double)), "adjoint alloc") &&
              adj_ok(cudaMalloc(&b->du_part, 3 * ((size_t)blocks_for(b->cells, 128) + 1) * sizeof(double)), "adjoint alloc");
    b->rev_blocks = (int)blocks_for(b->cells, 128);
    if (ok && temperature)
        ok = adj_ok(cudaMalloc(&b->temperature, n * sizeof(float)), "adjoint alloc") &&
             adj_ok(cudaMemcpy(b->temperature, temperature, n * sizeof(float), cudaMemcpyHostToDevice), "temperature upload");
    if (ok) ok = adj_ok(cudaMemcpy(b->solid, obstacle, n, cudaMemcpyHostToDevice), "mask upload");
    if (!ok) {
        delete b;
        return 0;
    }
    b->geo.nx = cfg->nx;
    b->geo.ny = cfg->ny;
    b->geo.nz = cfg->nz;
    b->geo.cells = b->cells;
    for (int f = 0; f < 6; ++f) b->geo.kind[f] = cfg->face_kind[f];
    b->geo.solid = b->solid;
    const long long h = g_next_adj++;
    g_adj[h] = b;
    *out_handle = h;
    return 1;
}

AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_set_probes(long long handle, int count, const int* cells, const float* targets) {
    std::lock_guard<std::mutex> lk(g_adj_mutex);
    g_adj_error.clear();
    Brick* b = find_brick(handle);
    if (!b || count < 1 || !cells || !targets) {
        g_adj_error = "adjoint_set_probes: unknown handle, no probes or null arrays";
        return 0;
    }
    std::vector<long long> c(count);
    std::vector<uint8_t> solid(b->cells);
    if (!adj_ok(cudaMemcpy(solid.data(), b->solid, b->cells, cudaMemcpyDeviceToHost), "mask read")) return 0;
    for (int k = 0; k < count; ++k) {
        if (cells[k] < 0 || cells[k] >= b->cells || solid[cells[k]]) {
            g_adj_error = "adjoint_set_probes: probe " + std::to_string(k) + " is outside the brick or solid";
            return 0;
        }
        c[k] = cells[k];
    }
    for (void* p : {(void*)b->probe_cells, (void*)b->probe_target, (void*)b->probe_u, (void*)b->probe_loss})
        if (p) cudaFree(p);
    b->probe_cells = nullptr;
    b->probe_target = b->probe_u = nullptr;
    b->probe_loss = nullptr;
    b->nprobe = 0;
    if (!adj_ok(cudaMalloc(&b->probe_cells, count * sizeof(long long)), "probe alloc") ||
        !adj_ok(cudaMalloc(&b->probe_target, 3 * count * sizeof(float)), "probe alloc") ||
        !adj_ok(cudaMalloc(&b->probe_u, 3 * count * sizeof(float)), "probe alloc") ||
        !adj_ok(cudaMalloc(&b->probe_loss, count * sizeof(double)), "probe alloc") ||
        !adj_ok(cudaMemcpy(b->probe_cells, c.data(), count * sizeof(long long), cudaMemcpyHostToDevice), "probe upload") ||
        !adj_ok(cudaMemcpy(b->probe_target, targets, 3 * count * sizeof(float), cudaMemcpyHostToDevice), "probe upload"))
        return 0;
    b->nprobe = count;
    return 1;
}

// Forward run (no checkpoints kept): loss and probe velocities. precision 0
// runs the FP32 model the gradient is taken of, 1 the same model in FP64.
AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_forward(long long handle, const float* force_soa, const float* inflow,
                                                       int precision, double* out_loss, float* out_probe_u) {
    std::lock_guard<std::mutex> lk(g_adj_mutex);
    g_adj_error.clear();
    Brick* b = find_brick(handle);
    if (!b || !inflow || b->nprobe < 1 || (precision != 0 && precision != 1)) {
        g_adj_error = "adjoint_forward: unknown handle, null inflow, no probes or bad precision";
        return 0;
    }
    cudaStream_t s = current_stream();
    if (!upload_force(*b, force_soa, s)) return 0;
    const int N = b->cfg.steps;
    const Geo G = b->geo;
    if (precision == 0) {
        if (!launch_step<float>(*b, inflow, true, nullptr, b->st[0], s)) return 0;
        int cur = 0;
        for (int n = 2; n <= N; ++n) {
            if (!launch_step<float>(*b, inflow, false, b->st[cur], b->st[cur ^ 1], s)) return 0;
            cur ^= 1;
        }
        adj_probe_kernel<float><<<blocks_for(b->nprobe, 64), 64, 0, s>>>(G, b->st[cur], inflow[0], inflow[1], inflow[2],
                                                                          b->nprobe, b->probe_cells, b->probe_target,
                                                                          b->probe_u, b->probe_loss);
    } else {
        for (int k = 0; k < 2; ++k)
            if (!b->st64[k] && !adj_ok(cudaMalloc(&b->st64[k], b->state_elems * sizeof(double)), "fp64 state alloc")) return 0;
        if (!launch_step<double>(*b, inflow, true, nullptr, b->st64[0], s)) return 0;
        int cur = 0;
        for (int n = 2; n <= N; ++n) {
            if (!launch_step<double>(*b, inflow, false, b->st64[cur], b->st64[cur ^ 1], s)) return 0;
            cur ^= 1;
        }
        adj_probe_kernel<double><<<blocks_for(b->nprobe, 64), 64, 0, s>>>(G, b->st64[cur], inflow[0], inflow[1], inflow[2],
                                                                           b->nprobe, b->probe_cells, b->probe_target,
                                                                           b->probe_u, b->probe_loss);
    }
    count_launch();
    if (!adj_ok(cudaGetLastError(), "probe kernel")) return 0;
    std::vector<double> pl(b->nprobe);
    if (!adj_ok(cudaMemcpyAsync(pl.data(), b->probe_loss, b->nprobe * sizeof(double), cudaMemcpyDeviceToHost, s), "loss read"))
        return 0;
    if (out_probe_u &&
        !adj_ok(cudaMemcpyAsync(out_probe_u, b->probe_u, 3 * b->nprobe * sizeof(float), cudaMemcpyDeviceToHost, s), "probe read"))
        return 0;
    if (!adj_ok(cudaStreamSynchronize(s), "forward sync")) return 0;
    double loss = 0.0;
    for (double v : pl) loss += v;
    if (out_loss) *out_loss = loss;
    return 1;
}

// Loss and its gradient with respect to the body-force field (3 x cells, SoA,
// FP64) and the inflow vector (3, FP64): forward run with checkpoints, then
// the reverse sweep segment by segment.
AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_gradient(long long handle, const float* force_soa, const float* inflow,
                                                        double* out_loss, double* out_grad_force, double* out_grad_inflow) {
    std::lock_guard<std::mutex> lk(g_adj_mutex);
    g_adj_error.clear();
    Brick* b = find_brick(handle);
    if (!b || !inflow || b->nprobe < 1) {
        g_adj_error = "adjoint_gradient: unknown handle, null inflow or no probes";
        return 0;
    }
    const auto t0 = std::chrono::steady_clock::now();
    cudaStream_t s = current_stream();
    const int N = b->cfg.steps, K = b->cfg.checkpoint_every;
    const Geo G = b->geo;
    const size_t bytes = b->state_elems * sizeof(float);
    // checkpoint and segment states, allocated at the first gradient call
    // (forward-only use needs neither)
    if (b->ckpt.empty()) {
        const int segments = (N + K - 1) / K;
        b->ckpt.assign(segments, nullptr);
        b->seg.assign(2 * std::max(0, K - 1), nullptr);
        bool got = true;
        for (int j = 1; got && j < segments; ++j) got = adj_ok(cudaMalloc(&b->ckpt[j], bytes), "checkpoint alloc");
        for (size_t j = 0; got && j < b->seg.size(); ++j) got = adj_ok(cudaMalloc(&b->seg[j], bytes), "segment alloc");
        if (got && !b->side) got = adj_ok(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking), "side stream");
        if (!got) {
            for (float* p : b->ckpt)
                if (p) cudaFree(p);
            for (float* p : b->seg)
                if (p) cudaFree(p);
            b->ckpt.clear();
            b->seg.clear();
            return 0;
        }
    }
    cudaEvent_t ev[6];
    for (auto& e : ev) cudaEventCreate(&e);
    const size_t du_bytes = 3 * ((size_t)b->rev_blocks + 1) * sizeof(double);
    bool ok = upload_force(*b, force_soa, s) && adj_ok(cudaMemsetAsync(b->du_part, 0, du_bytes, s), "clear") &&
              adj_ok(cudaMemsetAsync(b->grad_f, 0, 3 * b->cells * sizeof(double), s), "clear");
    // forward with checkpoints s_{jK}
    cudaEventRecord(ev[0], s);
    int cur = 0;
    ok = ok && launch_step<float>(*b, inflow, true, nullptr, b->st[0], s);
    if (ok && K == 1 && N >= 2) ok = adj_ok(cudaMemcpyAsync(b->ckpt[1], b->st[0], bytes, cudaMemcpyDeviceToDevice, s), "ckpt");
    for (int n = 2; ok && n <= N; ++n) {
        ok = launch_step<float>(*b, inflow, false, b->st[cur], b->st[cur ^ 1], s);
        cur ^= 1;
        if (ok && n % K == 0 && n < N)
            ok = adj_ok(cudaMemcpyAsync(b->ckpt[n / K], b->st[cur], bytes, cudaMemcpyDeviceToDevice, s), "checkpoint");
    }
    cudaEventRecord(ev[1], s);
    // loss and the seed of lambda_N
    if (ok) {
        adj_probe_kernel<float><<<blocks_for(b->nprobe, 64), 64, 0, s>>>(G, b->st[cur], inflow[0], inflow[1], inflow[2],
                                                                          b->nprobe, b->probe_cells, b->probe_target,
                                                                          b->probe_u, b->probe_loss);
        count_launch();
        ok = adj_ok(cudaMemsetAsync(b->lam[0], 0, bytes, s), "lambda clear");
    }
    if (ok) {
        adj_seed_kernel<<<1, 32, 0, s>>>(G, b->st[cur], inflow[0], inflow[1], inflow[2], b->nprobe, b->probe_cells,
                                          b->probe_target, b->lam[0], b->du_part + 3 * (size_t)b->rev_blocks);
        count_launch();
        ok = adj_ok(cudaGetLastError(), "seed kernel");
    }
    // reverse sweep over segments: segment j covers calls jK+1 .. min((j+1)K, N)
    // and needs s_{jK} .. s_{(j+1)K-1} (s_0 = the initial equilibrium). The
    // states of segment j - 1 are recomputed on the side stream, into the
    // other of two buffer sets, while segment j is reversed on s: the
    // recomputation reads only checkpoint j - 1, so the two run side by side.
    int lc = 0;
    double rec_ms = 0.0, rev_ms = 0.0;
    const int segments = (N + K - 1) / K;
    const int per = std::max(0, K - 1);
    cudaStream_t s2 = b->side;
    std::vector<cudaEvent_t> evw(segments), evr(segments), eve(segments);  // on s: before / after the wait, after the reverse
    cudaEvent_t rec_done[2], rev_done[2], fwd_done;
    bool rev_used[2] = {false, false};
    for (int k = 0; k < segments; ++k) {
        cudaEventCreate(&evw[k]);
        cudaEventCreate(&evr[k]);
        cudaEventCreate(&eve[k]);
    }
    for (int k = 0; k < 2; ++k) {
        cudaEventCreateWithFlags(&rec_done[k], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&rev_done[k], cudaEventDisableTiming);
    }
    cudaEventCreateWithFlags(&fwd_done, cudaEventDisableTiming);
    // the side stream starts after the forward (force field, checkpoints)
    ok = ok && adj_ok(cudaEventRecord(fwd_done, s), "sweep fork") && adj_ok(cudaStreamWaitEvent(s2, fwd_done, 0), "sweep fork");
    auto recompute = [&](int j, int set) {
        const int first = j * K + 1, last = std::min((j + 1) * K, N);
        if (rev_used[set] && !adj_ok(cudaStreamWaitEvent(s2, rev_done[set], 0), "segment reuse")) return false;
        const float* prev = j > 0 ? b->ckpt[j] : nullptr;
        for (int m = 1; m <= last - first; ++m) {
            float* dst = b->seg[(size_t)set * per + m - 1];
            if (!(m == 1 && j == 0 ? launch_step<float>(*b, inflow, true, nullptr, dst, s2)
                                   : launch_step<float>(*b, inflow, false, prev, dst, s2)))
                return false;
            prev = dst;
        }
        return adj_ok(cudaEventRecord(rec_done[set], s2), "segment done");
    };
    if (ok && segments > 0) ok = recompute(segments - 1, 0);
    for (int j = segments - 1, idx = 0; ok && j >= 0; --j, ++idx) {
        const int set = idx % 2;
        if (j > 0) ok = recompute(j - 1, set ^ 1);
        const int first = j * K + 1, last = std::min((j + 1) * K, N);
        // states[m] = s_{jK + m} for m = 1 .. last - first (s_{jK} = ckpt[j])
        std::vector<const float*> states(last - first + 1, nullptr);
        states[0] = j > 0 ? b->ckpt[j] : nullptr;
        for (int m = 1; m <= last - first; ++m) states[m] = b->seg[(size_t)set * per + m - 1];
        ok = ok && adj_ok(cudaEventRecord(evw[idx], s), "sweep event") && adj_ok(cudaStreamWaitEvent(s, rec_done[set], 0), "segment wait") &&
             adj_ok(cudaEventRecord(evr[idx], s), "sweep event");
        for (int n = last; ok && n >= first; --n) {
            const int m = n - first;  // input state of call n is states[m]
            StepArgs<float> a = step_args<float>(*b, inflow, states[m], nullptr);
            // the reverse launch writes every fluid slot of lam[lc ^ 1] (scatter)
            if (n == 1)
                adj_reverse_kernel<true><<<blocks_for(b->cells, 128), 128, 0, s>>>(a, b->lam[lc], b->lam[lc ^ 1], b->grad_f,
                                                                                   b->du_part);
            else
                adj_reverse_kernel<false><<<blocks_for(b->cells, 128), 128, 0, s>>>(a, b->lam[lc], b->lam[lc ^ 1], b->grad_f,
                                                                                    b->du_part);
            count_launch();
            ok = adj_ok(cudaGetLastError(), "reverse kernel");
            lc ^= 1;
        }
        ok = ok && adj_ok(cudaEventRecord(eve[idx], s), "sweep event") && adj_ok(cudaEventRecord(rev_done[set], s), "sweep event");
        rev_used[set] = true;
    }
    if (ok) ok = adj_ok(cudaStreamSynchronize(s), "sweep sync");
    for (int k = 0; ok && k < segments; ++k) {
        rec_ms += elapsed(evw[k], evr[k]);
        rev_ms += elapsed(evr[k], eve[k]);
    }
    for (int k = 0; k < segments; ++k) {
        cudaEventDestroy(evw[k]);
        cudaEventDestroy(evr[k]);
        cudaEventDestroy(eve[k]);
    }
    for (int k = 0; k < 2; ++k) {
        cudaEventDestroy(rec_done[k]);
        cudaEventDestroy(rev_done[k]);
    }
    cudaEventDestroy(fwd_done);
    std::vector<double> pl(b->nprobe), du(3 * ((size_t)b->rev_blocks + 1));
    if (ok) ok = adj_ok(cudaMemcpyAsync(pl.data(), b->probe_loss, b->nprobe * sizeof(double), cudaMemcpyDeviceToHost, s),
                        "loss read") &&
                 adj_ok(cudaMemcpyAsync(du.data(), b->du_part, du_bytes, cudaMemcpyDeviceToHost, s), "gradient read");
    if (ok && out_grad_force)
        ok = adj_ok(cudaMemcpyAsync(out_grad_force, b->grad_f, 3 * b->cells * sizeof(double), cudaMemcpyDeviceToHost, s),
                    "gradient read");
    if (ok) ok = adj_ok(cudaStreamSynchronize(s), "gradient sync");
    if (ok) {
        b->fwd_ms = elapsed(ev[0], ev[1]);
        b->recompute_ms = rec_ms;
        b->rev_ms = rev_ms;
        b->fwd_steps = N;
        b->rev_steps = N;
        b->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (!ok) return 0;
    double loss = 0.0, gu[3] = {0.0, 0.0, 0.0};
    for (double v : pl) loss += v;
    for (size_t k = 0; k < du.size(); ++k) gu[k % 3] += du[k];
    if (out_loss) *out_loss = loss;
    if (out_grad_inflow) {
        out_grad_inflow[0] = gu[0];
        out_grad_inflow[1] = gu[1];
        out_grad_inflow[2] = gu[2];
    }
    return 1;
}

// Device times of the last gradient call: forward (with checkpoint copies),
// segment recomputation and reverse launches, per call, and the wall time.
AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_timing(long long handle, double* fwd_ms_per_step, double* recompute_ms_per_step,
                                                      double* rev_ms_per_step, double* total_ms) {
    std::lock_guard<std::mutex> lk(g_adj_mutex);
    Brick* b = find_brick(handle);
    if (!b || b->fwd_steps == 0) return 0;
    if (fwd_ms_per_step) *fwd_ms_per_step = b->fwd_ms / b->fwd_steps;
    if (recompute_ms_per_step) *recompute_ms_per_step = b->recompute_ms / b->rev_steps;
    if (rev_ms_per_step) *rev_ms_per_step = b->rev_ms / b->rev_steps;
    if (total_ms) *total_ms = b->total_ms;
    return 1;
}

AERO_LBM_B200_EXPORT void aero_lbm_b200_adjoint_destroy(long long handle) {
    std::lock_guard<std::mutex> lk(g_adj_mutex);
    auto it = g_adj.find(handle);
    if (it == g_adj.end()) return;
    cudaStreamSynchronize(current_stream());
    delete it->second;
    g_adj.erase(it);
}

AERO_LBM_B200_EXPORT const char* aero_lbm_b200_adjoint_last_error(void) { return g_adj_error.c_str(); }

// One cell's collision and its vector-Jacobian product on the host CPU
// (precision 0 float, 1 double), for checking the reverse sweep against
// finite differences without a GPU.
AERO_LBM_B200_EXPORT int aero_lbm_b200_adjoint_collide_vjp_host(int precision, const AeroLbmB200AdjointConfig* cfg,
                                                                const double* f_in, double temperature,
                                                                const double* cell_force, const double* lam_out,
                                                                double* f_out, double* lam_in, double* lam_force) {
    if (!cfg || !f_in || !cell_force || !lam_out || !f_out || !lam_in || !lam_force) return 0;
    const CollideParams cp = params_of(*cfg);
    if (precision == 0) {
        float f[27], fo[27], lo[27], li[27], lf[3];
        for (int q = 0; q < 27; ++q) { f[q] = (float)f_in[q]; lo[q] = (float)lam_out[q]; }
        CollideTape<float> t;
        collide_fwd<float>(f, cp, (float)temperature, (float)cell_force[0], (float)cell_force[1], (float)cell_force[2], fo, t);
        collide_vjp<float>(t, cp, lo, li, lf);
        for (int q = 0; q < 27; ++q) { f_out[q] = fo[q]; lam_in[q] = li[q]; }
        for (int a = 0; a < 3; ++a) lam_force[a] = lf[a];
    } else {
        double f[27], fo[27], lo[27], li[27], lf[3];
        for (int q = 0; q < 27; ++q) { f[q] = f_in[q]; lo[q] = lam_out[q]; }
        CollideTape<double> t;
        collide_fwd<double>(f, cp, temperature, cell_force[0], cell_force[1], cell_force[2], fo, t);
        collide_vjp<double>(t, cp, lo, li, lf);
        for (int q = 0; q < 27; ++q) { f_out[q] = fo[q]; lam_in[q] = li[q]; }
        for (int a = 0; a < 3; ++a) lam_force[a] = lf[a];
    }
    return 1;
}

}  // extern "C"
