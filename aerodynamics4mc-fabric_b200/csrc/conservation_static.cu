// Allocation-free FP64 conservation sums.
//
// Some callers of this library cannot call cudaMalloc: a real-time game thread
// (the mod's simulation worker drives the native step once per tick) must not
// block on it, because cudaMalloc and cudaFree can synchronise the whole
// device and stall the tick; and an embedding that budgets all device memory
// up front forbids allocations once it is running. aero_lbm_b200_conservation_sums
// allocates its partial-sum scratch on first use; this entry point allocates
// nothing: its scratch is the file-scope device array below.
//
// The array holds the per-block partial sums of a one-block-per-256-cells
// pass plus the four results, so it bounds the brick size:
// kStaticMaxCells = 2,097,152 cells (a 128^3 brick); larger contexts are
// rejected with an error. It is 256 KiB, held by every GPU that loads the
// library until the process exits.
//
// Host code never uses the array's name as a device address (on the host it is
// only a stand-in). The first call on each device, with that device current,
// looks up the array's device address with cudaGetSymbolAddress and caches it;
// make that first call on a device before any stream capture. Every call
// writes every partial it later reads and then the four results, so nothing
// has to be cleared between calls; the array keeps the last call's values.
// All calls share the one array: calls that overlap on the GPU (from several
// host threads, or on several streams) race on it and must be serialised by
// the caller. The entry point itself serialises with the runtime lock and
// synchronises the library stream before returning.
#include <mutex>

#include "../../include/aero_lbm_b200.h"
#include "ip_launch.h"
#include "runtime_internal.h"

namespace aero {
namespace {

constexpr int kStaticThreads = 256;
constexpr long long kStaticMaxCells = 2097152;  // 128^3
constexpr int kStaticMaxBlocks = (int)(kStaticMaxCells / kStaticThreads);
constexpr int kStaticResult = kStaticMaxBlocks * 4;  // index of the 4 results

static __device__ __align__(256) double g_conservation_scratch[kStaticMaxBlocks * 4 + 4];

constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_setup_mutex;

// Device address of the scratch array on the context's device `dev` (looked
// up once per device, with that device current). The call is rejected when
// another device is current: the context's memory, the library stream and
// the scratch all live on `dev`.
double* scratch_for_device(int dev, std::string& err) {
    if (dev < 0 || dev >= kMaxDevices) {
        err = "the context's device " + std::to_string(dev) + " is outside the first " + std::to_string(kMaxDevices) +
              " devices the scratch table covers";
        return nullptr;
    }
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) {
        err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return nullptr;
    }
    if (cur != dev) {
        err = "device " + std::to_string(cur) + " is current but the context lives on device " + std::to_string(dev) +
              "; make that device current first";
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        double* p = nullptr;
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_conservation_scratch);
        if (e != cudaSuccess || !p) {
            err = std::string("cudaGetSymbolAddress(conservation scratch): ") + cudaGetErrorString(e);
            return nullptr;
        }
        g_scratch_ptr[dev] = p;
    }
    return g_scratch_ptr[dev];
}

__device__ __forceinline__ double warp_sum_s(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void block_sum4_s(double (&v)[4]) {
    __shared__ double sh[4][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = warp_sum_s(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) sh[k][warp] = v[k];
    }
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = warp_sum_s(lane < nw ? sh[k][lane] : 0.0);
    }
}

__device__ __forceinline__ void add_cell(const float (&f)[27], double (&acc)[4]) {
    RawMoments m;
    raw_moments27<false>(f, m);
    acc[0] += (double)m.r000;
    acc[1] += (double)m.r100;
    acc[2] += (double)m.r010;
    acc[3] += (double)m.r001;
}

// One cell per thread, one block per 256 cells; partials[block] <- block sums.
__global__ void static_sums_ab_kernel(int nx, int ny, int nz, const float* __restrict__ g,
                                      const uint32_t* __restrict__ flags, const uint8_t* __restrict__ obstacle,
                                      const float* __restrict__ ref_p, const FaceParams* __restrict__ F,
                                      double* __restrict__ partials, int direct) {
    const long long cells = (long long)nx * ny * nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (cell < cells) {
        const uint32_t w = flags[cell];
        if (!(w & kFlagSelfSolid)) {
            const int z = (int)(cell % nz), y = (int)((cell / nz) % ny), x = (int)(cell / ((long long)ny * nz));
            float f[27];
            if (direct) {  // g holds the streamed state itself (after a halo exchange)
#pragma unroll
                for (int q = 0; q < 27; ++q) f[q] = g[(long long)q * cells + cell];
            } else {
                const PullView v{g, obstacle, ref_p, F, cells, nx, ny, nz};
                pull27(v, w, cell, x, y, z, f);
            }
            add_cell(f, acc);
        }
    }
    block_sum4_s(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) partials[blockIdx.x * 4 + k] = acc[k];
    }
}

template <class S>
__global__ void static_sums_ip_kernel(const typename S::T* __restrict__ f, IpArgs a, double* __restrict__ partials) {
    const PadGeom G = a.g;
    const long long cells = (long long)G.nx * G.ny * G.nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (cell < cells) {
        const uint32_t w = a.flags_prev[cell];
        if (!(w & kFlagSelfSolid)) {
            int x, y, z;
            cell_coords(G, cell, x, y, z);
            const int own = pad_index(G, x, y, z);
            const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
            float fl[27];
            ip_pull<S>(f, a, G, o, own, w, a.parity, fl);
            add_cell(fl, acc);
        }
    }
    block_sum4_s(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) partials[blockIdx.x * 4 + k] = acc[k];
    }
}

// partials[kStaticResult + k] <- sum of the first `blocks` partials.
__global__ void static_sums_reduce_kernel(double* __restrict__ partials, int blocks) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) {
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] += partials[i * 4 + k];
    }
    block_sum4_s(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) partials[kStaticResult + k] = acc[k];
    }
}

}  // namespace
}  // namespace aero

using namespace aero;

extern "C" {

// Same result as aero_lbm_b200_conservation_sums (FP64 {sum rho, sum rho u}
// over fluid cells of the context's current streamed state, into a host
// array of 4 doubles), computed without allocating: see the file comment for
// who needs this, the size limit and the sharing rules of its static scratch.
AERO_LBM_B200_EXPORT int aero_lbm_b200_conservation_sums_noalloc(long long context_key, double* out4) {
    std::lock_guard<std::recursive_mutex> lk(runtime_mutex());
    clear_error();
    Context* c = find_context(context_key);
    if (!c || !c->initialized || !out4) {
        set_error("conservation_sums_noalloc: no initialized context or null output");
        return 0;
    }
    if (c->cells > kStaticMaxCells) {
        set_error("conservation_sums_noalloc: context has " + std::to_string(c->cells) +
                  " cells; the static scratch covers at most 2097152 (a 128^3 brick)");
        return 0;
    }
    std::string err;
    double* scratch = scratch_for_device(c->device, err);
    if (!scratch) {
        set_error("conservation_sums_noalloc: " + err);
        return 0;
    }
    cudaStream_t s = current_stream();
    const int blocks = (int)((c->cells + kStaticThreads - 1) / kStaticThreads);
    if (c->layout == 0) {
        const float* g = c->f_ready ? c->g[1 - c->cur] : c->g[c->cur];
        static_sums_ab_kernel<<<blocks, kStaticThreads, 0, s>>>(c->nx, c->ny, c->nz, g, c->flags[c->slot],
                                                                c->obstacle[c->slot], c->ref_p[c->slot],
                                                                c->d_face[c->slot], scratch, c->f_ready ? 1 : 0);
    } else {
        if (!join_fill(*c, s)) return 0;  // the last call's pending face pre-fill first
        IpArgs a{};
        a.g = make_pad_geom(c->nx, c->ny, c->nz, c->periodic_mask);
        a.parity = c->parity;
        a.flags_prev = c->flags[c->slot];
        a.obstacle_cur = c->obstacle[c->slot];
        a.ref_p_prev = c->ref_p[c->slot];
        a.face_prev = c->d_face[c->slot];
        a.cur = c->fields(c->slot);
        a.sc = Fp16Scale{c->fp16_scale, c->fp16_scale > 0.0f ? 1.0f / c->fp16_scale : 0.0f};
        if (c->ip_variant == kIpF16Fast)
            static_sums_ip_kernel<StoreF16Dev><<<blocks, kStaticThreads, 0, s>>>(static_cast<const __half*>(c->ip), a, scratch);
        else if (c->ip_variant == kIpI16Fast)
            static_sums_ip_kernel<StoreI16Dev><<<blocks, kStaticThreads, 0, s>>>(static_cast<const short*>(c->ip), a, scratch);
        else
            static_sums_ip_kernel<StoreF32><<<blocks, kStaticThreads, 0, s>>>(static_cast<const float*>(c->ip), a, scratch);
    }
    count_launch();
    if (!cuda_ok(cudaGetLastError(), "conservation_sums_noalloc kernel")) return 0;
    static_sums_reduce_kernel<<<1, 256, 0, s>>>(scratch, blocks);
    count_launch();
    if (!cuda_ok(cudaGetLastError(), "conservation_sums_noalloc reduce")) return 0;
    if (!cuda_ok(cudaMemcpyAsync(out4, scratch + kStaticResult, 4 * sizeof(double), cudaMemcpyDeviceToHost, s),
                 "conservation_sums_noalloc copy")) return 0;
    return cuda_ok(cudaStreamSynchronize(s), "conservation_sums_noalloc sync") ? 1 : 0;
}

}  // extern "C"
