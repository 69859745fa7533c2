// Per-context operations between or around steps (see context_ops.cuh).
// Built with --fmad=false: the shifted pull evaluates the face rules
// operation by operation, like the reference-order step kernel.
// Each is one or two small launches on the caller's stream; none is on the
// per-step path except the overlays (a sparse scatter after the ingest) and
// the cylinder force (one read pass, only under that benchmark preset).
#include "context_ops.cuh"

#include "d3q27_step.cuh"

namespace aero {
namespace {

constexpr int kOverlayChannels = 6;  // vx, vy, vz, p, T, source (jni.cpp:75-81)

// thermal: 0 the overlay's temperature is the collision's field; 1 it is the
// transport's reference temperature and the overlay's source replaces the
// cell's; 2 as 1 but the cell keeps its fan-driven source (9-channel packets:
// thermal_source_term, jni.cpp:1783-1797, ignores the stored source then)
__global__ void apply_overlays_kernel(const int* __restrict__ cells, const float* __restrict__ values, int count,
                                      CellFields f, long long n_cells, int thermal) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int cell = cells[i];
    if (cell < 0 || (long long)cell >= n_cells) return;
    const float* v = values + (long long)i * kOverlayChannels;
    f.ref_ux[cell] = isfinite(v[0]) ? v[0] : 0.0f;
    f.ref_uy[cell] = isfinite(v[1]) ? v[1] : 0.0f;
    f.ref_uz[cell] = isfinite(v[2]) ? v[2] : 0.0f;
    f.ref_p[cell] = clampf_dev(v[3], -0.03f, 0.03f);
    if (thermal) {
        f.ref_temperature[cell] = clampf_dev(v[4], -1.0f, 1.0f);
        if (thermal == 1) f.thermal_source[cell] = clampf_dev(v[5], -0.006f, 0.006f);
    } else {
        f.temperature[cell] = clampf_dev(v[4], -1.0f, 1.0f);
    }
}

__device__ __forceinline__ bool shifted_source(int x, int y, int z, int dx, int dy, int dz, int nx, int ny, int nz,
                                               int& sx, int& sy, int& sz) {
    sx = x + dx; sy = y + dy; sz = z + dz;
    return sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz;
}

__global__ void shift_f32_kernel(const float* __restrict__ src, float* __restrict__ dst, int nx, int ny, int nz, int comps,
                                 int dx, int dy, int dz, float fill, int populations) {
    const long long cells = (long long)nx * ny * nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    int x, y, z, sx, sy, sz;
    cell_xyz32(cell, ny, nz, x, y, z);
    const bool in = shifted_source(x, y, z, dx, dy, dz, nx, ny, nz, sx, sy, sz);
    const long long scell = ((long long)sx * ny + sy) * nz + sz;
    for (int k = 0; k < comps; ++k) {
        const float rest = populations ? feq27(k, 1.0f, 0.0f, 0.0f, 0.0f) : fill;
        dst[(long long)k * cells + cell] = in ? src[(long long)k * cells + scell] : rest;
    }
}

__global__ void shift_u8_kernel(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst, int nx, int ny, int nz,
                                int dx, int dy, int dz) {
    const long long cells = (long long)nx * ny * nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    int x, y, z, sx, sy, sz;
    cell_xyz32(cell, ny, nz, x, y, z);
    dst[cell] = shifted_source(x, y, z, dx, dy, dz, nx, ny, nz, sx, sy, sz) ? src[((long long)sx * ny + sy) * nz + sz] : 0;
}

__global__ void shift_materialise_ab_kernel(int nx, int ny, int nz, const float* __restrict__ g,
                                            const uint32_t* __restrict__ flags, const uint8_t* __restrict__ obstacle,
                                            const float* __restrict__ ref_p, const FaceParams* __restrict__ F, int dx,
                                            int dy, int dz, float* __restrict__ f_out) {
    const long long cells = (long long)nx * ny * nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    int x, y, z, sx, sy, sz;
    cell_xyz32(cell, ny, nz, x, y, z);
    float f[27];
    if (shifted_source(x, y, z, dx, dy, dz, nx, ny, nz, sx, sy, sz)) {
        const long long scell = ((long long)sx * ny + sy) * nz + sz;
        const PullView v{g, obstacle, ref_p, F, cells, nx, ny, nz};
        pull27(v, flags[scell], scell, sx, sy, sz, f);
    } else {
#pragma unroll
        for (int q = 0; q < 27; ++q) f[q] = feq27(q, 1.0f, 0.0f, 0.0f, 0.0f);
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) f_out[(long long)q * cells + cell] = f[q];
}

template <class S>
struct IpSideT {
    typename S::T* f;
    PadGeom g;
    const uint32_t* flags;
    int parity;
    Fp16Scale sc;
};

// tmp[q][x] = incoming population q of cell x + d (rest equilibrium outside
// the brick or on a solid cell, whose memory holds no populations).
template <class S>
__global__ void ip_gather_shifted_kernel(IpSideT<S> v, int dx, int dy, int dz, float* __restrict__ tmp) {
    const PadGeom G = v.g;
    const long long cells = (long long)G.nx * G.ny * G.nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    int x, y, z, sx, sy, sz;
    cell_xyz32(cell, G.ny, G.nz, x, y, z);
    bool live = shifted_source(x, y, z, dx, dy, dz, G.nx, G.ny, G.nz, sx, sy, sz);
    uint32_t w = 0;
    if (live) {
        w = v.flags[((long long)sx * G.ny + sy) * G.nz + sz];
        live = !(w & kFlagSelfSolid);
    }
    if (!live) {
#pragma unroll 1
        for (int q = 0; q < 27; ++q) tmp[(long long)q * cells + cell] = feq27(q, 1.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const NeighbourOffsets o = neighbour_offsets(G, sx, sy, sz);
    const int own = pad_index(G, sx, sy, sz);
#pragma unroll 1
    for (int q = 0; q < 27; ++q) {
        int c, d;
        incoming_slot(o, own, q, v.parity, (w >> q) & 1u, c, d);
        tmp[(long long)q * cells + cell] = S::load(v.f + (long long)d * G.pcells + c, q, v.sc);
    }
}

template <class S>
__global__ void ip_scatter_kernel(IpSideT<S> v, const float* __restrict__ tmp) {
    const PadGeom G = v.g;
    const long long cells = (long long)G.nx * G.ny * G.nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    const uint32_t w = v.flags[cell];
    if (w & kFlagSelfSolid) return;
    int x, y, z;
    cell_xyz32(cell, G.ny, G.nz, x, y, z);
    const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
    const int own = pad_index(G, x, y, z);
#pragma unroll 1
    for (int q = 0; q < 27; ++q) {
        int c, d;
        incoming_slot(o, own, q, v.parity, (w >> q) & 1u, c, d);
        S::store(v.f + (long long)d * G.pcells + c, q, tmp[(long long)q * cells + cell], v.sc);
    }
}

__global__ void gather_temperature_kernel(const float* __restrict__ t, const uint8_t* __restrict__ obstacle, int nx, int ny,
                                          int nz, OutBox b, float* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.count()) return;
    const int az = (int)(i % b.sz);
    const int ay = (int)((i / b.sz) % b.sy);
    const int ax = (int)(i / ((long long)b.sy * b.sz));
    const int x = min(nx - 1, b.ox + ax * b.stride), y = min(ny - 1, b.oy + ay * b.stride),
              z = min(nz - 1, b.oz + az * b.stride);
    const long long cell = ((long long)x * ny + y) * nz + z;
    float v = 0.0f;
    if (!obstacle[cell]) {
        v = clampf_dev(t[cell], -1.0f, 1.0f);
        if (!isfinite(v)) v = 0.0f;
    }
    out[i] = v;
}

__global__ void fill_rest_kernel(float* __restrict__ f, long long cells) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells * 27) return;
    f[i] = feq27((int)(i / cells), 1.0f, 0.0f, 0.0f, 0.0f);
}

struct CylinderGeom {
    float cx, cy, r2;
};

__global__ void cylinder_force_kernel(const float* __restrict__ post, const uint8_t* __restrict__ obstacle, int nx, int ny,
                                      int nz, CylinderGeom cyl, double* __restrict__ out3) {
    __shared__ double sh[3][32];
    const long long cells = (long long)nx * ny * nz;
    double acc[3] = {0.0, 0.0, 0.0};
    for (long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x; cell < cells;
         cell += (long long)gridDim.x * blockDim.x) {
        if (obstacle[cell]) continue;
        int x, y, z;
        cell_xyz32(cell, ny, nz, x, y, z);
#pragma unroll 1
        for (int q = 0; q < 27; ++q) {
            if (q == kRest27 || q_cz(q) != 0) continue;
            const int ex = x + q_cx(q), ey = y + q_cy(q);
            if (ex < 0 || ey < 0 || ex >= nx || ey >= ny) continue;
            if (!obstacle[((long long)ex * ny + ey) * nz + z]) continue;
            // no contraction: the disc test rounds like the reference's
            const float ddx = __fsub_rn((float)ex, cyl.cx), ddy = __fsub_rn((float)ey, cyl.cy);
            if (!(__fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)) <= cyl.r2)) continue;
            const double fq2 = 2.0 * (double)post[(long long)q * cells + cell];
            acc[0] += fq2 * (double)q_cx(q);
            acc[1] += fq2 * (double)q_cy(q);
        }
    }
    // The terms are floats scaled by 2 and summed in double: every partial sum
    // is exact at these magnitudes, so the order does not change the result.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_down_sync(0xffffffffu, acc[k], o);
        if (lane == 0) sh[k][warp] = acc[k];
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            double v = lane < nw ? sh[k][lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if (lane == 0) atomicAdd(out3 + k, v);
        }
    }
}

unsigned cell_blocks(long long cells) { return (unsigned)((cells + 127) / 128); }

template <class S>
IpSideT<S> side_of(const IpView& v) {
    return IpSideT<S>{static_cast<typename S::T*>(v.f), v.g, v.flags, v.parity, v.sc};
}

template <class S>
cudaError_t ip_gather_t(const IpView& v, int dx, int dy, int dz, float* tmp, cudaStream_t s) {
    const long long cells = (long long)v.g.nx * v.g.ny * v.g.nz;
    ip_gather_shifted_kernel<S><<<cell_blocks(cells), 128, 0, s>>>(side_of<S>(v), dx, dy, dz, tmp);
    count_launch();
    return cudaGetLastError();
}

template <class S>
cudaError_t ip_scatter_t(const IpView& v, const float* tmp, cudaStream_t s) {
    const long long cells = (long long)v.g.nx * v.g.ny * v.g.nz;
    ip_scatter_kernel<S><<<cell_blocks(cells), 128, 0, s>>>(side_of<S>(v), tmp);
    count_launch();
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_apply_overlays(const int* cells, const float* values, int count, CellFields f, long long n_cells,
                                  int thermal, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    apply_overlays_kernel<<<(unsigned)((count + 127) / 128), 128, 0, s>>>(cells, values, count, f, n_cells, thermal);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_shift_f32(const float* src, float* dst, BrickDims d, int comps, int dx, int dy, int dz, float fill,
                             bool populations, cudaStream_t s) {
    if (d.cells <= 0) return cudaSuccess;
    shift_f32_kernel<<<cell_blocks(d.cells), 128, 0, s>>>(src, dst, d.nx, d.ny, d.nz, comps, dx, dy, dz, fill,
                                                          populations ? 1 : 0);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_shift_u8(const uint8_t* src, uint8_t* dst, BrickDims d, int dx, int dy, int dz, cudaStream_t s) {
    if (d.cells <= 0) return cudaSuccess;
    shift_u8_kernel<<<cell_blocks(d.cells), 128, 0, s>>>(src, dst, d.nx, d.ny, d.nz, dx, dy, dz);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_shift_materialise_ab(BrickDims d, const float* g, const uint32_t* flags, const uint8_t* obstacle,
                                        const float* ref_p, const FaceParams* face, int dx, int dy, int dz, float* f_out,
                                        cudaStream_t s) {
    if (d.cells <= 0) return cudaSuccess;
    shift_materialise_ab_kernel<<<cell_blocks(d.cells), 128, 0, s>>>(d.nx, d.ny, d.nz, g, flags, obstacle, ref_p, face, dx,
                                                                     dy, dz, f_out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_ip_gather_shifted(int storage, const IpView& v, int dx, int dy, int dz, float* tmp, cudaStream_t s) {
    if (storage == 0) return ip_gather_t<StoreF32>(v, dx, dy, dz, tmp, s);
    if (storage == 1) return ip_gather_t<StoreF16Dev>(v, dx, dy, dz, tmp, s);
    return ip_gather_t<StoreI16Dev>(v, dx, dy, dz, tmp, s);
}

cudaError_t launch_ip_scatter(int storage, const IpView& v, const float* tmp, cudaStream_t s) {
    if (storage == 0) return ip_scatter_t<StoreF32>(v, tmp, s);
    if (storage == 1) return ip_scatter_t<StoreF16Dev>(v, tmp, s);
    return ip_scatter_t<StoreI16Dev>(v, tmp, s);
}

cudaError_t launch_fill_rest(float* f, long long cells, cudaStream_t s) {
    if (cells <= 0) return cudaSuccess;
    fill_rest_kernel<<<(unsigned)((cells * 27 + 255) / 256), 256, 0, s>>>(f, cells);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_gather_temperature(const float* t, const uint8_t* obstacle, BrickDims d, OutBox box, float* out,
                                      cudaStream_t s) {
    const long long n = box.count();
    if (n <= 0) return cudaSuccess;
    gather_temperature_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(t, obstacle, d.nx, d.ny, d.nz, box, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_cylinder_force(const float* post, const uint8_t* obstacle, BrickDims d, double* out3, cudaStream_t s) {
    // cylinder_benchmark_geometry (jni.cpp:201-212), evaluated in float on the host
    const float length_cells = (float)std::max(1, d.nx - 1);
    const float channel_height = (float)std::max(1, d.ny - 1);
    float diameter = std::max(2.5f, 0.1f / 2.2f * length_cells);
    diameter = std::min(diameter, std::max(2.5f, channel_height - 4.0f));
    const float radius = 0.5f * diameter;
    const CylinderGeom cyl{0.2f / 2.2f * length_cells, 0.0f + 0.2f / 0.41f * channel_height, radius * radius};
    cudaError_t e = cudaMemsetAsync(out3, 0, 3 * sizeof(double), s);
    if (e != cudaSuccess || d.cells <= 0) return e;
    const long long want = (d.cells + 255) / 256;
    const unsigned blocks = (unsigned)std::min<long long>(want, 4 * 148);
    cylinder_force_kernel<<<blocks, 256, 0, s>>>(post, obstacle, d.nx, d.ny, d.nz, cyl, out3);
    count_launch();
    return cudaGetLastError();
}

}  // namespace aero
