// Kernel templates of the FP32 D3Q27 brick step, shared by the two
// translation units that instantiate them: d3q27_exact.cu (reference-order
// collision, built with --fmad=false) and d3q27_fast.cu (factorised collision).
#pragma once

#include "collide27_exact.cuh"
#include "d3q27_kernels.cuh"

namespace aero {

__device__ __forceinline__ bool wrap_coord(int& c, int n, int lo, int hi) {
    if (c >= 0 && c < n) return true;
    if (c < 0 ? lo : hi) {
        c %= n;
        if (c < 0) c += n;
        return true;
    }
    return false;
}

__device__ __forceinline__ int oob_face(int sx, int sy, int sz, int nx, int ny, int nz) {
    if (sx < 0) return kFaceXMin;
    if (sx >= nx) return kFaceXMax;
    if (sy < 0) return kFaceYMin;
    if (sy >= ny) return kFaceYMax;
    if (sz < 0) return kFaceZMin;
    return kFaceZMax;
}

// Collide one fluid cell; false = non-finite input, the caller reseeds.
// (x, y, z): the cell's coordinates, for the runtime terms' edge layers;
// temperature: the cell's buoyancy temperature when the caller computed it
// (fused transport), else null (read from cur.temperature).
template <bool kExact>
__device__ __forceinline__ bool collide_cell(float (&f)[27], const CollideParams& cp, const CellFields& cur,
                                             const ForceField& force, long long cell, int x, int y, int z,
                                             const float* temperature = nullptr) {
    const float* tp = temperature ? temperature : cur.temperature + cell;
    CollideOut o;
    const float cfx = force.fx ? force.fx[cell] : 0.0f;
    const float cfy = force.fy ? force.fy[cell] : 0.0f;
    const float cfz = force.fz ? force.fz[cell] : 0.0f;
    CellExtras ex;
    const CellExtras* exp = nullptr;
    int d = 0;
    if (cp.runtime_terms) {
        d = edge_distance(x, y, z, cp.nx, cp.ny, cp.nz);
        ex.fan_mask = cur.fan_mask ? cur.fan_mask[cell] : 0.0f;
        ex.fan_x = cur.fan_mask ? cur.fan_ux[cell] : 0.0f;
        ex.fan_y = cur.fan_mask ? cur.fan_uy[cell] : 0.0f;
        ex.fan_z = cur.fan_mask ? cur.fan_uz[cell] : 0.0f;
        ex.noise = cp.fan_noise_amp * signed_noise((unsigned long long)cell, cp.step);
        ex.nudge = state_nudge_at(cp, d);
        ex.ref_x = cur.ref_ux[cell];
        ex.ref_y = cur.ref_uy[cell];
        ex.ref_z = cur.ref_uz[cell];
        exp = &ex;
    }
    const bool ok = kExact ? exact::collide27_exact(f, cp, tp, cfx, cfy, cfz, o, exp)
                           : collide27(f, cp, tp, cfx, cfy, cfz, o, exp);
    if (ok) record_u(cur, cell, o.ux, o.uy, o.uz);
    if (ok && cp.runtime_terms) {
        const float alpha = sponge_alpha_at(cp, d);
        if (alpha > 0.0f) {
            // sponge toward the rest state (jni.cpp:2401-2411)
            const float keep = 1.0f - alpha;
#pragma unroll
            for (int q = 0; q < 27; ++q) f[q] = keep * f[q] + alpha * feq27(q, 1.0f, 0.0f, 0.0f, 0.0f);
        }
    }
    return ok;
}

// Reseed a cell into the two-buffer state (out of line: rare path).
static __device__ __noinline__ void reseed_store_ab(float* __restrict__ g_out, long long cells, long long cell,
                                                     CellFields cur, float max_speed) {
    float rho, ux, uy, uz;
    reseed_state(ReseedSource{cur.ref_p, cur.ref_ux, cur.ref_uy, cur.ref_uz, cell}, max_speed, rho, ux, uy, uz);
    record_u(cur, cell, ux, uy, uz);
#pragma unroll 1
    for (int q = 0; q < 27; ++q) g_out[(long long)q * cells + cell] = feq27(q, rho, ux, uy, uz);
}

// ---------------------------------------------------------------- pull
struct PullView {
    const float* g;
    const uint8_t* obstacle;  // mask of the streaming call
    const float* ref_p;       // pressure proxy of the streaming call (equilibrium faces)
    const FaceParams* face;   // faces of the streaming call (device memory)
    long long cells;
    int nx, ny, nz;
};

// Face value for a source outside a non-bounce-back face
// (jni.cpp:1494-1602: equilibrium, symmetry, convective outflow).
static __device__ __noinline__ float face_value(const float* __restrict__ g, const uint8_t* __restrict__ obstacle,
                                         const float* __restrict__ ref_p, const FaceParams* __restrict__ Fp,
                                         long long cells, int nx, int ny, int nz, long long cell, int x, int y, int z,
                                         int q, int sx, int sy, int sz) {
    const FaceParams& F = *Fp;
    const PullView v{g, obstacle, ref_p, Fp, cells, nx, ny, nz};
    const int face = oob_face(sx, sy, sz, nx, ny, nz);
    const int kind = F.kind[face];
    const float bounced = v.g[(long long)q_opp(q) * v.cells + cell];
    auto idx = [&](int a, int b, int c) { return ((long long)a * ny + b) * nz + c; };
    switch (kind) {
        case kHydroBounceBack:
            return bounced;
        case kHydroMovingWall:
        case kHydroVelocity:
        case kHydroPressure: {
            float rho = 1.0f + clampf_dev(v.ref_p[cell], -0.03f, 0.03f);
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
        case kHydroSymmetry: {
            const int ix = min(max(sx, 0), nx - 1), iy = min(max(sy, 0), ny - 1), iz = min(max(sz, 0), nz - 1);
            const long long src = idx(ix, iy, iz);
            return v.obstacle[src] ? bounced : v.g[(long long)q * v.cells + src];
        }
        default:
            if (kind == kHydroInheritGame && F.disable_convective) return bounced;
            break;
    }
    // Convective outflow (jni.cpp:1494-1517); also the fall-through kinds.
    const int dx = (sx < 0 || sx >= nx) ? q_cx(q) : 0;
    const int dy = (sy < 0 || sy >= ny) ? q_cy(q) : 0;
    const int dz = (sz < 0 || sz >= nz) ? q_cz(q) : 0;
    const long long s1 = idx(min(max(x + dx, 0), nx - 1), min(max(y + dy, 0), ny - 1), min(max(z + dz, 0), nz - 1));
    if (v.obstacle[s1]) return bounced;
    const float f1 = v.g[(long long)q * v.cells + s1];
    const long long s2 = idx(min(max(x + 2 * dx, 0), nx - 1), min(max(y + 2 * dy, 0), ny - 1), min(max(z + 2 * dz, 0), nz - 1));
    if (v.obstacle[s2]) return f1;
    const float f2 = v.g[(long long)q * v.cells + s2];
    return f1 + 0.15f * (f1 - f2);
}

// Pull all 27 incoming populations of one cell: S(g) at this cell.
__device__ __forceinline__ void pull27(const PullView& v, uint32_t w, long long cell, int x, int y, int z,
                                       float (&f)[27]) {
    const long long cells = v.cells;
    if (w & kFlagSelfSolid) {
#pragma unroll
        for (int q = 0; q < 27; ++q) f[q] = __ldg(v.g + (long long)q_opp(q) * cells + cell);
        return;
    }
    const int nx = v.nx, ny = v.ny, nz = v.nz;
    if (!(w & kFlagFaceSpecial)) {
        // Sources are in range after the periodic wrap, or bounce-back.
        const long long yz = (long long)ny * nz;
        int xs[3] = {x + 1, x, x - 1}, ys[3] = {y + 1, y, y - 1}, zs[3] = {z + 1, z, z - 1};
        // wrap (a non-wrapping out-of-range source is always bounce-back here)
        if (xs[0] >= nx) xs[0] -= nx;
        if (xs[2] < 0) xs[2] += nx;
        if (ys[0] >= ny) ys[0] -= ny;
        if (ys[2] < 0) ys[2] += ny;
        if (zs[0] >= nz) zs[0] -= nz;
        if (zs[2] < 0) zs[2] += nz;
        const long long X[3] = {xs[0] * yz, xs[1] * yz, xs[2] * yz};
        const long long Y[3] = {(long long)ys[0] * nz, (long long)ys[1] * nz, (long long)ys[2] * nz};
#pragma unroll
        for (int q = 0; q < 27; ++q) {
            const bool bb = (w >> q) & 1u;
            const long long src = X[q / 9] + Y[(q / 3) % 3] + zs[q % 3];
            const long long a = bb ? (long long)q_opp(q) * cells + cell : (long long)q * cells + src;
            f[q] = __ldg(v.g + a);
        }
        return;
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) {
        if ((w >> q) & 1u) {
            f[q] = v.g[(long long)q_opp(q) * cells + cell];
            continue;
        }
        int sx = x - q_cx(q), sy = y - q_cy(q), sz = z - q_cz(q);
        const bool inx = wrap_coord(sx, nx, v.face->wrap_lo[0], v.face->wrap_hi[0]);
        const bool iny = wrap_coord(sy, ny, v.face->wrap_lo[1], v.face->wrap_hi[1]);
        const bool inz = wrap_coord(sz, nz, v.face->wrap_lo[2], v.face->wrap_hi[2]);
        if (inx && iny && inz) {
            f[q] = v.g[(long long)q * cells + ((long long)sx * ny + sy) * nz + sz];
        } else {
            f[q] = face_value(v.g, v.obstacle, v.ref_p, v.face, cells, nx, ny, nz, cell, x, y, z, q, sx, sy, sz);
        }
    }
}

// ---------------------------------------------------------------- init + collide
template <bool kExact>
__global__ void __launch_bounds__(128) init_collide_kernel(int nx, int ny, int nz, CellFields cur, ForceField force,
                                                           CollideParams cp, float* __restrict__ g_out) {
    const long long cells = (long long)nx * ny * nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    float f[27];
    const bool solid = cur.obstacle[cell] != 0;
    // initialize_distributions (jni.cpp:1752-1781)
    float rho = 1.0f, ux = 0.0f, uy = 0.0f, uz = 0.0f;
    if (!solid) {
        rho = clampf_dev(1.0f + cur.ref_p[cell], 0.97f, 1.03f);
        ux = cur.ref_ux[cell]; uy = cur.ref_uy[cell]; uz = cur.ref_uz[cell];
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) f[q] = feq27(q, rho, ux, uy, uz);
    if (solid) record_u(cur, cell, 0.0f, 0.0f, 0.0f);
    int x, y, z;
    cell_xyz32(cell, ny, nz, x, y, z);
    if (!solid && !collide_cell<kExact>(f, cp, cur, force, cell, x, y, z)) {
        reseed_store_ab(g_out, cells, cell, cur, cp.max_speed);
        return;
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) g_out[(long long)q * cells + cell] = f[q];
}

template <bool kExact>
cudaError_t launch_init_collide_t(BrickDims d, CellFields cur, ForceField force, CollideParams cp, float* g_out,
                                cudaStream_t stream) {
    if (d.cells <= 0) return cudaSuccess;
    const int block = 128;
    const long long grid = (d.cells + block - 1) / block;
    init_collide_kernel<kExact><<<(unsigned)grid, block, 0, stream>>>(d.nx, d.ny, d.nz, cur, force, cp, g_out);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------- fused step (two buffers)
template <bool kExact>
__global__ void __launch_bounds__(128) step_ab_kernel(int nx, int ny, int nz, const float* __restrict__ g_in,
                                                      float* __restrict__ g_out, const uint32_t* __restrict__ flags_prev,
                                                      const uint8_t* __restrict__ obstacle_prev,
                                                      const float* __restrict__ ref_p_prev,
                                                      const FaceParams* __restrict__ F, CellFields cur,
                                                      ForceField force, CollideParams cp) {
    const long long cells = (long long)nx * ny * nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    int x, y, z;
    cell_xyz32(cell, ny, nz, x, y, z);
    float f[27];
    const PullView v{g_in, obstacle_prev, ref_p_prev, F, cells, nx, ny, nz};
    pull27(v, flags_prev[cell], cell, x, y, z, f);
    if (cur.obstacle[cell]) record_u(cur, cell, 0.0f, 0.0f, 0.0f);
    if (!cur.obstacle[cell] && !collide_cell<kExact>(f, cp, cur, force, cell, x, y, z)) {
        reseed_store_ab(g_out, cells, cell, cur, cp.max_speed);
        return;
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) g_out[(long long)q * cells + cell] = f[q];
}

template <bool kExact>
cudaError_t launch_step_ab_t(BrickDims d, const float* g_in, float* g_out, const uint32_t* flags_prev,
                           const uint8_t* obstacle_prev, const float* ref_p_prev, const FaceParams* face_prev,
                           CellFields cur, ForceField force, CollideParams cp, cudaStream_t stream) {
    if (d.cells <= 0) return cudaSuccess;
    const int block = 128;
    const long long grid = (d.cells + block - 1) / block;
    step_ab_kernel<kExact><<<(unsigned)grid, block, 0, stream>>>(d.nx, d.ny, d.nz, g_in, g_out, flags_prev, obstacle_prev,
                                                        ref_p_prev, face_prev, cur, force, cp);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------- collide only (two buffers)
// The call after a halo exchange: the streamed state f (the pull of the last
// call, with the exchanged slabs written in) already sits in f_io; collide
// it in place.
template <bool kExact>
__global__ void __launch_bounds__(128) collide_ab_kernel(int nx, int ny, int nz, float* __restrict__ f_io,
                                                         CellFields cur, ForceField force, CollideParams cp) {
    const long long cells = (long long)nx * ny * nz;
    const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= cells) return;
    if (cur.obstacle[cell]) {
        // the reference collides no solid cell; its f stays as streamed
        record_u(cur, cell, 0.0f, 0.0f, 0.0f);
        return;
    }
    float f[27];
#pragma unroll
    for (int q = 0; q < 27; ++q) f[q] = f_io[(long long)q * cells + cell];
    int x, y, z;
    cell_xyz32(cell, ny, nz, x, y, z);
    if (!collide_cell<kExact>(f, cp, cur, force, cell, x, y, z)) {
        reseed_store_ab(f_io, cells, cell, cur, cp.max_speed);
        return;
    }
#pragma unroll
    for (int q = 0; q < 27; ++q) f_io[(long long)q * cells + cell] = f[q];
}

template <bool kExact>
cudaError_t launch_collide_ab_t(BrickDims d, float* f_io, CellFields cur, ForceField force, CollideParams cp,
                                cudaStream_t stream) {
    if (d.cells <= 0) return cudaSuccess;
    const int block = 128;
    collide_ab_kernel<kExact><<<(unsigned)((d.cells + block - 1) / block), block, 0, stream>>>(d.nx, d.ny, d.nz, f_io,
                                                                                             cur, force, cp);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------- output
// write_output / strided extract semantics (jni.cpp:2535-2581, 9385-9446).
__device__ __forceinline__ void macro_out(const float (&f)[27], bool solid, float scale, float* o) {
    if (solid) { o[0] = o[1] = o[2] = o[3] = 0.0f; return; }
    RawMoments m;
    raw_moments27<false>(f, m);
    float rho = m.r000;
    if (!(isfinite(rho) && isfinite(m.r100) && isfinite(m.r010) && isfinite(m.r001))) {
        o[0] = o[1] = o[2] = o[3] = 0.0f;
        return;
    }
    rho = clampf_dev(rho, 0.97f, 1.03f);
    float ux = m.r100 / rho, uy = m.r010 / rho, uz = m.r001 / rho;
    if (!(isfinite(ux) && isfinite(uy) && isfinite(uz))) ux = uy = uz = 0.0f;
    if (fabsf(rho - 1.0f) < 1e-6f) rho = 1.0f;
    if (fabsf(ux) < 1e-7f) ux = 0.0f;
    if (fabsf(uy) < 1e-7f) uy = 0.0f;
    if (fabsf(uz) < 1e-7f) uz = 0.0f;
    o[0] = ux * scale;
    o[1] = uy * scale;
    o[2] = uz * scale;
    o[3] = clampf_dev(rho - 1.0f, -0.03f, 0.03f);
}

template <bool kExact>
__global__ void output_ab_kernel(int nx, int ny, int nz, const float* __restrict__ g, const uint32_t* __restrict__ flags,
                                 const uint8_t* __restrict__ obstacle, const float* __restrict__ ref_p,
                                 const FaceParams* __restrict__ F, OutBox b, int out_ch, float scale,
                                 float* __restrict__ out, int direct) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.count()) return;
    const int az = (int)(i % b.sz);
    const int ay = (int)((i / b.sz) % b.sy);
    const int ax = (int)(i / ((long long)b.sy * b.sz));
    const int x = min(nx - 1, b.ox + ax * b.stride), y = min(ny - 1, b.oy + ay * b.stride),
              z = min(nz - 1, b.oz + az * b.stride);
    const long long cells = (long long)nx * ny * nz;
    const long long cell = ((long long)x * ny + y) * nz + z;
    float f[27];
    const PullView v{g, obstacle, ref_p, F, cells, nx, ny, nz};
    const uint32_t w = flags[cell];
    if (direct) {  // g holds the streamed state itself
#pragma unroll
        for (int q = 0; q < 27; ++q) f[q] = g[(long long)q * cells + cell];
    } else {
        pull27(v, w, cell, x, y, z, f);
    }
    float o[4];
    if (kExact) exact::macro_out_exact(f, (w & kFlagSelfSolid) != 0, scale, o);
    else macro_out(f, (w & kFlagSelfSolid) != 0, scale, o);
    float* dst = out + i * out_ch;
    dst[0] = o[0]; dst[1] = o[1]; dst[2] = o[2]; dst[3] = o[3];
    for (int c = 4; c < out_ch; ++c) dst[c] = 0.0f;
}

template <bool kExact>
cudaError_t launch_output_ab_t(BrickDims d, const float* g, const uint32_t* flags, const uint8_t* obstacle,
                             const float* ref_p, const FaceParams* face, OutBox box, int out_channels,
                             float velocity_scale, float* out, cudaStream_t stream, int direct = 0) {
    const long long n = box.count();
    if (n <= 0) return cudaSuccess;
    const int block = 128;
    output_ab_kernel<kExact><<<(unsigned)((n + block - 1) / block), block, 0, stream>>>(
        d.nx, d.ny, d.nz, g, flags, obstacle, ref_p, face, box, out_channels, velocity_scale, out, direct);
    count_launch();
    return cudaGetLastError();
}

}  // namespace aero
