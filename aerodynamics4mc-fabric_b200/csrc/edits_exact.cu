// Block edits and the boundary-reference shell of an in-place brick (see
// edits.cuh). Built with --fmad=false: the shell's arithmetic rounds
// operation by operation, like the oracle's float instantiation.
#include "edits.cuh"

namespace aero {
namespace {

__global__ void patch_mask_kernel(uint8_t* __restrict__ next, long long n_cells, const int* __restrict__ cells,
                                  const uint8_t* __restrict__ solid, int count) {
    // one thread walks the patches in order: duplicates resolve like the
    // reference's sequential loop, and block edits are few
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int i = 0; i < count; ++i) {
        const int c = cells[i];
        if (c >= 0 && (long long)c < n_cells) next[c] = solid[i] ? 1 : 0;
    }
}

template <class S>
__global__ void patch_reset_kernel(typename S::T* __restrict__ f, IpArgs a, const int* __restrict__ cells, int count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const PadGeom G = a.g;
    const long long n_cells = (long long)G.nx * G.ny * G.nz;
    const int cell = cells[i];
    if (cell < 0 || (long long)cell >= n_cells) return;
    const uint32_t w = a.flags_prev[cell];
    if (w & kFlagSelfSolid) {
        if (!a.solid_f) return;  // without the store every solid cell is at rest already
#pragma unroll 1
        for (int q = 0; q < 27; ++q) a.solid_f[(long long)q * n_cells + cell] = feq27(q, 1.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    int x, y, z;
    cell_xyz32(cell, G.ny, G.nz, x, y, z);
    const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
    const int own = pad_index(G, x, y, z);
#pragma unroll 1
    for (int q = 0; q < 27; ++q) {
        int c, d;
        incoming_slot(o, own, q, a.parity, (w >> q) & 1u, c, d);
        S::store(f + (long long)d * G.pcells + c, q, feq27(q, 1.0f, 0.0f, 0.0f, 0.0f), a.sc);
    }
}

template <class S>
__global__ void shell_relax_kernel(typename S::T* __restrict__ f, IpArgs a, const ShellCell* __restrict__ shell, int count,
                                   int layers, float relaxation) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const ShellCell sc = shell[i];
    const PadGeom G = a.g;
    const uint32_t w = a.flags_prev[sc.cell];
    if (w & kFlagSelfSolid) return;
    int x, y, z;
    cell_xyz32(sc.cell, G.ny, G.nz, x, y, z);
    const NeighbourOffsets o = neighbour_offsets(G, x, y, z);
    const int own = pad_index(G, x, y, z);
    float fl[27];
    long long slot[27];
    float rho = 0.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
#pragma unroll 1
    for (int q = 0; q < 27; ++q) {
        int c, d;
        incoming_slot(o, own, q, a.parity, (w >> q) & 1u, c, d);
        slot[q] = (long long)d * G.pcells + c;
        fl[q] = S::load(f + slot[q], q, a.sc);
        rho += fl[q];
        jx += fl[q] * (float)q_cx(q);
        jy += fl[q] * (float)q_cy(q);
        jz += fl[q] * (float)q_cz(q);
    }
    if (!(isfinite(rho) && isfinite(jx) && isfinite(jy) && isfinite(jz))) return;
    rho = clampf_dev(rho, 0.97f, 1.03f);
    float ux = jx / rho, uy = jy / rho, uz = jz / rho;
    const float s2 = ux * ux + uy * uy + uz * uz;
    if (!isfinite(s2) || s2 > a.cp.max_speed * a.cp.max_speed) {
        if (!isfinite(s2) || s2 <= 0.0f) {
            ux = uy = uz = 0.0f;
        } else {
            const float k = a.cp.max_speed / sqrtf(s2);
            ux *= k; uy *= k; uz *= k;
        }
    }
    const float t = 1.0f - (float)(sc.layer - 1) / fmaxf(1.0f, (float)layers);
    const float alpha = clampf_dev(relaxation * t * t, 0.0f, 0.5f);
    const float rho_t = clampf_dev(1.0f + clampf_dev(sc.p, -0.03f, 0.03f), 0.97f, 1.03f);
    const float nux = ux + alpha * (sc.ux - ux), nuy = uy + alpha * (sc.uy - uy), nuz = uz + alpha * (sc.uz - uz);
    const float nrho = rho + alpha * (rho_t - rho);
#pragma unroll 1
    for (int q = 0; q < 27; ++q) {
        const float v = fl[q] + (feq27(q, nrho, nux, nuy, nuz) - feq27(q, rho, ux, uy, uz));
        S::store(f + slot[q], q, v, a.sc);
    }
}

template <class S>
cudaError_t reset_t(void* f, const IpArgs& a, const int* cells, int count, cudaStream_t s) {
    patch_reset_kernel<S><<<(unsigned)((count + 127) / 128), 128, 0, s>>>(static_cast<typename S::T*>(f), a, cells, count);
    count_launch();
    return cudaGetLastError();
}

template <class S>
cudaError_t shell_t(void* f, const IpArgs& a, const ShellCell* shell, int count, int layers, float relaxation,
                    cudaStream_t s) {
    shell_relax_kernel<S><<<(unsigned)((count + 127) / 128), 128, 0, s>>>(static_cast<typename S::T*>(f), a, shell, count,
                                                                         layers, relaxation);
    count_launch();
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_patch_mask(const uint8_t* cur, uint8_t* next, long long n_cells, const int* cells,
                              const uint8_t* solid, int count, cudaStream_t s) {
    if (cur != next) {
        cudaError_t e = cudaMemcpyAsync(next, cur, (size_t)n_cells, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return e;
    }
    if (count <= 0) return cudaSuccess;
    patch_mask_kernel<<<1, 32, 0, s>>>(next, n_cells, cells, solid, count);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_patch_reset(int storage, void* f, const IpArgs& a, const int* cells, int count, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    if (storage == 0) return reset_t<StoreF32>(f, a, cells, count, s);
    if (storage == 1) return reset_t<StoreF16Dev>(f, a, cells, count, s);
    return reset_t<StoreI16Dev>(f, a, cells, count, s);
}

cudaError_t launch_shell_relax(int storage, void* f, const IpArgs& a, const ShellCell* shell, int count, int layers,
                               float relaxation, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    if (storage == 0) return shell_t<StoreF32>(f, a, shell, count, layers, relaxation, s);
    if (storage == 1) return shell_t<StoreF16Dev>(f, a, shell, count, layers, relaxation, s);
    return shell_t<StoreI16Dev>(f, a, shell, count, layers, relaxation, s);
}

}  // namespace aero
