// Halo exchange between overlapping bricks (see halo_exact.cu).
#pragma once

#include <cuda_runtime.h>

#include "d3q27_kernels.cuh"
#include "inplace27.cuh"

namespace aero {

// One direction of the exchange: per axis the source start, destination
// start and size (cells).
struct HaloSlab {
    int src[3], dst[3], size[3];
};

// halo_exchange_slab_bounds with the reference's halo clamp
// (max(1, min(halo_layers, n / 2 - 1)), core n - 2 halo > 0).
bool halo_slabs(int n, int halo_layers, int ox, int oy, int oz, HaloSlab& first_to_second, HaloSlab& second_to_first);

// An in-place context as the exchange sees it.
struct HaloIpSide {
    void* f;
    PadGeom g;
    const uint32_t* flags;  // classification of the last call (bounce bits, solid cells)
    int parity;             // parity of the next step
    Fp16Scale sc;
    float* solid_f;         // populations of solid cells (IpArgs::solid_f), or null
};

// storage: 0 FP32, 1 IEEE-half deviations, 2 16-bit fixed point (both sides alike).
cudaError_t launch_halo_ip(int storage, const HaloIpSide& a, const HaloIpSide& b, const HaloSlab& ab,
                           const HaloSlab& ba, cudaStream_t s);
cudaError_t launch_materialise_ab(BrickDims d, const float* g, const uint32_t* flags, const uint8_t* obstacle,
                                  const float* ref_p, const FaceParams* face, float* f_out, cudaStream_t s);
// comps component-major arrays of `cells` floats each, copied along one slab.
cudaError_t launch_halo_soa(const float* a, float* b, long long cells, int ny, int nz, int comps, const HaloSlab& ab,
                            cudaStream_t s);

// Many exchanges in one launch: each job copies one slab in one direction.
// The jobs live in device memory (the caller uploads them); jobs of one launch
// must not write what another reads (true for the face slabs of a brick
// world: writes go to the outermost layer along the exchange axis, reads come
// from inner layers).
struct HaloIpJob {
    HaloIpSide src, dst;
    HaloSlab slab;
};
struct HaloSoaJob {
    const float* src;
    float* dst;
    long long cells;
    int ny, nz;
    HaloSlab slab;
};
// max_slab: the largest slab (cells) of the jobs (sets the grid).
cudaError_t launch_halo_ip_batch(int storage, const HaloIpJob* jobs, int njobs, int max_slab, cudaStream_t s);
cudaError_t launch_halo_soa_batch(const HaloSoaJob* jobs, int njobs, int max_slab, cudaStream_t s);

}  // namespace aero
