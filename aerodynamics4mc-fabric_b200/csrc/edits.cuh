// Block edits and the boundary-reference shell of an in-place brick
// (aero_lbm_patch_d3q27_f16_static_cells_rect, aero_lbm_set/clear_d3q27_f16_
// boundary_shell_rect; native/src/aero_lbm_jni.cpp:4725-4778, 6156-6260,
// 6443-6540, 9905-10037).
#pragma once

#include <cuda_runtime.h>

#include "d3q27_inplace.cuh"

namespace aero {

// The mask of the next call: next[c] = cur[c], then next[cells[i]] = solid[i]
// for every in-range patch (later patches of the same cell win, as the
// reference's host loop does).
cudaError_t launch_patch_mask(const uint8_t* cur, uint8_t* next, long long n_cells, const int* cells,
                              const uint8_t* solid, int count, cudaStream_t s);

// Reset every patched cell to rest: a cell fluid in the classification the
// next step streams with gets rest populations in its incoming slots, a
// solid one in the solid-cell store (storage 0 FP32, 1 IEEE half, 2 fixed
// point).
cudaError_t launch_patch_reset(int storage, void* f, const IpArgs& a, const int* cells, int count, cudaStream_t s);

// One shell cell: its layer (1 = outermost) and the target state.
struct ShellCell {
    int cell;
    int layer;
    float ux, uy, uz, p;
};

// Relax the macroscopic state of each shell cell toward its target before
// the next collision: with rho = sum f, u = j / clamp(rho), speed clamp,
// alpha = clamp(relaxation * t^2, 0, 0.5), t = 1 - (layer - 1) / layers, the
// populations move by feq(rho + alpha (rho_t - rho), u + alpha (u_t - u)) -
// feq(rho, u), which sets the cell's mass and momentum to the nudged values
// and keeps its non-equilibrium part (the nudge of jni.cpp:4536-4551 written
// as an equilibrium shift for the cumulant collision).
cudaError_t launch_shell_relax(int storage, void* f, const IpArgs& a, const ShellCell* shell, int count, int layers,
                               float relaxation, cudaStream_t s);

}  // namespace aero
