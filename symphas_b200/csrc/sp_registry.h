/*
 * sp_registry.h -- table of the fused-step kernels built into the library.
 *
 * Each entry is one (model, form, dimension, dtype, stencil point set) lowered
 * at build time into one or more kernel instantiations that differ only in
 * their tile shape; sp_create looks the description up here, the way SymPhas
 * resolves model_X_t<D, SolverFT<Stencil..>> at compile time
 * (sol/inc/modelmacros.h:597-626, examples/solvers/solverft.h:219-239), and
 * sp_autotune picks the fastest tile shape on the current GPU.
 */
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <vector>

namespace sp {

struct KernelKey {
  int model, form, dim, dtype, lp, gp, bp;
};
// kernel keys carry a point set of a 4th-order stencil (Stencil2d4h) as
// SP_PTS4 + points: its point counts overlap the 2nd-order ones (lap 9, bilap 21)
constexpr int SP_PTS4 = 1000;

struct KernelInfo {
  int nf;       // fields
  int ns;       // staged operands
  int R;        // halo in y and z (stencil reach of the lowered model)
  int hx;       // halo in x (R rounded up to 16 bytes, or the stage ring)
  int tx, ty;   // tile
  int spt, pd;  // rows per thread, TMA stages in flight
  int threads;  // threads per CTA
  size_t smem;  // dynamic shared memory per CTA
  // launches one fused step; `params` is StepParams<T> (3D) or Step2Params<T>
  // (2D); `grid` is ignored for 2D (persistent grid from `ctas`)
  cudaError_t (*launch)(const void* params, dim3 grid, cudaStream_t s);
  // CTAs of this kernel resident per SM (for sizing grids)
  int (*occupancy)();
  // x halo inside the TMA box (-1: the field's x halo); a kernel that takes
  // its x neighbours from elsewhere loads the bare rows
  int box_hx = -1;
  // nonzero: the kernel runs only on 3D grids of this x extent, periodic in x
  int nx_only = 0;
  // steps one launch can advance (temporally blocked kernels: > 1); such a
  // kernel runs only on 2D grids periodic on both axes whose x extents are
  // multiples of x_multiple
  int kt = 1;
  int x_multiple = 1;
};

// appends a tile variant for `key` (the first registered is the default)
void register_kernel(const KernelKey& key, const KernelInfo& info);
const std::vector<KernelInfo>* find_kernels(const KernelKey& key);
void register_all_kernels();

}  // namespace sp
