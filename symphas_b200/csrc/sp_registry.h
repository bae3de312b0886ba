/*
 * sp_registry.h -- table of the fused-step kernels built into the library.
 *
 * Each entry is one (model, form, dimension, dtype, stencil point set) lowered
 * at build time into a kernel instantiation; sp_create looks its description
 * up here, the way SymPhas resolves model_X_t<D, SolverFT<Stencil..>> at
 * compile time (sol/inc/modelmacros.h:597-626, examples/solvers/solverft.h:219-239).
 */
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace sp {

struct KernelKey {
  int model, form, dim, dtype, lp, gp, bp;
};

struct KernelInfo {
  int nf;       // fields
  int ns;       // staged operands
  int R;        // halo in y and z (stencil reach of the lowered model)
  int hx;       // halo in x (R rounded up to 16 bytes)
  int tx, ty;   // tile
  int threads;  // threads per CTA
  size_t smem;  // dynamic shared memory per CTA
  // launches one fused step; `params` is StepParams<T> (3D) or Step2Params<T>
  // (2D); `grid` is ignored for 2D (persistent grid from `ctas`)
  cudaError_t (*launch)(const void* params, dim3 grid, cudaStream_t s);
  // CTAs of this kernel resident per SM (for sizing persistent grids)
  int (*occupancy)();
};

void register_kernel(const KernelKey& key, const KernelInfo& info);
const KernelInfo* find_kernel(const KernelKey& key);
void register_all_kernels();

}  // namespace sp
