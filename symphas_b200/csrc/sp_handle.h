/*
 * sp_handle.h -- the handle behind the C ABI (private to the library): device
 * buffers, per-instance geometry, the chosen kernel and its launch state.
 */
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/symphas_b200.h"
#include "sp_registry.h"

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
// geometry and parameters of one instance: every instance of a batch has the
// same, the members of an ensemble each their own
struct InstGeo {
  int n[3] = {1, 1, 1};
  long long pitch = 0, ly = 0, lz = 1, plane = 0, felems = 0;
  size_t off = 0;  // element offset of the instance's field 0 in each buffer
  int model = 0;   // SP_MODEL_* of the instance
  int kind = 0;    // 0 = first model of the kernel, 1 = second (ensembles)
  double dt = 0.0;
  double coeff[8] = {1, 1, 1, 1, 1, 1, 1, 1};
  long long sites() const { return (long long)n[0] * n[1] * n[2]; }
};

struct sp_handle {
  sp_desc d{};
  std::vector<InstGeo> geo;  // [batch]
  bool ensemble = false;     // members differ in size, model or parameters
  const sp::KernelInfo* ki = nullptr;   // the chosen tile variant
  std::vector<sp::KernelInfo> variants;  // every tile shape built for this kernel
  int variant = 0;
  int nf = 1, batch = 1, dim = 2;
  int h[3] = {0, 0, 0};  // halo of every instance
  // geometry of instance 0 (the geometry of every instance of a 3D batch)
  int n[3] = {1, 1, 1};
  long long pitch = 0, ly = 0, lz = 1, plane = 0, felems = 0;
  size_t esz = 8;
  char* buf[2] = {nullptr, nullptr};
  CUtensorMap* maps_d[2] = {nullptr, nullptr};
  void** outs_d[2] = {nullptr, nullptr};
  int cur = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sms = 148;
  // 3D grid
  int ntx = 1, nty = 1, nzc = 1, zchunk = 1;
  // 2D persistent grid
  void* inst2_d = nullptr;
  int2* items_d = nullptr;
  int nitems = 0;
  int* ctr_d = nullptr;
  int grid2 = 1;
  // scratch for reductions
  double* partial_d = nullptr;
  size_t partial_n = 0;
  double* result_d = nullptr;
  double* result_h = nullptr;
  int* err_d = nullptr;
  // graphs replaying GRAPH_STEPS steps from each buffer parity
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  bool graphs = true;  // false once capture failed on this stream
  long long launches = 0;
  // mass conservation of field 0 (sp_conserve_mass): every `conserve_every`
  // steps, restore each instance's mass to its target (2 doubles per instance:
  // the target mass and the energy reduced alongside it)
  int conserve_every = 0, since_conserve = 0;
  unsigned long long conserve_passes = 0;  // seeds the stochastic rounding
  double* mass_target_d = nullptr;
  double* cons_d = nullptr;  // [2] the latest reduction
  std::string err;
};

// padded field `f` of instance `inst` in buffer `which`, and its interior origin
inline char* field_base(sp_handle* H, int which, int inst, int f) {
  const InstGeo& g = H->geo[inst];
  return H->buf[which] + (g.off + size_t(f) * g.felems) * H->esz;
}
inline char* field_origin(sp_handle* H, int which, int inst, int f) {
  const InstGeo& g = H->geo[inst];
  return field_base(H, which, inst, f) +
         size_t((H->dim == 3 ? H->h[2] : 0) * g.plane + H->h[1] * g.pitch + H->h[0]) * H->esz;
}
