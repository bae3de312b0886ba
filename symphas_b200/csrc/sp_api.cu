/*
 * sp_api.cu -- implementation of the C ABI declared in include/symphas_b200.h.
 *
 * Host-side plumbing only: validation, device buffers, TMA descriptors, the
 * step loop (with CUDA-graph replay of long step sequences), uploads,
 * downloads and reductions.  The numerical work is in the kernels of
 * sp_kernels.cuh, instantiated in sp_inst_*.cu.
 */
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/symphas_b200.h"
#include "sp_aux.cuh"
#include "sp_kernels.cuh"
#include "sp_registry.h"

namespace sp {

// ---------------------------------------------------------------------------
// kernel registry
// ---------------------------------------------------------------------------
namespace {
using KeyT = std::tuple<int, int, int, int, int, int, int>;
std::map<KeyT, std::vector<KernelInfo>>& table() {
  static std::map<KeyT, std::vector<KernelInfo>> t;
  return t;
}
KeyT tup(const KernelKey& k) { return KeyT{k.model, k.form, k.dim, k.dtype, k.lp, k.gp, k.bp}; }
}  // namespace

void register_kernel(const KernelKey& key, const KernelInfo& info) {
  table()[tup(key)].push_back(info);
}
const std::vector<KernelInfo>* find_kernels(const KernelKey& key) {
  auto it = table().find(tup(key));
  return it == table().end() ? nullptr : &it->second;
}
// the built-in kernel sets (sp_inst_exact.cu, sp_inst_fused.cu,
// sp_inst_wide.cu); weak, so a program that compiles this runtime with only
// its own models (the C++ front end, symphas_model.hpp) links without them
void register_exact_kernels() __attribute__((weak));
void register_fused_kernels() __attribute__((weak));
void register_wide_kernels() __attribute__((weak));
void register_all_kernels() {
  static std::once_flag once;
  std::call_once(once, [] {
    if (register_exact_kernels) register_exact_kernels();
    if (register_fused_kernels) register_fused_kernels();
    if (register_wide_kernels) register_wide_kernels();
  });
}

// ---------------------------------------------------------------------------
// seeded initial values: SplitMix64 counter stream, bit-identical to the oracle
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_seed(T* org, int dim, int n0, int n1, int n2, int h0, int h1, int h2,
                       long long pitch, long long plane, unsigned long long seed, double lo,
                       double hi) {
  const long long total = (long long)n0 * n1 * (dim == 3 ? n2 : 1);
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    unsigned long long z = seed + (unsigned long long)(id + 1) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    const double u = __dmul_rn(double(z >> 11), 1.0 / 9007199254740992.0);
    const double v = __dadd_rn(lo, __dmul_rn(__dsub_rn(hi, lo), u));
    const long long i = id % n0, j = (id / n0) % n1, k = id / ((long long)n0 * n1);
    org[(k + (dim == 3 ? h2 : 0)) * plane + (j + h1) * pitch + (i + h0)] = T(v);
  }
}

}  // namespace sp

#include "sp_handle.h"

namespace {

constexpr int GRAPH_STEPS = 32;
constexpr int RED_THREADS = 256;

thread_local std::string g_create_error;

int fail(sp_handle* H, int code, const std::string& msg) {
  if (H) H->err = msg;
  return code;
}
int cuda_fail(sp_handle* H, cudaError_t e, const char* what) {
  return fail(H, SP_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define SP_CUDA(H, call)                              \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(H, e_, #call); \
  } while (0)

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiled) nullptr;
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

int energy_kind(int model) {
  switch (model) {
    case SP_MODEL_AMK:
    case SP_MODEL_BMK: return 1;
    case SP_MODEL_C: return 2;
    default: return 0;
  }
}


// padded layout of an instance of extents n: x padded to whole 16-byte units
// past the halo, each field rounded up to 64 elements (256 or 512 bytes)
void set_geometry(sp_handle* H, InstGeo& g, const int n[3]) {
  for (int a = 0; a < 3; ++a) g.n[a] = (a < H->dim) ? n[a] : 1;
  const int va = int(16 / H->esz);
  g.pitch = ((g.n[0] + 2 * H->h[0] + va - 1) / va) * va;
  g.ly = g.n[1] + 2 * H->h[1];
  g.lz = H->dim == 3 ? g.n[2] + 2 * H->h[2] : 1;
  g.plane = g.pitch * g.ly;
  g.felems = ((g.plane * g.lz + 63) / 64) * 64;
}

int check_err_flag(sp_handle* H) {
  int e = 0;
  SP_CUDA(H, cudaMemcpyAsync(&e, H->err_d, sizeof(int), cudaMemcpyDeviceToHost, H->stream));
  SP_CUDA(H, cudaStreamSynchronize(H->stream));
  if (e != 0) {
    cudaMemsetAsync(H->err_d, 0, sizeof(int), H->stream);
    // a CTA that gave up left the 2D work queue without re-arming it
    if (H->ctr_d) cudaMemsetAsync(H->ctr_d, 0, 2 * sizeof(int), H->stream);
    return fail(H, SP_ETIMEOUT, "a kernel gave up waiting for a TMA tile (device error flag set)");
  }
  return SP_OK;
}

// one launch of the configured kernel: `steps` steps (1 unless the kernel is
// temporally blocked; then at most its kt), from the current buffer into the
// other; `advance` false leaves the current buffer current (timing runs)
template <class T>
int launch_step_t(sp_handle* H, int rhs_only, double* partial, int steps, bool advance) {
  const int src = H->cur, dst = H->cur ^ 1;
  const double divh = 1.0 / H->d.h;
  const double divh2 = divh * divh, divh3 = divh * divh2, divh4 = divh2 * divh2;
  cudaError_t e;
  if (H->dim == 3) {
    sp::StepParams<T> p{};
    p.maps = H->maps_d[src];
    p.out = reinterpret_cast<T* const*>(H->outs_d[dst]);
    for (int a = 0; a < 3; ++a) {
      p.n[a] = H->n[a];
      p.h[a] = H->h[a];
      p.per[a] = H->d.boundary[2 * a] == SP_PERIODIC;
    }
    p.pitch = H->pitch;
    p.plane = H->plane;
    p.ntx = H->ntx;
    p.nty = H->nty;
    p.zchunk = H->zchunk;
    p.rhs_only = rhs_only;
    p.dt = T(H->d.dt);
    p.divh2 = T(divh2);
    p.divh3 = T(divh3);
    p.divh4 = T(divh4);
    for (int i = 0; i < 8; ++i) p.coef[i] = T(H->d.coeff[i]);
    p.partial = partial;
    p.err = H->err_d;
    e = H->ki->launch(&p, dim3(H->ntx * H->nty, H->nzc, H->batch), H->stream);
  } else {
    sp::Step2Params<T> p{};
    p.maps = H->maps_d[src];
    p.out = reinterpret_cast<T* const*>(H->outs_d[dst]);
    p.inst = static_cast<const sp::Inst2<T>*>(H->inst2_d);
    p.items = H->items_d;
    p.nitems = H->nitems;
    p.ctr = H->ctr_d;
    p.rhs_only = rhs_only;
    p.hx = H->h[0];
    p.hy = H->h[1];
    p.partial = partial;
    p.err = H->err_d;
    p.in = reinterpret_cast<const T* const*>(H->outs_d[src]);
    p.tsteps = steps;
    e = H->ki->launch(&p, dim3(H->grid2), H->stream);
  }
  if (e != cudaSuccess) return cuda_fail(H, e, "fused step launch");
  ++H->launches;
  if (!rhs_only && advance) H->cur = dst;
  return SP_OK;
}

int launch_step(sp_handle* H, int rhs_only, double* partial, int steps = 1, bool advance = true) {
  if (steps < 1 || steps > H->ki->kt || (rhs_only && steps != 1))
    return fail(H, SP_EINVAL, "steps per launch outside the kernel's range");
  return H->esz == 4 ? launch_step_t<float>(H, rhs_only, partial, steps, advance)
                     : launch_step_t<double>(H, rhs_only, partial, steps, advance);
}

template <class T>
int fill_halo_t(sp_handle* H, int which, int inst, int f) {
  const InstGeo& g = H->geo[inst];
  sp::HaloParams<T> p{};
  p.org = reinterpret_cast<T*>(field_base(H, which, inst, f));
  p.dim = H->dim;
  for (int a = 0; a < 3; ++a) {
    p.n[a] = g.n[a];
    p.h[a] = H->h[a];
  }
  p.pitch = g.pitch;
  p.plane = g.plane;
  for (int s = 0; s < 6; ++s) {
    p.bc[s] = H->d.boundary[s];
    p.bv[s] = T(H->d.boundary_value[s]);
  }
  const long long L0 = g.n[0] + 2LL * H->h[0], L1 = g.n[1] + 2LL * H->h[1];
  const long long n2 = H->dim == 3 ? g.n[2] : 1, h2 = H->dim == 3 ? H->h[2] : 0;
  const long long cells = 2 * h2 * L0 * L1 + n2 * 2 * H->h[1] * L0 + n2 * g.n[1] * 2 * H->h[0];
  const int blocks = int(std::min<long long>(H->sms * 4LL, (cells + 255) / 256));
  sp::k_fill_halo<T><<<blocks, 256, 0, H->stream>>>(p);
  SP_CUDA(H, cudaGetLastError());
  return SP_OK;
}

// every instance's halo of field f in one launch (instances of equal extents)
template <class T>
int fill_halo_batch_t(sp_handle* H, int which, int f) {
  const InstGeo& g = H->geo[0];
  sp::HaloParams<T> p{};
  p.org = reinterpret_cast<T*>(field_base(H, which, 0, f));
  p.dim = H->dim;
  for (int a = 0; a < 3; ++a) {
    p.n[a] = g.n[a];
    p.h[a] = H->h[a];
  }
  p.pitch = g.pitch;
  p.plane = g.plane;
  for (int s = 0; s < 6; ++s) {
    p.bc[s] = H->d.boundary[s];
    p.bv[s] = T(H->d.boundary_value[s]);
  }
  p.inst_stride = (long long)H->nf * g.felems;
  const long long L0 = g.n[0] + 2LL * H->h[0], L1 = g.n[1] + 2LL * H->h[1];
  const long long n2 = H->dim == 3 ? g.n[2] : 1, h2 = H->dim == 3 ? H->h[2] : 0;
  const long long cells = 2 * h2 * L0 * L1 + n2 * 2 * H->h[1] * L0 + n2 * g.n[1] * 2 * H->h[0];
  const int blocks = int(std::min<long long>(std::max(1LL, H->sms * 4LL / H->batch) , (cells + 255) / 256));
  sp::k_fill_halo<T><<<dim3(std::max(blocks, 1), H->batch), 256, 0, H->stream>>>(p);
  SP_CUDA(H, cudaGetLastError());
  return SP_OK;
}

int fill_halo(sp_handle* H, int which, int inst, int f) {
  return H->esz == 4 ? fill_halo_t<float>(H, which, inst, f)
                     : fill_halo_t<double>(H, which, inst, f);
}

// after new interior values: the halo of the current buffer, and the constant
// (Dirichlet) halo of the other buffer, which the step kernels never write
int refresh_halos(sp_handle* H, int inst, int f) {
  if (int rc = fill_halo(H, H->cur ^ 1, inst, f)) return rc;
  return fill_halo(H, H->cur, inst, f);
}

int validate(const sp_desc* d, std::string& why) {
  if (!d) return why = "null description", SP_EINVAL;
  if (d->dim != 2 && d->dim != 3) return why = "dim must be 2 or 3", SP_EINVAL;
  for (int a = 0; a < d->dim; ++a)
    if (d->n[a] < 4 || d->n[a] > (1 << 16)) return why = "each extent must be in [4, 65536]", SP_EINVAL;
  if (d->dtype != SP_F32 && d->dtype != SP_F64) return why = "dtype must be SP_F32 or SP_F64", SP_EINVAL;
  if (d->form != SP_FORM_EXACT && d->form != SP_FORM_FUSED) return why = "form must be exact or fused", SP_EINVAL;
  if (!(d->h > 0.0)) return why = "grid spacing h must be positive", SP_EINVAL;
  if (d->batch < 1) return why = "batch must be >= 1", SP_EINVAL;
  if (d->accuracy != 0 && d->accuracy != 2 && d->accuracy != 4)
    return why = "accuracy must be 2 (Stencil2d2h / Stencil3d2h) or 4 (Stencil2d4h)", SP_EINVAL;
  if (d->accuracy == 4 && d->dim != 2)
    return why = "4th-order stencils are two-dimensional (Stencil2d4h)", SP_EINVAL;
  for (int a = 0; a < d->dim; ++a) {
    const int l = d->boundary[2 * a], r = d->boundary[2 * a + 1];
    if ((l != SP_PERIODIC && l != SP_DIRICHLET) || (r != SP_PERIODIC && r != SP_DIRICHLET))
      return why = "boundary must be SP_PERIODIC or SP_DIRICHLET", SP_EINVAL;
    if ((l == SP_PERIODIC) != (r == SP_PERIODIC))
      return why = "a periodic axis must be periodic on both sides", SP_EINVAL;
  }
  return SP_OK;
}

void release(sp_handle* H) {
  if (!H) return;
  if (H->stream) cudaStreamSynchronize(H->stream);
  for (int k = 0; k < 2; ++k) {
    if (H->gexec[k]) cudaGraphExecDestroy(H->gexec[k]);
    cudaFree(H->buf[k]);
    cudaFree(H->maps_d[k]);
    cudaFree(H->outs_d[k]);
  }
  cudaFree(H->inst2_d);
  cudaFree(H->items_d);
  cudaFree(H->ctr_d);
  cudaFree(H->partial_d);
  cudaFree(H->result_d);
  cudaFree(H->err_d);
  cudaFree(H->mass_target_d);
  cudaFree(H->cons_d);
  if (H->result_h) cudaFreeHost(H->result_h);
  if (H->own_stream && H->stream) cudaStreamDestroy(H->stream);
  delete H;
}

template <class T>
int setup_2d_t(sp_handle* H) {
  std::vector<sp::Inst2<T>> ip(H->batch);
  const double divh = 1.0 / H->d.h;
  const double divh2 = divh * divh, divh3 = divh * divh2, divh4 = divh2 * divh2;
  const int tx = H->ki->tx, ty = H->ki->ty;
  for (int i = 0; i < H->batch; ++i) {
    const InstGeo& g = H->geo[i];
    sp::Inst2<T>& q = ip[i];
    q.n[0] = g.n[0];
    q.n[1] = g.n[1];
    q.per[0] = H->d.boundary[0] == SP_PERIODIC;
    q.per[1] = H->d.boundary[2] == SP_PERIODIC;
    q.pitch = g.pitch;
    q.ntx = (g.n[0] + tx - 1) / tx;
    q.kind = g.kind;
    q.dt = T(g.dt);
    q.divh2 = T(divh2);
    q.divh3 = T(divh3);
    q.divh4 = T(divh4);
    for (int c = 0; c < 8; ++c) q.coef[c] = T(g.coeff[c]);
  }
  cudaFree(H->inst2_d);
  cudaFree(H->items_d);
  H->inst2_d = nullptr;
  H->items_d = nullptr;
  SP_CUDA(H, cudaMalloc(&H->inst2_d, sizeof(sp::Inst2<T>) * H->batch));
  SP_CUDA(H, cudaMemcpy(H->inst2_d, ip.data(), sizeof(sp::Inst2<T>) * H->batch,
                        cudaMemcpyHostToDevice));
  // work items (instance, tile); the persistent CTAs take them in this order,
  // so the costlier ones go first (the second model of an ensemble stages an
  // operand, and larger instances hold more tiles) and the cheap ones fill
  // the tail of the step
  std::vector<int> order(H->batch);
  for (int i = 0; i < H->batch; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    const InstGeo &gx = H->geo[x], &gy = H->geo[y];
    if (gx.kind != gy.kind) return gx.kind > gy.kind;
    return gx.sites() > gy.sites();
  });
  std::vector<int2> items;
  for (int i : order) {
    const int tiles = ip[i].ntx * ((H->geo[i].n[1] + ty - 1) / ty);
    // the tile's coordinates packed as x | y << 16 (sp::Step2Params::items)
    for (int t = 0; t < tiles; ++t)
      items.push_back(make_int2(i, (t % ip[i].ntx) | ((t / ip[i].ntx) << 16)));
  }
  H->nitems = int(items.size());
  H->ntx = ip[0].ntx;
  H->nty = (H->geo[0].n[1] + ty - 1) / ty;
  if (H->batch > 1) {
    SP_CUDA(H, cudaMalloc(&H->items_d, sizeof(int2) * items.size()));
    SP_CUDA(H, cudaMemcpy(H->items_d, items.data(), sizeof(int2) * items.size(),
                          cudaMemcpyHostToDevice));
  }
  if (!H->ctr_d) {
    SP_CUDA(H, cudaMalloc(&H->ctr_d, 2 * sizeof(int)));
    SP_CUDA(H, cudaMemset(H->ctr_d, 0, 2 * sizeof(int)));
  }
  const int occ = H->ki->occupancy();
  H->grid2 = std::max(1, std::min(H->sms * occ, H->nitems));
  return SP_OK;
}

// whether tile variant v can run this handle's grid (row kernels need every
// instance to be a 3D grid of their x extent, periodic in x)
bool applicable(const sp_handle* H, int v) {
  const sp::KernelInfo& k = H->variants[v];
  if (k.kt > 1) {
    // temporally blocked: 2D, periodic on both axes, x extents in whole copies
    if (H->dim != 2) return false;
    for (int s = 0; s < 4; ++s)
      if (H->d.boundary[s] != SP_PERIODIC) return false;
    for (const InstGeo& g : H->geo)
      if (g.n[0] % k.x_multiple != 0) return false;
  }
  if (k.nx_only == 0) return true;
  if (H->dim != 3 || H->d.boundary[0] != SP_PERIODIC) return false;
  for (const InstGeo& g : H->geo)
    if (g.n[0] != k.nx_only) return false;
  return true;
}

// TMA descriptors of every field of both buffers (box = the tile plus its
// halo), output origins, grid sizing and scratch: everything that depends on
// the chosen tile shape.
int configure(sp_handle* H, int variant) {
  SP_CUDA(H, cudaStreamSynchronize(H->stream));
  H->variant = variant;
  H->ki = &H->variants[variant];
  const int R = H->ki->R;
  H->ntx = (H->n[0] + H->ki->tx - 1) / H->ki->tx;
  H->nty = (H->n[1] + H->ki->ty - 1) / H->ki->ty;
  for (int k = 0; k < 2; ++k)
    if (H->gexec[k]) {
      cudaGraphExecDestroy(H->gexec[k]);
      H->gexec[k] = nullptr;
    }

  EncodeTiled enc = encode_fn();
  if (!enc) return fail(H, SP_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const int cnt = H->batch * H->nf;
  for (int k = 0; k < 2; ++k) {
    std::vector<CUtensorMap> maps(cnt);
    std::vector<void*> outs(cnt);
    for (int i = 0; i < H->batch; ++i)
      for (int f = 0; f < H->nf; ++f) {
        const int idx = i * H->nf + f;
        const InstGeo& g = H->geo[i];
        void* base = field_base(H, k, i, f);
        outs[idx] = base;
        const cuuint32_t bw =
            cuuint32_t(H->ki->tx + 2 * (H->ki->box_hx < 0 ? H->h[0] : H->ki->box_hx));
        const cuuint32_t bh = cuuint32_t(H->ki->ty + 2 * R);
        const CUtensorMapDataType dt =
            H->esz == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
        CUresult r;
        if (H->dim == 3) {
          cuuint64_t gdim[3] = {cuuint64_t(g.pitch), cuuint64_t(g.ly), cuuint64_t(g.lz)};
          cuuint64_t gstr[2] = {cuuint64_t(g.pitch * H->esz), cuuint64_t(g.plane * H->esz)};
          cuuint32_t box[3] = {bw, bh, 1};
          cuuint32_t es[3] = {1, 1, 1};
          r = enc(&maps[idx], dt, 3, base, gdim, gstr, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        } else {
          cuuint64_t gdim[2] = {cuuint64_t(g.pitch), cuuint64_t(g.ly)};
          cuuint64_t gstr[1] = {cuuint64_t(g.pitch * H->esz)};
          cuuint32_t box[2] = {bw, bh};
          cuuint32_t es[2] = {1, 1};
          r = enc(&maps[idx], dt, 2, base, gdim, gstr, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        }
        if (r != CUDA_SUCCESS) {
          char b[128];
          snprintf(b, sizeof b, "cuTensorMapEncodeTiled failed (CUresult %d)", int(r));
          return fail(H, SP_ECUDA, b);
        }
      }
    if (!H->maps_d[k]) SP_CUDA(H, cudaMalloc(&H->maps_d[k], sizeof(CUtensorMap) * cnt));
    SP_CUDA(H, cudaMemcpy(H->maps_d[k], maps.data(), sizeof(CUtensorMap) * cnt,
                          cudaMemcpyHostToDevice));
    if (!H->outs_d[k]) SP_CUDA(H, cudaMalloc(&H->outs_d[k], sizeof(void*) * cnt));
    SP_CUDA(H, cudaMemcpy(H->outs_d[k], outs.data(), sizeof(void*) * cnt, cudaMemcpyHostToDevice));
  }

  size_t partial_n = 2 * size_t(H->sms) * 8;
  if (H->dim == 3) {
    // z planes per CTA: as many z chunks as fit one wave of resident CTAs
    // (each chunk re-reads 2R planes, so longer chunks waste less)
    const int occ = H->ki->occupancy();
    const long long tiles = (long long)H->ntx * H->nty * H->batch;
    const long long slots = (long long)H->sms * occ;
    int chunks = int(std::max(1LL, slots / tiles));
    chunks = std::min(chunks, std::max(1, H->n[2] / std::max(4, 2 * R)));
    H->zchunk = (H->n[2] + chunks - 1) / chunks;
    if (const char* zc = getenv("SP_ZCHUNK")) {
      const int v = atoi(zc);
      if (v > 0) H->zchunk = std::min(v, H->n[2]);
    }
    H->nzc = (H->n[2] + H->zchunk - 1) / H->zchunk;
    partial_n = std::max(partial_n, size_t(H->ntx) * H->nty * H->nzc * H->batch);
  } else {
    int rc = H->esz == 4 ? setup_2d_t<float>(H) : setup_2d_t<double>(H);
    if (rc) return rc;
    partial_n = std::max(partial_n, size_t(H->grid2));
  }
  if (partial_n > H->partial_n) {
    cudaFree(H->partial_d);
    H->partial_d = nullptr;
    H->partial_n = partial_n;
    SP_CUDA(H, cudaMalloc(&H->partial_d, sizeof(double) * partial_n));
  }
  return SP_OK;
}

// fastest tile shape of each (kernel key, extents, batch) found so far
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int, int, int, int, int, int, int, int, int>, int> g_tuned;

// the kernel-key code of a point count: 4th-order point sets are offset
int pts_code(const sp_desc& d, int pts) { return d.accuracy == 4 ? sp::SP_PTS4 + pts : pts; }

std::tuple<int, int, int, int, int, int, int, int, int, int, int> tune_key(const sp_handle* H) {
  const sp_desc& d = H->d;
  return {d.model, d.form, d.dim, d.dtype, pts_code(d, d.lap_pts), pts_code(d, d.gradlap_pts),
          pts_code(d, d.bilap_pts), H->n[0], H->n[1], H->n[2], H->batch};
}

// kernel model of an ensemble: one model shared by every member, or the
// two-model kernel for members of models AMK and BMK (kind 0 and 1)
int ensemble_model(const sp_member* m, int count, std::string& why) {
  bool amk = false, bmk = false, same = true;
  for (int i = 0; i < count; ++i) {
    same = same && m[i].model == m[0].model;
    amk = amk || m[i].model == SP_MODEL_AMK;
    bmk = bmk || m[i].model == SP_MODEL_BMK;
  }
  if (same) return m[0].model;
  for (int i = 0; i < count; ++i)
    if (m[i].model != SP_MODEL_AMK && m[i].model != SP_MODEL_BMK)
      return why = "an ensemble mixes models only of SP_MODEL_AMK and SP_MODEL_BMK", -1;
  return SP_ENSEMBLE_AMK_BMK;
}

// a handle over `desc` (a batch of identical instances), or, when `members`
// is given, over `count` members that each have their own extents, model,
// time step and coefficients (desc then supplies dim, dtype, form, stencil,
// boundaries and h)
int create(const sp_desc* desc, const sp_member* members, int count, sp_handle* H) {
  std::string why;
  sp_desc dd{};
  if (desc) dd = *desc;
  if (members) {
    if (!desc) return fail(H, SP_EINVAL, "null description");
    if (count < 1) return fail(H, SP_EINVAL, "an ensemble needs at least one member");
    if (desc->dim != 2) return fail(H, SP_EINVAL, "ensembles are two-dimensional");
    for (int i = 0; i < count; ++i) {
      for (int a = 0; a < 2; ++a)
        if (members[i].n[a] < 4 || members[i].n[a] > (1 << 16))
          return fail(H, SP_EINVAL, "each extent must be in [4, 65536]");
      if (!std::isfinite(members[i].dt)) return fail(H, SP_EINVAL, "dt must be finite");
    }
    const int model = ensemble_model(members, count, why);
    if (model < 0) return fail(H, SP_EINVAL, why);
    dd.model = model;
    dd.n[0] = members[0].n[0];
    dd.n[1] = members[0].n[1];
    dd.batch = count;
    dd.dt = members[0].dt;
    for (int c = 0; c < 8; ++c) dd.coeff[c] = members[0].coeff[c];
    H->ensemble = true;
  }
  if (int rc = validate(desc ? &dd : nullptr, why)) return fail(H, rc, why);
  sp::register_all_kernels();
  H->d = dd;
  H->dim = dd.dim;
  H->batch = dd.batch;
  H->esz = dd.dtype == SP_F32 ? 4 : 8;
  const sp::KernelKey key{dd.model,
                          dd.form,
                          dd.dim,
                          dd.dtype,
                          pts_code(dd, dd.lap_pts),
                          pts_code(dd, dd.gradlap_pts),
                          pts_code(dd, dd.bilap_pts)};
  const std::vector<sp::KernelInfo>* vs = sp::find_kernels(key);
  if (!vs || vs->empty()) {
    char b[256];
    snprintf(b, sizeof b,
             "no fused kernel built for model %d form %d dim %d dtype %d stencil %dd%dh<%d,%d,%d>",
             dd.model, dd.form, dd.dim, dd.dtype, dd.dim, dd.accuracy == 4 ? 4 : 2, dd.lap_pts,
             dd.gradlap_pts, dd.bilap_pts);
    return fail(H, SP_EINVAL, b);
  }
  H->variants = *vs;
  H->ki = &H->variants[0];
  H->nf = H->ki->nf;
  const int R = H->ki->R;
  H->h[0] = H->ki->hx;
  H->h[1] = R;
  H->h[2] = H->dim == 3 ? R : 0;
  for (const sp::KernelInfo& v : H->variants)
    if (v.hx != H->h[0] || v.R != R || v.nf != H->nf)
      return fail(H, SP_EINVAL, "tile variants of one kernel disagree on the halo");
  H->geo.resize(H->batch);
  size_t off = 0;
  for (int i = 0; i < H->batch; ++i) {
    InstGeo& g = H->geo[i];
    set_geometry(H, g, members ? members[i].n : dd.n);
    for (int a = 0; a < H->dim; ++a)
      if (g.n[a] < 2 * R)
        return fail(H, SP_EINVAL, "an extent is smaller than twice the stencil reach");
    g.off = off;
    off += size_t(H->nf) * g.felems;
    g.model = members ? members[i].model : dd.model;
    g.kind = (dd.model == SP_ENSEMBLE_AMK_BMK && g.model == SP_MODEL_BMK) ? 1 : 0;
    g.dt = members ? members[i].dt : dd.dt;
    for (int c = 0; c < 8; ++c) g.coeff[c] = members ? members[i].coeff[c] : dd.coeff[c];
  }
  const InstGeo& g0 = H->geo[0];
  for (int a = 0; a < 3; ++a) H->n[a] = g0.n[a];
  H->pitch = g0.pitch;
  H->ly = g0.ly;
  H->lz = g0.lz;
  H->plane = g0.plane;
  H->felems = g0.felems;

  int dev = 0;
  SP_CUDA(H, cudaGetDevice(&dev));
  SP_CUDA(H, cudaDeviceGetAttribute(&H->sms, cudaDevAttrMultiProcessorCount, dev));
  SP_CUDA(H, cudaStreamCreateWithFlags(&H->stream, cudaStreamNonBlocking));
  H->own_stream = true;

  const size_t bytes = off * H->esz;
  for (int k = 0; k < 2; ++k) {
    if (cudaMalloc(&H->buf[k], bytes) != cudaSuccess)
      return fail(H, SP_ENOMEM, "device allocation of the field buffers failed");
    SP_CUDA(H, cudaMemset(H->buf[k], 0, bytes));
  }
  SP_CUDA(H, cudaMalloc(&H->result_d, sizeof(double) * (2 + H->batch)));
  SP_CUDA(H, cudaMallocHost(&H->result_h, sizeof(double) * (2 + H->batch)));
  SP_CUDA(H, cudaMalloc(&H->err_d, sizeof(int)));
  SP_CUDA(H, cudaMemset(H->err_d, 0, sizeof(int)));

  // tile shape: an explicit choice (SP_TILE), else the one sp_autotune found
  // for this kernel and size in this process, else the first registered
  int variant = 0;
  if (!H->ensemble) {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    auto it = g_tuned.find(tune_key(H));
    if (it != g_tuned.end()) variant = it->second;
  }
  if (const char* t = getenv("SP_TILE")) variant = atoi(t);
  if (variant < 0 || variant >= int(H->variants.size()) || !applicable(H, variant)) variant = 0;
  if (int rc = configure(H, variant)) return rc;
  SP_CUDA(H, cudaDeviceSynchronize());
  return SP_OK;
}

int check_field(sp_handle* H, int inst, int field, size_t bytes) {
  if (!H) return SP_EINVAL;
  if (inst < 0 || inst >= H->batch) return fail(H, SP_EINVAL, "instance index out of range");
  if (field < 0 || field >= H->nf) return fail(H, SP_EINVAL, "field index out of range");
  const size_t need = size_t(H->geo[inst].sites()) * H->esz;
  if (bytes != need) return fail(H, SP_EINVAL, "byte count does not match the interior size");
  return SP_OK;
}

cudaMemcpy3DParms interior_copy(sp_handle* H, int which, int inst, int field, void* other,
                                bool to_device, cudaMemcpyKind kind) {
  const InstGeo& g = H->geo[inst];
  cudaMemcpy3DParms p{};
  cudaPitchedPtr dev = make_cudaPitchedPtr(field_base(H, which, inst, field), g.pitch * H->esz,
                                           g.pitch, g.ly);
  cudaPitchedPtr com = make_cudaPitchedPtr(other, g.n[0] * H->esz, g.n[0], g.n[1]);
  cudaPos dpos = make_cudaPos(H->h[0] * H->esz, H->h[1], H->dim == 3 ? H->h[2] : 0);
  if (to_device) {
    p.srcPtr = com;
    p.dstPtr = dev;
    p.dstPos = dpos;
  } else {
    p.srcPtr = dev;
    p.srcPos = dpos;
    p.dstPtr = com;
  }
  p.extent = make_cudaExtent(g.n[0] * H->esz, g.n[1], g.n[2]);
  p.kind = kind;
  return p;
}

int upload(sp_handle* H, int inst, int field, const void* src, size_t bytes, cudaMemcpyKind k) {
  if (int rc = check_field(H, inst, field, bytes)) return rc;
  cudaMemcpy3DParms p = interior_copy(H, H->cur, inst, field, const_cast<void*>(src), true, k);
  SP_CUDA(H, cudaMemcpy3DAsync(&p, H->stream));
  return refresh_halos(H, inst, field);
}

int download(sp_handle* H, int which, int inst, int field, void* dst, size_t bytes,
             cudaMemcpyKind k, bool wait) {
  if (int rc = check_field(H, inst, field, bytes)) return rc;
  cudaMemcpy3DParms p = interior_copy(H, which, inst, field, dst, false, k);
  SP_CUDA(H, cudaMemcpy3DAsync(&p, H->stream));
  if (wait) return check_err_flag(H);
  return SP_OK;
}

int capture_graph(sp_handle* H) {
  const int parity = H->cur;
  cudaGraph_t g = nullptr;
  if (H->stream == nullptr || cudaStreamBeginCapture(H->stream, cudaStreamCaptureModeThreadLocal) !=
                                  cudaSuccess) {
    cudaGetLastError();
    H->graphs = false;  // e.g. the legacy default stream cannot be captured
    return SP_OK;
  }
  int rc = SP_OK;
  const long long before = H->launches;
  for (int i = 0; i < GRAPH_STEPS && rc == SP_OK; ++i) rc = launch_step(H, 0, nullptr, H->ki->kt);
  cudaError_t e = cudaStreamEndCapture(H->stream, &g);
  H->launches = before;
  H->cur = parity;
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(H, e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&H->gexec[parity], g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(H, e, "cudaGraphInstantiate");
  return SP_OK;
}

// queue the FP64 (mass, energy) reduction of a field into out[0..1] (device)
template <class T>
int enqueue_reduce_t(sp_handle* H, int inst, int field, double* out) {
  const InstGeo& g = H->geo[inst];
  sp::ReduceParams<T> p{};
  p.f0 = reinterpret_cast<const T*>(field_base(H, H->cur, inst, field));
  p.e0 = reinterpret_cast<const T*>(field_base(H, H->cur, inst, 0));
  p.e1 = H->nf > 1 ? reinterpret_cast<const T*>(field_base(H, H->cur, inst, 1)) : nullptr;
  p.dim = H->dim;
  for (int a = 0; a < 3; ++a) {
    p.n[a] = g.n[a];
    p.h[a] = H->h[a];
  }
  p.pitch = g.pitch;
  p.plane = g.plane;
  p.energy_kind = energy_kind(g.model);
  p.c1 = g.coeff[0];
  p.c2 = g.coeff[1];
  p.kappa = g.model == SP_MODEL_C ? 1.0 : g.coeff[1];
  p.gamma = g.coeff[0];
  p.h_sp = H->d.h;
  p.partial = H->partial_d;
  const long long total = g.sites();
  int blocks = int(std::min<long long>((total + RED_THREADS - 1) / RED_THREADS,
                                       (long long)(H->partial_n / 2)));
  blocks = std::max(blocks, 1);
  sp::k_reduce<T, RED_THREADS><<<blocks, RED_THREADS, 0, H->stream>>>(p);
  SP_CUDA(H, cudaGetLastError());
  sp::k_finish<RED_THREADS><<<1, RED_THREADS, 0, H->stream>>>(H->partial_d, blocks, 2, out);
  SP_CUDA(H, cudaGetLastError());
  return SP_OK;
}

int enqueue_reduce(sp_handle* H, int inst, int field, double* out) {
  return H->esz == 4 ? enqueue_reduce_t<float>(H, inst, field, out)
                     : enqueue_reduce_t<double>(H, inst, field, out);
}

// restore the mass of field 0 of every instance to its target (no host wait)
int conserve_pass(sp_handle* H) {
  for (int i = 0; i < H->batch; ++i) {
    if (int rc = enqueue_reduce(H, i, 0, H->cons_d)) return rc;
    const InstGeo& g = H->geo[i];
    sp::ShiftParams sh{};
    sh.dim = H->dim;
    for (int a = 0; a < 3; ++a) {
      sh.n[a] = g.n[a];
      sh.h[a] = H->h[a];
    }
    sh.pitch = g.pitch;
    sh.plane = g.plane;
    sh.pass = ++H->conserve_passes;
    const long long cells = (g.n[0] + 2LL * H->h[0]) * (g.n[1] + 2LL * H->h[1]) *
                            (H->dim == 3 ? g.n[2] + 2LL * H->h[2] : 1);
    const int blocks = int(std::min<long long>(H->sms * 8LL, (cells + 255) / 256));
    if (H->esz == 4)
      sp::k_mass_shift<float><<<blocks, 256, 0, H->stream>>>(
          reinterpret_cast<float*>(field_base(H, H->cur, i, 0)), sh, H->cons_d,
          H->mass_target_d + 2 * i, double(g.sites()));
    else
      sp::k_mass_shift<double><<<blocks, 256, 0, H->stream>>>(
          reinterpret_cast<double*>(field_base(H, H->cur, i, 0)), sh, H->cons_d,
          H->mass_target_d + 2 * i, double(g.sites()));
    SP_CUDA(H, cudaGetLastError());
  }
  return SP_OK;
}

// sp_step without mass conservation: graph-replayed chunks, then single launches
int step_plain(sp_handle* H, int nsteps);

int reduce(sp_handle* H, int inst, int field, double* mass, double* energy) {
  if (int rc = enqueue_reduce(H, inst, field, H->result_d)) return rc;
  SP_CUDA(H, cudaMemcpyAsync(H->result_h, H->result_d, 2 * sizeof(double),
                             cudaMemcpyDeviceToHost, H->stream));
  if (int rc = check_err_flag(H)) return rc;
  double hd = 1.0;
  for (int a = 0; a < H->dim; ++a) hd *= H->d.h;
  if (mass) *mass = H->result_h[0];
  if (energy) *energy = H->result_h[1] * hd;
  if (!std::isfinite(H->result_h[0]) || !std::isfinite(H->result_h[1]))
    return fail(H, SP_ENONFINITE, "the field holds NaN or Inf");
  return SP_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int sp_create(const sp_desc* desc, sp_handle** out) {
  return sp_create_ensemble(desc, nullptr, 0, out);
}

int sp_create_ensemble(const sp_desc* desc, const sp_member* members, int count,
                       sp_handle** out) {
  g_create_error.clear();
  if (!out) return SP_EINVAL;
  *out = nullptr;
  sp_handle* H = new sp_handle();
  int rc = create(desc, members, count, H);
  if (rc != SP_OK) {
    g_create_error = H->err;
    release(H);
    return rc;
  }
  *out = H;
  return SP_OK;
}

const char* sp_create_error(void) { return g_create_error.c_str(); }

int sp_upload(sp_handle* h, int inst, int field, const void* host, size_t bytes) {
  if (!h || !host) return SP_EINVAL;
  return upload(h, inst, field, host, bytes, cudaMemcpyHostToDevice);
}

}  // extern "C"

namespace {
// the batch's instances share their extents and sit one after another
bool uniform_batch(const sp_handle* H) {
  for (int i = 0; i < H->batch; ++i) {
    const InstGeo& g = H->geo[i];
    for (int a = 0; a < 3; ++a)
      if (g.n[a] != H->geo[0].n[a]) return false;
    if (g.off != size_t(i) * H->nf * H->geo[0].felems) return false;
  }
  return true;
}

template <class T>
int batch_copy_t(sp_handle* H, int field, void* dense, size_t bytes, bool to_field) {
  if (field < 0 || field >= H->nf) return fail(H, SP_EINVAL, "field index out of range");
  if (!uniform_batch(H))
    return fail(H, SP_EINVAL, "batched copies need instances of equal extents");
  const InstGeo& g = H->geo[0];
  const long long total = (long long)H->batch * g.sites();
  if (bytes != size_t(total) * sizeof(T))
    return fail(H, SP_EINVAL, "byte count does not match batch x interior size");
  const int blocks = int(std::min<long long>(H->sms * 8LL, (total + 255) / 256));
  sp::k_batch_copy<T><<<blocks, 256, 0, H->stream>>>(
      reinterpret_cast<T*>(field_base(H, H->cur, 0, field)), (long long)H->nf * g.felems,
      g.pitch, g.plane, g.n[0], g.n[1], g.n[2], H->h[0], H->h[1], H->h[2],
      static_cast<T*>(dense), total, to_field ? 1 : 0);
  SP_CUDA(H, cudaGetLastError());
  if (!to_field) return SP_OK;
  // as refresh_halos, for every instance at once
  if (int rc = fill_halo_batch_t<T>(H, H->cur ^ 1, field)) return rc;
  return fill_halo_batch_t<T>(H, H->cur, field);
}
}  // namespace

extern "C" {

int sp_upload_batch_device(sp_handle* h, int field, const void* dev, size_t bytes) {
  if (!h || !dev) return SP_EINVAL;
  void* d = const_cast<void*>(dev);
  return h->esz == 4 ? batch_copy_t<float>(h, field, d, bytes, true)
                     : batch_copy_t<double>(h, field, d, bytes, true);
}

int sp_download_batch_device(sp_handle* h, int field, void* dev, size_t bytes) {
  if (!h || !dev) return SP_EINVAL;
  return h->esz == 4 ? batch_copy_t<float>(h, field, dev, bytes, false)
                     : batch_copy_t<double>(h, field, dev, bytes, false);
}

int sp_upload_device(sp_handle* h, int inst, int field, const void* dev, size_t bytes) {
  if (!h || !dev) return SP_EINVAL;
  return upload(h, inst, field, dev, bytes, cudaMemcpyDeviceToDevice);
}

int sp_fill_uniform(sp_handle* H, int inst, int field, uint64_t seed, double lo, double hi) {
  if (!H) return SP_EINVAL;
  if (inst < 0 || inst >= H->batch) return fail(H, SP_EINVAL, "instance index out of range");
  if (int rc = check_field(H, inst, field, size_t(H->geo[inst].sites()) * H->esz)) return rc;
  const InstGeo& g = H->geo[inst];
  char* base = field_base(H, H->cur, inst, field);
  if (H->esz == 4)
    sp::k_seed<float><<<H->sms * 4, 256, 0, H->stream>>>(
        reinterpret_cast<float*>(base), H->dim, g.n[0], g.n[1], g.n[2], H->h[0], H->h[1],
        H->h[2], g.pitch, g.plane, seed, lo, hi);
  else
    sp::k_seed<double><<<H->sms * 4, 256, 0, H->stream>>>(
        reinterpret_cast<double*>(base), H->dim, g.n[0], g.n[1], g.n[2], H->h[0], H->h[1],
        H->h[2], g.pitch, g.plane, seed, lo, hi);
  SP_CUDA(H, cudaGetLastError());
  return refresh_halos(H, inst, field);
}

int sp_step(sp_handle* H, int nsteps) {
  if (!H || nsteps < 0) return SP_EINVAL;
  if (H->conserve_every <= 0) return step_plain(H, nsteps);
  // a pass falls due after every conserve_every steps (sp_step_mass counts too)
  do {
    if (H->since_conserve >= H->conserve_every) {
      if (int rc = conserve_pass(H)) return rc;
      H->since_conserve = 0;
    }
    const int k = std::min(nsteps, H->conserve_every - H->since_conserve);
    if (int rc = step_plain(H, k)) return rc;
    nsteps -= k;
    H->since_conserve += k;
  } while (nsteps > 0 || H->since_conserve >= H->conserve_every);
  return SP_OK;
}

int sp_conserve_mass(sp_handle* H, int every) {
  if (!H || every < 0) return SP_EINVAL;
  if (every > 0) {
    for (int a = 0; a < H->dim; ++a)
      if (H->d.boundary[2 * a] != SP_PERIODIC)
        return fail(H, SP_EINVAL, "mass conservation needs periodic boundaries on every axis");
    if (!H->mass_target_d) SP_CUDA(H, cudaMalloc(&H->mass_target_d, 2 * sizeof(double) * H->batch));
    if (!H->cons_d) SP_CUDA(H, cudaMalloc(&H->cons_d, 2 * sizeof(double)));
    for (int i = 0; i < H->batch; ++i)
      if (int rc = enqueue_reduce(H, i, 0, H->mass_target_d + 2 * i)) return rc;
    if (int rc = check_err_flag(H)) return rc;
  }
  H->conserve_every = every;
  H->since_conserve = 0;
  return SP_OK;
}

}  // extern "C"

namespace {
int step_plain(sp_handle* H, int nsteps) {
  // a graph replays GRAPH_STEPS launches of kt steps each
  const int kt = H->ki->kt, chunk = GRAPH_STEPS * kt;
  while (nsteps > 0) {
    if (nsteps >= chunk && H->graphs && !H->gexec[H->cur])
      if (int rc = capture_graph(H)) return rc;
    if (nsteps >= chunk && H->gexec[H->cur]) {
      SP_CUDA(H, cudaGraphLaunch(H->gexec[H->cur], H->stream));
      H->launches += GRAPH_STEPS;
      nsteps -= chunk;
    } else {
      const int s = std::min(kt, nsteps);
      if (int rc = launch_step(H, 0, nullptr, s)) return rc;
      nsteps -= s;
    }
  }
  return SP_OK;
}
}  // namespace

extern "C" {

int sp_step_mass(sp_handle* H, int nsteps, double* mass) {
  if (!H || nsteps < 1 || !mass) return SP_EINVAL;
  if (H->dim == 2 && H->batch > 1)
    return fail(H, SP_EINVAL, "fused mass reduction needs dim 3 or a single 2D instance");
  if (int rc = sp_step(H, nsteps - 1)) return rc;
  if (int rc = launch_step(H, 0, H->partial_d)) return rc;
  if (H->conserve_every > 0) ++H->since_conserve;  // its pass runs before the next step
  const int per = H->dim == 3 ? H->ntx * H->nty * H->nzc : H->grid2;
  for (int i = 0; i < H->batch; ++i) {
    sp::k_finish<RED_THREADS><<<1, RED_THREADS, 0, H->stream>>>(H->partial_d + size_t(i) * per,
                                                               per, 1, H->result_d + i);
    SP_CUDA(H, cudaGetLastError());
  }
  SP_CUDA(H, cudaMemcpyAsync(H->result_h, H->result_d, sizeof(double) * H->batch,
                             cudaMemcpyDeviceToHost, H->stream));
  if (int rc = check_err_flag(H)) return rc;
  for (int i = 0; i < H->batch; ++i) mass[i] = H->result_h[i];
  return SP_OK;
}

int sp_eval_rhs(sp_handle* H, int inst, int field, void* host, size_t bytes) {
  if (!H || !host) return SP_EINVAL;
  if (int rc = check_field(H, inst, field, bytes)) return rc;
  if (int rc = launch_step(H, 1, nullptr)) return rc;
  return download(H, H->cur ^ 1, inst, field, host, bytes, cudaMemcpyDeviceToHost, true);
}

int sp_download(sp_handle* h, int inst, int field, void* host, size_t bytes) {
  if (!h || !host) return SP_EINVAL;
  return download(h, h->cur, inst, field, host, bytes, cudaMemcpyDeviceToHost, true);
}

int sp_download_device(sp_handle* h, int inst, int field, void* dev, size_t bytes) {
  if (!h || !dev) return SP_EINVAL;
  return download(h, h->cur, inst, field, dev, bytes, cudaMemcpyDeviceToDevice, false);
}

int sp_reduce(sp_handle* H, int inst, int field, double* mass, double* energy) {
  if (!H) return SP_EINVAL;
  if (inst < 0 || inst >= H->batch || field < 0 || field >= H->nf)
    return fail(H, SP_EINVAL, "instance or field index out of range");
  return reduce(H, inst, field, mass, energy);
}

int sp_autotune(sp_handle* H, int reps) {
  if (!H || reps < 1) return SP_EINVAL;
  if (H->variants.size() < 2) return SP_OK;
  const long long launches = H->launches;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  SP_CUDA(H, cudaEventCreate(&e0));
  SP_CUDA(H, cudaEventCreate(&e1));
  int best = H->variant;
  float best_ms = 1e30f;
  int rc = SP_OK;
  for (int v = 0; v < int(H->variants.size()) && rc == SP_OK; ++v) {
    if (!applicable(H, v)) continue;
    if ((rc = configure(H, v))) break;
    // one-step kernels: right-hand-side launches, the same loads and stores
    // as a step; temporally blocked ones: launches of kt whole steps into the
    // other buffer, which is not made current.  Either leaves the state of
    // the model untouched; the time is taken per step.
    const int kt = H->ki->kt;
    auto once = [&]() { return kt > 1 ? launch_step(H, 0, nullptr, kt, false) : launch_step(H, 1, nullptr); };
    for (int i = 0; i < 2 && rc == SP_OK; ++i) rc = once();
    cudaEventRecord(e0, H->stream);
    for (int i = 0; i < reps && rc == SP_OK; ++i) rc = once();
    cudaEventRecord(e1, H->stream);
    if (rc) break;
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = fail(H, SP_ECUDA, "autotune timing failed");
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= float(kt);
    if (ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  H->launches = launches;
  if (rc) return rc;
  if ((rc = configure(H, best))) return rc;
  if (!H->ensemble) {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    g_tuned[tune_key(H)] = best;
  }
  return check_err_flag(H);
}

int sp_steps_per_launch(const sp_handle* H, int* kt) {
  if (!H || !kt) return SP_EINVAL;
  *kt = H->ki->kt;
  return SP_OK;
}

int sp_kernel_info(const sp_handle* H, int info[8]) {
  if (!H || !info) return SP_EINVAL;
  info[0] = H->ki->tx;
  info[1] = H->ki->ty;
  info[2] = H->ki->spt;
  info[3] = H->ki->pd;
  info[4] = H->variant;
  info[5] = int(H->variants.size());
  info[6] = H->ki->threads;
  info[7] = H->dim == 3 ? H->zchunk : H->grid2;
  return SP_OK;
}

int sp_set_dt(sp_handle* H, double dt) {
  if (!H) return SP_EINVAL;
  if (!std::isfinite(dt)) return fail(H, SP_EINVAL, "dt must be finite");
  if (H->ensemble) return fail(H, SP_EINVAL, "the members of an ensemble keep their own dt");
  if (dt == H->d.dt) return SP_OK;
  for (InstGeo& g : H->geo) g.dt = dt;
  SP_CUDA(H, cudaStreamSynchronize(H->stream));
  H->d.dt = dt;
  for (int k = 0; k < 2; ++k)
    if (H->gexec[k]) {
      cudaGraphExecDestroy(H->gexec[k]);
      H->gexec[k] = nullptr;
    }
  if (H->dim == 2) {
    cudaFree(H->inst2_d);
    cudaFree(H->items_d);
    cudaFree(H->ctr_d);
    H->inst2_d = nullptr;
    H->items_d = nullptr;
    H->ctr_d = nullptr;
    return H->esz == 4 ? setup_2d_t<float>(H) : setup_2d_t<double>(H);
  }
  return SP_OK;
}

int sp_set_stream(sp_handle* H, void* stream) {
  if (!H) return SP_EINVAL;
  SP_CUDA(H, cudaStreamSynchronize(H->stream));
  if (H->own_stream) cudaStreamDestroy(H->stream);
  H->stream = static_cast<cudaStream_t>(stream);
  H->own_stream = false;
  H->graphs = true;
  for (int k = 0; k < 2; ++k)
    if (H->gexec[k]) {
      cudaGraphExecDestroy(H->gexec[k]);
      H->gexec[k] = nullptr;
    }
  return SP_OK;
}

int sp_synchronize(sp_handle* H) {
  if (!H) return SP_EINVAL;
  return check_err_flag(H);
}

int sp_test_wait_timeout(sp_handle* H, long long cycles, int dirty_queue) {
  if (!H || cycles < 0 || cycles > (1LL << 31)) return SP_EINVAL;
  int* queue = dirty_queue ? H->ctr_d : nullptr;
  if (dirty_queue && !queue) return fail(H, SP_EINVAL, "the handle has no 2D work queue");
  sp::k_wait_probe<<<1, 32, 0, H->stream>>>(H->err_d, queue, cycles);
  SP_CUDA(H, cudaGetLastError());
  return SP_OK;
}

long long sp_launch_count(const sp_handle* H) { return H ? H->launches : -1; }

int sp_field_geometry(const sp_handle* H, int inst, int field, void** dev_origin,
                      long long* pitch, long long* plane, int halo[3]) {
  if (!H) return SP_EINVAL;
  sp_handle* M = const_cast<sp_handle*>(H);
  if (inst < 0 || inst >= H->batch || field < 0 || field >= H->nf)
    return fail(M, SP_EINVAL, "instance or field index out of range");
  if (dev_origin) *dev_origin = field_origin(M, H->cur, inst, field);
  if (pitch) *pitch = H->geo[inst].pitch;
  if (plane) *plane = H->geo[inst].plane;
  if (halo)
    for (int a = 0; a < 3; ++a) halo[a] = H->h[a];
  return SP_OK;
}

const char* sp_last_error(const sp_handle* h) { return h ? h->err.c_str() : "null handle"; }

void sp_destroy(sp_handle* h) { release(h); }

}  // extern "C"
