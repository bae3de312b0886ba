/*
 * sp_noalloc.cu -- FP64 mass and free-energy sums for callers that cannot
 * allocate device memory.
 *
 * sp_reduce uses a scratch buffer that sp_create allocates with cudaMalloc.
 * Some callers can do neither: an application whose device memory is owned by
 * another allocator (a framework's caching pool that has reserved the GPU, an
 * embedding host with a fixed memory budget), or a time-stepping loop that must
 * not stall, since cudaMalloc and cudaFree can synchronise the whole device.
 * sp_reduce_fields_noalloc does the same reduction on fields the caller already
 * holds in device memory and writes the sums to device memory the caller
 * provides; its only scratch is the file-scope array below, which every GPU
 * that loads this library keeps until the process exits.
 */
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>

#include "../../include/symphas_b200.h"
#include "sp_common.cuh"

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_BLOCKS = SP_NOALLOC_BLOCKS_PER_INSTANCE;
constexpr int NA_MAX_INST = SP_NOALLOC_MAX_INSTANCES;

// per-block (mass, energy) partials of every instance of one call:
// NA_MAX_INST * NA_BLOCKS * 2 doubles = 128 KiB.  Every call overwrites the
// slots it uses before reading them, so nothing needs clearing between calls.
static __device__ __align__(256) double sp_noalloc_scratch[NA_MAX_INST * NA_BLOCKS * 2];

struct NaParams {
  const void* fields;  // [batch][nf][n2][n1][n0], compact, periodic
  int f64;
  int dim, nf;
  int n[3];
  int energy_kind;  // 0 Landau(c1, c2), 1 Landau with kappa, 2 model C
  double c1, c2, kappa, gamma, h;
  double* partial;  // the device address of sp_noalloc_scratch
  double* out;      // [batch][2]
};

template <class T>
__device__ __forceinline__ double ld(const NaParams& p, long long i) {
  return double(static_cast<const T*>(p.fields)[i]);
}

template <class T>
__global__ void __launch_bounds__(NA_THREADS) k_noalloc_partial(const NaParams p) {
  __shared__ double red[32];
  const long long n0 = p.n[0], n1 = p.n[1], n2 = p.dim == 3 ? p.n[2] : 1;
  const long long cnt = n0 * n1 * n2;
  const int inst = blockIdx.y;
  const long long base = (long long)inst * p.nf * cnt;
  const double ih = 1.0 / p.h;
  double ms = 0.0, es = 0.0;
  for (long long id = blockIdx.x * (long long)NA_THREADS + threadIdx.x; id < cnt;
       id += (long long)gridDim.x * NA_THREADS) {
    const long long i = id % n0, j = (id / n0) % n1, k = id / (n0 * n1);
    const long long ip = (i + 1 == n0) ? id - i : id + 1;
    const long long jp = (j + 1 == n1) ? id - j * n0 : id + n0;
    const long long kp = (k + 1 == n2) ? id - k * n0 * n1 : id + n0 * n1;
    ms += ld<T>(p, base + id);
    double e = 0.0;
    for (int f = 0; f < p.nf; ++f) {
      const long long b = base + f * cnt;
      const double v = ld<T>(p, b + id);
      const double gx = (ld<T>(p, b + ip) - v) * ih, gy = (ld<T>(p, b + jp) - v) * ih;
      double g2 = gx * gx + gy * gy;
      if (p.dim == 3) {
        const double gz = (ld<T>(p, b + kp) - v) * ih;
        g2 += gz * gz;
      }
      const double v2 = v * v;
      if (p.energy_kind == 0)
        e += -0.5 * p.c1 * v2 + 0.25 * p.c2 * v2 * v2 + 0.5 * g2;
      else
        e += -0.5 * v2 + 0.25 * v2 * v2 + 0.5 * p.kappa * g2;
    }
    if (p.energy_kind == 2 && p.nf > 1) {
      const double a = ld<T>(p, base + id), c = ld<T>(p, base + cnt + id);
      e += p.gamma * a * a * c * c;
    }
    es += e;
  }
  const double m = sp::block_sum<NA_THREADS>(ms, red);
  __syncthreads();
  const double en = sp::block_sum<NA_THREADS>(es, red);
  if (threadIdx.x == 0) {
    double* slot = p.partial + (size_t(inst) * NA_BLOCKS + blockIdx.x) * 2;
    slot[0] = m;
    slot[1] = en;
  }
}

__global__ void __launch_bounds__(NA_THREADS) k_noalloc_finish(const NaParams p) {
  __shared__ double red[32];
  const int inst = blockIdx.x;
  const double* part = p.partial + size_t(inst) * NA_BLOCKS * 2;
  double hd = p.h * p.h;
  if (p.dim == 3) hd *= p.h;
  for (int s = 0; s < 2; ++s) {
    double v = 0.0;
    for (int i = threadIdx.x; i < NA_BLOCKS; i += NA_THREADS) v += part[2 * i + s];
    const double t = sp::block_sum<NA_THREADS>(v, red);
    if (threadIdx.x == 0) p.out[2 * inst + s] = s ? t * hd : t;
    __syncthreads();
  }
}

// device address of the scratch array, looked up once per device.  Host
// threads may make their first calls on a device at the same time: each looks
// the address up (the runtime answers both alike) and stores it; the atomic
// slots make those concurrent stores and loads well defined.
constexpr int NA_MAX_DEVICES = 64;
std::atomic<double*> g_scratch[NA_MAX_DEVICES] = {};

int energy_kind_of(int model) {
  switch (model) {
    case SP_MODEL_AMK:
    case SP_MODEL_BMK: return 1;
    case SP_MODEL_C: return 2;
    default: return 0;
  }
}

thread_local char g_msg[256];

int na_fail(int code, const char* msg) {
  snprintf(g_msg, sizeof g_msg, "%s", msg);
  return code;
}

}  // namespace

extern "C" {

int sp_reduce_fields_noalloc(const void* fields, int dtype, int dim, const int n[3], int model,
                             const double coeff[8], double h, int batch, double* out,
                             void* stream) {
  g_msg[0] = 0;
  if (!fields || !n || !out) return na_fail(SP_EINVAL, "null pointer argument");
  if (model != SP_MODEL_A && model != SP_MODEL_B && model != SP_MODEL_C && model != SP_MODEL_AMK &&
      model != SP_MODEL_BMK)
    return na_fail(SP_EINVAL,
                   "model must be SP_MODEL_A, SP_MODEL_B, SP_MODEL_C, SP_MODEL_AMK or SP_MODEL_BMK");
  if (dtype != SP_F32 && dtype != SP_F64) return na_fail(SP_EINVAL, "dtype must be SP_F32 or SP_F64");
  if (dim != 2 && dim != 3) return na_fail(SP_EINVAL, "dim must be 2 or 3");
  for (int a = 0; a < dim; ++a)
    if (n[a] < 1) return na_fail(SP_EINVAL, "extents must be positive");
  if (!(h > 0.0) || !std::isfinite(h))
    return na_fail(SP_EINVAL, "grid spacing h must be positive and finite");
  if (batch < 1 || batch > NA_MAX_INST) {
    char b[160];
    snprintf(b, sizeof b,
             "batch %d is outside 1..%d: the static scratch holds the partial sums of at "
             "most %d instances per call",
             batch, NA_MAX_INST, NA_MAX_INST);
    return na_fail(SP_EINVAL, b);
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES)
    return na_fail(SP_ECUDA, "no current CUDA device");
  double* scratch = g_scratch[dev].load(std::memory_order_relaxed);
  if (!scratch) {
    // first call on this device: the host-side name of the array is not a
    // device address; ask the runtime for the address on the current device
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, sp_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      snprintf(g_msg, sizeof g_msg, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return SP_ECUDA;
    }
    scratch = static_cast<double*>(ptr);
    g_scratch[dev].store(scratch, std::memory_order_relaxed);
  }
  NaParams p{};
  p.fields = fields;
  p.f64 = dtype == SP_F64;
  p.dim = dim;
  p.nf = model == SP_MODEL_C ? 2 : 1;
  for (int a = 0; a < 3; ++a) p.n[a] = a < dim ? n[a] : 1;
  p.energy_kind = energy_kind_of(model);
  p.c1 = coeff ? coeff[0] : 1.0;
  p.c2 = coeff ? coeff[1] : 1.0;
  p.kappa = model == SP_MODEL_C ? 1.0 : p.c2;
  p.gamma = p.c1;
  p.h = h;
  p.partial = scratch;
  p.out = out;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const dim3 grid(NA_BLOCKS, batch);
  if (p.f64)
    k_noalloc_partial<double><<<grid, NA_THREADS, 0, s>>>(p);
  else
    k_noalloc_partial<float><<<grid, NA_THREADS, 0, s>>>(p);
  k_noalloc_finish<<<batch, NA_THREADS, 0, s>>>(p);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    snprintf(g_msg, sizeof g_msg, "kernel launch: %s", cudaGetErrorString(e));
    return SP_ECUDA;
  }
  return SP_OK;
}

const char* sp_noalloc_error(void) { return g_msg; }

}  // extern "C"
