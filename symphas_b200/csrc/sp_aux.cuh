/*
 * sp_aux.cuh -- auxiliary kernels around the fused step: halo fill after an
 * upload, FP64 mass/energy reductions and the deterministic finishing sum.
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sp_common.cuh"
#include "sp_tma.cuh"

namespace sp {

// ---------------------------------------------------------------------------
// halo fill (after an upload): Dirichlet sides take their constant, the rest
// of the halo takes periodic images -- the same rule as the oracle
// ---------------------------------------------------------------------------
template <class T>
struct HaloParams {
  T* org;
  int dim;
  int n[3], h[3];
  long long pitch, plane;
  int bc[6];
  T bv[6];
  long long inst_stride;  // elements between instances of a batched launch (grid y)
};

// The halo cells only, enumerated as (a) the whole halo planes in z, (b) the
// whole halo rows in y of the interior planes, (c) the halo columns in x of
// the interior rows.
template <class T>
__global__ void k_fill_halo(HaloParams<T> p) {
  p.org += blockIdx.y * p.inst_stride;  // instance blockIdx.y of a batch
  const long long L0 = p.n[0] + 2 * p.h[0], L1 = p.n[1] + 2 * p.h[1];
  const int n2 = (p.dim == 3) ? p.n[2] : 1, h2 = (p.dim == 3) ? p.h[2] : 0;
  const long long A = 2LL * h2 * L0 * L1;            // halo planes
  const long long B = (long long)n2 * 2 * p.h[1] * L0;  // halo rows of interior planes
  const long long Cc = (long long)n2 * p.n[1] * 2 * p.h[0];  // halo columns
  const long long total = A + B + Cc;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    long long i, j, k;  // padded coordinates
    if (id < A) {
      const long long q = id / (L0 * L1), r = id % (L0 * L1);
      k = q < h2 ? q : n2 + q;
      j = r / L0;
      i = r % L0;
    } else if (id < A + B) {
      const long long e = id - A, q = e / L0;
      i = e % L0;
      const long long row = q % (2 * p.h[1]);
      k = h2 + q / (2 * p.h[1]);
      j = row < p.h[1] ? row : p.n[1] + row;
    } else {
      const long long e = id - A - B, col = e % (2 * p.h[0]), q = e / (2 * p.h[0]);
      i = col < p.h[0] ? col : p.n[0] + col;
      j = p.h[1] + q % p.n[1];
      k = h2 + q / p.n[1];
    }
    long long c[3] = {i - p.h[0], j - p.h[1], (p.dim == 3) ? k - p.h[2] : 0};
    int dir = -1;
    T dval = T(0);
    for (int a = 0; a < p.dim; ++a) {
      if (c[a] < 0 && p.bc[2 * a] == 1) {
        dir = 2 * a;
        dval = p.bv[2 * a];
      }
      if (c[a] >= p.n[a] && p.bc[2 * a + 1] == 1) {
        dir = 2 * a + 1;
        dval = p.bv[2 * a + 1];
      }
    }
    const long long idx = k * p.plane + j * p.pitch + i;
    if (dir >= 0) {
      p.org[idx] = dval;
      continue;
    }
    long long w[3] = {0, 0, 0};
    for (int a = 0; a < p.dim; ++a) {
      long long v = c[a] % p.n[a];
      if (v < 0) v += p.n[a];
      w[a] = v + p.h[a];
    }
    p.org[idx] = p.org[w[2] * p.plane + w[1] * p.pitch + w[0]];
  }
}

// ---------------------------------------------------------------------------
// one field of every instance of a batch (equal extents) to or from a dense
// array [instance][z][y][x] in device memory: interiors only
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_batch_copy(T* org, long long inst_stride, long long pitch, long long plane,
                             int n0, int n1, int n2, int h0, int h1, int h2, T* dense,
                             long long total, int to_field) {
  const long long sites = (long long)n0 * n1 * n2;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const long long i = id / sites, s = id - i * sites;
    const long long x = s % n0, yz = s / n0, y = yz % n1, z = yz / n1;
    T* f = org + i * inst_stride + (z + h2) * plane + (y + h1) * pitch + (x + h0);
    if (to_field)
      *f = dense[id];
    else
      dense[id] = *f;
  }
}

// ---------------------------------------------------------------------------
// FP64 reductions: mass of one field and the free energy of the system
// ---------------------------------------------------------------------------
template <class T>
struct ReduceParams {
  const T* f0;  // field whose mass is summed
  const T* e0;  // fields of the energy (e1 may be null)
  const T* e1;
  int dim;
  int n[3], h[3];
  long long pitch, plane;
  int energy_kind;  // 0 Landau(c1,c2), 1 Landau with kappa, 2 model C
  double c1, c2, kappa, gamma, h_sp;
  double* partial;  // [2 * gridDim.x]
};

template <class T, int NT>
__global__ void __launch_bounds__(NT) k_reduce(const ReduceParams<T> p) {
  __shared__ double red[32];
  const long long nx = p.n[0], ny = p.n[1], nz = (p.dim == 3) ? p.n[2] : 1;
  const long long total = nx * ny * nz;
  const double ih = 1.0 / p.h_sp;
  double ms = 0.0, es = 0.0;
  for (long long id = blockIdx.x * (long long)NT + threadIdx.x; id < total;
       id += (long long)gridDim.x * NT) {
    const long long i = id % nx, j = (id / nx) % ny, k = id / (nx * ny);
    const long long o = (k + (p.dim == 3 ? p.h[2] : 0)) * p.plane + (j + p.h[1]) * p.pitch +
                        (i + p.h[0]);
    ms += double(p.f0[o]);
    double e = 0.0;
    for (int f = 0; f < (p.e1 ? 2 : 1); ++f) {
      const T* g = f ? p.e1 : p.e0;
      const double v = double(g[o]);
      const double gx = (double(g[o + 1]) - v) * ih, gy = (double(g[o + p.pitch]) - v) * ih;
      double g2 = gx * gx + gy * gy;
      if (p.dim == 3) {
        const double gz = (double(g[o + p.plane]) - v) * ih;
        g2 += gz * gz;
      }
      const double v2 = v * v;
      if (p.energy_kind == 0)
        e += -0.5 * p.c1 * v2 + 0.25 * p.c2 * v2 * v2 + 0.5 * g2;
      else
        e += -0.5 * v2 + 0.25 * v2 * v2 + 0.5 * p.kappa * g2;
    }
    if (p.energy_kind == 2 && p.e1) {
      const double a = double(p.e0[o]), b = double(p.e1[o]);
      e += p.gamma * a * a * b * b;
    }
    es += e;
  }
  const double m = block_sum<NT>(ms, red);
  __syncthreads();
  const double e = block_sum<NT>(es, red);
  if (threadIdx.x == 0) {
    p.partial[2 * blockIdx.x] = m;
    p.partial[2 * blockIdx.x + 1] = e;
  }
}

// sums `count` groups of `stride` partials in a fixed order (deterministic)
template <int NT>
__global__ void __launch_bounds__(NT)
    k_finish(const double* partial, int count, int stride, double* out) {
  __shared__ double red[32];
  for (int s = 0; s < stride; ++s) {
    double v = 0.0;
    for (int i = threadIdx.x; i < count; i += NT) v += partial[size_t(i) * stride + s];
    const double t = block_sum<NT>(v, red);
    if (threadIdx.x == 0) out[s] = t;
    __syncthreads();
  }
}

// Mass-restoring shift of one field: every cell of the padded box, interior
// and halo, becomes value + s with s = (target - mass) / sites.  In FP32 a
// shift far below one ulp would round away at nearly every cell, so the sum
// is rounded stochastically instead: each cell takes the float just below or
// just above value + s with the probabilities that make its expectation
// value + s exactly (the restored mass is then within about sqrt(|N s| ulp) of
// the target).  The uniform draw hashes the interior site a cell shows (its
// periodic source for a halo cell) and the pass number, so a halo image
// rounds exactly like its source.  FP64 adds s.
struct ShiftParams {
  int dim;
  int n[3], h[3];
  long long pitch, plane;
  unsigned long long pass;
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

template <class T>
__global__ void k_mass_shift(T* base, const ShiftParams p, const double* mass,
                             const double* target, double sites) {
  const double s = (*target - *mass) / sites;
  const long long L0 = p.n[0] + 2 * p.h[0], L1 = p.n[1] + 2 * p.h[1];
  const long long L2 = (p.dim == 3) ? p.n[2] + 2 * p.h[2] : 1;
  const long long total = L0 * L1 * L2;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const long long i = id % L0, j = (id / L0) % L1, k = id / (L0 * L1);
    T& cell = base[k * p.plane + j * p.pitch + i];
    if constexpr (sizeof(T) == 8) {
      cell += s;
    } else {
      long long c[3] = {i - p.h[0], j - p.h[1], (p.dim == 3) ? k - p.h[2] : 0};
      for (int a = 0; a < p.dim; ++a) {
        c[a] %= p.n[a];
        if (c[a] < 0) c[a] += p.n[a];
      }
      const unsigned long long key =
          (unsigned long long)((c[2] * p.n[1] + c[1]) * p.n[0] + c[0]);
      const double v = double(cell) + s;
      const float f = float(v);
      const float lo = double(f) > v ? nextafterf(f, -INFINITY) : f;
      const float hi = double(f) > v ? f : nextafterf(f, INFINITY);
      const double frac = (v - double(lo)) / (double(hi) - double(lo));
      const double u = double(mix64(key * 0x9E3779B97F4A7C15ULL ^ (p.pass << 1)) >> 11) *
                       (1.0 / 9007199254740992.0);
      cell = T(u < frac ? hi : lo);
    }
  }
}

// The failure path of a step kernel, on its own: one warp waits on an
// mbarrier that nothing will complete (no copy is in flight), gives up after
// `limit` SM cycles as a step kernel gives up on a TMA tile, and sets the
// device error flag.  With `queue` it first takes an item from the 2D work
// queue and leaves without re-arming it, as a CTA that gave up mid-step does.
__global__ void k_wait_probe(int* err, int* queue, long long limit) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    tma::mbar_init(&bar, 1);
    tma::fence_barrier_init();
    if (queue) atomicAdd(queue, 1);
  }
  __syncwarp();
  const bool ok = tma::mbar_wait_limit(&bar, 0, limit, 20000u);
  if (!ok && threadIdx.x == 0) atomicExch(err, KERR_TMA_TIMEOUT);
}

}  // namespace sp
