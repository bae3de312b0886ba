/*
 * sp_regional.cu -- regional systems: SolverFT on SolverSystemFDwSD, whose
 * RegionalGrid keeps only a window of the domain (datatypes/inc/grid.h:2038-2158)
 * and moves it after the field (update_regional_system,
 * sol/inc/boundarysystem.h:438-471).
 *
 * The window is a handle of its own (sp_create over the window's interior),
 * so the fused step kernels do the stepping: its halo is the window's 3-deep
 * rim, constant at `empty` (SP_DIRICHLET), except along an axis that the
 * window spans from origin 0, which is periodic -- there the reference's rim
 * takes periodic images (regional_update_boundary,
 * datatypes/inc/boundaryupdatedata.h:1397-1431).
 *
 * Moving the window and searching for the next one:
 *   - k_reg_min: the minimum of the window (grid::min_value,
 *     sol/inc/boundarysystem.h:372-376);
 *   - k_reg_mask: one byte per cell of the window's buffer as the reference
 *     lays it out (dims incl. rim, x-fastest): value >= cutoff
 *     (compare_cutoff, datatypes/inc/gridfunctions.h:1471-1479).  Rim cells
 *     read `empty`, or along periodic axes the image the reference's rim holds
 *     at that moment: the value before the last step (the boundary update
 *     runs after the window check, boundarysystem.h:474-478);
 *   - the searches (get_view, get_view_resized, get_view_resized_periodic,
 *     adjust_region, resize_adjust_region; gridfunctions.h:1873-2238) run on
 *     the host over that mask, cell for cell in the reference's order;
 *   - k_reg_remap: a new window of `empty` with the interior copied from the
 *     old one modulo the domain (adjust_region_to_from, gridfunctions.h:1662-1683);
 *   - k_reg_shift: the in-place origin shift of a window that keeps its dims
 *     (adjust_origin_to_from, gridfunctions.h:1770-1852): a cell becomes
 *     empty by the test of the last axis alone, any other takes the buffer
 *     value at its index + the shift's offset, rim cells included; written
 *     here as a gather from the old state;
 *   - k_reg_gather / k_reg_scatter: whole-domain fields in and out.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/symphas_b200.h"
#include "sp_handle.h"

namespace {

constexpr int BD = 3;  // BOUNDARY_DEPTH, the rim of a window

// ---------------------------------------------------------------------------
// device side
// ---------------------------------------------------------------------------
template <class T>
struct RegView {
  const T* cur;   // interior origin of the window's field, present state
  const T* prev;  // the same in the other buffer: the state before the last step
  long long pitch, plane;
  int D;
  int c[3];    // window interior extents
  int d[3];    // window dims, rim included
  int per[3];  // axis periodic (the window spans the domain from origin 0)
  T rim;       // value of a rim cell along a constant axis
};

__device__ __forceinline__ int wrap_mod(long long a, int n) {
  long long r = a % n;
  return int(r < 0 ? r + n : r);
}

// value of cell r (window buffer coordinates, rim included) as the
// reference's buffer holds it
template <class T>
__device__ __forceinline__ T reg_value(const RegView<T>& v, const int r[3]) {
  bool out_const = false, out_per = false;
  int l[3] = {0, 0, 0};
  for (int a = 0; a < v.D; ++a) {
    l[a] = r[a] - BD;
    if (l[a] < 0 || l[a] >= v.c[a]) {
      if (v.per[a]) {
        out_per = true;
        l[a] = wrap_mod(l[a], v.c[a]);
      } else {
        out_const = true;
      }
    }
  }
  if (out_const) return v.rim;
  const T* src = out_per ? v.prev : v.cur;
  return src[(long long)l[2] * v.plane + (long long)l[1] * v.pitch + l[0]];
}

template <class T>
__global__ void k_reg_mask(RegView<T> v, T cutoff, unsigned char* mask, long long len) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const int r[3] = {int(i % v.d[0]), int((i / v.d[0]) % v.d[1]),
                      int(i / ((long long)v.d[0] * v.d[1]))};
    mask[i] = reg_value(v, r) >= cutoff ? 1 : 0;
  }
}

template <class T>
__global__ void k_reg_min(RegView<T> v, T* partial) {
  __shared__ T sm[256];
  const long long len = (long long)v.c[0] * v.c[1] * (v.D == 3 ? v.c[2] : 1);
  T m = v.cur[0];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const long long x = i % v.c[0], y = (i / v.c[0]) % v.c[1], z = i / ((long long)v.c[0] * v.c[1]);
    const T e = v.cur[z * v.plane + y * v.pitch + x];
    m = e < m ? e : m;
  }
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s && sm[threadIdx.x + s] < sm[threadIdx.x]) sm[threadIdx.x] = sm[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

struct Geo {
  int D;
  int n[3];   // domain interior
  int o[3];   // window origin
  int c[3];   // window interior
};

// compact window interior <- whole-domain interior
template <class T>
__global__ void k_reg_gather(Geo g, const T* global, T* win) {
  const long long len = (long long)g.c[0] * g.c[1] * g.c[2];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const long long l[3] = {i % g.c[0], (i / g.c[0]) % g.c[1], i / ((long long)g.c[0] * g.c[1])};
    long long gi = 0, s = 1;
    for (int a = 0; a < g.D; ++a) {
      gi += wrap_mod(g.o[a] + l[a], g.n[a]) * s;
      s *= g.n[a];
    }
    win[i] = global[gi];
  }
}

// whole-domain interior <- window interior, `empty` elsewhere
template <class T>
__global__ void k_reg_scatter(Geo g, RegView<T> v, T empty, T* global) {
  const long long len = (long long)g.n[0] * g.n[1] * g.n[2];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const long long p[3] = {i % g.n[0], (i / g.n[0]) % g.n[1], i / ((long long)g.n[0] * g.n[1])};
    bool in = true;
    long long off = 0;
    const long long st[3] = {1, v.pitch, v.plane};
    for (int a = 0; a < g.D; ++a) {
      const int l = wrap_mod(p[a] - g.o[a], g.n[a]);
      in = in && l < g.c[a];
      off += l * st[a];
    }
    global[i] = in ? v.cur[off] : empty;
  }
}

// adjust_region_to_from: new compact interior from the old window, modulo the
// domain; delta = normalised new origin - normalised old origin per axis
template <class T>
__global__ void k_reg_remap(Geo gn, RegView<T> old, int dx, int dy, int dz, T empty, T* win) {
  const int delta[3] = {dx, dy, dz};
  const long long len = (long long)gn.c[0] * gn.c[1] * gn.c[2];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const long long l[3] = {i % gn.c[0], (i / gn.c[0]) % gn.c[1], i / ((long long)gn.c[0] * gn.c[1])};
    bool in = true;
    long long off = 0;
    const long long st[3] = {1, old.pitch, old.plane};
    for (int a = 0; a < gn.D; ++a) {
      long long q = l[a] + delta[a];
      q = q < 0 ? q + gn.n[a] : (q >= gn.n[a] ? q - gn.n[a] : q);
      in = in && q >= 0 && q < old.c[a];
      off += q * st[a];
    }
    win[i] = in ? old.cur[off] : empty;
  }
}

// adjust_origin_to_from, in place (window dims kept): shift s per axis
template <class T>
__global__ void k_reg_shift(RegView<T> v, int sx, int sy, int sz, T empty, T* win) {
  const int s[3] = {sx, sy, sz};
  const int L = v.D - 1;
  const int dirL = s[L] >= 0 ? 1 : -1;
  const int ovL = v.c[L] - (s[L] < 0 ? -s[L] : s[L]);
  long long st[3] = {1, v.d[0], (long long)v.d[0] * v.d[1]};
  long long off = 0, bo = 0, blen = 1;
  for (int a = 0; a < v.D; ++a) {
    off += s[a] * st[a];
    bo += BD * st[a];
    blen *= v.d[a];
  }
  const long long len = (long long)v.c[0] * v.c[1] * (v.D == 3 ? v.c[2] : 1);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len;
       i += (long long)gridDim.x * blockDim.x) {
    const long long p[3] = {i % v.c[0], (i / v.c[0]) % v.c[1], i / ((long long)v.c[0] * v.c[1])};
    const bool set_empty = dirL > 0 ? (p[L] >= ovL) : (p[L] < v.c[L] - ovL);
    long long idx = 0;
    for (int a = 0; a < v.D; ++a) idx += p[a] * st[a];
    const long long src = idx + off + bo;
    T val = empty;
    if (!set_empty && src >= 0 && src < blen) {
      const int r[3] = {int(src % v.d[0]), int((src / v.d[0]) % v.d[1]),
                        int(src / ((long long)v.d[0] * v.d[1]))};
      val = reg_value(v, r);
    }
    win[i] = val;
  }
}

// ---------------------------------------------------------------------------
// host search over the mask (the reference's order, cell for cell)
// ---------------------------------------------------------------------------
struct Search {
  int D;
  int G[3], o[3], d[3];
  const unsigned char* m;  // window buffer mask (null: no interior)

  long stride(int a) const {
    long s = 1;
    for (int i = 0; i < a; ++i) s *= d[i];
    return s;
  }
  long interior(long c[3]) const {
    long len = 1;
    for (int a = 0; a < D; ++a) {
      c[a] = d[a] - 2 * BD;
      if (c[a] <= 0) len = 0;
      len *= std::max(c[a], 0L);
    }
    return m ? len : 0;
  }
  bool at(const long pos[3], const long st[3]) const {
    long idx = 0;
    for (int a = 0; a < D; ++a) idx += (pos[a] + BD) * st[a];
    return m[idx] != 0;
  }

  // get_view (gridfunctions.h:1962-1986 with get_view_intervals :1945-1960):
  // buffer entries 0 .. len(interior)-1, rim cells among them, at positions
  // (n / stride) % interior_dims
  void view_fixed(int origin[3]) const {
    long c[3], iv[3][2], st[3];
    const long len = interior(c);
    for (int a = 0; a < D; ++a) {
      iv[a][0] = c[a];
      iv[a][1] = 0;
      st[a] = stride(a);
    }
    for (long n = 0; n < len; ++n)
      if (m[n])
        for (int a = 0; a < D; ++a) {
          const long p = (n / st[a]) % c[a];
          iv[a][0] = std::min(iv[a][0], p);
          iv[a][1] = std::max(iv[a][1], p);
        }
    for (int a = 0; a < D; ++a) {
      const long dims = iv[a][1] - iv[a][0] + 1 + 2 * BD;
      const long delta = d[a] - dims;
      origin[a] = int(o[a] + (iv[a][0] - delta / 2));
    }
  }

  // get_view_resized (:1873-1913), in the serial order of its loop
  void view_resized(int origin[3], int dims[3]) const {
    long c[3], iv[3][2], st[3];
    const long len = interior(c);
    for (int a = 0; a < D; ++a) {
      iv[a][0] = d[a];
      iv[a][1] = 0;
      st[a] = stride(a);
    }
    for (long n = 0; n < len; ++n) {
      long pos[3], rem = n, idx = 0;
      for (int a = 0; a < D; ++a) {
        pos[a] = rem % c[a] + BD;
        rem /= c[a];
        idx += pos[a] * st[a];
      }
      if (!m[idx]) continue;
      bool inside = true;
      for (int a = 0; a < D; ++a) inside = inside && pos[a] >= iv[a][0] && pos[a] < iv[a][1];
      if (inside) continue;
      for (int a = 0; a < D; ++a) {
        if (pos[a] >= iv[a][0])
          iv[a][1] = std::max(pos[a], iv[a][1]);
        else
          iv[a][0] = std::min(pos[a], iv[a][0]);
      }
    }
    for (int a = 0; a < D; ++a) {
      origin[a] = int(iv[a][0] - BD + o[a]);
      dims[a] = int(std::max(0L, iv[a][1] - iv[a][0] + 1 + 2 * BD));
    }
  }

  // get_view_resized_periodic (:1988-2163): the window is the whole domain
  void view_periodic(int origin[3], int dims_out[3]) const {
    long c[3], st[3];
    const long len = interior(c);
    for (int a = 0; a < D; ++a) st[a] = stride(a);
    long start = -1;
    for (long n = 0; n < len && start < 0; ++n) {
      long pos[3] = {0, 0, 0}, rem = n;
      for (int a = 0; a < D; ++a) {
        pos[a] = rem % c[a];
        rem /= c[a];
      }
      if (at(pos, st)) start = n;
    }
    if (start < 0) {
      for (int a = 0; a < D; ++a) dims_out[a] = 0;
      return;
    }
    long iv[3][2], iu[3][2];
    {
      long rem = start;
      for (int a = 0; a < D; ++a) {
        iu[a][0] = iu[a][1] = rem % c[a];
        rem /= c[a];
      }
    }
    bool grown;
    do {
      for (int a = 0; a < D; ++a) {
        iv[a][0] = iu[a][0];
        iv[a][1] = iu[a][1];
      }
      for (int i = 0; i < D; ++i) {
        bool right = true;
        long pos[3] = {0, 0, 0};
        for (int j = 0; j < D; ++j) {
          pos[j] = (j == i) ? iu[j][1] + 1 : iu[j][0];
          // a negative entry wraps with the extent of axis i, as written there
          pos[j] = (pos[j] >= c[j]) ? pos[j] - c[j] : (pos[j] < 0) ? c[i] + pos[j] : pos[j];
        }
        long sd[2] = {1, 1};
        int ns = 0;
        for (int j = 0; j < D; ++j)
          if (j != i) sd[ns++] = iu[j][1] - iu[j][0] + 1;
        long slen = 1;
        for (int q = 0; q < ns; ++q) slen *= sd[q];
        const long steps = c[i] - (iu[i][1] - iu[i][0] + 1);
        bool found[2] = {true, false};
        long last[2] = {iu[i][0], iu[i][1]};
        for (long n = 0; n < steps; ++n) {
          for (long k = 0; k < slen && !found[right ? 1 : 0]; ++k) {
            const long sp[2] = {k % sd[0], ns > 1 ? k / sd[0] : 0};
            int q = 0;
            for (int j = 0; j < D; ++j) {
              if (j == i) continue;
              const long p = sp[q++] + iu[j][0];
              pos[j] = (p < 0) ? p + c[j] : (p >= c[j]) ? p - c[j] : p;
            }
            if (at(pos, st)) found[right ? 1 : 0] = true;
          }
          if (right) {
            if (found[1]) {
              iu[i][1] = (pos[i] < iu[i][1]) ? pos[i] + c[i] : pos[i];
              ++last[1];
            }
            pos[i] = (last[0] <= 0) ? c[i] + last[0] - 1 : last[0] - 1;
            found[0] = false;
            right = false;
          } else {
            if (found[0]) {
              iu[i][0] = (pos[i] > iu[i][0]) ? pos[i] - c[i] : pos[i];
              --last[0];
            }
            pos[i] = (last[1] >= c[i] - 1) ? last[1] + 1 - c[i] : last[1] + 1;
            found[1] = false;
            right = true;
          }
        }
      }
      grown = false;
      for (int a = 0; a < D; ++a) grown = grown || !(iv[a][0] <= iu[a][0] && iv[a][1] >= iu[a][1]);
    } while (grown);
    for (int a = 0; a < D; ++a) {
      origin[a] = int(iu[a][0] + o[a]);
      dims_out[a] = int(std::max(0L, iu[a][1] - iu[a][0] + 1 + 2 * BD));
    }
  }

  // adjust_region (:2166-2176, mode 0) or resize_adjust_region (:2194-2238,
  // mode 1): the window the next move goes to
  void target(int mode, double factor, double rel_eps, int no[3], int nd[3]) const {
    for (int a = 0; a < 3; ++a) {
      no[a] = o[a];
      nd[a] = d[a];
    }
    if (mode == 0) {
      int origin[3] = {0, 0, 0};
      view_fixed(origin);
      for (int a = 0; a < D; ++a) {
        const int delta = G[a] - 2 * BD;
        no[a] = origin[a] + ((origin[a] < 0) ? delta : (origin[a] >= delta) ? -delta : 0);
      }
      return;
    }
    int origin[3] = {0, 0, 0}, dims[3] = {0, 0, 0};
    bool whole = true;
    for (int a = 0; a < D; ++a) whole = whole && G[a] == d[a];
    if (whole)
      view_periodic(origin, dims);
    else
      view_resized(origin, dims);
    bool same = true;
    for (int a = 0; a < D; ++a) {
      const int dim0 = std::min(G[a], int(dims[a] * factor));
      no[a] = origin[a] - (dim0 - dims[a]) / 2;
      no[a] += (no[a] < 0) ? (G[a] - 2 * BD) : 0;
      nd[a] = dim0;
      if (std::abs(nd[a] - d[a]) / double(d[a]) > rel_eps) same = false;
    }
    if (same)
      for (int a = 0; a < D; ++a) {
        no[a] = origin[a] - (d[a] - dims[a]) / 2;
        no[a] += (no[a] < 0) ? (G[a] - 2 * BD) : 0;
        nd[a] = d[a];
      }
  }
};

}  // namespace

// ---------------------------------------------------------------------------
// the regional system
// ---------------------------------------------------------------------------
struct sp_regional {
  sp_desc gd{};  // the whole domain
  sp_regional_params p{};
  int D = 2;
  int G[3] = {1, 1, 1}, o[3] = {0, 0, 0}, d[3] = {1, 1, 1};
  double empty = 0.0, cutoff = 0.0, time = 0.0;
  int next_resize = 0;
  sp_handle* w = nullptr;  // the window (null while it has no interior)
  void* stream = nullptr;  // stream given to every window handle, or null
  // device scratch, grown on demand and kept: whole-domain staging, a compact
  // window, the cutoff mask, the minimum's partials (every use waits for its
  // work before returning, so each call may reuse them)
  struct Scratch {
    void* p = nullptr;
    size_t cap = 0;
  } dom, win, msk, red;
  size_t esz = 8;
  std::string err;
};

namespace {

thread_local std::string g_reg_create_error;

int rfail(sp_regional* R, int code, const std::string& msg) {
  if (R) R->err = msg;
  return code;
}
#define SP_RCUDA(R, call)                                                          \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) return rfail(R, SP_ECUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

template <class P>
int grow(sp_regional* R, sp_regional::Scratch& s, size_t bytes, P** out) {
  if (s.cap < bytes) {
    if (s.p) cudaFree(s.p);  // waits for the work that used it
    s.p = nullptr;
    s.cap = 0;
    SP_RCUDA(R, cudaMalloc(&s.p, bytes));
    s.cap = bytes;
  }
  *out = static_cast<P*>(s.p);
  return SP_OK;
}

int blocks_for(long long n) { return int(std::max(1LL, std::min<long long>(148LL * 8, (n + 255) / 256))); }

long long interior_cells(const sp_regional* R, const int d[3]) {
  long long len = 1;
  for (int a = 0; a < R->D; ++a) len *= std::max(0, d[a] - 2 * BD);
  return len;
}

bool has_interior(const sp_regional* R, const int d[3]) {
  for (int a = 0; a < R->D; ++a)
    if (d[a] - 2 * BD <= 0) return false;
  return true;
}

template <class T>
RegView<T> view_of(const sp_regional* R) {
  RegView<T> v{};
  sp_handle* H = R->w;
  v.cur = reinterpret_cast<const T*>(field_origin(H, H->cur, 0, 0));
  v.prev = reinterpret_cast<const T*>(field_origin(H, H->cur ^ 1, 0, 0));
  v.pitch = H->geo[0].pitch;
  v.plane = H->geo[0].plane;
  v.D = R->D;
  for (int a = 0; a < 3; ++a) {
    v.c[a] = a < R->D ? R->d[a] - 2 * BD : 1;
    v.d[a] = a < R->D ? R->d[a] : 1;
    v.per[a] = a < R->D && R->o[a] == 0 && R->d[a] == R->G[a];
  }
  v.rim = T(H->d.boundary_value[0]);
  return v;
}

Geo geo_of(const sp_regional* R, const int o[3], const int d[3]) {
  Geo g{};
  g.D = R->D;
  for (int a = 0; a < 3; ++a) {
    g.n[a] = a < R->D ? R->gd.n[a] : 1;
    g.o[a] = a < R->D ? o[a] : 0;
    g.c[a] = a < R->D ? d[a] - 2 * BD : 1;
  }
  return g;
}

// the other buffer takes the present state: rim images read from it before
// the next step then hold the values the window was moved with
int sync_prev(sp_regional* R, sp_handle* H) {
  const size_t bytes = size_t(H->geo[0].felems) * H->nf * H->esz;
  SP_RCUDA(R, cudaMemcpyAsync(H->buf[H->cur ^ 1] + H->geo[0].off * H->esz,
                              H->buf[H->cur] + H->geo[0].off * H->esz, bytes,
                              cudaMemcpyDeviceToDevice, H->stream));
  return SP_OK;
}

// a handle over the window (o, d) with rim value `empty`
int make_window(sp_regional* R, const int o[3], const int d[3], sp_handle** out) {
  *out = nullptr;
  if (!has_interior(R, d)) return SP_OK;
  sp_desc wd = R->gd;
  wd.batch = 1;
  for (int a = 0; a < R->D; ++a) {
    wd.n[a] = d[a] - 2 * BD;
    const bool per = o[a] == 0 && d[a] == R->G[a];
    wd.boundary[2 * a] = wd.boundary[2 * a + 1] = per ? SP_PERIODIC : SP_DIRICHLET;
    wd.boundary_value[2 * a] = wd.boundary_value[2 * a + 1] = R->empty;
  }
  if (int rc = sp_create(&wd, out))
    return rfail(R, rc, std::string("window handle: ") + sp_create_error());
  if (R->stream)
    if (int rc = sp_set_stream(*out, R->stream)) {
      const std::string why = sp_last_error(*out);
      sp_destroy(*out);
      *out = nullptr;
      return rfail(R, rc, "window stream: " + why);
    }
  return SP_OK;
}

template <class T>
int min_t(sp_regional* R, double* out) {
  *out = R->empty;
  if (!R->w) return SP_OK;
  const RegView<T> v = view_of<T>(R);
  const int blocks = blocks_for(interior_cells(R, R->d));
  T* part = nullptr;
  if (int rc = grow(R, R->red, sizeof(T) * blocks, &part)) return rc;
  k_reg_min<T><<<blocks, 256, 0, R->w->stream>>>(v, part);
  std::vector<T> h(blocks);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), part, sizeof(T) * blocks, cudaMemcpyDeviceToHost, R->w->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(R->w->stream);
  if (e != cudaSuccess) return rfail(R, SP_ECUDA, std::string("window minimum: ") + cudaGetErrorString(e));
  T m = h[0];
  for (T x : h) m = x < m ? x : m;
  // std::min(*e, empty)
  *out = (R->empty < double(m)) ? R->empty : double(m);
  return SP_OK;
}

template <class T>
int mask_t(sp_regional* R, std::vector<unsigned char>& mask) {
  mask.clear();
  if (!R->w) return SP_OK;
  const RegView<T> v = view_of<T>(R);
  const long long len = (long long)v.d[0] * v.d[1] * v.d[2];
  mask.resize(size_t(len));
  unsigned char* m = nullptr;
  if (int rc = grow(R, R->msk, size_t(len), &m)) return rc;
  k_reg_mask<T><<<blocks_for(len), 256, 0, R->w->stream>>>(v, T(R->cutoff), m, len);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(mask.data(), m, size_t(len), cudaMemcpyDeviceToHost, R->w->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(R->w->stream);
  if (e != cudaSuccess) return rfail(R, SP_ECUDA, std::string("window mask: ") + cudaGetErrorString(e));
  return SP_OK;
}

// compact window values -> field of window handle H, halo refreshed, the
// other buffer in step; waits for the copies
int put_window(sp_regional* R, sp_handle* H, const void* dev, long long cells) {
  if (int rc = sp_upload_device(H, 0, 0, dev, size_t(cells) * R->esz))
    return rfail(R, rc, std::string("window upload: ") + sp_last_error(H));
  if (int rc = sync_prev(R, H)) return rc;
  if (int rc = sp_synchronize(H)) return rfail(R, rc, std::string("window upload: ") + sp_last_error(H));
  return SP_OK;
}

// adjust_region_to_from (and adjust_origin_to_from_replace): a new window
// handle whose interior is copied from the old window modulo the domain; on
// failure the regional system is left as it was
template <class T>
int replace_t(sp_regional* R, const int no[3], const int nd[3]) {
  sp_handle* nw = nullptr;
  if (int rc = make_window(R, no, nd, &nw)) return rc;
  int rc = SP_OK;
  if (nw) {
    const Geo gn = geo_of(R, no, nd);
    const long long cells = interior_cells(R, nd);
    int delta[3] = {0, 0, 0};
    RegView<T> ov{};
    if (R->w) {
      if (sp_synchronize(R->w) != SP_OK) rc = rfail(R, SP_ECUDA, sp_last_error(R->w));
      ov = view_of<T>(R);
      for (int a = 0; a < R->D; ++a) {
        const int wrap = R->G[a] - 2 * BD;
        const long on = R->o[a] - wrap * std::lround(double(R->o[a]) / wrap);
        const long nn = no[a] - wrap * std::lround(double(no[a]) / wrap);
        delta[a] = int(nn - on);
      }
    } else {
      // no old interior: every cell takes `empty`
      ov.cur = reinterpret_cast<const T*>(field_origin(nw, nw->cur, 0, 0));
    }
    T* tmp = nullptr;
    if (rc == SP_OK) rc = grow(R, R->win, sizeof(T) * size_t(cells), &tmp);
    if (rc == SP_OK) {
      k_reg_remap<T><<<blocks_for(cells), 256, 0, nw->stream>>>(gn, ov, delta[0], delta[1],
                                                                 delta[2], T(R->empty), tmp);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) rc = rfail(R, SP_ECUDA, std::string("window remap: ") + cudaGetErrorString(e));
    }
    if (rc == SP_OK) rc = put_window(R, nw, tmp, cells);
  }
  if (rc != SP_OK) {
    if (nw) sp_destroy(nw);
    return rc;
  }
  if (R->w) sp_destroy(R->w);
  R->w = nw;
  std::copy(no, no + 3, R->o);
  std::copy(nd, nd + 3, R->d);
  return SP_OK;
}

// adjust_origin_to_from: dims kept
template <class T>
int shift_t(sp_regional* R, const int no[3]) {
  bool skip = true, replace = false;
  int s[3] = {0, 0, 0};
  for (int a = 0; a < R->D; ++a) {
    s[a] = no[a] - R->o[a];
    skip = skip && s[a] == 0;
  }
  if (skip) return SP_OK;
  for (int a = 0; a < R->D; ++a) replace = replace || std::abs(s[a]) + R->d[a] > R->G[a];
  if (replace || !R->w) return replace_t<T>(R, no, R->d);
  const long long cells = interior_cells(R, R->d);
  T* tmp = nullptr;
  if (int rc = grow(R, R->win, sizeof(T) * size_t(cells), &tmp)) return rc;
  const RegView<T> v = view_of<T>(R);
  k_reg_shift<T><<<blocks_for(cells), 256, 0, R->w->stream>>>(v, s[0], s[1], s[2], T(R->empty), tmp);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(R->w->stream);
  if (e != cudaSuccess) return rfail(R, SP_ECUDA, std::string("window shift: ") + cudaGetErrorString(e));
  const int rc = put_window(R, R->w, tmp, cells);
  if (rc == SP_OK) std::copy(no, no + 3, R->o);
  return rc;
}

// RegionalGrid::adjust(select_region) (grid.h:2118-2128)
int move(sp_regional* R, const int no[3], const int nd[3]) {
  bool same_d = true, same_o = true;
  for (int a = 0; a < R->D; ++a) {
    same_d = same_d && nd[a] == R->d[a];
    same_o = same_o && no[a] == R->o[a];
  }
  if (same_d && same_o) return SP_OK;
  if (same_d) return R->esz == 4 ? shift_t<float>(R, no) : shift_t<double>(R, no);
  return R->esz == 4 ? replace_t<float>(R, no, nd) : replace_t<double>(R, no, nd);
}

int search_target(sp_regional* R, int mode, double rel_eps, int no[3], int nd[3]) {
  std::vector<unsigned char> mask;
  if (int rc = R->esz == 4 ? mask_t<float>(R, mask) : mask_t<double>(R, mask)) return rc;
  Search s{};
  s.D = R->D;
  for (int a = 0; a < 3; ++a) {
    s.G[a] = R->G[a];
    s.o[a] = R->o[a];
    s.d[a] = R->d[a];
  }
  s.m = mask.empty() ? nullptr : mask.data();
  s.target(mode, R->p.padding_factor, rel_eps, no, nd);
  return SP_OK;
}

// update_regional_system (boundarysystem.h:438-471)
int update(sp_regional* R) {
  int no[3], nd[3];
  if (R->next_resize == 0) {
    double m0 = 0.0;
    if (int rc = R->esz == 4 ? min_t<float>(R, &m0) : min_t<double>(R, &m0)) return rc;
    R->cutoff = m0 + R->p.cutoff_eps;
    R->empty = m0;
    if (int rc = search_target(R, 1, 0.0, no, nd)) return rc;
    if (int rc = move(R, no, nd)) return rc;
    ++R->next_resize;
  } else if (R->next_resize > 0) {
    const int cur = int(R->time / R->p.resize_delta);
    if (cur >= R->next_resize) {
      if (int rc = search_target(R, R->p.fixed ? 0 : 1, 0.05, no, nd)) return rc;
      if (int rc = move(R, no, nd)) return rc;
      R->next_resize = cur + 1;
    }
  }
  return SP_OK;
}

bool update_due(const sp_regional* R, double t) {
  if (R->next_resize == 0) return true;
  return R->next_resize > 0 && int(t / R->p.resize_delta) >= R->next_resize;
}

}  // namespace

extern "C" {

int sp_regional_create(const sp_desc* desc, const sp_regional_params* params, sp_regional** out) {
  if (!out) return SP_EINVAL;
  *out = nullptr;
  g_reg_create_error.clear();
  if (!desc || !params) return g_reg_create_error = "null argument", SP_EINVAL;
  if (desc->batch != 1) return g_reg_create_error = "a regional system has batch 1", SP_EINVAL;
  if (desc->model == SP_MODEL_C)
    return g_reg_create_error = "single-field models only (each field of SymPhas's multi-field "
                                "models has a window of its own)", SP_EINVAL;
  if (desc->dim != 2 && desc->dim != 3) return g_reg_create_error = "dim must be 2 or 3", SP_EINVAL;
  for (int s = 0; s < 2 * desc->dim; ++s)
    if (desc->boundary[s] != SP_PERIODIC)
      return g_reg_create_error = "the domain of a regional system is periodic on every side", SP_EINVAL;
  if (!(params->resize_delta > 0.0) || !(params->padding_factor > 0.0) || !(params->cutoff_eps >= 0.0))
    return g_reg_create_error = "resize_delta and padding_factor must be > 0, cutoff_eps >= 0", SP_EINVAL;
  sp_regional* R = new sp_regional;
  R->gd = *desc;
  R->p = *params;
  R->D = desc->dim;
  R->esz = desc->dtype == SP_F32 ? 4 : 8;
  for (int a = 0; a < 3; ++a) {
    R->G[a] = a < R->D ? desc->n[a] + 2 * BD : 1;
    R->o[a] = 0;
    R->d[a] = R->G[a];
  }
  R->empty = 0.0;  // REGIONAL_GRID_OUTER_VALUE (grid.h:2022)
  if (int rc = make_window(R, R->o, R->d, &R->w)) {
    g_reg_create_error = R->err;
    delete R;
    return rc;
  }
  if (R->w && R->w->nf != 1) {
    g_reg_create_error = "single-field models only (each field of SymPhas's multi-field models "
                         "has a window of its own)";
    sp_destroy(R->w);
    delete R;
    return SP_EINVAL;
  }
  *out = R;
  return SP_OK;
}

int sp_regional_upload(sp_regional* R, const void* host, size_t bytes) {
  if (!R || !host) return SP_EINVAL;
  const long long n = (long long)R->gd.n[0] * R->gd.n[1] * (R->D == 3 ? R->gd.n[2] : 1);
  if (bytes != size_t(n) * R->esz) return rfail(R, SP_EINVAL, "bytes must be the whole domain's interior");
  if (!R->w) return SP_OK;
  void* g = nullptr;
  void* win = nullptr;
  const long long cells = interior_cells(R, R->d);
  if (int rc = grow(R, R->dom, bytes, &g)) return rc;
  if (int rc = grow(R, R->win, size_t(cells) * R->esz, &win)) return rc;
  cudaError_t e = cudaMemcpyAsync(g, host, bytes, cudaMemcpyHostToDevice, R->w->stream);
  if (e == cudaSuccess) {
    const Geo gg = geo_of(R, R->o, R->d);
    if (R->esz == 4)
      k_reg_gather<float><<<blocks_for(cells), 256, 0, R->w->stream>>>(gg, (const float*)g, (float*)win);
    else
      k_reg_gather<double><<<blocks_for(cells), 256, 0, R->w->stream>>>(gg, (const double*)g, (double*)win);
    e = cudaGetLastError();
  }
  const int rc = e == cudaSuccess
                     ? put_window(R, R->w, win, cells)
                     : rfail(R, SP_ECUDA, std::string("regional upload: ") + cudaGetErrorString(e));
  return rc;
}

int sp_regional_download(sp_regional* R, void* host, size_t bytes) {
  if (!R || !host) return SP_EINVAL;
  const long long n = (long long)R->gd.n[0] * R->gd.n[1] * (R->D == 3 ? R->gd.n[2] : 1);
  if (bytes != size_t(n) * R->esz) return rfail(R, SP_EINVAL, "bytes must be the whole domain's interior");
  if (!R->w) {
    for (long long i = 0; i < n; ++i) {
      if (R->esz == 4)
        static_cast<float*>(host)[i] = float(R->empty);
      else
        static_cast<double*>(host)[i] = R->empty;
    }
    return SP_OK;
  }
  void* g = nullptr;
  if (int rc = grow(R, R->dom, bytes, &g)) return rc;
  const Geo gg = geo_of(R, R->o, R->d);
  if (R->esz == 4)
    k_reg_scatter<float><<<blocks_for(n), 256, 0, R->w->stream>>>(gg, view_of<float>(R), float(R->empty), (float*)g);
  else
    k_reg_scatter<double><<<blocks_for(n), 256, 0, R->w->stream>>>(gg, view_of<double>(R), R->empty, (double*)g);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(host, g, bytes, cudaMemcpyDeviceToHost, R->w->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(R->w->stream);
  if (e != cudaSuccess) return rfail(R, SP_ECUDA, std::string("regional download: ") + cudaGetErrorString(e));
  return SP_OK;
}

int sp_regional_step(sp_regional* R, int nsteps) {
  if (!R || nsteps < 0) return SP_EINVAL;
  const double dt = R->gd.dt;
  int i = 0;
  while (i < nsteps) {
    if (int rc = update(R)) return rc;
    // the iterations after this one whose window check does nothing run
    // together, time accumulating step by step as in run_model
    int k = 1;
    double t = R->time + dt;
    while (i + k < nsteps && !update_due(R, t)) {
      t += dt;
      ++k;
    }
    if (R->w)
      if (int rc = sp_step(R->w, k)) return rfail(R, rc, sp_last_error(R->w));
    for (int j = 0; j < k; ++j) R->time += dt;
    i += k;
  }
  return SP_OK;
}

int sp_regional_adjust(sp_regional* R, const int origin[3], const int dims[3]) {
  if (!R || !origin || !dims) return SP_EINVAL;
  int no[3] = {0, 0, 0}, nd[3] = {1, 1, 1};
  for (int a = 0; a < R->D; ++a) {
    if (dims[a] < 0 || dims[a] > R->G[a])
      return rfail(R, SP_EINVAL, "window dims must be in [0, domain extent + 6]");
    if (dims[a] > 2 * BD && dims[a] - 2 * BD < 4)
      return rfail(R, SP_EINVAL, "a window interior below 4 cells is not supported");
    no[a] = origin[a];
    nd[a] = dims[a];
  }
  return move(R, no, nd);
}

int sp_regional_window(const sp_regional* R, int origin[3], int dims[3], double state[4]) {
  if (!R) return SP_EINVAL;
  for (int a = 0; a < 3; ++a) {
    if (origin) origin[a] = R->o[a];
    if (dims) dims[a] = R->d[a];
  }
  if (state) {
    state[0] = R->empty;
    state[1] = R->cutoff;
    state[2] = R->time;
    state[3] = R->next_resize;
  }
  return SP_OK;
}

int sp_regional_set_dt(sp_regional* R, double dt) {
  if (!R) return SP_EINVAL;
  if (R->w)
    if (int rc = sp_set_dt(R->w, dt)) return rfail(R, rc, sp_last_error(R->w));
  R->gd.dt = dt;
  return SP_OK;
}

int sp_regional_set_stream(sp_regional* R, void* stream) {
  if (!R) return SP_EINVAL;
  if (R->w)
    if (int rc = sp_set_stream(R->w, stream)) return rfail(R, rc, sp_last_error(R->w));
  R->stream = stream;
  return SP_OK;
}

sp_handle* sp_regional_handle(sp_regional* R) { return R ? R->w : nullptr; }

const char* sp_regional_error(const sp_regional* R) {
  return R ? R->err.c_str() : g_reg_create_error.c_str();
}

void sp_regional_destroy(sp_regional* R) {
  if (!R) return;
  if (R->w) sp_destroy(R->w);
  for (sp_regional::Scratch* sc : {&R->dom, &R->win, &R->msk, &R->red})
    if (sc->p) cudaFree(sc->p);
  delete R;
}

int sp_region_search(int dim, const int G[3], const int origin[3], const int dims[3],
                     const unsigned char* mask, int mode, double factor, double rel_eps,
                     int new_origin[3], int new_dims[3]) {
  if ((dim != 2 && dim != 3) || !G || !origin || !dims || !new_origin || !new_dims) return SP_EINVAL;
  if (mode != 0 && mode != 1) return SP_EINVAL;
  Search s{};
  s.D = dim;
  for (int a = 0; a < 3; ++a) {
    s.G[a] = a < dim ? G[a] : 1;
    s.o[a] = a < dim ? origin[a] : 0;
    s.d[a] = a < dim ? dims[a] : 1;
  }
  s.m = mask;
  s.target(mode, factor, rel_eps, new_origin, new_dims);
  return SP_OK;
}

}  // extern "C"
