/*
 * sp_kernels.cuh -- fused forward-Euler step kernels for sm_100a.
 *
 * One launch = one SolverFT iteration of every field of every instance: it
 * reads each field once from HBM (TMA tiles into shared memory), evaluates
 * the lowered EVOLUTION right-hand sides, applies psi + dt * dframe, writes
 * the result once, and refreshes the periodic halo of the output in the same
 * pass (a site within the stencil reach of a periodic face also stores its
 * image into the halo).  This replaces, per step, the reference's halo pass
 * (datatypes/inc/boundaryupdate.h:154-356), its temporaries for derivatives of
 * expressions (sym/inc/expressionderivatives.h:1546-1588), the evaluation into
 * dframe (examples/solvers/solverft.h:90-103) and the Euler pass (:46-50).
 *
 * Device layout of a field: x-fastest, interior n[0] x n[1] (x n[2]) inside a
 * halo of h[0] cells in x (the stencil reach rounded up to 16 bytes, so every
 * TMA box starts aligned) and R cells in y and z; rows are padded to a
 * multiple of 16 bytes.  Fields ping-pong between two buffers.
 *
 * 3D: a CTA owns a TX x TY column of the xy-plane and marches through a chunk
 * of z; field planes stream through a ring of 2R+2 shared-memory slots, each
 * filled by one TMA box load one plane ahead of use; staged operands (the
 * fused form) live in a ring of 2RS+1 planes.
 * 2D: a persistent grid pulls TX x TY tiles from an atomic work queue that may
 * span many independent instances of different sizes and models (the
 * ensemble); the next tile's TMA load overlaps the current tile's compute.
 */
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "sp_expr.cuh"
#include "sp_tma.cuh"

namespace sp {

constexpr int ceil_to(int a, int b) { return (a + b - 1) / b * b; }
constexpr int imax(int a, int b) { return a > b ? a : b; }

enum : int { KERR_NONE = 0, KERR_TMA_TIMEOUT = 1 };

// x halo (elements) for a stencil reach R: R rounded up to 16 bytes
template <class T>
constexpr int halo_x(int R) {
  return ceil_to(R > 0 ? R : 1, 16 / (int)sizeof(T));
}

template <class T>
struct StepParams {
  const CUtensorMap* maps;  // input tensor maps, [inst * nf + f]
  T* const* out;            // output padded origins, [inst * nf + f]
  int n[3];                 // interior extents
  int h[3];                 // halo widths
  long long pitch, plane;   // padded row and plane, in elements
  int per[3];               // 1 = periodic axis: store halo images
  int ntx, nty, zchunk;     // tiles along x and y; z planes per CTA
  int rhs_only;             // 1 = store dframe instead of stepping
  T dt, divh2, divh3, divh4;
  T coef[8];
  double* partial;  // per-CTA FP64 sum of the new field 0, or null
  int* err;         // device error flag
};

template <class T>
struct Inst2 {  // one instance of the 2D persistent kernel
  int n[2];
  int per[2];
  long long pitch;
  int ntx;
  int kind;  // 0 = first model, 1 = second model
  T dt, divh2, divh3, divh4;
  T coef[8];
};

template <class T>
struct Step2Params {
  const CUtensorMap* maps;  // input tensor maps, [inst * nf + f]
  T* const* out;            // output padded origins, [inst * nf + f]
  const Inst2<T>* inst;     // [ninst]
  const int2* items;        // [nitems] (instance, tile) or null: instance 0, tile = item
  int nitems;
  int* ctr;  // [0] work-queue counter, [1] finished-CTA counter; both are
             // zero on entry and the last CTA to finish zeroes them again
  int rhs_only;
  int hx, hy;       // common halo of every instance
  double* partial;  // per-CTA FP64 sum of the new field 0 (single instance), or null
  int* err;
};

// Evaluation context of one site: shared-memory offsets of the field planes
// (NZ planes centred at ZR) and staged-operand planes, all relative to `base`.
template <class T, int DIM, int LP, int GP, int BP, int NF, int NZ, int ZR, int PW, int NS,
          int NSZ, int SZR, int SW>
struct Ctx {
  using value_type = T;
  static constexpr int dim = DIM, lap_points = LP, gradlap_points = GP, bilap_points = BP;
  const T* base;
  int fo[NF][NZ];
  int so[NS > 0 ? NS : 1][NSZ > 0 ? NSZ : 1];
  T divh2, divh3, divh4;
  const T* cf;
  template <int I, int X, int Y, int Z>
  __device__ __forceinline__ T var() const {
    static_assert(I >= 1 && I <= NF, "field index");
    static_assert(Z + ZR >= 0 && Z + ZR < NZ, "z reach beyond the loaded planes");
    static_assert(DIM == 3 || Z == 0, "z offset in 2D");
    return base[fo[I - 1][Z + ZR] + Y * PW + X];
  }
  template <int K, int X, int Y, int Z>
  __device__ __forceinline__ T stg() const {
    static_assert(K >= 0 && K < NS, "stage index");
    static_assert(Z + SZR >= 0 && Z + SZR < NSZ, "z reach beyond the staged planes");
    return base[so[K][Z + SZR] + Y * SW + X];
  }
  __device__ __forceinline__ T coef(int i) const { return cf[i - 1]; }
};

// store v at interior (x,y,z) of a padded field and, along periodic axes, at
// its images in the halo that lie within the stencil reach R
template <class T, int DIM, int R>
__device__ __forceinline__ void store_with_images(T* org, int x, int y, int z, T v, const int* n,
                                                  const int* h, const int* per, long long pitch,
                                                  long long plane) {
  long long xs[2], ys[2], zs[2];
  int cx = 1, cy = 1, cz = 1;
  xs[0] = x + h[0];
  ys[0] = y + h[1];
  zs[0] = (DIM == 3) ? z + h[2] : 0;
  if (R > 0) {
    if (per[0]) {
      if (x < R) xs[cx++] = xs[0] + n[0];
      else if (x >= n[0] - R) xs[cx++] = xs[0] - n[0];
    }
    if (per[1]) {
      if (y < R) ys[cy++] = ys[0] + n[1];
      else if (y >= n[1] - R) ys[cy++] = ys[0] - n[1];
    }
    if (DIM == 3 && per[2]) {
      if (z < R) zs[cz++] = zs[0] + n[2];
      else if (z >= n[2] - R) zs[cz++] = zs[0] - n[2];
    }
  }
  for (int k = 0; k < cz; ++k)
    for (int j = 0; j < cy; ++j)
      for (int i = 0; i < cx; ++i) org[zs[k] * plane + ys[j] * pitch + xs[i]] = v;
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < NT / 32; ++i) s += red[i];
  return s;
}

// ---------------------------------------------------------------------------
// tile configuration: TX x TY sites per CTA (per plane in 3D), SPT consecutive
// rows per thread, PD planes (3D) or tiles (2D) of TMA prefetch in flight
// ---------------------------------------------------------------------------
template <int TX_, int TY_, int SPT_, int PD_>
struct TileCfg {
  static constexpr int TX = TX_, TY = TY_, SPT = SPT_, PD = PD_;
  static_assert(TY % SPT == 0, "rows per thread must divide the tile height");
  static constexpr int NT = TX * TY / SPT;
  static_assert(NT % 32 == 0 && NT <= 1024, "threads per CTA");
};

// ---------------------------------------------------------------------------
// 3D: z-marching fused step
// ---------------------------------------------------------------------------
template <class M, class T, int LP, int GP, int BP, class TC>
struct Fd3 {
  static constexpr int TX = TC::TX, TY = TC::TY, SPT = TC::SPT, PD = TC::PD, NT = TC::NT;
  static constexpr int NF = M::nf, NS = M::ns, R = M::R, RS = M::RS;
  static constexpr int HXA = halo_x<T>(R);
  static constexpr int PW = TX + 2 * HXA, PH = TY + 2 * R;
  static constexpr int PLANE = ceil_to(PW * PH, 128 / (int)sizeof(T));
  static constexpr int NSLOT = 2 * R + 1 + PD;
  static constexpr int SW = TX + 2 * RS, SH = TY + 2 * RS, SPL = ceil_to(SW * SH, 32);
  static constexpr int NSR = NS > 0 ? 2 * RS + 1 : 0;
  static constexpr int RD = imax(M::r_direct, 0);  // z reach of the rhs into fields
  static constexpr int RI = imax(M::r_stage, 0);   // z reach of a stage into fields
  static constexpr size_t SMEM =
      256 + sizeof(T) * (size_t(NF) * NSLOT * PLANE + size_t(NS) * NSR * SPL);
  static_assert(NSLOT <= 32, "barrier header holds 32 slots");
  static_assert(PW <= 256 && PH <= 256, "TMA box limit");
  static_assert((PW * sizeof(T)) % 16 == 0, "TMA box rows must be whole 16-byte units");
};

template <class M, class T, int LP, int GP, int BP, class TC>
__global__ void __launch_bounds__(TC::NT)
    k_fd3d(const __grid_constant__ StepParams<T> p, const __grid_constant__ M m) {
  using K = Fd3<M, T, LP, GP, BP, TC>;
  constexpr int TX = K::TX, SPT = K::SPT, PD = K::PD, NF = K::NF, NS = K::NS, R = K::R,
                RS = K::RS, HXA = K::HXA, PW = K::PW, PH = K::PH, PLANE = K::PLANE,
                NSLOT = K::NSLOT, SW = K::SW, SPL = K::SPL, NSR = K::NSR, NT = K::NT,
                RD = K::RD, RI = K::RI;
  constexpr uint32_t TXB = uint32_t(NF * PW * PH * sizeof(T));

  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  T* fbuf = reinterpret_cast<T*>(smem_raw + 256);
  T* sbuf = fbuf + NF * NSLOT * PLANE;
  __shared__ double red[32];

  const int tid = threadIdx.x, tx = tid % TX, row0 = (tid / TX) * SPT;
  const int tile = blockIdx.x;
  const int x0 = (tile % p.ntx) * TX, y0 = (tile / p.ntx) * K::TY;
  const int zb = blockIdx.y * p.zchunk;
  const int ze = min(zb + p.zchunk, p.n[2]);
  const int inst = blockIdx.z;
  const CUtensorMap* maps = p.maps + inst * NF;
  const int nplanes = (ze - zb) + 2 * R;

  if (tid == 0) {
    for (int s = 0; s < NSLOT; ++s) tma::mbar_init(&bars[s], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();

  // plane sequence q <-> z = zb - R + q, slot q % NSLOT, phase (q / NSLOT) & 1
  auto issue = [&](int q) {
    const int s = q % NSLOT;
    tma::mbar_arrive_expect_tx(&bars[s], TXB);
    const int zz = zb - R + q + p.h[2];
#pragma unroll
    for (int f = 0; f < NF; ++f)
      tma::load_3d(fbuf + (f * NSLOT + s) * PLANE, maps + f, &bars[s], x0 + p.h[0] - HXA,
                   y0 + p.h[1] - R, zz);
  };
  if (tid == 0) {
    const int pro = min(2 * R + PD, nplanes);
    for (int q = 0; q < pro; ++q) issue(q);
  }

  const int x = x0 + tx;
  double msum = 0.0;

  for (int z = zb; z < ze; ++z) {
    const int qz = z - zb + R;
    if (tid == 0 && qz + R + PD < nplanes) issue(qz + R + PD);
    bool bad = false;
    for (int q = (z == zb) ? 0 : qz + R; q <= qz + R; ++q)
      bad |= !tma::mbar_wait(&bars[q % NSLOT], (q / NSLOT) & 1);
    if (__syncthreads_or(bad)) {
      if (tid == 0) atomicExch(p.err, KERR_TMA_TIMEOUT);
      return;
    }

    if constexpr (NS > 0) {
      using CS = Ctx<T, 3, LP, GP, BP, NF, 2 * RI + 1, RI, PW, 1, 1, 0, SW>;
      for (int zs = (z == zb) ? z - RS : z + RS; zs <= z + RS; ++zs) {
        const int qs = zs - zb + R;
        const int sslot = (zs - zb + RS) % NSR;
        int fslot[2 * RI + 1];
#pragma unroll
        for (int dz = -RI; dz <= RI; ++dz) fslot[dz + RI] = ((qs + dz) % NSLOT) * PLANE;
        for (int c = tid; c < SW * K::SH; c += NT) {
          const int sy = c / SW, sx = c % SW;
          CS ctx;
          ctx.base = fbuf;
          const int cell = (sy - RS + R) * PW + (sx - RS + HXA);
#pragma unroll
          for (int f = 0; f < NF; ++f)
#pragma unroll
            for (int dz = -RI; dz <= RI; ++dz)
              ctx.fo[f][dz + RI] = f * NSLOT * PLANE + fslot[dz + RI] + cell;
          ctx.divh2 = p.divh2;
          ctx.divh3 = p.divh3;
          ctx.divh4 = p.divh4;
          ctx.cf = p.coef;
          sbuf[sslot * SPL + c] = eval(m.s0, ctx);
          if constexpr (NS > 1) sbuf[(NSR + sslot) * SPL + c] = eval(m.s1, ctx);
        }
      }
      __syncthreads();
    }

    {
      using CO = Ctx<T, 3, LP, GP, BP, NF, 2 * RD + 1, RD, PW, NS, (NS > 0 ? 2 * RS + 1 : 1),
                     (NS > 0 ? RS : 0), SW>;
      CO c0;
      c0.base = fbuf;
      const int cell = (row0 + R) * PW + tx + HXA;
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int dz = -RD; dz <= RD; ++dz)
          c0.fo[f][dz + RD] = (f * NSLOT + (qz + dz) % NSLOT) * PLANE + cell;
      if constexpr (NS > 0) {
        const int scell = int(sbuf - fbuf) + (row0 + RS) * SW + tx + RS;
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
          for (int dz = -RS; dz <= RS; ++dz)
            c0.so[k][dz + RS] = (k * NSR + (z + dz - zb + RS) % NSR) * SPL + scell;
      }
      c0.divh2 = p.divh2;
      c0.divh3 = p.divh3;
      c0.divh4 = p.divh4;
      c0.cf = p.coef;
#pragma unroll
      for (int k = 0; k < SPT; ++k) {
        CO ctx = c0;
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
          for (int dz = 0; dz < 2 * RD + 1; ++dz) ctx.fo[f][dz] += k * PW;
        if constexpr (NS > 0) {
#pragma unroll
          for (int kk = 0; kk < NS; ++kk)
#pragma unroll
            for (int dz = 0; dz < 2 * RS + 1; ++dz) ctx.so[kk][dz] += k * SW;
        }
        const int y = y0 + row0 + k;
        const T r0 = eval(m.r0, ctx);
        T r1 = T(0);
        if constexpr (NF > 1) r1 = eval(m.r1, ctx);
        if (x < p.n[0] && y < p.n[1]) {
          const T v0c = ctx.template var<1, 0, 0, 0>();
          const T v0 = p.rhs_only ? r0 : v0c + p.dt * r0;
          store_with_images<T, 3, R>(p.out[inst * NF], x, y, z, v0, p.n, p.h, p.per, p.pitch,
                                     p.plane);
          msum += double(v0);
          if constexpr (NF > 1) {
            const T v1c = ctx.template var<2, 0, 0, 0>();
            const T v1 = p.rhs_only ? r1 : v1c + p.dt * r1;
            store_with_images<T, 3, R>(p.out[inst * NF + 1], x, y, z, v1, p.n, p.h, p.per,
                                       p.pitch, p.plane);
          }
        }
      }
    }
    __syncthreads();
  }

  if (p.partial) {
    const double s = block_sum<NT>(msum, red);
    if (tid == 0)
      p.partial[(size_t(blockIdx.z) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
  }
}

// ---------------------------------------------------------------------------
// 2D: persistent tile-queue fused step over one or many instances
// ---------------------------------------------------------------------------
template <class M0, class M1, class T, int LP, int GP, int BP, class TC>
struct Fd2 {
  static_assert(M0::nf == M1::nf, "models of one launch share the field count");
  static constexpr int TX = TC::TX, TY = TC::TY, SPT = TC::SPT, PD = TC::PD, NT = TC::NT;
  static constexpr int NF = M0::nf;
  static constexpr int NS = imax(M0::ns, M1::ns);
  static constexpr int R = imax(M0::R, M1::R);
  static constexpr int RS = imax(M0::RS, M1::RS);
  static_assert(M0::ns == 0 || M0::RS == RS, "staged models of one launch share the reach");
  static_assert(M1::ns == 0 || M1::RS == RS, "staged models of one launch share the reach");
  static constexpr int HXA = halo_x<T>(R);
  static constexpr int PW = TX + 2 * HXA, PH = TY + 2 * R;
  static constexpr int PLANE = ceil_to(PW * PH, 128 / (int)sizeof(T));
  static constexpr int NQ = PD + 1;  // tile slots: the current one and PD in flight
  static constexpr int SW = TX + 2 * RS, SH = TY + 2 * RS, SPL = ceil_to(SW * SH, 32);
  static constexpr size_t SMEM = 256 + sizeof(T) * (size_t(NQ) * NF * PLANE + size_t(NS) * SPL);
  static_assert(NQ <= 16, "barrier header holds 16 slots");
  static_assert(PW <= 256 && PH <= 256, "TMA box limit");
  static_assert((PW * sizeof(T)) % 16 == 0, "TMA box rows must be whole 16-byte units");
};

template <class K, class M, class T, int LP, int GP, int BP>
__device__ __forceinline__ void fd2_tile(const Step2Params<T>& p, const M& m,
                                         const Inst2<T>& ip, int ii, const T* fbuf, T* sbuf,
                                         int slot, int x0, int y0, double& msum) {
  constexpr int TX = K::TX, SPT = K::SPT, NF = K::NF, R = K::R, RS = K::RS, HXA = K::HXA,
                PW = K::PW, PLANE = K::PLANE, SW = K::SW, NT = K::NT;
  constexpr int NS = M::ns;
  const int tid = threadIdx.x, tx = tid % TX, row0 = (tid / TX) * SPT;
  if constexpr (NS > 0) {
    using CS = Ctx<T, 2, LP, GP, BP, NF, 1, 0, PW, 1, 1, 0, SW>;
    for (int c = tid; c < SW * K::SH; c += NT) {
      const int sy = c / SW, sx = c % SW;
      CS ctx;
      ctx.base = fbuf;
      const int cell = (sy - RS + R) * PW + (sx - RS + HXA);
#pragma unroll
      for (int f = 0; f < NF; ++f) ctx.fo[f][0] = (slot * NF + f) * PLANE + cell;
      ctx.divh2 = ip.divh2;
      ctx.divh3 = ip.divh3;
      ctx.divh4 = ip.divh4;
      ctx.cf = ip.coef;
      sbuf[c] = eval(m.s0, ctx);
      if constexpr (NS > 1) sbuf[K::SPL + c] = eval(m.s1, ctx);
    }
    __syncthreads();
  }
  using CO = Ctx<T, 2, LP, GP, BP, NF, 1, 0, PW, NS, 1, 0, SW>;
  CO c0;
  c0.base = fbuf;
  const int cell = (row0 + R) * PW + tx + HXA;
#pragma unroll
  for (int f = 0; f < NF; ++f) c0.fo[f][0] = (slot * NF + f) * PLANE + cell;
  if constexpr (NS > 0) {
    const int scell = int(sbuf - fbuf) + (row0 + RS) * SW + tx + RS;
#pragma unroll
    for (int k = 0; k < NS; ++k) c0.so[k][0] = k * K::SPL + scell;
  }
  c0.divh2 = ip.divh2;
  c0.divh3 = ip.divh3;
  c0.divh4 = ip.divh4;
  c0.cf = ip.coef;
  const int x = x0 + tx;
  const int h[3] = {p.hx, p.hy, 0};
  const int n3[3] = {ip.n[0], ip.n[1], 1};
  const int per3[3] = {ip.per[0], ip.per[1], 0};
#pragma unroll
  for (int k = 0; k < SPT; ++k) {
    CO ctx = c0;
#pragma unroll
    for (int f = 0; f < NF; ++f) ctx.fo[f][0] += k * PW;
    if constexpr (NS > 0) {
#pragma unroll
      for (int kk = 0; kk < NS; ++kk) ctx.so[kk][0] += k * SW;
    }
    const int y = y0 + row0 + k;
    const T r0 = eval(m.r0, ctx);
    T r1 = T(0);
    if constexpr (NF > 1) r1 = eval(m.r1, ctx);
    if (x < ip.n[0] && y < ip.n[1]) {
      const T v0c = ctx.template var<1, 0, 0, 0>();
      const T v0 = p.rhs_only ? r0 : v0c + ip.dt * r0;
      store_with_images<T, 2, R>(p.out[ii * NF], x, y, 0, v0, n3, h, per3, ip.pitch, 0);
      msum += double(v0);
      if constexpr (NF > 1) {
        const T v1c = ctx.template var<2, 0, 0, 0>();
        const T v1 = p.rhs_only ? r1 : v1c + ip.dt * r1;
        store_with_images<T, 2, R>(p.out[ii * NF + 1], x, y, 0, v1, n3, h, per3, ip.pitch, 0);
      }
    }
  }
}

template <class M0, class M1, class T, int LP, int GP, int BP, class TC>
__global__ void __launch_bounds__(TC::NT)
    k_fd2d(const __grid_constant__ Step2Params<T> p, const __grid_constant__ M0 m0,
           const __grid_constant__ M1 m1) {
  using K = Fd2<M0, M1, T, LP, GP, BP, TC>;
  constexpr int TX = K::TX, TY = K::TY, PD = K::PD, NQ = K::NQ, NF = K::NF, R = K::R,
                HXA = K::HXA, PW = K::PW, PH = K::PH, PLANE = K::PLANE, NT = K::NT;
  constexpr uint32_t TXB = uint32_t(NF * PW * PH * sizeof(T));

  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);      // [16]
  int2* items = reinterpret_cast<int2*>(smem_raw + 128);        // [16]
  T* fbuf = reinterpret_cast<T*>(smem_raw + 256);
  T* sbuf = fbuf + NQ * NF * PLANE;
  __shared__ double red[32];
  const int tid = threadIdx.x;

  auto fetch = [&]() -> int2 {
    const int t = atomicAdd(&p.ctr[0], 1);
    if (t >= p.nitems) return make_int2(-1, 0);
    return p.items ? p.items[t] : make_int2(0, t);
  };
  auto issue = [&](int2 it, int slot) {
    const Inst2<T>& ip = p.inst[it.x];
    const int x0 = (it.y % ip.ntx) * TX, y0 = (it.y / ip.ntx) * TY;
    tma::mbar_arrive_expect_tx(&bars[slot], TXB);
#pragma unroll
    for (int f = 0; f < NF; ++f)
      tma::load_2d(fbuf + (slot * NF + f) * PLANE, p.maps + it.x * NF + f, &bars[slot],
                   x0 + p.hx - HXA, y0 + p.hy - R);
  };

  if (tid == 0) {
    for (int s = 0; s < NQ; ++s) tma::mbar_init(&bars[s], 1);
    tma::fence_barrier_init();
    for (int s = 0; s < PD; ++s) {
      const int2 it = fetch();
      items[s] = it;
      if (it.x >= 0) issue(it, s);
    }
  }
  __syncthreads();

  double msum = 0.0;
  for (int it = 0;; ++it) {
    const int slot = it % NQ;
    const volatile int* vi = reinterpret_cast<volatile int*>(&items[slot]);
    const int2 cur = make_int2(vi[0], vi[1]);
    if (cur.x < 0) break;
    if (tid == 0) {
      const int2 nxt = fetch();
      const int ns = (it + PD) % NQ;
      items[ns] = nxt;
      if (nxt.x >= 0) issue(nxt, ns);
    }
    const bool bad = !tma::mbar_wait(&bars[slot], (it / NQ) & 1);
    if (__syncthreads_or(bad)) {
      if (tid == 0) atomicExch(p.err, KERR_TMA_TIMEOUT);
      return;
    }
    const Inst2<T>& ip = p.inst[cur.x];
    const int x0 = (cur.y % ip.ntx) * TX, y0 = (cur.y / ip.ntx) * TY;
    if (ip.kind == 0)
      fd2_tile<K, M0, T, LP, GP, BP>(p, m0, ip, cur.x, fbuf, sbuf, slot, x0, y0, msum);
    else
      fd2_tile<K, M1, T, LP, GP, BP>(p, m1, ip, cur.x, fbuf, sbuf, slot, x0, y0, msum);
    __syncthreads();
  }
  if (tid == 0) {
    // the last CTA to leave the queue re-arms it for the next launch
    __threadfence();
    if (atomicAdd(&p.ctr[1], 1) == int(gridDim.x) - 1) {
      p.ctr[0] = 0;
      p.ctr[1] = 0;
      __threadfence();
    }
  }
  if (p.partial) {
    const double s = block_sum<NT>(msum, red);
    if (tid == 0) p.partial[blockIdx.x] = s;
  }
}

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
};

template <class T>
__global__ void k_fill_halo(const HaloParams<T> p) {
  const long long L0 = p.n[0] + 2 * p.h[0], L1 = p.n[1] + 2 * p.h[1];
  const long long L2 = (p.dim == 3) ? p.n[2] + 2 * p.h[2] : 1;
  const long long total = L0 * L1 * L2;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const long long i = id % L0, j = (id / L0) % L1, k = id / (L0 * L1);
    long long c[3] = {i - p.h[0], j - p.h[1], (p.dim == 3) ? k - p.h[2] : 0};
    bool outside = false;
    for (int a = 0; a < p.dim; ++a)
      if (c[a] < 0 || c[a] >= p.n[a]) outside = true;
    if (!outside) continue;
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

}  // namespace sp
