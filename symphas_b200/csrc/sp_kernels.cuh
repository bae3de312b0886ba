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
 * of z; field planes stream through a ring of 2R+1+PD shared-memory slots,
 * each filled by one TMA box load PD planes ahead of use; staged operands
 * (the fused form) live in a ring of 2RS+1 planes.
 * 2D: a persistent grid pulls TX x TY tiles from an atomic work queue that may
 * span many independent instances of different sizes and models (the
 * ensemble); PD tiles are in flight while one is computed.
 * In both, a thread evaluates W consecutive x-sites (Vec<T,W>) on SPT
 * consecutive rows, so shared-memory words are 8 or 16 bytes wide and
 * neighbouring rows' loads are shared.
 */
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "sp_common.cuh"
#include "sp_expr.cuh"
#include "sp_tma.cuh"

namespace sp {

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
  const int2* items;        // [nitems] (instance, tile x | tile y << 16), or null:
                            // instance 0, linear tile index = item
  int nitems;
  int* ctr;  // [0] work-queue counter, [1] finished-CTA counter; both are
             // zero on entry and the last CTA to finish zeroes them again
  int rhs_only;
  int hx, hy;       // common halo of every instance
  double* partial;  // per-CTA FP64 sum of the new field 0 (single instance), or null
  int* err;
  // temporally blocked kernels (sp_tb2.cuh): input padded origins,
  // [inst * nf + f], and the steps of this launch (1 .. the kernel's KT)
  const T* const* in;
  int tsteps;
};

// ---------------------------------------------------------------------------
// tile configuration: TX x TY sites per CTA (per plane in 3D), W consecutive
// x-sites and SPT consecutive rows per thread, PD planes (3D) or tiles (2D) of
// TMA prefetch in flight
// ---------------------------------------------------------------------------
template <int TX_, int TY_, int SPT_, int PD_, int W_>
struct TileCfg {
  static constexpr int TX = TX_, TY = TY_, SPT = SPT_, PD = PD_, W = W_;
  static_assert(TX % W == 0 && TY % SPT == 0, "tile must split into thread groups");
  static constexpr int TXT = TX / W;  // threads along a row
  static constexpr int NT = TXT * (TY / SPT);
  static_assert(NT % 32 == 0 && NT <= 1024, "threads per CTA");
};

// halo geometry shared by the kernels and the host: x halo HXA covers the
// stencil reach R and the stage ring (RSA = RS rounded up to W, plus the
// stage's own reach RI), rounded up to 16 bytes.  With W > 2 the ring's column
// groups are wider than the RS columns the output reads from them: only those
// RS columns need their stencil inside the halo (RS + RI), the group's other
// lanes are computed from whatever lies next to the row in shared memory and
// are never read, so W = 2 and W = 4 tiles share one field layout.
template <class T, int W, int R, int NS, int RS, int RI>
struct HaloGeom {
  static constexpr int RSA = NS > 0 ? ceil_to(imax(RS, 1), W) : 0;
  static constexpr int RX = W > 2 ? imax(RS, 1) : RSA;
  static constexpr int HXA = ceil_to(imax(imax(R, 1), NS > 0 ? RX + RI : 0),
                                     imax(16 / (int)sizeof(T), W));
};

// Store the W values of one site group at interior (x, y, z) (x a multiple of
// W).  Interior groups take one vector store; groups within the stencil reach
// of a periodic face also store their images into the halo, element by element.
template <class T, int W, int DIM, int R>
__device__ __forceinline__ void store_group(T* org, int x, int y, int z, const vec_t<T, W>& v,
                                            const int* n, const int* h, const int* per,
                                            long long pitch, long long plane) {
  if (x + W <= n[0] && n[0] % W == 0) {
    // whole group: it and each of its periodic images is one vector store
    int xs[2] = {x + h[0], 0}, ys[2] = {y + h[1], 0}, zs[2] = {DIM == 3 ? z + h[2] : 0, 0};
    int cx = 1, cy = 1, cz = 1;
    if (R > 0) {
      if (per[0]) {
        if (x < R) xs[cx++] = xs[0] + n[0];
        else if (x + W > n[0] - R) xs[cx++] = xs[0] - n[0];
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
        for (int i = 0; i < cx; ++i)
          *reinterpret_cast<vec_t<T, W>*>(org + (long long)zs[k] * plane +
                                          (long long)ys[j] * pitch + xs[i]) = v;
    return;
  }
  // ragged end of a row: element by element
#pragma unroll
  for (int j = 0; j < W; ++j) {
    const int xj = x + j;
    if (xj >= n[0]) break;
    const T s = lane(v, j);
    long long xs[2], ys[2], zs[2];
    int cx = 1, cy = 1, cz = 1;
    xs[0] = xj + h[0];
    ys[0] = y + h[1];
    zs[0] = (DIM == 3) ? z + h[2] : 0;
    if (per[0]) {
      if (xj < R) xs[cx++] = xs[0] + n[0];
      else if (xj >= n[0] - R) xs[cx++] = xs[0] - n[0];
    }
    if (per[1]) {
      if (y < R) ys[cy++] = ys[0] + n[1];
      else if (y >= n[1] - R) ys[cy++] = ys[0] - n[1];
    }
    if (DIM == 3 && per[2]) {
      if (z < R) zs[cz++] = zs[0] + n[2];
      else if (z >= n[2] - R) zs[cz++] = zs[0] - n[2];
    }
    for (int k = 0; k < cz; ++k)
      for (int jj = 0; jj < cy; ++jj)
        for (int i = 0; i < cx; ++i) org[zs[k] * plane + ys[jj] * pitch + xs[i]] = s;
  }
}

// offset (in elements) of the periodic image of coordinate c along an axis of
// length n and halo stride `stride`, or 0 when c is farther than R from both
// faces; `w` is the width of the group stored at c
__device__ __forceinline__ long long image_offset(int per, int c, int w, int n, int R,
                                                  long long stride) {
  if (!per) return 0;
  if (c < R) return (long long)n * stride;
  if (c + w > n - R) return -(long long)n * stride;
  return 0;
}

// Vector store of v at p when `on`, as one predicated instruction.  Periodic
// images belong to the lanes at a face, and those lanes sit in every warp of
// a face tile: a branch around their stores would diverge every such warp,
// a predicated store costs each warp one issue slot.  p need only be a valid
// address when `on`.
__device__ __forceinline__ void st_if(float* p, const Vec<float, 2>& v, bool on) {
  asm volatile(
      "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %3, 0;\n\t"
      "@q st.global.v2.f32 [%0], {%1, %2};\n\t}" ::"l"(p),
      "f"(v.v[0]), "f"(v.v[1]), "r"(int(on))
      : "memory");
}
__device__ __forceinline__ void st_if(float* p, const Vec<float, 4>& v, bool on) {
  asm volatile(
      "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %5, 0;\n\t"
      "@q st.global.v4.f32 [%0], {%1, %2, %3, %4};\n\t}" ::"l"(p),
      "f"(v.v[0]), "f"(v.v[1]), "f"(v.v[2]), "f"(v.v[3]), "r"(int(on))
      : "memory");
}
__device__ __forceinline__ void st_if(double* p, const Vec<double, 2>& v, bool on) {
  asm volatile(
      "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %3, 0;\n\t"
      "@q st.global.v2.f64 [%0], {%1, %2};\n\t}" ::"l"(p),
      "d"(v.v[0]), "d"(v.v[1]), "r"(int(on))
      : "memory");
}
template <class T, class V>
__device__ __forceinline__ void st_if(T* p, const V& v, bool on) {
  if (on) *reinterpret_cast<V*>(p) = v;
}

// A whole W-group at b (padded address of an interior site) and its periodic
// images (offsets xo, yo, zo; 0 where there is none); `in` says whether the
// group exists.  xany: some lane of the block has an x image (block-uniform);
// yo is uniform across a warp (a warp holds whole rows) and zo across the
// block (one plane), so only the x images are predicated per lane and the
// other cases are uniform branches.
template <class T, class V>
__device__ __forceinline__ void put_images_pred(T* b, const V& v, bool in, bool xany,
                                                long long xo, long long yo, long long zo) {
  const bool xi = in && xo != 0;
  st_if(b, v, in);
  if (xany) st_if(b + xo, v, xi);
  if (yo != 0) {
    st_if(b + yo, v, in);
    if (xany) st_if(b + xo + yo, v, xi);
  }
  if (zo != 0) {
    st_if(b + zo, v, in);
    if (xany) st_if(b + zo + xo, v, xi);
    if (yo != 0) {
      st_if(b + zo + yo, v, in);
      if (xany) st_if(b + zo + xo + yo, v, xi);
    }
  }
}

// (s + d) mod N for 0 <= s < N and |d| < N, without a division
template <int N>
__device__ __forceinline__ int wrap(int s, int d) {
  int r = s + d;
  r += (r < 0) ? N : 0;
  r -= (r >= N) ? N : 0;
  return r;
}

template <class T, int W>
__device__ __forceinline__ double vsum(const vec_t<T, W>& v, int x, int n0) {
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < W; ++j)
    if (x + j < n0) s += double(lane(v, j));
  return s;
}

// ---------------------------------------------------------------------------
// 3D: z-marching fused step
//
// The march is a pipeline over z: iteration zi computes the staged operands
// of plane zi + RS (if the model stages any) and, once zi >= zb, the output
// of plane zi.  The field planes it needs lie in the window [zi + L, zi + U],
// so the shared-memory ring holds U - L + 1 planes plus PD in flight.
// ---------------------------------------------------------------------------
template <class M, class T, int LP, int GP, int BP, class TC, bool EXACT>
struct Fd3 {
  static constexpr int TX = TC::TX, TY = TC::TY, SPT = TC::SPT, PD = TC::PD, W = TC::W,
                       TXT = TC::TXT, NT = TC::NT;
  static constexpr int NF = M::nf, NS = M::ns, R = M::R, RS = NS > 0 ? M::RS : 0;
  static constexpr int RD = imax(M::r_direct, 0);  // reach of the rhs into fields
  static constexpr int RI = imax(M::r_stage, 0);   // reach of a stage into fields
  static constexpr int U = imax(RD, NS > 0 ? RS + RI : 0);        // newest plane needed
  static constexpr int L = NS > 0 ? (RS - RI < -RD ? RS - RI : -RD) : -RD;  // oldest
  static constexpr int WARM = 2 * RS;  // iterations that only compute stages
  using G = HaloGeom<T, W, R, NS, RS, RI>;
  static constexpr int RSA = G::RSA, HXA = G::HXA;
  static constexpr int PW = TX + 2 * HXA, PH = TY + 2 * R;
  static constexpr int PLANE = ceil_to(PW * PH, 128 / (int)sizeof(T));
  // One barrier per plane, at the end of the iteration.  The output of plane
  // zi reads staged planes zi - RS .. zi + RS: the in-plane neighbours only at
  // zi (staged by the previous iteration, behind its barrier), and the other
  // planes only at the thread's own sites, which the thread itself staged.  So
  // the stage of plane zi + RS and the output of plane zi need no barrier
  // between them, and the stage ring holds just the 2 RS + 1 planes read.
  // Field ring: the U - L planes the next iteration still reads and PD in
  // flight; the plane issued after the barrier reuses the slot of plane zi + L,
  // which no later iteration reads.
  static constexpr int NSLOT = (U - L) + PD;
  static constexpr int SW = TX + 2 * RSA, SH = TY + 2 * RS, SPL = ceil_to(SW * SH, 32);
  static constexpr int NSR = NS > 0 ? 2 * RS + 1 : 0;
  static constexpr int SWC = SW / W;        // column groups of a stage row
  static constexpr int XC = 2 * RSA / W;    // extra column groups left and right
  static constexpr int NE = 2 * RS * SWC + TY * XC;  // stage cells beyond one per row group
  static constexpr int NX = (NE + NT - 1) / NT;       // of them, per thread at most
  static constexpr size_t SMEM =
      256 + sizeof(T) * (size_t(NF) * NSLOT * PLANE + size_t(NS) * NSR * SPL);
  static_assert(U == R, "the newest plane needed is R ahead");
  static_assert(R - WARM + L <= 0, "prologue planes fit in the ring");
  static_assert(PD >= 1, "at least one plane in flight");
  // staged planes are read off the own site only at z offsets other than 0
  // (the 7-point Laplacian of the fused form)
  static_assert(NS == 0 || LP == 7, "staged operands under the 7-point Laplacian only");
  static_assert(NSLOT <= 32, "barrier header holds 32 slots");
  static_assert(PW <= 256 && PH <= 256, "TMA box limit");
  static_assert((PW * sizeof(T)) % 16 == 0, "TMA box rows must be whole 16-byte units");
  static_assert(NX <= 4, "extra stage cells per thread");
};

// Stage cells of a tile.  Each thread stages the cells of its own output
// sites (stage row row0 + k + RS, column group txt + RSA / W), so a staged
// value at the thread's own site is one the thread wrote itself.  The ring
// around them -- the RS rows above and below (every column group) and the
// XC / 2 column groups left and right of each inner row -- is shared out:
// thread tid takes ring cells tid, tid + NT, ... (row -1 marks none).
template <int NE, int NT, int NX, int TY, int RS, int SWC, int XC, int TXT>
__device__ __forceinline__ void extra_cells(int tid, int (&xsr)[NX > 0 ? NX : 1],
                                            int (&xsc)[NX > 0 ? NX : 1]) {
#pragma unroll
  for (int j = 0; j < (NX > 0 ? NX : 1); ++j) {
    const int e = tid + j * NT;
    xsr[j] = -1;
    xsc[j] = 0;
    if constexpr (NE > 0) {
      if (e >= NE) continue;
      if (e < 2 * RS * SWC) {
        const int r = e / SWC;
        xsr[j] = r < RS ? r : TY + r;
        xsc[j] = e % SWC;
      } else {
        const int e2 = e - 2 * RS * SWC, cc = e2 % XC;
        xsr[j] = RS + e2 / XC;
        xsc[j] = cc < XC / 2 ? cc : TXT + cc;
      }
    }
  }
}

template <class M, class T, int LP, int GP, int BP, class TC, bool EXACT>
__global__ void __launch_bounds__(TC::NT)
    k_fd3d(const __grid_constant__ StepParams<T> p, const __grid_constant__ M m) {
  pdl_enter();
  using K = Fd3<M, T, LP, GP, BP, TC, EXACT>;
  constexpr int TX = K::TX, TY = K::TY, SPT = K::SPT, PD = K::PD, W = K::W, TXT = K::TXT,
                NF = K::NF, NS = K::NS, R = K::R, RS = K::RS, RSA = K::RSA, HXA = K::HXA,
                PW = K::PW, PH = K::PH, PLANE = K::PLANE, NSLOT = K::NSLOT, SW = K::SW,
                SPL = K::SPL, NSR = K::NSR, NT = K::NT, RD = K::RD, RI = K::RI, U = K::U,
                WARM = K::WARM, SWC = K::SWC, XC = K::XC, NE = K::NE, NX = K::NX, L = K::L;
  constexpr int NX1 = NX > 0 ? NX : 1;
  constexpr uint32_t TXB = uint32_t(NF * PW * PH * sizeof(T));
  using V = vec_t<T, W>;
  constexpr int SO = NS > 1 ? 2 : 1;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  T* fbuf = reinterpret_cast<T*>(smem_raw + 256);
  T* sbuf = fbuf + NF * NSLOT * PLANE;
  __shared__ double red[32];

  const int tid = threadIdx.x, txt = tid % TXT, tg = tid / TXT, row0 = tg * SPT;
  const int tile = blockIdx.x;
  const int x0 = (tile % p.ntx) * TX, y0 = (tile / p.ntx) * TY;
  const int zb = blockIdx.y * p.zchunk;
  const int ze = min(zb + p.zchunk, p.n[2]);
  const int inst = blockIdx.z;
  const CUtensorMap* maps = p.maps + inst * NF;
  // field planes of this CTA: z = zb - R + q for q in [0, nplanes)
  const int nplanes = (ze - 1 + U) - (zb - R) + 1;
  const V vdivh2(p.divh2), vdivh3(p.divh3), vdivh4(p.divh4), vdt(p.dt);
  T coef[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) coef[i] = p.coef[i];

  // output rows of this thread: pointers at plane 0 and which need halo images
  const int x = x0 + txt * W;
  const bool xin = x < p.n[0];
  // whole W-groups (every group but a ragged row end) store as vectors, their
  // periodic images too
  const bool vec_ok = (p.n[0] % W == 0) && (x + W <= p.n[0]);
  const long long xo = image_offset(p.per[0], x, W, p.n[0], R, 1);
  T* orow[SPT][NF];
  bool rowin[SPT];
  long long yo[SPT];
#pragma unroll
  for (int k = 0; k < SPT; ++k) {
    const int y = y0 + row0 + k;
    rowin[k] = xin && y < p.n[1];
    yo[k] = image_offset(p.per[1], y, 1, p.n[1], R, p.pitch);
#pragma unroll
    for (int f = 0; f < NF; ++f)
      orow[k][f] = p.out[inst * NF + f] + (long long)(y + p.h[1]) * p.pitch + (x + p.h[0]);
  }
  // `plain`: the whole tile lies inside the domain, away from every periodic
  // face, in whole vectors: its stores are straight-line code.  The same for
  // every thread of the block.
  const bool plain = (p.n[0] % W == 0) && x0 + TX <= p.n[0] && y0 + TY <= p.n[1] &&
                     (!p.per[0] || (x0 >= R && x0 + TX <= p.n[0] - R)) &&
                     (!p.per[1] || (y0 >= R && y0 + TY <= p.n[1] - R));
  const bool ragged = xin && !vec_ok;  // a group cut by the end of the row
  // some thread of the block has an x image (the same for every thread)
  const bool xany = p.per[0] && (x0 < R || x0 + TX + W > p.n[0] - R);
  const bool do_mass = p.partial != nullptr;
  // the stage cells beyond this thread's row groups, if any
  int xsr[NX1], xsc[NX1];
  extra_cells<NE, NT, NX, TY, RS, SWC, XC, TXT>(tid, xsr, xsc);

  if (tid == 0) {
    for (int s = 0; s < NSLOT; ++s) tma::mbar_init(&bars[s], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();

  auto issue = [&](int q) {
    const int s = q % NSLOT;
    tma::mbar_arrive_expect_tx(&bars[s], TXB);
    const int zz = zb - R + q + p.h[2];
#pragma unroll
    for (int f = 0; f < NF; ++f)
      tma::load_3d(fbuf + (f * NSLOT + s) * PLANE, maps + f, &bars[s], x0 + p.h[0] - HXA,
                   y0 + p.h[1] - R, zz);
  };
  const int zi0 = zb - WARM;
  // Plane sequence number q(z) = z - (zb - R), ring slot q % NSLOT, barrier
  // phase (q / NSLOT) & 1.  Iteration zi waits for q(zi + U), issues plane
  // q(zi + U + PD) after its barrier, reads the field planes zi + L .. zi + U and the staged
  // planes zi - RS .. zi + RS, and writes staged plane zi + RS.  The slots and
  // phases are advanced by one per iteration (no divisions), and the planes
  // read are kept as windows of pointers shifted by one plane per iteration.
  constexpr int NPW = U - L + 1;                // field planes read per iteration
  constexpr int NSW = NS > 0 ? 2 * RS + 1 : 1;  // staged planes read per iteration
  const int q0 = zi0 - (zb - R);                // q of plane zi0 (>= 0)
  if (tid == 0) {
    const int pro = min(q0 + U + PD, nplanes);
    for (int q = 0; q < pro; ++q) issue(q);
  }
  // every plane the first iteration reads except the newest, which the first
  // iteration waits for like any other
  bool bad0 = false;
  for (int q = 0; q < q0 + U; ++q) bad0 |= !tma::mbar_wait(&bars[q % NSLOT], (q / NSLOT) & 1);

  const T* const fend = fbuf + NSLOT * PLANE;
  const T* pw[NPW];  // field plane zi + L + j, field 0
  pw[0] = fbuf + (((q0 + L) % NSLOT + NSLOT) % NSLOT) * PLANE;
#pragma unroll
  for (int j = 1; j < NPW; ++j) pw[j] = pw[j - 1] + PLANE == fend ? fbuf : pw[j - 1] + PLANE;
  const T* ps[NSW];  // staged plane zi - RS + j, operand 0
  if constexpr (NS > 0) {
    // staged planes count from zb - RS: plane zi0 - RS + j is number j - 2 RS
    const T* const send = sbuf + NSR * SPL;
    ps[0] = sbuf + (((-2 * RS) % NSR + NSR) % NSR) * SPL;
#pragma unroll
    for (int j = 1; j < NSW; ++j) ps[j] = ps[j - 1] + SPL == send ? sbuf : ps[j - 1] + SPL;
  }
  int qw = q0 + U, wslot = qw % NSLOT, wph = (qw / NSLOT) & 1;  // plane waited for
  int qn = q0 + U + PD, nslot = qn % NSLOT;                      // plane issued

  double msum = 0.0;
  for (int zi = zi0; zi < ze; ++zi) {
    bool bad = !tma::mbar_wait(&bars[wslot], wph);
    if (zi == zi0) bad |= bad0;

    if constexpr (NS > 0) {
      using CS = Ctx<T, W, !EXACT, 3, LP, GP, BP, NF, 2 * RI + 1, RI, PW, 1, 1, 0, SW>;
      T* sdst = const_cast<T*>(ps[NSW - 1]);
      CS c0;
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int dz = -RI; dz <= RI; ++dz) c0.fo[f][dz + RI] = pw[RS + dz - L] + f * NSLOT * PLANE;
      c0.divh2 = vdivh2;
      c0.divh3 = vdivh3;
      c0.divh4 = vdivh4;
      c0.cf = coef;
      // stage cell (sr, column group c): field row sr - RS + R, x = c*W - RSA + HXA.
      // All of this thread's cells are evaluated before any is stored, so the
      // loads are not ordered behind stores the compiler cannot disambiguate.
      auto cell = [&](int sr, int c, V (&o)[SO]) {
        CS ctx = c0;
        const int off = (sr - RS + R) * PW + c * W - RSA + HXA;
#pragma unroll
        for (int f = 0; f < NF; ++f)
#pragma unroll
          for (int dz = 0; dz < 2 * RI + 1; ++dz) ctx.fo[f][dz] += off;
        o[0] = eval(m.s0, ctx);
        if constexpr (NS > 1) o[1] = eval(m.s1, ctx);
      };
      V sv[SPT + NX1][SO];
#pragma unroll
      for (int k = 0; k < SPT; ++k) cell(row0 + k + RS, txt + RSA / W, sv[k]);
#pragma unroll
      for (int j = 0; j < NX; ++j)
        if (xsr[j] >= 0) cell(xsr[j], xsc[j], sv[SPT + j]);
      auto put = [&](int sr, int c, const V (&o)[SO]) {
        *reinterpret_cast<V*>(sdst + sr * SW + c * W) = o[0];
        if constexpr (NS > 1) *reinterpret_cast<V*>(sdst + NSR * SPL + sr * SW + c * W) = o[1];
      };
#pragma unroll
      for (int k = 0; k < SPT; ++k) put(row0 + k + RS, txt + RSA / W, sv[k]);
#pragma unroll
      for (int j = 0; j < NX; ++j)
        if (xsr[j] >= 0) put(xsr[j], xsc[j], sv[SPT + j]);
    }

    if (zi >= zb) {
      const int z = zi;
      using CO = Ctx<T, W, !EXACT, 3, LP, GP, BP, NF, 2 * RD + 1, RD, PW, NS,
                     (NS > 0 ? 2 * RS + 1 : 1), (NS > 0 ? RS : 0), SW>;
      CO c0;
      const int cell = (row0 + R) * PW + txt * W + HXA;
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int dz = -RD; dz <= RD; ++dz) c0.fo[f][dz + RD] = pw[dz - L] + f * NSLOT * PLANE + cell;
      if constexpr (NS > 0) {
        const int scell = (row0 + RS) * SW + txt * W + RSA;
#pragma unroll
        for (int k = 0; k < NS; ++k)
#pragma unroll
          for (int dz = -RS; dz <= RS; ++dz) c0.so[k][dz + RS] = ps[dz + RS] + k * NSR * SPL + scell;
      }
      c0.divh2 = vdivh2;
      c0.divh3 = vdivh3;
      c0.divh4 = vdivh4;
      c0.cf = coef;
      V nv[SPT][NF];
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
        const V r0 = eval(m.r0, ctx);
        nv[k][0] = p.rhs_only ? r0 : fmadd<!EXACT>(vdt, r0, ctx.template var<1, 0, 0, 0>());
        if constexpr (NF > 1) {
          const V r1 = eval(m.r1, ctx);
          nv[k][1] = p.rhs_only ? r1 : fmadd<!EXACT>(vdt, r1, ctx.template var<2, 0, 0, 0>());
        }
      }
      const long long zoff = (long long)(z + p.h[2]) * p.plane;
      const long long zo = image_offset(p.per[2], z, 1, p.n[2], R, p.plane);
      if (plain && zo == 0) {
#pragma unroll
        for (int k = 0; k < SPT; ++k)
#pragma unroll
          for (int f = 0; f < NF; ++f) *reinterpret_cast<V*>(orow[k][f] + zoff) = nv[k][f];
      } else {
        // a tile at a face or the end of the domain: every group and its
        // images as predicated stores (no divergence); a group cut by the end
        // of a row element by element
#pragma unroll
        for (int k = 0; k < SPT; ++k) {
#pragma unroll
          for (int f = 0; f < NF; ++f)
            put_images_pred(orow[k][f] + zoff, nv[k][f], rowin[k] && vec_ok, xany, xo, yo[k], zo);
          if (ragged && rowin[k]) {
#pragma unroll
            for (int f = 0; f < NF; ++f)
              store_group<T, W, 3, R>(p.out[inst * NF + f], x, y0 + row0 + k, z, nv[k][f], p.n,
                                      p.h, p.per, p.pitch, p.plane);
          }
        }
      }
      if (do_mass) {
#pragma unroll
        for (int k = 0; k < SPT; ++k)
          if (rowin[k]) msum += vsum<T, W>(nv[k][0], x, p.n[0]);
      }
    }

    // the one barrier of the iteration: staged plane zi + RS written, every
    // read of this iteration done
    if (__syncthreads_or(bad)) {
      if (tid == 0) {
        atomicExch(p.err, KERR_TMA_TIMEOUT);
        tma::drain(bars, NSLOT, zi == zi0 ? 0 : qw, min(qn - 1, nplanes - 1));
      }
      return;
    }
    if (tid == 0 && qn < nplanes) {
      tma::mbar_arrive_expect_tx(&bars[nslot], TXB);
#pragma unroll
      for (int f = 0; f < NF; ++f)
        tma::load_3d(fbuf + (f * NSLOT + nslot) * PLANE, maps + f, &bars[nslot],
                     x0 + p.h[0] - HXA, y0 + p.h[1] - R, zb - R + qn + p.h[2]);
    }

    // advance the windows, the waited-for and the issued plane by one
    {
      const T* nw = pw[NPW - 1] + PLANE == fend ? fbuf : pw[NPW - 1] + PLANE;
#pragma unroll
      for (int j = 0; j < NPW - 1; ++j) pw[j] = pw[j + 1];
      pw[NPW - 1] = nw;
    }
    if constexpr (NS > 0) {
      const T* const send = sbuf + NSR * SPL;
      const T* nw = ps[NSW - 1] + SPL == send ? sbuf : ps[NSW - 1] + SPL;
#pragma unroll
      for (int j = 0; j < NSW - 1; ++j) ps[j] = ps[j + 1];
      ps[NSW - 1] = nw;
    }
    ++qw;
    if (++wslot == NSLOT) {
      wslot = 0;
      wph ^= 1;
    }
    ++qn;
    if (++nslot == NSLOT) nslot = 0;
  }
  __syncthreads();

  if (p.partial) {
    const double s = block_sum<NT>(msum, red);
    if (tid == 0)
      p.partial[(size_t(blockIdx.z) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
  }
}

// ---------------------------------------------------------------------------
// 2D: persistent tile-queue fused step over one or many instances.
// One barrier per tile: the tile ring keeps PD tiles in flight plus two being
// read, and the stage buffer alternates between two copies.
// ---------------------------------------------------------------------------
template <class M0, class M1, class T, int LP, int GP, int BP, class TC, bool EXACT>
struct Fd2 {
  static constexpr bool exact = EXACT;
  static_assert(M0::nf == M1::nf, "models of one launch share the field count");
  static constexpr int TX = TC::TX, TY = TC::TY, SPT = TC::SPT, PD = TC::PD, W = TC::W,
                       TXT = TC::TXT, NT = TC::NT;
  static constexpr int NF = M0::nf;
  static constexpr int NS = imax(M0::ns, M1::ns);
  static constexpr int R = imax(M0::R, M1::R);
  static constexpr int RS = NS > 0 ? imax(M0::ns ? M0::RS : 0, M1::ns ? M1::RS : 0) : 0;
  static constexpr int RI = imax(imax(M0::r_stage, M1::r_stage), 0);
  static_assert(M0::ns == 0 || M0::RS == RS, "staged models of one launch share the reach");
  static_assert(M1::ns == 0 || M1::RS == RS, "staged models of one launch share the reach");
  using G = HaloGeom<T, W, R, NS, RS, RI>;
  static constexpr int RSA = G::RSA, HXA = G::HXA;
  static constexpr int PW = TX + 2 * HXA, PH = TY + 2 * R;
  static constexpr int PLANE = ceil_to(PW * PH, 128 / (int)sizeof(T));
  static constexpr int NQ = PD + 2;  // tile slots: PD in flight, the one staged, the one output
  static constexpr int SW = TX + 2 * RSA, SH = TY + 2 * RS, SPL = ceil_to(SW * SH, 32);
  static constexpr int SWC = SW / W, XC = 2 * RSA / W;
  static constexpr int NE = 2 * RS * SWC + TY * XC;
  static constexpr int NX = (NE + NT - 1) / NT, NX1 = NX > 0 ? NX : 1;
  static constexpr size_t SMEM =
      256 + sizeof(T) * (size_t(NQ) * NF * PLANE + size_t(2) * NS * SPL);
  static_assert(NQ <= 16, "barrier header holds 16 slots");
  static_assert(PW <= 256 && PH <= 256, "TMA box limit");
  static_assert((PW * sizeof(T)) % 16 == 0, "TMA box rows must be whole 16-byte units");
  static_assert(NX <= 4, "extra stage cells per thread");
};

// staged operands of model M for one tile
template <class K, class M, class T, int LP, int GP, int BP>
__device__ __forceinline__ void fd2_stage(const M& m, const Inst2<T>& ip, const T* fbuf, T* sbuf,
                                          int slot, const int (&xsr)[K::NX1],
                                          const int (&xsc)[K::NX1]) {
  constexpr int SPT = K::SPT, W = K::W, TXT = K::TXT, NF = K::NF, R = K::R, RS = K::RS,
                RSA = K::RSA, HXA = K::HXA, PW = K::PW, PLANE = K::PLANE, SW = K::SW;
  constexpr int NS = M::ns;
  constexpr int SO = NS > 1 ? 2 : 1;
  using V = vec_t<T, W>;
  using CS = Ctx<T, W, !K::exact, 2, LP, GP, BP, NF, 1, 0, PW, 1, 1, 0, SW>;
  const int tid = threadIdx.x, txt = tid % TXT, row0 = (tid / TXT) * SPT;
  T coef[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) coef[i] = ip.coef[i];
  CS c0;
#pragma unroll
  for (int f = 0; f < NF; ++f) c0.fo[f][0] = fbuf + (slot * NF + f) * PLANE;
  c0.divh2 = V(ip.divh2);
  c0.divh3 = V(ip.divh3);
  c0.divh4 = V(ip.divh4);
  c0.cf = coef;
  auto cell = [&](int sr, int c, V (&o)[SO]) {
    CS ctx = c0;
    const int off = (sr - RS + R) * PW + c * W - RSA + HXA;
#pragma unroll
    for (int f = 0; f < NF; ++f) ctx.fo[f][0] += off;
    o[0] = eval(m.s0, ctx);
    if constexpr (NS > 1) o[1] = eval(m.s1, ctx);
  };
  V sv[SPT + K::NX1][SO];
#pragma unroll
  for (int k = 0; k < SPT; ++k) cell(row0 + k + RS, txt + RSA / W, sv[k]);
#pragma unroll
  for (int j = 0; j < K::NX; ++j)
    if (xsr[j] >= 0) cell(xsr[j], xsc[j], sv[SPT + j]);
  auto put = [&](int sr, int c, const V (&o)[SO]) {
    *reinterpret_cast<V*>(sbuf + sr * SW + c * W) = o[0];
    if constexpr (NS > 1) *reinterpret_cast<V*>(sbuf + K::SPL + sr * SW + c * W) = o[1];
  };
#pragma unroll
  for (int k = 0; k < SPT; ++k) put(row0 + k + RS, txt + RSA / W, sv[k]);
#pragma unroll
  for (int j = 0; j < K::NX; ++j)
    if (xsr[j] >= 0) put(xsr[j], xsc[j], sv[SPT + j]);
}

// right-hand sides, Euler update and stores of model M for one tile
template <class K, class M, class T, int LP, int GP, int BP>
__device__ __forceinline__ void fd2_out(const Step2Params<T>& p, const M& m, const Inst2<T>& ip,
                                        int ii, const T* fbuf, const T* sbuf, int slot, int x0,
                                        int y0, double& msum) {
  constexpr int TX = K::TX, TY = K::TY, SPT = K::SPT, W = K::W, TXT = K::TXT, NF = K::NF, R = K::R, RS = K::RS,
                RSA = K::RSA, HXA = K::HXA, PW = K::PW, PLANE = K::PLANE, SW = K::SW;
  constexpr int NS = M::ns;
  using V = vec_t<T, W>;
  const int tid = threadIdx.x, txt = tid % TXT, row0 = (tid / TXT) * SPT;
  T coef[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) coef[i] = ip.coef[i];
  const int n0 = ip.n[0], n1 = ip.n[1];
  const long long pitch = ip.pitch;
  using CO = Ctx<T, W, !K::exact, 2, LP, GP, BP, NF, 1, 0, PW, NS, 1, 0, SW>;
  CO c0;
  const int cell = (row0 + R) * PW + txt * W + HXA;
#pragma unroll
  for (int f = 0; f < NF; ++f) c0.fo[f][0] = fbuf + (slot * NF + f) * PLANE + cell;
  if constexpr (NS > 0) {
    const int scell = int(sbuf - fbuf) + (row0 + RS) * SW + txt * W + RSA;
#pragma unroll
    for (int k = 0; k < NS; ++k) c0.so[k][0] = fbuf + k * K::SPL + scell;
  }
  const V vdt(ip.dt);
  c0.divh2 = V(ip.divh2);
  c0.divh3 = V(ip.divh3);
  c0.divh4 = V(ip.divh4);
  c0.cf = coef;
  const int x = x0 + txt * W;
  V nv[SPT][NF];
#pragma unroll
  for (int k = 0; k < SPT; ++k) {
    CO ctx = c0;
#pragma unroll
    for (int f = 0; f < NF; ++f) ctx.fo[f][0] += k * PW;
    if constexpr (NS > 0) {
#pragma unroll
      for (int kk = 0; kk < NS; ++kk) ctx.so[kk][0] += k * SW;
    }
    const V r0 = eval(m.r0, ctx);
    nv[k][0] = p.rhs_only ? r0 : fmadd<!K::exact>(vdt, r0, ctx.template var<1, 0, 0, 0>());
    if constexpr (NF > 1) {
      const V r1 = eval(m.r1, ctx);
      nv[k][1] = p.rhs_only ? r1 : fmadd<!K::exact>(vdt, r1, ctx.template var<2, 0, 0, 0>());
    }
  }
  const bool vec_ok = (n0 % W == 0) && (x + W <= n0);
  const long long xo = image_offset(ip.per[0], x, W, n0, R, 1);
  const int h[3] = {p.hx, p.hy, 0};
  const int n3[3] = {n0, n1, 1};
  const int per3[3] = {ip.per[0], ip.per[1], 0};
  T* out[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) out[f] = p.out[ii * NF + f];
  const int yr0 = y0 + row0;
  // the whole tile inside the domain, away from every periodic face, in whole
  // vectors: straight-line stores (the same for every thread of the block)
  const bool plain = (n0 % W == 0) && x0 + TX <= n0 && y0 + TY <= n1 &&
                     (!ip.per[0] || (x0 >= R && x0 + TX <= n0 - R)) &&
                     (!ip.per[1] || (y0 >= R && y0 + TY <= n1 - R));
  if (plain) {
    T* b0 = nullptr;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      b0 = out[f] + (long long)(yr0 + p.hy) * pitch + x + p.hx;
#pragma unroll
      for (int k = 0; k < SPT; ++k) *reinterpret_cast<V*>(b0 + k * pitch) = nv[k][f];
    }
  } else {
    // a tile at a face or the end of the domain: whole groups and their
    // images as predicated stores (no divergence); a group cut by the end of
    // a row element by element
    const bool ragged = x < n0 && !vec_ok;
    const bool xany = ip.per[0] && (x0 < R || x0 + TX + W > n0 - R);
#pragma unroll
    for (int k = 0; k < SPT; ++k) {
      const int y = y0 + row0 + k;
      const bool in = x < n0 && y < n1;
      const long long yo = image_offset(ip.per[1], y, 1, n1, R, pitch);
#pragma unroll
      for (int f = 0; f < NF; ++f)
        put_images_pred(out[f] + (long long)(y + p.hy) * pitch + x + p.hx, nv[k][f],
                        in && vec_ok, xany, xo, yo, 0LL);
      if (ragged && in) {
#pragma unroll
        for (int f = 0; f < NF; ++f)
          store_group<T, W, 2, R>(out[f], x, y, 0, nv[k][f], n3, h, per3, pitch, 0);
      }
    }
  }
  if (p.partial) {
#pragma unroll
    for (int k = 0; k < SPT; ++k)
      if (x < n0 && y0 + row0 + k < n1) msum += vsum<T, W>(nv[k][0], x, n0);
  }
}

template <class M0, class M1, class T, int LP, int GP, int BP, class TC, bool EXACT>
__global__ void __launch_bounds__(TC::NT)
    k_fd2d(const __grid_constant__ Step2Params<T> p, const __grid_constant__ M0 m0,
           const __grid_constant__ M1 m1) {
  using K = Fd2<M0, M1, T, LP, GP, BP, TC, EXACT>;
  constexpr int TX = K::TX, TY = K::TY, PD = K::PD, NQ = K::NQ, NF = K::NF, R = K::R,
                HXA = K::HXA, PW = K::PW, PH = K::PH, PLANE = K::PLANE, NT = K::NT,
                NS = K::NS, RS = K::RS, SWC = K::SWC, XC = K::XC, NE = K::NE, TXT = K::TXT;
  constexpr uint32_t TXB = uint32_t(NF * PW * PH * sizeof(T));

  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);  // [16]
  int2* items = reinterpret_cast<int2*>(smem_raw + 128);    // [16]
  T* fbuf = reinterpret_cast<T*>(smem_raw + 256);
  T* sbuf = fbuf + NQ * NF * PLANE;
  __shared__ double red[32];
  const int tid = threadIdx.x;

  int xsr[K::NX1], xsc[K::NX1];
  extra_cells<NE, NT, K::NX, TY, RS, SWC, XC, TXT>(tid, xsr, xsc);

  // before any global access: the work-queue counter the previous grid
  // re-arms, the fields it wrote and the buffer it was still reading
  pdl_enter();

  // When every CTA has many items (ensembles), they are taken from the queue
  // in batches of 4, one batch requested ahead (thread 0 only): the atomic's
  // result is needed a batch later, so its round trip to L2 stays off the path
  // of the tile loop, and the one counter sees a quarter of the atomics.
  // Batches never overlap, so a CTA that finds an item past the end holds no
  // valid item in its next batch.  With few items per CTA, batches and items
  // held ahead would unbalance the tail: those launches take one item at a
  // time, when they need it -- except a single instance (no item list), whose
  // tiles all cost the same: its CTAs take a fixed round-robin share, so no
  // queue round trip to L2 lies on the path of a launch of a few tiles per CTA.
  const bool many = p.nitems >= 64 * int(gridDim.x);
  const bool fixed_share = !many && !p.items;
  constexpr int QB = 4;
  int qcur = 0, qend = 0, qnext = 0, qown = int(blockIdx.x);
  if (tid == 0 && many) qnext = atomicAdd(&p.ctr[0], QB);
  auto fetch = [&]() -> int2 {
    if (fixed_share) {
      const int t = qown;
      qown += int(gridDim.x);
      return t < p.nitems ? make_int2(0, t) : make_int2(-1, 0);
    }
    if (qcur == qend) {
      if (many) {
        qcur = qnext;
        qend = qnext + QB;
        qnext = atomicAdd(&p.ctr[0], QB);
      } else {
        qcur = atomicAdd(&p.ctr[0], 1);
        qend = qcur + 1;
      }
    }
    const int t = qcur++;
    if (t >= p.nitems) return make_int2(-1, 0);
    return p.items ? p.items[t] : make_int2(0, t);
  };
  // tile coordinates of an item: packed by the host in an item list (no
  // division per tile), a linear index otherwise
  auto tile_xy = [&](int t, int ntx) -> int2 {
    if (p.items) return make_int2(t & 0xffff, t >> 16);
    return make_int2(t % ntx, t / ntx);
  };
  auto issue = [&](int2 it, int slot) {
    const Inst2<T>& ip = p.inst[it.x];
    const int2 tc = tile_xy(it.y, ip.ntx);
    const int x0 = tc.x * TX, y0 = tc.y * TY;
    tma::mbar_arrive_expect_tx(&bars[slot], TXB);
#pragma unroll
    for (int f = 0; f < NF; ++f)
      tma::load_2d(fbuf + (slot * NF + f) * PLANE, p.maps + it.x * NF + f, &bars[slot],
                   x0 + p.hx - HXA, y0 + p.hy - R);
  };

  // Tile j of this CTA's sequence lives in ring slot j % NQ (barrier phase
  // (j / NQ) & 1) and stages into copy j & 1 of the stage buffer.  Iteration
  // it stages tile it + 1 and writes the output of tile it, staged by the
  // previous iteration: the two are independent, so one barrier per tile, at
  // the end of the iteration, orders everything.  The ring holds tiles it and
  // it + 1 and PD in flight; iteration it issues tile it + 1 + PD into the slot
  // of tile it - 1, which every thread finished with before the last barrier.
  auto item_at = [&](int j) -> int2 {
    const volatile int* v = reinterpret_cast<volatile int*>(&items[j % NQ]);
    return make_int2(v[0], v[1]);
  };
  auto stage = [&](int2 t, int j) {
    if constexpr (NS > 0) {
      const Inst2<T>& ip = p.inst[t.x];
      T* sb = sbuf + (j & 1) * NS * K::SPL;
      if (ip.kind == 0) {
        if constexpr (M0::ns > 0)
          fd2_stage<K, M0, T, LP, GP, BP>(m0, ip, fbuf, sb, j % NQ, xsr, xsc);
      } else {
        if constexpr (M1::ns > 0)
          fd2_stage<K, M1, T, LP, GP, BP>(m1, ip, fbuf, sb, j % NQ, xsr, xsc);
      }
    }
  };
  // error path: record, wait (bounded) for tiles first .. first + PD still in
  // flight, leave
  auto give_up = [&](int first) {
    if (tid == 0) {
      atomicExch(p.err, KERR_TMA_TIMEOUT);
      for (int j = first; j <= first + PD; ++j)
        if (item_at(j).x >= 0) tma::mbar_wait(&bars[j % NQ], (j / NQ) & 1);
    }
  };

  if (tid == 0) {
    for (int s = 0; s < NQ; ++s) tma::mbar_init(&bars[s], 1);
    tma::fence_barrier_init();
    for (int s = 0; s <= PD; ++s) {
      const int2 t = fetch();
      items[s] = t;
      if (t.x >= 0) issue(t, s);
    }
  }
  __syncthreads();
  {
    const int2 t0 = item_at(0);
    bool bad = false;
    if (t0.x >= 0) {
      bad = !tma::mbar_wait(&bars[0], 0);
      if (!bad) stage(t0, 0);
    }
    if (__syncthreads_or(bad)) {
      give_up(0);
      return;
    }
  }

  double msum = 0.0;
  for (int it = 0;; ++it) {
    const int2 cur = item_at(it);
    if (cur.x < 0) break;
    const int2 nxt = item_at(it + 1);
    if (tid == 0) {
      const int2 t = fetch();
      const int ns = (it + 1 + PD) % NQ;
      items[ns] = t;
      if (t.x >= 0) issue(t, ns);
    }
    bool bad = false;
    if (nxt.x >= 0) {
      bad = !tma::mbar_wait(&bars[(it + 1) % NQ], ((it + 1) / NQ) & 1);
      if (!bad) stage(nxt, it + 1);
    }
    {
      const Inst2<T>& ip = p.inst[cur.x];
      const T* sb = sbuf + (it & 1) * (NS > 0 ? NS : 1) * K::SPL;
      const int2 tc = tile_xy(cur.y, ip.ntx);
      const int x0 = tc.x * TX, y0 = tc.y * TY;
      if (ip.kind == 0)
        fd2_out<K, M0, T, LP, GP, BP>(p, m0, ip, cur.x, fbuf, sb, it % NQ, x0, y0, msum);
      else
        fd2_out<K, M1, T, LP, GP, BP>(p, m1, ip, cur.x, fbuf, sb, it % NQ, x0, y0, msum);
    }
    if (__syncthreads_or(bad)) {
      give_up(it + 1);
      return;
    }
  }
  __syncthreads();
  if (tid == 0 && !fixed_share) {
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

}  // namespace sp
