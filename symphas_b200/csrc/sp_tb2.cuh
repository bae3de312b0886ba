/*
 * sp_tb2.cuh -- temporally blocked 2D fused step: up to KT Euler steps of
 * SolverFT::step (examples/solvers/solverft.h:46-103) per launch, for grids
 * periodic on both axes.
 *
 * A CTA takes a TX x TY tile of an instance from the same work queue as the
 * one-step kernel (k_fd2d) and loads the tile with a margin of KT * R rows and
 * columns around it (R: the model's reach per step), wrapped around the
 * periodic faces, so that the stored halo is not needed.  It then runs the
 * steps in shared memory, each step on a region R smaller than the last on
 * every side: the staged operands (mu of a conserved model) on the region the
 * step's right-hand side reads, then psi + dt * rhs into a second buffer.
 * The last step writes the tile (and its periodic images, as every step
 * kernel does) to the output buffer.  Every site of every step is evaluated
 * by the same expression code as the one-step kernels, in the same order, so
 * s steps of this kernel give the bits of s launches of k_fd2d.
 *
 * Per step, the tile's fields cross HBM once per KT steps instead of once per
 * step; the price is the margin: the regions of the early steps are larger
 * than the tile.  Which depth pays is measured (sp_autotune), per model and
 * grid.
 *
 * Loads are 16-byte cp.async copies (no TMA box: the margin wraps around the
 * faces, which a tiled box cannot do), double-buffered so the next tile's
 * copy overlaps this tile's steps.  Columns are handled in groups of 16 bytes,
 * so the x extent of every instance must be a multiple of 16 bytes.
 *
 * A launch runs `p.tsteps` (1..KT) steps: the last tsteps of the KT-step
 * schedule, so its regions are exactly as large as tsteps steps need.
 */
#pragma once

#include "sp_kernels.cuh"

namespace sp {

// TX x TY tile, up to KT steps per launch, NT threads, W sites per thread
// group, SR consecutive rows per work item (their shared neighbour rows are
// loaded once)
template <int TX_, int TY_, int KT_, int NT_, int W_, int SR_ = 4>
struct TbCfg {
  static constexpr int TX = TX_, TY = TY_, KT = KT_, NT = NT_, W = W_, SR = SR_;
};

template <class M0, class M1, class T, int LP, int GP, int BP, class TC, bool EXACT>
struct Fd2T {
  static constexpr bool exact = EXACT;
  static_assert(M0::nf == M1::nf, "models of one launch share the field count");
  static constexpr int TX = TC::TX, TY = TC::TY, KT = TC::KT, NT = TC::NT, W = TC::W,
                       SR = TC::SR;
  static constexpr int NF = M0::nf;
  static constexpr int NS = imax(M0::ns, M1::ns);
  static constexpr int R = imax(M0::R, M1::R);
  static constexpr int RS = NS > 0 ? imax(M0::ns ? M0::RS : 0, M1::ns ? M1::RS : 0) : 0;
  static constexpr int RI = imax(imax(M0::r_stage, M1::r_stage), 0);
  static_assert(M0::ns == 0 || M0::RS == RS, "staged models of one launch share the reach");
  static_assert(M1::ns == 0 || M1::RS == RS, "staged models of one launch share the reach");
  static constexpr int LC = 16 / (int)sizeof(T);  // elements per 16-byte copy
  static constexpr int HT = KT * R;                // margin of valid input around the tile
  // columns held on each side: the margin rounded up to whole copies, and one
  // W-group more, because each step's region is rounded out to whole groups
  // and those extra sites read up to R further
  static constexpr int HX = ceil_to(ceil_to(HT, W) + W, LC);
  static constexpr int HY = HT;
  static constexpr int PW = TX + 2 * HX, PH = TY + 2 * HY;
  // SR - 1 rows below the region: the last work item of a region whose row
  // count is not a multiple of SR reads them (and does not store its rows
  // beyond the region)
  static constexpr int PLANE = ceil_to(PW * (PH + SR - 1), 32);
  static constexpr int GW = PW / LC;  // copies per row
  // planes: input (two tiles, double-buffered) and the step buffer per field,
  // and the staged operands
  static constexpr size_t SMEM = 128 + sizeof(T) * (size_t(3 * NF + NS) * PLANE);
  // the field layout of the one-step kernels of the same key (their x halo)
  static constexpr int HXA = HaloGeom<T, W, R, NS, RS, RI>::HXA;
  static_assert(TX % W == 0 && TX % LC == 0, "whole groups and copies per tile row");
  static_assert(SR >= 1 && TY % SR == 0, "the tile's rows split into work items");
  static_assert(W <= LC && LC % W == 0, "a group lies inside one 16-byte copy");
  static_assert(R <= W, "one extra group covers the reach of the rounded-out sites");
  static_assert(KT >= 1 && KT <= 8, "steps per launch");
  static_assert(NT % 32 == 0 && NT <= 1024, "threads per CTA");
  static_assert(SMEM <= 227 * 1024, "shared memory of one CTA");
};

template <class T>
__device__ __forceinline__ void tb_cp16(T* dst, const T* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void tb_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void tb_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// v mod n for v within a few multiples of n (the margin is small against n)
__device__ __forceinline__ int tb_wrap(int v, int n) {
  while (v < 0) v += n;
  while (v >= n) v -= n;
  return v;
}

// staged operands of model M on the tile grown by HS sites (rows exact,
// columns rounded out to whole groups): src holds NF field planes, sb NS
// stage planes, all of pitch PW with the tile origin at (HY, HX)
template <class K, class M, class T, int LP, int GP, int BP, int HS>
__device__ __forceinline__ void tb_stage(const M& m, const Inst2<T>& ip, const T* src, T* sb) {
  constexpr int W = K::W, PW = K::PW, PLANE = K::PLANE, NF = K::NF, NT = K::NT;
  constexpr int NS = M::ns;
  constexpr int HG = (HS + W - 1) / W, SR = K::SR;
  constexpr int NR = K::TY + 2 * HS, NG = K::TX / W + 2 * HG, NRB = (NR + SR - 1) / SR,
                CNT = NRB * NG;
  using V = vec_t<T, W>;
  using CS = Ctx<T, W, !K::exact, 2, LP, GP, BP, NF, 1, 0, PW, 1, 1, 0, PW>;
  T coef[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) coef[i] = ip.coef[i];
  CS c0;
  c0.divh2 = V(ip.divh2);
  c0.divh3 = V(ip.divh3);
  c0.divh4 = V(ip.divh4);
  c0.cf = coef;
#pragma unroll 1
  for (int i = threadIdx.x; i < CNT; i += NT) {
    const int rb = i / NG, g = i - rb * NG;
    const int off = (rb * SR - HS + K::HY) * PW + (g - HG) * W + K::HX;
    // every row of the item before any store: the rows share loads
    V s0[SR], s1[SR];
#pragma unroll
    for (int k = 0; k < SR; ++k) {
      CS ctx = c0;
#pragma unroll
      for (int f = 0; f < NF; ++f) ctx.fo[f][0] = src + f * PLANE + off + k * PW;
      s0[k] = eval(m.s0, ctx);
      if constexpr (NS > 1) s1[k] = eval(m.s1, ctx);
    }
#pragma unroll
    for (int k = 0; k < SR; ++k) {
      if (NR % SR != 0 && rb * SR + k >= NR) break;
      *reinterpret_cast<V*>(sb + off + k * PW) = s0[k];
      if constexpr (NS > 1) *reinterpret_cast<V*>(sb + PLANE + off + k * PW) = s1[k];
    }
  }
}

// right-hand sides and Euler update of model M on the tile grown by HO sites,
// into the step buffer dst (same geometry as src)
template <class K, class M, class T, int LP, int GP, int BP, int HO>
__device__ __forceinline__ void tb_update(const M& m, const Inst2<T>& ip, const T* src,
                                          const T* sb, T* dst) {
  constexpr int W = K::W, PW = K::PW, PLANE = K::PLANE, NF = K::NF, NT = K::NT, NS = K::NS;
  constexpr int HG = (HO + W - 1) / W, SR = K::SR;
  constexpr int NR = K::TY + 2 * HO, NG = K::TX / W + 2 * HG, NRB = (NR + SR - 1) / SR,
                CNT = NRB * NG;
  using V = vec_t<T, W>;
  using CO = Ctx<T, W, !K::exact, 2, LP, GP, BP, NF, 1, 0, PW, NS, 1, 0, PW>;
  T coef[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) coef[i] = ip.coef[i];
  CO c0;
  c0.divh2 = V(ip.divh2);
  c0.divh3 = V(ip.divh3);
  c0.divh4 = V(ip.divh4);
  c0.cf = coef;
  const V vdt(ip.dt);
#pragma unroll 1
  for (int i = threadIdx.x; i < CNT; i += NT) {
    const int rb = i / NG, g = i - rb * NG;
    const int off = (rb * SR - HO + K::HY) * PW + (g - HG) * W + K::HX;
    V n0[SR], n1[SR];
#pragma unroll
    for (int k = 0; k < SR; ++k) {
      CO ctx = c0;
#pragma unroll
      for (int f = 0; f < NF; ++f) ctx.fo[f][0] = src + f * PLANE + off + k * PW;
      if constexpr (NS > 0) {
#pragma unroll
        for (int q = 0; q < NS; ++q) ctx.so[q][0] = sb + q * PLANE + off + k * PW;
      }
      const V r0 = eval(m.r0, ctx);
      n0[k] = fmadd<!K::exact>(vdt, r0, ctx.template var<1, 0, 0, 0>());
      if constexpr (NF > 1) {
        const V r1 = eval(m.r1, ctx);
        n1[k] = fmadd<!K::exact>(vdt, r1, ctx.template var<2, 0, 0, 0>());
      }
    }
#pragma unroll
    for (int k = 0; k < SR; ++k) {
      if (NR % SR != 0 && rb * SR + k >= NR) break;
      *reinterpret_cast<V*>(dst + off + k * PW) = n0[k];
      if constexpr (NF > 1) *reinterpret_cast<V*>(dst + PLANE + off + k * PW) = n1[k];
    }
  }
}

// the last step: right-hand sides (and the Euler update unless rhs_only) on
// the tile itself, stored with their periodic images to the output fields
template <class K, class M, class T, int LP, int GP, int BP>
__device__ __forceinline__ void tb_final(const Step2Params<T>& p, const M& m, const Inst2<T>& ip,
                                         int ii, const T* src, const T* sb, int x0, int y0,
                                         double& msum) {
  constexpr int W = K::W, PW = K::PW, PLANE = K::PLANE, NF = K::NF, NT = K::NT, NS = K::NS,
                R = K::R, TX = K::TX, TY = K::TY;
  constexpr int SR = K::SR, NG = TX / W, CNT = (TY / SR) * NG;
  using V = vec_t<T, W>;
  using CO = Ctx<T, W, !K::exact, 2, LP, GP, BP, NF, 1, 0, PW, NS, 1, 0, PW>;
  T coef[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) coef[i] = ip.coef[i];
  CO c0;
  c0.divh2 = V(ip.divh2);
  c0.divh3 = V(ip.divh3);
  c0.divh4 = V(ip.divh4);
  c0.cf = coef;
  const V vdt(ip.dt);
  const int n0 = ip.n[0], n1 = ip.n[1];
  const long long pitch = ip.pitch;
  T* out[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) out[f] = p.out[ii * NF + f];
  const int h[3] = {p.hx, p.hy, 0};
  const int n3[3] = {n0, n1, 1};
  const int per3[3] = {1, 1, 0};
  // the whole tile inside the instance and R away from every face: plain
  // vector stores (uniform across the block)
  const bool plain =
      x0 >= R && x0 + TX <= n0 - R && y0 >= R && y0 + TY <= n1 - R;
  const bool rhs_only = p.rhs_only != 0;
#pragma unroll 1
  for (int i = threadIdx.x; i < CNT; i += NT) {
    const int rb = i / NG, g = i - rb * NG;
    const int off = (rb * SR + K::HY) * PW + g * W + K::HX;
    V nv[SR][NF];
#pragma unroll
    for (int k = 0; k < SR; ++k) {
      CO ctx = c0;
#pragma unroll
      for (int f = 0; f < NF; ++f) ctx.fo[f][0] = src + f * PLANE + off + k * PW;
      if constexpr (NS > 0) {
#pragma unroll
        for (int q = 0; q < NS; ++q) ctx.so[q][0] = sb + q * PLANE + off + k * PW;
      }
      const V r0 = eval(m.r0, ctx);
      nv[k][0] = rhs_only ? r0 : fmadd<!K::exact>(vdt, r0, ctx.template var<1, 0, 0, 0>());
      if constexpr (NF > 1) {
        const V r1 = eval(m.r1, ctx);
        nv[k][1] = rhs_only ? r1 : fmadd<!K::exact>(vdt, r1, ctx.template var<2, 0, 0, 0>());
      }
    }
    const int x = x0 + g * W;
#pragma unroll
    for (int k = 0; k < SR; ++k) {
      const int y = y0 + rb * SR + k;
      if (plain) {
#pragma unroll
        for (int f = 0; f < NF; ++f)
          *reinterpret_cast<V*>(out[f] + (long long)(y + p.hy) * pitch + x + p.hx) = nv[k][f];
      } else if (x < n0 && y < n1) {
#pragma unroll
        for (int f = 0; f < NF; ++f)
          store_group<T, W, 2, R>(out[f], x, y, 0, nv[k][f], n3, h, per3, pitch, 0);
      }
      if (p.partial && x < n0 && y < n1) msum += vsum<T, W>(nv[k][0], x, n0);
    }
  }
}

// KT-step schedule of one tile, from step KT - tsteps on: step j reads a
// margin of (KT - j) R, stages on (KT - j) R - RI and updates on
// (KT - j - 1) R; the last step writes the output
template <class K, class M, class T, int LP, int GP, int BP, int J>
__device__ __forceinline__ void tb_steps(const Step2Params<T>& p, const M& m, const Inst2<T>& ip,
                                         int ii, T* a, T* b, T* sb, int x0, int y0, int first,
                                         double& msum) {
  constexpr int KT = K::KT, R = K::R;
  if constexpr (J < KT) {
    if (J >= first) {
      constexpr int HIN = (KT - J) * R;
      if constexpr (M::ns > 0) {
        tb_stage<K, M, T, LP, GP, BP, HIN - K::RI>(m, ip, a, sb);
        __syncthreads();
      }
      if constexpr (J == KT - 1) {
        tb_final<K, M, T, LP, GP, BP>(p, m, ip, ii, a, sb, x0, y0, msum);
      } else {
        tb_update<K, M, T, LP, GP, BP, HIN - R>(m, ip, a, sb, b);
        __syncthreads();
      }
      tb_steps<K, M, T, LP, GP, BP, J + 1>(p, m, ip, ii, b, a, sb, x0, y0, first, msum);
    } else {
      tb_steps<K, M, T, LP, GP, BP, J + 1>(p, m, ip, ii, a, b, sb, x0, y0, first, msum);
    }
  }
}

template <class M0, class M1, class T, int LP, int GP, int BP, class TC, bool EXACT>
__global__ void __launch_bounds__(TC::NT)
    k_fd2t(const __grid_constant__ Step2Params<T> p, const __grid_constant__ M0 m0,
           const __grid_constant__ M1 m1) {
  using K = Fd2T<M0, M1, T, LP, GP, BP, TC, EXACT>;
  constexpr int TX = K::TX, TY = K::TY, NF = K::NF, NT = K::NT, LC = K::LC, PW = K::PW,
                PH = K::PH, PLANE = K::PLANE, GW = K::GW, HX = K::HX, HY = K::HY, KT = K::KT;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  int2* slots = reinterpret_cast<int2*>(smem_raw);  // [2]: the item of each input buffer
  T* inb = reinterpret_cast<T*>(smem_raw + 128);    // [2][NF] planes
  T* mid = inb + 2 * NF * PLANE;                    // [NF]
  T* sbuf = mid + NF * PLANE;                       // [NS]
  __shared__ double red[32];
  const int tid = threadIdx.x;

  pdl_enter();

  // the work queue of k_fd2d: batches of 4 items per atomic when every CTA
  // has many, one at a time otherwise, a fixed share for a single instance
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
  auto tile_xy = [&](int t, int ntx) -> int2 {
    if (p.items) return make_int2(t & 0xffff, t >> 16);
    return make_int2(t % ntx, t / ntx);
  };
  // the tile with its margin, wrapped around the periodic faces, into input
  // buffer `buf` (every thread issues its share of 16-byte copies)
  auto load = [&](int2 it, int buf) {
    const Inst2<T>& ip = p.inst[it.x];
    const int2 tc = tile_xy(it.y, ip.ntx);
    const int xs = tc.x * TX - HX, ys = tc.y * TY - HY;
    const int n0 = ip.n[0], n1 = ip.n[1];
    const long long pitch = ip.pitch;
    constexpr int CNT = NF * PH * GW;
#pragma unroll 1
    for (int i = tid; i < CNT; i += NT) {
      const int f = NF > 1 ? i / (PH * GW) : 0;
      const int rem = i - f * (PH * GW);
      const int r = rem / GW, c = rem - r * GW;
      const int y = tb_wrap(ys + r, n1), x = tb_wrap(xs + c * LC, n0);
      tb_cp16(inb + (buf * NF + f) * PLANE + r * PW + c * LC,
              p.in[it.x * NF + f] + (long long)(y + p.hy) * pitch + (x + p.hx));
    }
  };

  const int first = KT - p.tsteps;  // the schedule's first step of this launch
  double msum = 0.0;
  if (tid == 0) slots[0] = fetch();
  __syncthreads();
  int2 cur = slots[0];
  if (cur.x >= 0) load(cur, 0);
  tb_commit();
  int buf = 0;
  while (cur.x >= 0) {
    if (tid == 0) slots[buf ^ 1] = fetch();
    // every thread is done with the previous tile (its buffers are free) and
    // sees the next item
    __syncthreads();
    const int2 nxt = slots[buf ^ 1];
    if (nxt.x >= 0) load(nxt, buf ^ 1);
    tb_commit();
    tb_wait<1>();  // this thread's copies of the current tile have landed
    __syncthreads();  // and everyone's
    const Inst2<T>& ip = p.inst[cur.x];
    const int2 tc = tile_xy(cur.y, ip.ntx);
    T* a = inb + buf * NF * PLANE;
    if (ip.kind == 0)
      tb_steps<K, M0, T, LP, GP, BP, 0>(p, m0, ip, cur.x, a, mid, sbuf, tc.x * TX, tc.y * TY,
                                        first, msum);
    else
      tb_steps<K, M1, T, LP, GP, BP, 0>(p, m1, ip, cur.x, a, mid, sbuf, tc.x * TX, tc.y * TY,
                                        first, msum);
    cur = nxt;
    buf ^= 1;
  }
  tb_wait<0>();
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
