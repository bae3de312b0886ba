/*
 * sp_ch.cuh -- lowering of the conserved-dynamics pattern of the fused form:
 *
 *     d psi / dt = M * lap(mu),   mu = P(psi) - K * lap(psi)     (3D, 7-point lap)
 *
 * with P any pointwise sub-tree of the model (no derivative) and M, K pointwise
 * constants -- model B (Cahn-Hilliard, the SymPhas MB of
 * examples/models/modeldefinitions.h:48-51 in fused form) and its mobility /
 * gradient-coefficient variant.  The tree is recognised at compile time
 * (ChPattern); P, M and K are still evaluated by the generic evaluator, and
 * every floating-point operation mirrors the generic fused evaluation
 * (sp_expr.cuh) operand for operand, so this kernel gives the same bits as the
 * generic kernel and the autotuner may choose either.
 *
 * What differs is the execution: a thread owns W x SPT sites of a column and
 * keeps the z-neighbours it needs (psi at z, z+1, z+2 and mu at z-1, z, z+1)
 * in registers, so shared memory is read only for in-plane neighbours, through
 * per-plane row pointers with compile-time offsets; mu needs a ring of three
 * planes.  The TMA pipeline (field planes in flight, one barrier per plane) is
 * the generic kernel's.
 */
#pragma once

#include <type_traits>

#include "sp_kernels.cuh"

namespace sp {

// ---------------------------------------------------------------------------
// pattern recognition on the lowered model type
// ---------------------------------------------------------------------------
template <class E>
struct IsPointwise {  // no derivative and no stage anywhere below
  static constexpr bool value =
      ex::Reach<E>::field <= 0 && ex::Reach<E>::stage < 0 && ex::Reach<E>::max_var <= 1;
};

template <class R0>
struct ChRhs {
  static constexpr bool ok = false;
};
template <>
struct ChRhs<ex::Lap<ex::StageRef<0>>> {  // lap(mu)
  static constexpr bool ok = true, has_m = false;
  using Mob = ex::Lit;
  __device__ static Mob mob(const ex::Lap<ex::StageRef<0>>&) { return ex::Lit(1.0); }
};
template <class MExpr>
struct ChRhs<ex::Mul<MExpr, ex::Lap<ex::StageRef<0>>>> {  // M * lap(mu)
  static constexpr bool ok = IsPointwise<MExpr>::value && ex::Reach<MExpr>::field < 0;
  static constexpr bool has_m = true;
  using Mob = MExpr;
  __device__ static const Mob& mob(const ex::Mul<MExpr, ex::Lap<ex::StageRef<0>>>& e) {
    return e.a;
  }
};

template <class S0>
struct ChStage {
  static constexpr bool ok = false;
};
template <class E>
struct IsMul {
  static constexpr bool value = false;
};
template <class A, class B>
struct IsMul<ex::Mul<A, B>> {
  static constexpr bool value = true;
};
// (a product minus lap(psi) is evaluated as one FMA by the generic evaluator,
// so that shape is left to the generic kernel)
template <class P>
struct ChStage<ex::Sub<P, ex::Lap<ex::Var<1>>>> {  // P(psi) - lap(psi)
  static constexpr bool ok = IsPointwise<P>::value && !IsMul<P>::value, has_k = false;
  using Kx = ex::Lit;
  __device__ static const P& pw(const ex::Sub<P, ex::Lap<ex::Var<1>>>& e) { return e.a; }
  __device__ static Kx kappa(const ex::Sub<P, ex::Lap<ex::Var<1>>>&) { return ex::Lit(1.0); }
};
template <class P, class KExpr>
struct ChStage<ex::Sub<P, ex::Mul<KExpr, ex::Lap<ex::Var<1>>>>> {  // P(psi) - K lap(psi)
  static constexpr bool ok = IsPointwise<P>::value && IsPointwise<KExpr>::value &&
                             ex::Reach<KExpr>::field < 0;
  static constexpr bool has_k = true;
  using Kx = KExpr;
  __device__ static const P& pw(const ex::Sub<P, ex::Mul<KExpr, ex::Lap<ex::Var<1>>>>& e) {
    return e.a;
  }
  __device__ static const Kx& kappa(const ex::Sub<P, ex::Mul<KExpr, ex::Lap<ex::Var<1>>>>& e) {
    return e.b.a;
  }
};

template <class M>
struct ChPattern {
  static constexpr bool ok = M::nf == 1 && M::ns == 1 && ChRhs<decltype(M::r0)>::ok &&
                             ChStage<decltype(M::s0)>::ok;
};

// pointwise evaluation context: psi and the coefficients live in registers
template <class T, int W>
struct PwCtx {
  using scalar_type = T;
  using value_type = vec_t<T, W>;
  static constexpr bool contract = true;
  static constexpr int dim = 3, lap_points = 7, gradlap_points = 10, bilap_points = 25;
  value_type psi;
  value_type divh2, divh3, divh4;
  const T* cf;
  template <int I, int X, int Y, int Z>
  __device__ __forceinline__ value_type var() const {
    static_assert(I == 1 && X == 0 && Y == 0 && Z == 0, "pointwise sub-tree");
    return psi;
  }
  template <int K, int X, int Y, int Z>
  __device__ __forceinline__ value_type stg() const {
    static_assert(K < 0, "pointwise sub-tree");
    return psi;
  }
  __device__ __forceinline__ value_type coef(int i) const { return value_type(cf[i - 1]); }
};

// x-direction pair sum of a W-group at p (p W-aligned): lanes j hold
// p[j-1] + p[j+1], built lane by lane from aligned loads (no register shuffles)
template <class T, int W>
__device__ __forceinline__ vec_t<T, W> xsum(const T* p) {
  const vec_t<T, W> a = load_at<T, W, -W>(p), c = load_at<T, W, 0>(p), b = load_at<T, W, W>(p);
  vec_t<T, W> r;
  if constexpr (W == 1) {
    r = a + b;
  } else {
#pragma unroll
    for (int j = 0; j < W; ++j) {
      const T l = (j == 0) ? a.v[W - 1] : c.v[j - 1];
      const T h = (j == W - 1) ? b.v[0] : c.v[j + 1];
      r.v[j] = l + h;
    }
  }
  return r;
}

// 7-point Laplacian from its three pair sums and the centre, in the generic
// fused evaluator's order: fma(-6 divh2, c, ((sx + sy) + sz) * divh2)
template <class V>
__device__ __forceinline__ V lap7(const V& sx, const V& sy, const V& sz, const V& c,
                                  const V& m6divh2, const V& divh2) {
  return fmadd<true>(m6divh2, c, ((sx + sy) + sz) * divh2);
}

template <class M, class T, class TC>
struct Ch3 {
  static constexpr int TX = TC::TX, TY = TC::TY, SPT = TC::SPT, PD = TC::PD, W = TC::W,
                       TXT = TC::TXT, NT = TC::NT;
  static constexpr int R = 2, RS = 1, RI = 1;
  using G = HaloGeom<T, W, R, 1, RS, RI>;
  static constexpr int RSA = G::RSA, HXA = G::HXA;
  static constexpr int PW = TX + 2 * HXA, PH = TY + 2 * R;
  static constexpr int PLANE = ceil_to(PW * PH, 128 / (int)sizeof(T));
  // field window z .. z+2, one spare plane, PD in flight
  static constexpr int NSLOT = 3 + 1 + PD;
  static constexpr int SW = TX + 2 * RSA, SH = TY + 2 * RS, SPL = ceil_to(SW * SH, 32);
  static constexpr int NSR = 3;  // mu planes z, z+1 and the spare
  static constexpr int SWC = SW / W, XC = 2 * RSA / W;
  static constexpr int NE = 2 * RS * SWC + TY * XC;
  static constexpr size_t SMEM = 256 + sizeof(T) * (size_t(NSLOT) * PLANE + size_t(NSR) * SPL);
  static_assert(ChPattern<M>::ok, "model is not of the conserved M lap(P - K lap) form");
  static_assert(M::R == R && M::RS == RS, "reach of the pattern");
  static_assert(NE <= NT, "one extra stage cell per thread at most");
  static_assert(PW <= 256 && PH <= 256 && (PW * sizeof(T)) % 16 == 0, "TMA box");
};

template <class M, class T, class TC>
__global__ void __launch_bounds__(TC::NT)
    k_ch3d(const __grid_constant__ StepParams<T> p, const __grid_constant__ M m) {
  pdl_enter();
  using K = Ch3<M, T, TC>;
  constexpr int TX = K::TX, TY = K::TY, SPT = K::SPT, PD = K::PD, W = K::W, TXT = K::TXT,
                R = K::R, RS = K::RS, RSA = K::RSA, HXA = K::HXA, PW = K::PW, PH = K::PH,
                PLANE = K::PLANE, NSLOT = K::NSLOT, SW = K::SW, SPL = K::SPL, NSR = K::NSR,
                NT = K::NT, SWC = K::SWC, XC = K::XC, NE = K::NE;
  constexpr uint32_t TXB = uint32_t(PW * PH * sizeof(T));
  using V = vec_t<T, W>;
  using RH = ChRhs<decltype(M::r0)>;
  using SG = ChStage<decltype(M::s0)>;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  T* fbuf = reinterpret_cast<T*>(smem_raw + 256);
  T* sbuf = fbuf + NSLOT * PLANE;
  __shared__ double red[32];

  const int tid = threadIdx.x, txt = tid % TXT, tg = tid / TXT, row0 = tg * SPT;
  const int tile = blockIdx.x;
  const int x0 = (tile % p.ntx) * TX, y0 = (tile / p.ntx) * TY;
  const int zb = blockIdx.y * p.zchunk;
  const int ze = min(zb + p.zchunk, p.n[2]);
  const CUtensorMap* map = p.maps + blockIdx.z;
  const int nplanes = (ze - 1 + R) - (zb - R) + 1;

  T coef[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) coef[i] = p.coef[i];
  PwCtx<T, W> pc;
  pc.divh2 = V(p.divh2);
  pc.divh3 = V(p.divh3);
  pc.divh4 = V(p.divh4);
  pc.cf = coef;
  const V divh2(p.divh2), vdt(p.dt);
  const V m6divh2 = V(-6.0) * divh2;
  // M and K are constants of the tree (coefficients, literals)
  const V mob = eval(RH::mob(m.r0), pc);
  const V kap = eval(SG::kappa(m.s0), pc);

  // output rows of this thread
  const int x = x0 + txt * W;
  const bool xin = x < p.n[0];
  const bool vec_ok = (p.n[0] % W == 0) && (x + W <= p.n[0]);
  const long long xo = image_offset(p.per[0], x, W, p.n[0], R, 1);
  T* orow[SPT];
  bool rowin[SPT];
  long long yo[SPT];
#pragma unroll
  for (int k = 0; k < SPT; ++k) {
    const int y = y0 + row0 + k;
    rowin[k] = xin && y < p.n[1];
    yo[k] = image_offset(p.per[1], y, 1, p.n[1], R, p.pitch);
    orow[k] = p.out[blockIdx.z] + (long long)(y + p.h[1]) * p.pitch + (x + p.h[0]);
  }
  // the whole tile inside the domain, away from every periodic face, in whole
  // vectors: straight-line stores (the same for every thread of the block)
  const bool plain = (p.n[0] % W == 0) && x0 + TX <= p.n[0] && y0 + TY <= p.n[1] &&
                     (!p.per[0] || (x0 >= R && x0 + TX <= p.n[0] - R)) &&
                     (!p.per[1] || (y0 >= R && y0 + TY <= p.n[1] - R));
  const bool ragged = xin && !vec_ok;
  const bool xany = p.per[0] && (x0 < R || x0 + TX + W > p.n[0] - R);
  const bool do_mass = p.partial != nullptr;
  // the mu cell beyond this thread's own ones, if any: own cells are stage
  // rows RS..TY+RS-1 and column groups RSA/W..RSA/W+TXT-1; the ring is the
  // rows above and below (all groups) and the column groups left and right
  int xsr = -1, xsc = 0;
  if (tid < NE) {
    if (tid < 2 * RS * SWC) {
      const int r = tid / SWC;
      xsr = r < RS ? r : TY + r;
      xsc = tid % SWC;
    } else {
      const int e = tid - 2 * RS * SWC;
      const int cc = e % XC;
      xsr = RS + e / XC;
      xsc = cc < XC / 2 ? cc : TXT + cc;
    }
  }
  // element offsets: own field cell (row row0, in the field tile), own mu cell,
  // and the extra mu cell with its field cell
  const int fown = (row0 + R) * PW + txt * W + HXA;
  const int sown = (row0 + RS) * SW + txt * W + RSA;
  const int sext = xsr * SW + xsc * W;
  const int fext = (xsr - RS + R) * PW + xsc * W - RSA + HXA;

  if (tid == 0) {
    for (int s = 0; s < NSLOT; ++s) tma::mbar_init(&bars[s], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
  auto issue = [&](int q) {
    const int s = q % NSLOT;
    tma::mbar_arrive_expect_tx(&bars[s], TXB);
    tma::load_3d(fbuf + s * PLANE, map, &bars[s], x0 + p.h[0] - HXA, y0 + p.h[1] - R,
                 zb - R + q + p.h[2]);
  };
  // plane sequence q(z) = z - (zb - R); iteration zi issues q(zi + R + PD)
  const int zi0 = zb - 2 * RS;
  if (tid == 0) {
    const int pro = min(zi0 + R + PD - (zb - R), nplanes);
    for (int q = 0; q < pro; ++q) issue(q);
  }

  // register queues of the own cells: psi at z-1.. and mu at z-1.., rotated
  // by the iteration's phase (zi - zi0) % 3
  V qpsi[3][SPT], qmu[3][SPT];
  double msum = 0.0;
  int zslot = 0;  // ring slot of plane zi (q(zi0) = 0)
  int mslot = 0;  // mu ring slot of plane zi + 1 at iteration zi

  auto body = [&](auto phase_tag, int zi) -> bool {
    constexpr int P = decltype(phase_tag)::value;
    constexpr int IM = P % 3, IC = (P + 1) % 3, IP = (P + 2) % 3;
    // wait for plane zi + 2 (all of 0..2 on the first iteration)
    const int qw = zi + R - (zb - R);
    bool bad = false;
    if (zi == zi0) {
      for (int q = 0; q <= qw; ++q) bad |= !tma::mbar_wait(&bars[q % NSLOT], (q / NSLOT) & 1);
    } else {
      bad = !tma::mbar_wait(&bars[wrap<NSLOT>(zslot, R)], (qw / NSLOT) & 1);
    }
    const T* f0 = fbuf + zslot * PLANE;                    // psi(zi)
    const T* f1 = fbuf + wrap<NSLOT>(zslot, 1) * PLANE;    // psi(zi+1)
    const T* f2 = fbuf + wrap<NSLOT>(zslot, 2) * PLANE;    // psi(zi+2)
    T* mw = sbuf + mslot * SPL;                            // mu(zi+1)
    const T* mr = sbuf + wrap<NSR>(mslot, -1) * SPL;       // mu(zi)
    if (zi == zi0) {
#pragma unroll
      for (int k = 0; k < SPT; ++k) {
        qpsi[IM][k] = load_at<T, W, 0>(f0 + fown + k * PW);
        qpsi[IC][k] = load_at<T, W, 0>(f1 + fown + k * PW);
      }
    }
    // ---- mu at z+1: own cells from the queues, the extra cell from shared memory
    {
      const T* c1 = f1 + fown;
      V mu[SPT];
#pragma unroll
      for (int k = 0; k < SPT; ++k) {
        qpsi[IP][k] = load_at<T, W, 0>(f2 + fown + k * PW);
        const V c = qpsi[IC][k];
        const V sx = xsum<T, W>(c1 + k * PW);
        const V sy = load_at<T, W, 0>(c1 + (k - 1) * PW) + load_at<T, W, 0>(c1 + (k + 1) * PW);
        const V sz = qpsi[IM][k] + qpsi[IP][k];
        const V l = lap7(sx, sy, sz, c, m6divh2, divh2);
        pc.psi = c;
        const V pw = eval(SG::pw(m.s0), pc);
        if constexpr (SG::has_k)
          mu[k] = fmadd<true>(-kap, l, pw);
        else
          mu[k] = pw - l;
      }
      V mue;
      if (xsr >= 0) {
        const T* e1 = f1 + fext;
        const V c = load_at<T, W, 0>(e1);
        const V sx = xsum<T, W>(e1);
        const V sy = load_at<T, W, -PW>(e1) + load_at<T, W, PW>(e1);
        const V sz = load_at<T, W, 0>(f0 + fext) + load_at<T, W, 0>(f2 + fext);
        const V l = lap7(sx, sy, sz, c, m6divh2, divh2);
        pc.psi = c;
        const V pw = eval(SG::pw(m.s0), pc);
        if constexpr (SG::has_k)
          mue = fmadd<true>(-kap, l, pw);
        else
          mue = pw - l;
      }
#pragma unroll
      for (int k = 0; k < SPT; ++k) {
        *reinterpret_cast<V*>(mw + sown + k * SW) = mu[k];
        qmu[IP][k] = mu[k];
      }
      if (xsr >= 0) *reinterpret_cast<V*>(mw + sext) = mue;
    }
    if (__syncthreads_or(bad)) return false;
    // ---- output at z = zi: psi + dt * M * lap(mu)
    if (zi >= zb) {
      const T* c0 = mr + sown;
      const long long zoff = (long long)(zi + p.h[2]) * p.plane;
      const long long zo = image_offset(p.per[2], zi, 1, p.n[2], R, p.plane);
      V nv[SPT];
#pragma unroll
      for (int k = 0; k < SPT; ++k) {
        const V sx = xsum<T, W>(c0 + k * SW);
        const V sy = load_at<T, W, 0>(c0 + (k - 1) * SW) + load_at<T, W, 0>(c0 + (k + 1) * SW);
        const V sz = qmu[IM][k] + qmu[IP][k];
        V r = lap7(sx, sy, sz, qmu[IC][k], m6divh2, divh2);
        if constexpr (RH::has_m) r = mob * r;
        nv[k] = p.rhs_only ? r : fmadd<true>(vdt, r, qpsi[IM][k]);
      }
      if (plain && zo == 0) {
#pragma unroll
        for (int k = 0; k < SPT; ++k) *reinterpret_cast<V*>(orow[k] + zoff) = nv[k];
      } else {
#pragma unroll
        for (int k = 0; k < SPT; ++k) {
          put_images_pred(orow[k] + zoff, nv[k], rowin[k] && vec_ok, xany, xo, yo[k], zo);
          if (ragged && rowin[k])
            store_group<T, W, 3, R>(p.out[blockIdx.z], x, y0 + row0 + k, zi, nv[k], p.n, p.h,
                                    p.per, p.pitch, p.plane);
        }
      }
      if (do_mass) {
#pragma unroll
        for (int k = 0; k < SPT; ++k)
          if (rowin[k]) msum += vsum<T, W>(nv[k], x, p.n[0]);
      }
    }
    return true;
  };

  // zi0, zi0+1 are the warm-up iterations (mu only); one barrier per plane
  int phase = 0;
  for (int zi = zi0; zi < ze; ++zi) {
    const int qn = zi + R + PD - (zb - R);
    if (tid == 0 && qn < nplanes) issue(qn);
    bool ok;
    if (phase == 0)
      ok = body(std::integral_constant<int, 0>{}, zi);
    else if (phase == 1)
      ok = body(std::integral_constant<int, 1>{}, zi);
    else
      ok = body(std::integral_constant<int, 2>{}, zi);
    if (!ok) {
      if (tid == 0) {
        atomicExch(p.err, KERR_TMA_TIMEOUT);
        tma::drain(bars, NSLOT, zi == zi0 ? 0 : zi + R - (zb - R), min(qn, nplanes - 1));
      }
      return;
    }
    phase = phase == 2 ? 0 : phase + 1;
    zslot = wrap<NSLOT>(zslot, 1);
    mslot = wrap<NSR>(mslot, 1);
  }
  __syncthreads();
  if (p.partial) {
    const double s = block_sum<NT>(msum, red);
    if (tid == 0)
      p.partial[(size_t(blockIdx.z) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
  }
}

}  // namespace sp
