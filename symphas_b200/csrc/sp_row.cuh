/*
 * sp_row.cuh -- row kernel for any fused FP32 model lowered onto 7-point
 * Laplacians with at most one staged operand (models A, B, C, AMK, BMK in
 * their fused forms), on grids whose x extent is one or two 128-site warp
 * rows (n_x = 128 or 256) and periodic in x.
 *
 * The data movement of the conserved-pattern row kernel (sp_chrow.cuh) with
 * the right-hand sides and the staged operand evaluated by the generic
 * evaluator (sp_expr.cuh) on a context of its own: a CTA owns whole x rows
 * (warp w: one row, lane l: the 4-site chunks x = 128 g + 4 l), the x
 * neighbours of a chunk come from warp shuffles (the periodic row wraps around
 * the warp), y neighbours from the rows in shared memory, z neighbours of the
 * staged operand from a register queue and of the fields from the TMA plane
 * ring.  The evaluator asks the context only for the offsets a 7-point
 * Laplacian reads and forms its sums in the same order as in the tile
 * kernels, so every site gets the same bits as there.
 */
#pragma once

#include "sp_ch.cuh"

namespace sp {

template <class M, int NXR_, int YW_, int PD_, int MINB_ = 1>
struct RowCfg {
  using T = float;
  static constexpr int NXR = NXR_, G = NXR_ / 128, YW = YW_, PD = PD_, MINB = MINB_;
  static constexpr int NT = 32 * YW, SPT = 1, TX = NXR;
  static constexpr int NF = M::nf, NS = M::ns, R = M::R;
  static constexpr int RD = imax(M::r_direct, 0);
  static constexpr int RS = NS > 0 ? M::RS : 0, RI = imax(M::r_stage, 0);
  static constexpr int RING = RS;                      // staged rows above and below the outputs
  static constexpr int TY = YW - 2 * RING;             // output rows per CTA
  static constexpr int U = imax(RD, NS > 0 ? RS + RI : 0);                    // newest plane read
  static constexpr int L = NS > 0 ? (RS - RI < -RD ? RS - RI : -RD) : -RD;    // oldest
  static constexpr int WARM = 2 * RS;  // iterations that only stage
  static constexpr int NPW = U - L + 1;
  static constexpr int PH = TY + 2 * R;  // field rows of a plane box (y0 - R ..)
  static constexpr int PLANE = NXR * PH;
  static constexpr int NSLOT = NPW + PD;
  static constexpr int MPL = NXR * YW;  // one staged plane
  static constexpr size_t SMEM =
      256 + sizeof(T) * (size_t(NF) * NSLOT * PLANE + (NS > 0 ? 2 * size_t(MPL) : 0));
  // the field layout of the tile kernels of the same key
  static constexpr int HXA = HaloGeom<T, 2, R, NS, RS, RI>::HXA;
  static_assert(NXR == 128 || NXR == 256, "rows of one warp, one or two chunks per lane");
  static_assert(NS <= 1 && RS <= 1 && RI <= 1 && RD <= 1, "7-point reach, one staged operand");
  static_assert(R - WARM + L <= 0, "prologue planes fit the ring");
  static_assert(TY >= 1 && NT <= 1024 && PH <= 256 && NSLOT <= 32, "shape");
  static_assert(MINB >= 1 && size_t(MINB) * (SMEM + 1024) <= 227 * 1024, "CTAs per SM");
};

// The values one row's evaluation reads: the fields' centres at planes
// z - 1, z, z + 1 (fc[.][0..2]) and rows y - 1, y + 1 at z, for all G chunks
// of the lane (the x neighbours at a row's ends come from the other chunk);
// the staged operand likewise.
template <int NF, int NS, int G>
struct RowData {
  using V = Vec<float, 4>;
  V fc[NF][3][G], fu[NF][G], fd[NF][G];
  V sc[NS > 0 ? NS : 1][3][G], su[NS > 0 ? NS : 1][G], sd[NS > 0 ? NS : 1][G];
};

// The evaluation context of chunk g over a RowData.  Offsets outside the
// 7-point reach do not compile.
template <int NF, int NS, int G, int g>
struct RowCtx {
  using scalar_type = float;
  using value_type = Vec<float, 4>;
  using V = value_type;
  static constexpr bool contract = true;
  static constexpr int dim = 3, lap_points = 7, gradlap_points = 10, bilap_points = 25;
  const RowData<NF, NS, G>& d;
  V divh2, divh3, divh4;
  const float* cf;
  int lane;

  // the site left of the chunk's first site and right of its last one
  __device__ __forceinline__ float left(const V (&c)[G]) const {
    const int lm = (lane + 31) & 31;
    if constexpr (G == 1) {
      return __shfl_sync(0xffffffffu, c[0].v[3], lm);
    } else {
      const float a = __shfl_sync(0xffffffffu, c[0].v[3], lm);
      const float b = __shfl_sync(0xffffffffu, c[1].v[3], lm);
      return (g == 0) == (lane == 0) ? b : a;
    }
  }
  __device__ __forceinline__ float right(const V (&c)[G]) const {
    const int lp = (lane + 1) & 31;
    if constexpr (G == 1) {
      return __shfl_sync(0xffffffffu, c[0].v[0], lp);
    } else {
      const float a = __shfl_sync(0xffffffffu, c[0].v[0], lp);
      const float b = __shfl_sync(0xffffffffu, c[1].v[0], lp);
      return (g == 0) == (lane == 31) ? b : a;
    }
  }
  template <int X, int Y, int Z>
  __device__ __forceinline__ V pick(const V (&c)[3][G], const V (&u)[G], const V (&dn)[G]) const {
    static_assert(Z >= -1 && Z <= 1, "z reach beyond one plane");
    static_assert(Z == 0 || (X == 0 && Y == 0), "7-point reach");
    if constexpr (X == 0 && Y == 0) {
      return c[Z + 1][g];
    } else if constexpr (X == 0 && Y == -1) {
      return u[g];
    } else if constexpr (X == 0 && Y == 1) {
      return dn[g];
    } else if constexpr (Y == 0 && X == -4) {  // the group left: only its last lane is read
      V r = c[1][g];
      r.v[3] = left(c[1]);
      return r;
    } else if constexpr (Y == 0 && X == 4) {  // the group right: only its first lane is read
      V r = c[1][g];
      r.v[0] = right(c[1]);
      return r;
    } else if constexpr (Y == 0 && X == -1) {
      V r;
      r.v[0] = left(c[1]);
      r.v[1] = c[1][g].v[0];
      r.v[2] = c[1][g].v[1];
      r.v[3] = c[1][g].v[2];
      return r;
    } else {
      static_assert(Y == 0 && X == 1, "7-point reach");
      V r;
      r.v[0] = c[1][g].v[1];
      r.v[1] = c[1][g].v[2];
      r.v[2] = c[1][g].v[3];
      r.v[3] = right(c[1]);
      return r;
    }
  }
  template <int I, int X, int Y, int Z>
  __device__ __forceinline__ V var() const {
    static_assert(I >= 1 && I <= NF, "field index");
    return pick<X, Y, Z>(d.fc[I - 1], d.fu[I - 1], d.fd[I - 1]);
  }
  template <int K, int X, int Y, int Z>
  __device__ __forceinline__ V stg() const {
    static_assert(K >= 0 && K < NS, "stage index");
    return pick<X, Y, Z>(d.sc[K], d.su[K], d.sd[K]);
  }
  __device__ __forceinline__ V coef(int i) const { return V(cf[i - 1]); }
};

template <class M, class KC>
__device__ __forceinline__ void row_step(const StepParams<float>& p, const M& m) {
  using T = float;
  using V = Vec<float, 4>;
  constexpr int NXR = KC::NXR, G = KC::G, TY = KC::TY, PD = KC::PD, PLANE = KC::PLANE,
                NSLOT = KC::NSLOT, MPL = KC::MPL, R = KC::R, NT = KC::NT, NF = KC::NF,
                NS = KC::NS, RING = KC::RING, U = KC::U, L = KC::L, WARM = KC::WARM,
                NPW = KC::NPW;
  constexpr uint32_t TXB = uint32_t(NF * PLANE * sizeof(T));
  using Data = RowData<NF, NS, G>;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  T* fbuf = reinterpret_cast<T*>(smem_raw + 256);  // [field][slot][PH][NXR]
  T* mbuf = fbuf + NF * NSLOT * PLANE;              // two staged planes, alternately
  __shared__ double red[32];

  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int xl = lane * 4;
  const int y0 = blockIdx.x * TY;
  const int zb = blockIdx.y * p.zchunk;
  const int ze = min(zb + p.zchunk, p.n[2]);
  const int inst = blockIdx.z;
  const CUtensorMap* maps = p.maps + inst * NF;
  // field planes of this CTA: z = zb - R + q for q in [0, nplanes)
  const int nplanes = (ze - 1 + U) - (zb - R) + 1;
  // warp w computes row y = y0 - RING + w: its field row in a plane box is
  // b = w - RING + R, its staged row w
  const int frow = (w - RING + R) * NXR;
  const int o = w - RING;  // output row, when 0 <= o < TY
  const int y = y0 + o;
  const bool oin = o >= 0 && o < TY && y < p.n[1];

  T coef[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) coef[i] = p.coef[i];
  const V divh2(p.divh2), divh3(p.divh3), divh4(p.divh4), vdt(p.dt);

  long long xo[G];
#pragma unroll
  for (int g = 0; g < G; ++g) xo[g] = image_offset(p.per[0], xl + 128 * g, 4, p.n[0], R, 1);
  const long long yo = oin ? image_offset(p.per[1], y, 1, p.n[1], R, p.pitch) : 0;
  const bool yimg = yo != 0;  // warp-uniform
  const bool do_mass = p.partial != nullptr;
  const bool rhs_only = p.rhs_only != 0;
  const bool zper = p.per[2] != 0;

  if (tid == 0) {
    for (int s = 0; s < NSLOT; ++s) tma::mbar_init(&bars[s], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
  auto issue = [&](int q) {
    const int s = q % NSLOT;
    tma::mbar_arrive_expect_tx(&bars[s], TXB);
#pragma unroll
    for (int f = 0; f < NF; ++f)
      tma::load_3d(fbuf + (f * NSLOT + s) * PLANE, maps + f, &bars[s], p.h[0], y0 - R + p.h[1],
                   zb - R + q + p.h[2]);
  };
  // plane sequence q(z) = z - (zb - R); iteration zi reads field planes zi + L
  // .. zi + U; the prologue issues every plane up to q(zi0 + U + PD), and
  // iteration zi > zi0 issues q(zi + U + PD) into the slot of plane
  // zi + L - 1, which the previous iteration read last, before its barrier
  const int zi0 = zb - WARM;
  const int q0 = zi0 - (zb - R);  // q of plane zi0 (>= 0)
  if (tid == 0) {
    const int pro = min(q0 + U + PD + 1, nplanes);
    for (int q = 0; q < pro; ++q) issue(q);
  }
  // every plane the first iteration reads except the newest, which the first
  // iteration waits for like any other
  bool bad0 = false;
  for (int q = 0; q < q0 + U; ++q) bad0 |= !tma::mbar_wait(&bars[q % NSLOT], (q / NSLOT) & 1);

  // per-plane state, advanced by one plane per iteration: element offsets of
  // planes zi + L + j in the ring, the slot and phase of plane zi + U, the
  // staged planes written and read, the output row in plane zi
  int po[NPW];
#pragma unroll
  for (int j = 0; j < NPW; ++j) po[j] = (((q0 + L + j) % NSLOT + NSLOT) % NSLOT) * PLANE;
  int wslot = (q0 + U) % NSLOT;
  uint32_t wph = uint32_t(((q0 + U) / NSLOT) & 1);
  int ow = ((zi0 + 1) & 1) * MPL, orr = (zi0 & 1) * MPL;
  T* oz[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f)
    oz[f] = p.out[inst * NF + f] + (long long)(y + p.h[1]) * p.pitch + (xl + p.h[0]) +
            (long long)(zi0 + p.h[2]) * p.plane;

  V qmu[3][G];  // the staged operand of row w at z - 1, z, z + 1 (rotated by phase)
  double msum = 0.0;

  auto ld = [&](const T* row, V (&v)[G]) {
#pragma unroll
    for (int g = 0; g < G; ++g) v[g] = *reinterpret_cast<const V*>(row + 128 * g + xl);
  };
  // plane zi + dz of field f, at this warp's field row + dy
  auto frow_at = [&](int f, int dz, int dy) -> const T* {
    return fbuf + f * NSLOT * PLANE + po[dz - L] + frow + dy * NXR;
  };

  auto body = [&](auto phase_tag, int zi) -> bool {
    constexpr int P = decltype(phase_tag)::value;
    [[maybe_unused]] constexpr int IM = P % 3, IC = (P + 1) % 3, IP = (P + 2) % 3;
    bool bad = !tma::mbar_wait(&bars[wslot], wph);
    if (zi == zi0) bad |= bad0;
    [[maybe_unused]] T* const mw = mbuf + ow;
    [[maybe_unused]] const T* const mr = mbuf + orr;
    // ---- staged operand at zi + 1 on this warp's row
    if constexpr (NS > 0) {
      Data d;
#pragma unroll
      for (int f = 0; f < NF; ++f) {
#pragma unroll
        for (int dz = 0; dz < 3; ++dz) ld(frow_at(f, dz, 0), d.fc[f][dz]);
        ld(frow_at(f, 1, -1), d.fu[f]);
        ld(frow_at(f, 1, 1), d.fd[f]);
      }
      const RowCtx<NF, NS, G, 0> c0{d, divh2, divh3, divh4, coef, lane};
      qmu[IP][0] = eval(m.s0, c0);
      if constexpr (G == 2) {
        const RowCtx<NF, NS, G, 1> c1{d, divh2, divh3, divh4, coef, lane};
        qmu[IP][1] = eval(m.s0, c1);
      }
#pragma unroll
      for (int g = 0; g < G; ++g) *reinterpret_cast<V*>(mw + w * NXR + 128 * g + xl) = qmu[IP][g];
    }
    // ---- output at z = zi
    if (zi >= zb && o >= 0 && o < TY) {  // warp-uniform
      const bool zf = zper && (zi < R || zi >= p.n[2] - R);
      const long long zo = zf ? image_offset(1, zi, 1, p.n[2], R, p.plane) : 0;
      const bool plain = !zf && !yimg;
      Data d;
#pragma unroll
      for (int f = 0; f < NF; ++f) {
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz)
          if (dz >= L && dz <= U) ld(frow_at(f, dz, 0), d.fc[f][dz + 1]);
        ld(frow_at(f, 0, -1), d.fu[f]);
        ld(frow_at(f, 0, 1), d.fd[f]);
      }
      if constexpr (NS > 0) {
#pragma unroll
        for (int g = 0; g < G; ++g) {
          d.sc[0][0][g] = qmu[IM][g];
          d.sc[0][1][g] = qmu[IC][g];
          d.sc[0][2][g] = qmu[IP][g];
        }
        ld(mr + (w - 1) * NXR, d.su[0]);
        ld(mr + (w + 1) * NXR, d.sd[0]);
      }
      V nv[NF][G];
      auto out = [&](const auto& c, int g) {
        const V r0 = eval(m.r0, c);
        nv[0][g] = rhs_only ? r0 : fmadd<true>(vdt, r0, d.fc[0][1][g]);
        if constexpr (NF > 1) {
          const V r1 = eval(m.r1, c);
          nv[1][g] = rhs_only ? r1 : fmadd<true>(vdt, r1, d.fc[1][1][g]);
        }
      };
      out(RowCtx<NF, NS, G, 0>{d, divh2, divh3, divh4, coef, lane}, 0);
      if constexpr (G == 2) out(RowCtx<NF, NS, G, 1>{d, divh2, divh3, divh4, coef, lane}, 1);
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int g = 0; g < G; ++g) {
          T* const b = oz[f] + 128 * g;
          if (plain) {
            st_if(b, nv[f][g], oin);
            st_if(b + xo[g], nv[f][g], oin && xo[g] != 0);
          } else {
            put_images_pred(b, nv[f][g], oin, true, xo[g], yo, zo);
          }
        }
      if (do_mass && oin) {
#pragma unroll
        for (int g = 0; g < G; ++g) msum += vsum<T, 4>(nv[0][g], xl + 128 * g, p.n[0]);
      }
    }
    return !__syncthreads_or(bad);
  };

  // WARM warm-up iterations (staging only); one barrier per plane; the body
  // is unrolled over the three phases of the staged-operand queue
  int zi = zi0;
  bool failed = false;
  auto step = [&](auto phase_tag) -> bool {  // false: stop
    if (zi >= ze) return false;
    const int qn = zi + U + PD - (zb - R);
    if (tid == 0 && zi > zi0 && qn < nplanes) issue(qn);
    if (!body(phase_tag, zi)) {
      if (tid == 0) {
        atomicExch(p.err, KERR_TMA_TIMEOUT);
        tma::drain(bars, NSLOT, zi == zi0 ? 0 : zi + U - (zb - R),
                   min(zi == zi0 ? q0 + U + PD : qn, nplanes - 1));
      }
      failed = true;
      return false;
    }
    const int nx = po[NPW - 1] + PLANE == NSLOT * PLANE ? 0 : po[NPW - 1] + PLANE;
#pragma unroll
    for (int j = 0; j < NPW - 1; ++j) po[j] = po[j + 1];
    po[NPW - 1] = nx;
    if (++wslot == NSLOT) {
      wslot = 0;
      wph ^= 1u;
    }
    const int t = ow;
    ow = orr;
    orr = t;
#pragma unroll
    for (int f = 0; f < NF; ++f) oz[f] += p.plane;
    ++zi;
    return true;
  };
  while (step(std::integral_constant<int, 0>{}) && step(std::integral_constant<int, 1>{}) &&
         step(std::integral_constant<int, 2>{})) {
  }
  if (failed) return;
  if (p.partial) {
    const double s = block_sum<NT>(msum, red);
    if (tid == 0)
      p.partial[(size_t(blockIdx.z) * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
  }
}

template <class M, class KC>
__global__ void __launch_bounds__(KC::NT)
    k_row(const __grid_constant__ StepParams<float> p, const __grid_constant__ M m) {
  pdl_enter();
  row_step<M, KC>(p, m);
}
template <class M, class KC>
__global__ void __launch_bounds__(KC::NT, KC::MINB)
    k_row_occ(const __grid_constant__ StepParams<float> p, const __grid_constant__ M m) {
  pdl_enter();
  row_step<M, KC>(p, m);
}

}  // namespace sp
