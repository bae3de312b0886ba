/*
 * sp_chrow.cuh -- row kernel of the conserved-dynamics pattern (sp_ch.cuh)
 *
 *     d psi / dt = M * lap(mu),   mu = P(psi) - K * lap(psi)     (3D, 7-point lap)
 *
 * for grids whose x extent is one or two 128-site warp rows (n_x = 128 or 256)
 * and periodic in x -- the 256^3 model B configuration among them.  Every
 * site is evaluated with the operations of the generic fused kernel in the
 * same order (lap7, the pointwise sub-trees through the generic evaluator),
 * so this is one more tile shape of the same kernel key and gives the same
 * bits.
 *
 * What differs is the data movement.  A CTA owns whole x rows: warp yw holds
 * SPT consecutive mu rows, lane l the four-site chunks x = 128 g + 4 l .. + 3
 * (g < G = n_x / 128), so every shared- and global-memory access of a chunk is
 * contiguous across the warp.  The x neighbours of a row are exchanged by warp
 * shuffles (periodic: the row wraps around the warp), so no x halo is loaded,
 * staged or computed; the CTA's mu rows (YW * SPT of them) cover its TY output
 * rows and the rows above and below, so the mu ring of the tile kernels is
 * just two more rows of the same loop; the z neighbours of psi and mu live in
 * register queues.  Shared memory holds the TMA ring of psi planes
 * (n_x x (TY + 4) boxes, no x halo) and two mu planes, from which only the
 * rows at warp boundaries are read back, one iteration later, behind the
 * single barrier per plane.  Periodic images are stored as by the other
 * kernels, so the fields keep their halo for every other consumer.
 */
#pragma once

#include "sp_ch.cuh"

namespace sp {

// QP: keep psi at z - 1 .. z + 1 of the warp's rows in a register queue
// (else read them from the plane ring, which holds them anyway); MINB: CTAs
// per SM the register allocation must leave room for (1: no constraint beyond
// one CTA)
template <class M, int NXR_, int YW_, int SPT_, int PD_, bool QP_ = true, int MINB_ = 1>
struct ChRow {
  using T = float;
  static constexpr int NXR = NXR_, G = NXR_ / 128, YW = YW_, SPT = SPT_, PD = PD_;
  static constexpr bool QP = QP_;
  static constexpr int W = 4 * G;  // sites per lane and row
  static constexpr int NT = 32 * YW;
  static constexpr int MR = YW * SPT;  // mu rows per CTA: TY outputs and one above and below
  static constexpr int TY = MR - 2, TX = NXR;
  static constexpr int R = 2, RS = 1, RI = 1;
  static constexpr int PH = MR + 2;       // psi rows of a plane box (mu rows +- 1)
  static constexpr int PLANE = NXR * PH;  // elements; rows are whole 16-byte units
  static constexpr int NSLOT = 3 + PD;    // psi planes z .. z+2 read, PD in flight
  static constexpr int MPL = NXR * MR;    // one mu plane
  static constexpr size_t SMEM =
      256 + sizeof(T) * (size_t(NSLOT) * PLANE + 2 * size_t(MPL));
  // the field layout of the tile kernels of the same key (their x halo)
  static constexpr int HXA = HaloGeom<T, 2, R, 1, RS, RI>::HXA;
  static constexpr int MINB = MINB_;
  static_assert(MINB >= 1 && size_t(MINB) * (SMEM + 1024) <= 227 * 1024,
                "the CTAs asked for fit the shared memory of an SM");
  static_assert(NXR == 128 || NXR == 256, "rows of one warp, one or two chunks per lane");
  static_assert(TY >= 1 && SPT >= 1, "at least one output row");
  static_assert(NT <= 1024, "threads per CTA");
  static_assert(PH <= 256, "TMA box");
  static_assert(NSLOT <= 32, "barrier header");
  static_assert(ChPattern<M>::ok, "model is not of the conserved M lap(P - K lap) form");
  static_assert(M::R == R && M::RS == RS, "reach of the pattern");
};

template <class M, class KC>
__device__ __forceinline__ void chrow_step(const StepParams<float>& p, const M& m) {
  using T = float;
  using V = Vec<float, 4>;
  constexpr int NXR = KC::NXR, G = KC::G, SPT = KC::SPT, TY = KC::TY, PD = KC::PD,
                PLANE = KC::PLANE, NSLOT = KC::NSLOT, MPL = KC::MPL, R = KC::R, NT = KC::NT;
  constexpr bool QP = KC::QP;
  constexpr uint32_t TXB = uint32_t(PLANE * sizeof(T));
  constexpr unsigned FULL = 0xffffffffu;
  using RH = ChRhs<decltype(M::r0)>;
  using SG = ChStage<decltype(M::s0)>;

  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  T* fbuf = reinterpret_cast<T*>(smem_raw + 256);
  T* mbuf = fbuf + NSLOT * PLANE;  // two mu planes, written and read alternately
  __shared__ double red[32];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int xl = lane * 4;    // chunk g of this lane: sites xl + 128 g .. + 3
  const int m0 = warp * SPT;  // first mu row of this warp (y = y0 - 1 + m)
  const int y0 = blockIdx.x * TY;
  const int zb = blockIdx.y * p.zchunk;
  const int ze = min(zb + p.zchunk, p.n[2]);
  const CUtensorMap* map = p.maps + blockIdx.z;
  const int nplanes = (ze - 1 + R) - (zb - R) + 1;

  T coef[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) coef[i] = p.coef[i];
  PwCtx<T, 4> pc;
  pc.divh2 = V(p.divh2);
  pc.divh3 = V(p.divh3);
  pc.divh4 = V(p.divh4);
  pc.cf = coef;
  const V divh2(p.divh2), vdt(p.dt);
  const V m6divh2 = V(-6.0) * divh2;
  const V mob = eval(RH::mob(m.r0), pc);
  const V kap = eval(SG::kappa(m.s0), pc);

  // a row in registers: G chunks per lane; in shared memory: NXR elements
  auto ld_row = [&](const T* row, V (&v)[G]) {
#pragma unroll
    for (int g = 0; g < G; ++g) v[g] = *reinterpret_cast<const V*>(row + 128 * g + xl);
  };
  // lane-wise x pair sums (left + right neighbour of each site) of a row; the
  // row is periodic, so its ends wrap around the warp: with two chunks, lane
  // 0's chunk 0 continues lane 31's chunk 1 and lane 0's chunk 1 lane 31's
  // chunk 0
  auto xsum_row = [&](const V (&c)[G], V (&s)[G]) {
    const int lm = (lane + 31) & 31, lp = (lane + 1) & 31;
    T l[G], r[G];
    if constexpr (G == 1) {
      l[0] = __shfl_sync(FULL, c[0].v[3], lm);
      r[0] = __shfl_sync(FULL, c[0].v[0], lp);
    } else {
      const T a = __shfl_sync(FULL, c[0].v[3], lm), b = __shfl_sync(FULL, c[1].v[3], lm);
      const T a2 = __shfl_sync(FULL, c[0].v[0], lp), b2 = __shfl_sync(FULL, c[1].v[0], lp);
      l[0] = lane == 0 ? b : a;
      l[1] = lane == 0 ? a : b;
      r[0] = lane == 31 ? b2 : a2;
      r[1] = lane == 31 ? a2 : b2;
    }
    // scalar adds: the operand pairs straddle the lanes' register pairs
#pragma unroll
    for (int g = 0; g < G; ++g) {
      s[g].v[0] = l[g] + c[g].v[1];
      s[g].v[1] = c[g].v[0] + c[g].v[2];
      s[g].v[2] = c[g].v[1] + c[g].v[3];
      s[g].v[3] = c[g].v[2] + r[g];
    }
  };

  // output rows: mu row m0 + k is output row o = m0 + k - 1 when 0 <= o < TY;
  // their addresses, whether they exist and their y images are fixed for the CTA
  long long xo[G];
#pragma unroll
  for (int g = 0; g < G; ++g) xo[g] = image_offset(p.per[0], xl + 128 * g, 4, p.n[0], R, 1);
  const bool do_mass = p.partial != nullptr;
  T* orow[SPT];
  bool oin[SPT];
  long long yo[SPT];
  bool yimg = false;  // some row of this warp has a y image (warp-uniform)
#pragma unroll
  for (int k = 0; k < SPT; ++k) {
    const int o = m0 + k - 1, y = y0 + o;
    oin[k] = o >= 0 && o < TY && y < p.n[1];
    yo[k] = oin[k] ? image_offset(p.per[1], y, 1, p.n[1], R, p.pitch) : 0;
    yimg |= yo[k] != 0;
    orow[k] = p.out[blockIdx.z] + (long long)(y + p.h[1]) * p.pitch + (xl + p.h[0]);
  }

  if (tid == 0) {
    for (int s = 0; s < NSLOT; ++s) tma::mbar_init(&bars[s], 1);
    tma::fence_barrier_init();
  }
  __syncthreads();
  auto issue = [&](int q) {
    const int s = q % NSLOT;
    tma::mbar_arrive_expect_tx(&bars[s], TXB);
    tma::load_3d(fbuf + s * PLANE, map, &bars[s], p.h[0], y0 - R + p.h[1], zb - R + q + p.h[2]);
  };
  // plane sequence q(z) = z - (zb - R); iteration zi reads psi planes zi ..
  // zi + 2; the prologue fills every slot (planes q = 0 .. NSLOT - 1) and
  // iteration zi > zi0 issues q(zi + R + PD) = q(zi - 1) + NSLOT into the slot
  // of plane zi - 1, which the previous iteration read last, before its barrier
  const int zi0 = zb - 2;
  if (tid == 0) {
    const int pro = min(NSLOT, nplanes);
    for (int q = 0; q < pro; ++q) issue(q);
  }

  // register queues of this warp's mu rows, rotated by the phase (zi - zi0) % 3:
  // psi and mu at planes z - 1, z, z + 1 relative to the output plane
  V qpsi[QP ? 3 : 1][SPT][G], qmu[3][SPT][G];
  double msum = 0.0;
  // per-plane state, advanced by one plane per iteration (no divisions, no
  // recomputation from zi): psi planes zi .. zi + 2 in the ring, the mbarrier
  // slot and phase of plane zi + 2, the mu planes written and read, and this
  // thread's output rows in plane zi
  // (element offsets into the shared arrays, so every access stays a
  // shared-memory access with a base the compiler knows)
  int o0 = 0, o1 = PLANE, o2 = 2 * PLANE;  // psi planes zi, zi+1, zi+2
  int wslot = 2;
  uint32_t wph = 0;
  int ow = ((zi0 + 1) & 1) * MPL;  // mu(zi+1), written now
  int orr = (zi0 & 1) * MPL;       // mu(zi), written last iteration
  T* oz[SPT];
#pragma unroll
  for (int k = 0; k < SPT; ++k) oz[k] = orow[k] + (long long)(zi0 + p.h[2]) * p.plane;
  const bool rhs_only = p.rhs_only != 0;
  const bool zper = p.per[2] != 0;
  const int rows = m0 * NXR + xl;  // this warp's first mu row (psi box row m0 + 1)

  auto body = [&](auto phase_tag, int zi) -> bool {
    constexpr int P = decltype(phase_tag)::value;
    constexpr int IM = P % 3, IC = (P + 1) % 3, IP = (P + 2) % 3;
    bool bad = false;
    if (zi == zi0) {
      for (int q = 0; q <= 2; ++q) bad |= !tma::mbar_wait(&bars[q], 0);
    } else {
      bad = !tma::mbar_wait(&bars[wslot], wph);
    }
    // psi at z = zi - 1 + j (j = 0, 1, 2) of row k: the queue, or the ring;
    // psi box row b holds y = y0 - 2 + b: mu row m has its centre at b = m + 1
    V pz[3][SPT][G];
    const T* const f0 = fbuf + o0;
    const T* const f1 = fbuf + o1;
    const T* const f2 = fbuf + o2;
    T* const mw = mbuf + ow;
    const T* const mr = mbuf + orr;
    if constexpr (QP) {
      if (zi == zi0) {
#pragma unroll
        for (int k = 0; k < SPT; ++k) {
          ld_row(f0 + rows + (k + 1) * NXR - xl, qpsi[IM][k]);
          ld_row(f1 + rows + (k + 1) * NXR - xl, qpsi[IC][k]);
        }
      }
#pragma unroll
      for (int k = 0; k < SPT; ++k) ld_row(f2 + rows + (k + 1) * NXR - xl, qpsi[IP][k]);
#pragma unroll
      for (int k = 0; k < SPT; ++k)
#pragma unroll
        for (int g = 0; g < G; ++g) {
          pz[0][k][g] = qpsi[IM][k][g];
          pz[1][k][g] = qpsi[IC][k][g];
          pz[2][k][g] = qpsi[IP][k][g];
        }
    } else {
#pragma unroll
      for (int k = 0; k < SPT; ++k) {
        ld_row(f0 + rows + (k + 1) * NXR - xl, pz[0][k]);
        ld_row(f1 + rows + (k + 1) * NXR - xl, pz[1][k]);
        ld_row(f2 + rows + (k + 1) * NXR - xl, pz[2][k]);
      }
    }
    // ---- mu at zi + 1 on this warp's rows
    {
      V above[G], below[G];
      ld_row(f1 + rows - xl, above);
      ld_row(f1 + rows + (SPT + 1) * NXR - xl, below);
#pragma unroll
      for (int k = 0; k < SPT; ++k) {
        V sx[G];
        xsum_row(pz[1][k], sx);
#pragma unroll
        for (int g = 0; g < G; ++g) {
          const V c = pz[1][k][g];
          const V sy = (k == 0 ? above[g] : pz[1][k - 1][g]) +
                       (k == SPT - 1 ? below[g] : pz[1][k + 1][g]);
          const V sz = pz[0][k][g] + pz[2][k][g];
          const V l = lap7(sx[g], sy, sz, c, m6divh2, divh2);
          pc.psi = c;
          const V pw = eval(SG::pw(m.s0), pc);
          V mu;
          if constexpr (SG::has_k)
            mu = fmadd<true>(-kap, l, pw);
          else
            mu = pw - l;
          qmu[IP][k][g] = mu;
          *reinterpret_cast<V*>(mw + rows + k * NXR + 128 * g) = mu;
        }
      }
    }
    // ---- output at z = zi: psi + dt * M * lap(mu)
    if (zi >= zb) {
      // periodic z images only on the planes within R of a z face
      const bool zf = zper && (zi < R || zi >= p.n[2] - R);
      const long long zo = zf ? image_offset(1, zi, 1, p.n[2], R, p.plane) : 0;
      const bool plain = !zf && !yimg;  // warp-uniform
#pragma unroll
      for (int k = 0; k < SPT; ++k) {
        const int o = m0 + k - 1;  // warp-uniform
        if (o < 0 || o >= TY) continue;
        V sx[G], up[G], dn[G];
        xsum_row(qmu[IC][k], sx);
        if (k == 0) ld_row(mr + rows - NXR - xl, up);
        if (k == SPT - 1) ld_row(mr + rows + SPT * NXR - xl, dn);
#pragma unroll
        for (int g = 0; g < G; ++g) {
          const V sy = (k == 0 ? up[g] : qmu[IC][k - 1][g]) + (k == SPT - 1 ? dn[g] : qmu[IC][k + 1][g]);
          const V sz = qmu[IM][k][g] + qmu[IP][k][g];
          V r = lap7(sx[g], sy, sz, qmu[IC][k][g], m6divh2, divh2);
          if constexpr (RH::has_m) r = mob * r;
          const V nv = rhs_only ? r : fmadd<true>(vdt, r, pz[0][k][g]);
          T* const b = oz[k] + 128 * g;
          if (plain) {
            st_if(b, nv, oin[k]);
            st_if(b + xo[g], nv, oin[k] && xo[g] != 0);
          } else {
            put_images_pred(b, nv, oin[k], true, xo[g], yo[k], zo);
          }
          if (do_mass && oin[k]) msum += vsum<T, 4>(nv, xl + 128 * g, p.n[0]);
        }
      }
    }
    return !__syncthreads_or(bad);
  };

  // zi0, zi0 + 1 are warm-up iterations (mu only); one barrier per plane; the
  // body is unrolled over the three phases of the register queues
  int zi = zi0;
  bool failed = false;
  auto step = [&](auto phase_tag) -> bool {  // false: stop
    if (zi >= ze) return false;
    const int qn = zi + R + PD - (zb - R);
    if (tid == 0 && zi > zi0 && qn < nplanes) issue(qn);
    if (!body(phase_tag, zi)) {
      if (tid == 0) {
        atomicExch(p.err, KERR_TMA_TIMEOUT);
        tma::drain(bars, NSLOT, zi == zi0 ? 0 : zi + R - (zb - R),
                   min(zi == zi0 ? NSLOT - 1 : qn, nplanes - 1));
      }
      failed = true;
      return false;
    }
    o0 = o1;
    o1 = o2;
    o2 = o2 + PLANE == NSLOT * PLANE ? 0 : o2 + PLANE;
    if (++wslot == NSLOT) {
      wslot = 0;
      wph ^= 1u;
    }
    const int t = ow;
    ow = orr;
    orr = t;
#pragma unroll
    for (int k = 0; k < SPT; ++k) oz[k] += p.plane;
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

// the kernel, with the occupancy hint only for shapes that ask for more than
// one CTA per SM (a hint of one changes the compiler's register choices)
template <class M, class KC>
__global__ void __launch_bounds__(KC::NT)
    k_chrow(const __grid_constant__ StepParams<float> p, const __grid_constant__ M m) {
  pdl_enter();
  chrow_step<M, KC>(p, m);
}
template <class M, class KC>
__global__ void __launch_bounds__(KC::NT, KC::MINB)
    k_chrow_occ(const __grid_constant__ StepParams<float> p, const __grid_constant__ M m) {
  pdl_enter();
  chrow_step<M, KC>(p, m);
}

}  // namespace sp
