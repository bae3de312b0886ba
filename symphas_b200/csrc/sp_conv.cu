/*
 * sp_conv.cu -- the learned jump of the surrogate path: BF16 tensor-core
 * implicit-GEMM 3x3 convolutions with circular padding (NHWC activations),
 * their weight gradient, the weight flip that turns the data gradient into a
 * forward convolution, and the Adam update.  No counterpart in SymPhas; the
 * finite-difference solver stays the judge of every jump.
 *
 * Forward, as a GEMM: rows = pixels (n, y, x), columns = output channels,
 * K = 9 taps x Cin, tap-major; A[p][t*Cin + c] = x[n, (y+dy) mod H, (x+dx) mod W, c]
 * is gathered tile by tile (16-byte cp.async, the circular wrap in the
 * address), B = weights [Cout][9*Cin].  mma.sync m16n8k16 (bf16 in, fp32
 * accumulate), ldmatrix fragments, two-stage cp.async pipeline.  The epilogue
 * adds the bias and an optional residual, stores the pre-activation z and,
 * when asked, gelu(z) (tanh form), both in bf16.
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstdlib>
#include <type_traits>

#include "../../include/symphas_b200.h"

namespace sp {
namespace conv {

constexpr int BM = 128, BN = 64, BK = 32, NTH = 128;  // 4 warps: 2 (m) x 2 (n)
constexpr int SA = BK + 8;                            // padded smem row (bf16): 80 B

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool pred) {
  const int sz = pred ? 16 : 0;  // zero-fill when out of range
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)),
               "l"(src), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ void ldmatrix_x4(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldmatrix_x2(uint32_t (&r)[2], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n"
               : "=r"(r[0]), "=r"(r[1])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4],
                                         const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
// gelu, tanh form, with the hardware tanh (tanh.approx.f32, about 2^-11
// relative): the activations are stored in bf16 (2^-8), so the result is the
// same function to within storage rounding, for a fraction of the epilogue's
// instructions
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu(float z) {
  const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
  const float hz = 0.5f * z;
  return fmaf(hz, tanh_fast(u), hz);
}

struct FwdParams {
  const __nv_bfloat16* x;    // [N][H][W][Cin]
  const __nv_bfloat16* w;    // [Cout][9][Cin]
  const float* bias;         // [Cout] or null
  const __nv_bfloat16* res;  // [N][H][W][Cout] added before the activation, or null
  __nv_bfloat16* z;          // pre-activation out [N][H][W][Cout], or null
  __nv_bfloat16* a;          // gelu(z) out, or null
  int n, h, wid, cin, cout;
};

// one CTA: 128 pixels x 64 output channels
__global__ void __launch_bounds__(NTH) k_conv3x3_fwd(const FwdParams p) {
  __shared__ __align__(128) __nv_bfloat16 sa[2][BM][SA];
  __shared__ __align__(128) __nv_bfloat16 sb[2][BN][SA];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = warp >> 1, wn = warp & 1;  // warp tile 64 x 32
  const long long npix = (long long)p.n * p.h * p.wid;
  const long long p0 = (long long)blockIdx.x * BM;
  const int co0 = blockIdx.y * BN;
  const int kchunks = p.cin / BK;  // per tap
  const int nk = 9 * kchunks;

  // each thread loads 4 16-byte chunks of A (128 rows x 4 chunks) and 2 of B
  // (64 rows x 4 chunks) per K step; the pixel coordinates of its A rows
  int arow[4], ay[4], ax[4];
  long long abase[4];
  bool aok[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = (tid + i * NTH) >> 2;
    arow[i] = r;
    const long long pix = p0 + r;
    aok[i] = pix < npix;
    const long long pp = aok[i] ? pix : 0;
    const int xx = int(pp % p.wid);
    const int yy = int((pp / p.wid) % p.h);
    const long long nn = pp / ((long long)p.wid * p.h);
    ax[i] = xx;
    ay[i] = yy;
    abase[i] = nn * p.h * p.wid;
  }
  auto load = [&](int stage, int kstep) {
    const int tap = kstep / kchunks, c0 = (kstep % kchunks) * BK;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int chunk = (tid + i * NTH) & 3;
      int yy = ay[i] + dy, xx = ax[i] + dx;
      yy += (yy < 0) ? p.h : 0;
      yy -= (yy >= p.h) ? p.h : 0;
      xx += (xx < 0) ? p.wid : 0;
      xx -= (xx >= p.wid) ? p.wid : 0;
      const __nv_bfloat16* src =
          p.x + ((abase[i] + (long long)yy * p.wid + xx) * p.cin + c0 + chunk * 8);
      cp_async16(&sa[stage][arow[i]][chunk * 8], src, aok[i]);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int r = (tid + i * NTH) >> 2, chunk = (tid + i * NTH) & 3;
      const int co = co0 + r;
      const bool ok = co < p.cout;
      const __nv_bfloat16* src = p.w + ((long long)(ok ? co : 0) * 9 * p.cin + tap * p.cin + c0 +
                                        chunk * 8);
      cp_async16(&sb[stage][r][chunk * 8], src, ok);
    }
    cp_async_commit();
  };

  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.f;

  load(0, 0);
  for (int ks = 0; ks < nk; ++ks) {
    const int st = ks & 1;
    if (ks + 1 < nk) {
      load(st ^ 1, ks + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      uint32_t af[4][4], bf[4][2];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = wm * 64 + i * 16 + (lane & 15);
        const int c = kk + (lane >> 4) * 8;
        ldmatrix_x4(af[i], &sa[st][r][c]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int r = wn * 32 + j * 8 + (lane & 7);
        const int c = kk + ((lane >> 3) & 1) * 8;
        ldmatrix_x2(bf[j], &sb[st][r][c]);
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma16816(acc[i][j], af[i], bf[j]);
    }
    __syncthreads();
  }

  // epilogue: fragment element e of tile (i, j) is row wm*64 + i*16 + lane/4
  // (+8 for e >= 2), column wn*32 + j*8 + (lane%4)*2 (+1 for odd e)
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const long long pix = p0 + wm * 64 + i * 16 + (lane >> 2) + half * 8;
      if (pix >= npix) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int co = co0 + wn * 32 + j * 8 + (lane & 3) * 2;
        if (co >= p.cout) continue;
        float v0 = acc[i][j][half * 2], v1 = acc[i][j][half * 2 + 1];
        if (p.bias) {
          v0 += p.bias[co];
          v1 += p.bias[co + 1];
        }
        const long long o = pix * p.cout + co;
        if (p.res) {
          const __nv_bfloat162 r = *reinterpret_cast<const __nv_bfloat162*>(p.res + o);
          v0 += __bfloat162float(r.x);
          v1 += __bfloat162float(r.y);
        }
        if (p.z) *reinterpret_cast<__nv_bfloat162*>(p.z + o) = __floats2bfloat162_rn(v0, v1);
        if (p.a)
          *reinterpret_cast<__nv_bfloat162*>(p.a + o) = __floats2bfloat162_rn(gelu(v0), gelu(v1));
      }
    }
}

}  // namespace conv
}  // namespace sp

namespace sp {
namespace conv {

__device__ __forceinline__ void ldmatrix_x4_t(uint32_t (&r)[4], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldmatrix_x2_t(uint32_t (&r)[2], const void* p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
               : "=r"(r[0]), "=r"(r[1])
               : "r"(smem_u32(p)));
}

// Weight gradient dw[co][t][c] += sum over pixels p of dy[p][co] * x[p + d_t][c],
// as a GEMM with rows (t, c) (a 32-channel block of one tap per CTA), columns
// co (64 per CTA) and K = pixels; each CTA sums `chunk` pixels and adds its
// fp32 tile into dw with atomics (split K).  Both operands are stored with
// the pixel (K) index outer, so their fragments come from ldmatrix.trans.
constexpr int WM = 32, WN = 64, WK = 32, WTH = 128;  // 4 warps along columns
constexpr int WSX = WM + 8, WSD = WN + 8;             // padded smem rows (bf16)

struct WgradParams {
  const __nv_bfloat16* x;   // [N][H][W][Cin]
  const __nv_bfloat16* dy;  // [N][H][W][Cout]
  float* dw;                // [Cout][9][Cin], accumulated
  int n, h, wid, cin, cout;
  long long chunk;          // pixels per CTA (multiple of WK)
};

__global__ void __launch_bounds__(WTH) k_conv3x3_wgrad(const WgradParams p) {
  __shared__ __align__(128) __nv_bfloat16 sx[2][WK][WSX];
  __shared__ __align__(128) __nv_bfloat16 sd[2][WK][WSD];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cblocks = p.cin / WM;
  const int tap = blockIdx.x / cblocks, c0 = (blockIdx.x % cblocks) * WM;
  const int dy_ = tap / 3 - 1, dx_ = tap % 3 - 1;
  const int co0 = blockIdx.y * WN;
  const long long npix = (long long)p.n * p.h * p.wid;
  const long long pb = (long long)blockIdx.z * p.chunk;
  const long long pe = pb + p.chunk < npix ? pb + p.chunk : npix;
  if (pb >= pe) return;
  const int nk = int((pe - pb + WK - 1) / WK);

  auto load = [&](int st, int ks) {
    const long long q0 = pb + (long long)ks * WK;
    {  // x: 32 pixels x 32 channels = 128 chunks of 16 B, one per thread
      const int r = tid >> 2, ch = tid & 3;
      const long long pix = q0 + r;
      const bool ok = pix < pe;
      // 32-bit division: the host keeps the pixel count below 2^31
      const uint32_t pp = uint32_t(ok ? pix : pb), t1 = pp / uint32_t(p.wid);
      const uint32_t nn32 = t1 / uint32_t(p.h);
      const int xx0 = int(pp - t1 * uint32_t(p.wid)), yy0 = int(t1 - nn32 * uint32_t(p.h));
      const long long nn = nn32;
      int yy = yy0 + dy_, xx = xx0 + dx_;
      yy += (yy < 0) ? p.h : 0;
      yy -= (yy >= p.h) ? p.h : 0;
      xx += (xx < 0) ? p.wid : 0;
      xx -= (xx >= p.wid) ? p.wid : 0;
      const __nv_bfloat16* src = p.x + (((nn * p.h + yy) * p.wid + xx) * p.cin + c0 + ch * 8);
      cp_async16(&sx[st][r][ch * 8], src, ok);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {  // dy: 32 pixels x 64 channels = 256 chunks
      const int idx = tid + i * WTH, r = idx >> 3, ch = idx & 7;
      const long long pix = q0 + r;
      const int co = co0 + ch * 8;
      const bool ok = pix < pe && co < p.cout;
      const __nv_bfloat16* src = p.dy + ((ok ? pix : pb) * p.cout + (ok ? co : 0));
      cp_async16(&sd[st][r][ch * 8], src, ok);
    }
    cp_async_commit();
  };

  float acc[2][2][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.f;

  load(0, 0);
  for (int ks = 0; ks < nk; ++ks) {
    const int st = ks & 1;
    if (ks + 1 < nk) {
      load(st ^ 1, ks + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < WK; kk += 16) {
      uint32_t af[2][4], bf[2][2];
      const int q = lane >> 3;
#pragma unroll
      for (int i = 0; i < 2; ++i)  // rows (channels) i*16 .. +15
        ldmatrix_x4_t(af[i], &sx[st][kk + (lane & 7) + (q >> 1) * 8][i * 16 + (q & 1) * 8]);
#pragma unroll
      for (int j = 0; j < 2; ++j)  // columns warp*16 + j*8 .. +7
        ldmatrix_x2_t(bf[j], &sd[st][kk + (lane & 7) + ((lane >> 3) & 1) * 8][warp * 16 + j * 8]);
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) mma16816(acc[i][j], af[i], bf[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int c = c0 + i * 16 + (lane >> 2) + half * 8;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int co = co0 + warp * 16 + j * 8 + (lane & 3) * 2;
        if (co >= p.cout) continue;
        float* d = p.dw + ((long long)co * 9 + tap) * p.cin + c;
        atomicAdd(d, acc[i][j][half * 2]);
        atomicAdd(d + 9LL * p.cin, acc[i][j][half * 2 + 1]);
      }
    }
}

// wf[c][t][co] = w[co][8 - t][c]: the forward weights of the data gradient
// x [pixel][c] = (bf16(psi[pixel]), 0, ..., 0): the network's input channels,
// one 16-byte store per thread and 8 channels
__global__ void k_embed0(const float* __restrict__ psi, __nv_bfloat16* __restrict__ x, int c8,
                         long long total) {
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const long long pix = id / c8;
    const int cc = int(id - pix * c8);
    __align__(16) __nv_bfloat16 v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = __float2bfloat16_rn(0.f);
    if (cc == 0) v[0] = __float2bfloat16_rn(psi[pix]);
    *reinterpret_cast<uint4*>(x + id * 8) = *reinterpret_cast<const uint4*>(v);
  }
}

// 2x2 average pooling of [N][H][W][C] bf16 (channels last): one thread per
// output pixel and 8 channels (16 bytes from each of the four inputs), the
// four values summed in fp32 row by row and scaled by 1/4
__global__ void k_avgpool2(const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ y,
                           int n, int h, int w, int c, long long total) {
  const int c8 = c / 8, wo = w / 2, ho = h / 2;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int cc = int(id % c8);
    const long long pix = id / c8;
    const int xo = int(pix % wo);
    const long long t = pix / wo;
    const int yo = int(t % ho);
    const long long nn = t / ho;
    const long long r0 = ((nn * h + 2 * yo) * w + 2 * xo) * c + cc * 8, r1 = r0 + (long long)w * c;
    const uint4 a = *reinterpret_cast<const uint4*>(x + r0);
    const uint4 b = *reinterpret_cast<const uint4*>(x + r0 + c);
    const uint4 d = *reinterpret_cast<const uint4*>(x + r1);
    const uint4 e = *reinterpret_cast<const uint4*>(x + r1 + c);
    const __nv_bfloat162* pa = reinterpret_cast<const __nv_bfloat162*>(&a);
    const __nv_bfloat162* pb = reinterpret_cast<const __nv_bfloat162*>(&b);
    const __nv_bfloat162* pd = reinterpret_cast<const __nv_bfloat162*>(&d);
    const __nv_bfloat162* pe = reinterpret_cast<const __nv_bfloat162*>(&e);
    __align__(16) __nv_bfloat162 o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 fa = __bfloat1622float2(pa[k]), fb = __bfloat1622float2(pb[k]);
      const float2 fd = __bfloat1622float2(pd[k]), fe = __bfloat1622float2(pe[k]);
      o[k] = __floats2bfloat162_rn((((fa.x + fb.x) + fd.x) + fe.x) * 0.25f,
                                   (((fa.y + fb.y) + fd.y) + fe.y) * 0.25f);
    }
    *reinterpret_cast<uint4*>(y + ((nn * ho + yo) * wo + xo) * c + cc * 8) =
        *reinterpret_cast<const uint4*>(o);
  }
}

__global__ void k_conv3x3_flip(const __nv_bfloat16* w, __nv_bfloat16* wf, int cin, int cout) {
  const long long total = 9LL * cin * cout;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int co = int(id % cout), t = int((id / cout) % 9);
    const long long c = id / (9LL * cout);
    wf[(c * 9 + t) * cout + co] = w[((long long)co * 9 + (8 - t)) * cin + c];
  }
}

// Adam (bias-corrected), fp32 master weights, bf16 copy for the convolutions
__global__ void k_adam(float* w, __nv_bfloat16* wb, const float* g, float* m, float* v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2,
                       float wd) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * w[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

int sms() {
  static int n = [] {
    int dev = 0, v = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
  }();
  return n;
}

}  // namespace conv
}  // namespace sp

extern "C" {

int sp_conv3x3_fwd(const void* x, const void* w, const float* bias, const void* res, void* z,
                   void* a, int n, int h, int w_, int cin, int cout, void* stream) {
  using namespace sp::conv;
  if (!x || !w || (!z && !a) || n < 1 || h < 1 || w_ < 1 || cin % BK != 0 || cout % 2 != 0 ||
      cout < 2)
    return SP_EINVAL;
  FwdParams p{static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(w), bias,
              static_cast<const __nv_bfloat16*>(res), static_cast<__nv_bfloat16*>(z),
              static_cast<__nv_bfloat16*>(a), n, h, w_, cin, cout};
  const long long npix = (long long)n * h * w_;
  dim3 grid(unsigned((npix + BM - 1) / BM), unsigned((cout + BN - 1) / BN));
  k_conv3x3_fwd<<<grid, NTH, 0, static_cast<cudaStream_t>(stream)>>>(p);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ECUDA;
}

int sp_conv3x3_wgrad(const void* x, const void* dy, float* dw, int n, int h, int w_, int cin,
                     int cout, void* stream) {
  using namespace sp::conv;
  if (!x || !dy || !dw || n < 1 || h < 1 || w_ < 1 || cin % WM != 0 || cout % 8 != 0)
    return SP_EINVAL;
  const long long npix = (long long)n * h * w_;
  if (npix >= (1LL << 31)) return SP_EINVAL;  // the kernel's pixel arithmetic is 32-bit
  const unsigned gx = unsigned(9 * (cin / WM)), gy = unsigned((cout + WN - 1) / WN);
  // enough pixel chunks for about four waves of CTAs
  long long want = (long long)sms() * 8 / (gx * gy);
  if (want < 1) want = 1;
  long long chunk = (npix + want - 1) / want;
  chunk = ((chunk + WK - 1) / WK) * WK;
  if (chunk < 1024) chunk = 1024;
  const unsigned gz = unsigned((npix + chunk - 1) / chunk);
  WgradParams p{static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(dy), dw,
                n, h, w_, cin, cout, chunk};
  k_conv3x3_wgrad<<<dim3(gx, gy, gz), WTH, 0, static_cast<cudaStream_t>(stream)>>>(p);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ECUDA;
}

int sp_embed_channel0_bf16(const float* psi, void* x, long long npix, int c, void* stream) {
  if (!psi || !x || npix < 1 || c < 8 || c % 8) return SP_EINVAL;
  if (reinterpret_cast<uintptr_t>(x) % 16 != 0) return SP_EINVAL;  // 16-byte stores
  const long long total = npix * (c / 8);
  const int blocks = int(total / 256 + 1 < 148LL * 16 ? total / 256 + 1 : 148LL * 16);
  sp::conv::k_embed0<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      psi, static_cast<__nv_bfloat16*>(x), c / 8, total);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ECUDA;
}

int sp_avgpool2_bf16(const void* x, void* y, int n, int h, int w_, int c, void* stream) {
  if (!x || !y || n < 1 || h < 2 || w_ < 2 || h % 2 || w_ % 2 || c < 8 || c % 8) return SP_EINVAL;
  if (reinterpret_cast<uintptr_t>(x) % 16 != 0 || reinterpret_cast<uintptr_t>(y) % 16 != 0)
    return SP_EINVAL;  // 16-byte loads and stores
  const long long total = (long long)n * (h / 2) * (w_ / 2) * (c / 8);
  const int blocks = int(total / 256 + 1 < 148LL * 16 ? total / 256 + 1 : 148LL * 16);
  sp::conv::k_avgpool2<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(x), static_cast<__nv_bfloat16*>(y), n, h, w_, c, total);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ECUDA;
}

int sp_conv3x3_flip(const void* w, void* wf, int cin, int cout, void* stream) {
  if (!w || !wf || cin < 1 || cout < 1) return SP_EINVAL;
  sp::conv::k_conv3x3_flip<<<256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(w), static_cast<__nv_bfloat16*>(wf), cin, cout);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ECUDA;
}

int sp_adam_step(float* w, void* wb, const float* g, float* m, float* v, long long n, float lr,
                 float b1, float b2, float eps, int step, float weight_decay, void* stream) {
  if (!w || !g || !m || !v || n < 1 || step < 1) return SP_EINVAL;
  const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
  const int blocks = int((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024);
  sp::conv::k_adam<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      w, static_cast<__nv_bfloat16*>(wb), g, m, v, n, lr, b1, b2, eps, c1, c2, weight_decay);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ECUDA;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The forward convolution on the 5th-generation tensor cores (tcgen05): the
// same implicit GEMM, a 128-pixel x BN-channel tile per CTA with its fp32
// accumulator in tensor memory.  Operands are gathered by cp.async (the
// circular wrap in the address) into shared memory in the K-major canonical
// layout without swizzle -- 8-row x 16-byte core matrices, K-adjacent core
// matrices 128 B apart (leading byte offset), row-adjacent ones 1 KiB apart
// (stride byte offset) -- in a ring of stages with a full and an empty
// mbarrier each; one thread issues the MMAs (M = 128, N = BN, K = 16 each,
// bf16 x bf16 -> fp32) of a stage once its copies have landed and commits
// them to the stage's empty barrier, whose (bounded) wait releases the stage
// to the producers.  Four warps read the accumulator back with tcgen05.ld for
// the epilogue.  The descriptor fields follow the PTX ISA's shared-memory and
// instruction descriptors for tcgen05.mma (as CUTLASS's cute/arch headers
// spell them out).
// ---------------------------------------------------------------------------
#include "sp_tma.cuh"

namespace sp {
namespace conv {

constexpr int TC_BM = 128, TC_BK = 64;

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
  // K-major, no swizzle: start >> 4, LBO = 128 B, SBO = 1024 B, version 1
  return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t(128 >> 4) << 16) |
         (uint64_t(1024 >> 4) << 32) | (uint64_t(1) << 46);
}

template <int BN>
__device__ __forceinline__ constexpr uint32_t umma_idesc() {
  // D fp32, A and B bf16, both K-major, N >> 3, M >> 4
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(BN >> 3) << 17) |
         (uint32_t(TC_BM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(addr));
}

template <int BN>
struct TcTile {
  // stages per CTA: about 100 KB of ring, so that two CTAs share an SM (one's
  // epilogue overlaps the other's main loop)
  static constexpr int S = BN == 32 ? 5 : BN == 64 ? 4 : 3;
  static constexpr int A_BYTES = TC_BM * TC_BK * 2, B_BYTES = BN * TC_BK * 2;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int NBAR = 2 * S + 1;  // full[S], empty[S], done
  static constexpr int SMEM = S * STAGE + NBAR * 8 + 16;
  static constexpr int COLS = BN;  // TMEM columns (a power of two >= 32)
};

// Warp roles (160 threads): warps 0-3 gather the operands of each K step
// (64 taps x channels) into the stage ring, arriving on full[s] as their
// copies land (cp.async.mbarrier.arrive.noinc), and after the main loop read
// the accumulator back (warp w: TMEM lanes 32w..32w+31 = pixels) for the
// epilogue; warp 4 allocates the tensor memory and one of its threads issues
// the MMAs of each stage once full[s] completes, committing to empty[s] (the
// stage may be refilled) and, after the last, to done.
template <int BN>
__global__ void __launch_bounds__(160) k_conv3x3_fwd_tc(const FwdParams p, int* err) {
  using TT = TcTile<BN>;
  constexpr int S = TT::S;
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * TT::STAGE);
  uint64_t* empty = full + S;
  uint64_t* done = empty + S;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long npix = (long long)p.n * p.h * p.wid;
  const long long p0 = (long long)blockIdx.x * TC_BM;
  const int co0 = blockIdx.y * BN;
  const int K = 9 * p.cin, nk = (K + TC_BK - 1) / TC_BK;

  if (warp == 4) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TT::COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      tma::mbar_init(&full[s], 128);
      tma::mbar_init(&empty[s], 1);
    }
    tma::mbar_init(done, 1);
    tma::fence_barrier_init();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  bool bad = false;

  if (warp < 4) {
    // producer: this thread's k chunk (8 channels) j of every K step, its 8
    // pixel rows tid / 8 + 16 i of A and BN / 16 channel rows of B
    const int j = tid & 7;
    int ry[8], rx[8];
    long long rbase[8];
    bool rok[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const long long pix = p0 + (tid >> 3) + 16 * i;
      rok[i] = pix < npix;
      const long long pp = rok[i] ? pix : 0;
      rx[i] = int(pp % p.wid);
      ry[i] = int((pp / p.wid) % p.h);
      rbase[i] = (pp / ((long long)p.wid * p.h)) * p.h * p.wid;
    }
    for (int ks = 0; ks < nk; ++ks) {
      const int s = ks % S;
      if (ks >= S) bad |= !tma::mbar_wait(&empty[s], uint32_t((ks / S - 1) & 1));
      unsigned char* sa = smem + s * TT::STAGE;
      unsigned char* sb = sa + TT::A_BYTES;
      const int k = ks * TC_BK + j * 8;
      const bool kok = k < K;
      const int tap = kok ? k / p.cin : 0, c = kok ? k - tap * p.cin : 0;
      const int dy = tap / 3 - 1, dx = tap % 3 - 1;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int r = (tid >> 3) + 16 * i;
        int yy = ry[i] + dy, xx = rx[i] + dx;
        yy += (yy < 0) ? p.h : 0;
        yy -= (yy >= p.h) ? p.h : 0;
        xx += (xx < 0) ? p.wid : 0;
        xx -= (xx >= p.wid) ? p.wid : 0;
        const __nv_bfloat16* src = p.x + ((rbase[i] + (long long)yy * p.wid + xx) * p.cin + c);
        cp_async16(sa + (r >> 3) * 1024 + j * 128 + (r & 7) * 16, src, rok[i] && kok);
      }
#pragma unroll
      for (int i = 0; i < BN / 16; ++i) {
        const int r = (tid >> 3) + 16 * i;
        const __nv_bfloat16* src = p.w + ((long long)(co0 + r) * K + (kok ? k : 0));
        cp_async16(sb + (r >> 3) * 1024 + j * 128 + (r & 7) * 16, src, kok);
      }
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(
                       smem_u32(&full[s]))
                   : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");

    // epilogue: accumulator rows (pixels) 32 warp .. 32 warp + 31
    bad |= !tma::mbar_wait(done, 0);
    __syncwarp();  // tcgen05.ld is warp-collective
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const long long pix = p0 + 32 * warp + lane;
#pragma unroll
    for (int c16 = 0; c16 < BN / 16; ++c16) {
      uint32_t v[16];
      tmem_ld16(tmem + (uint32_t(32 * warp) << 16) + uint32_t(c16 * 16), v);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (pix < npix && !bad) {
        const int cob = co0 + c16 * 16;
        const long long o = pix * p.cout + cob;
        __align__(16) __nv_bfloat162 zz[8], aa[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          float v0 = __uint_as_float(v[2 * e]), v1 = __uint_as_float(v[2 * e + 1]);
          if (p.bias) {
            v0 += p.bias[cob + 2 * e];
            v1 += p.bias[cob + 2 * e + 1];
          }
          if (p.res) {
            const __nv_bfloat162 r = *reinterpret_cast<const __nv_bfloat162*>(p.res + o + 2 * e);
            v0 += __bfloat162float(r.x);
            v1 += __bfloat162float(r.y);
          }
          zz[e] = __floats2bfloat162_rn(v0, v1);
          if (p.a) aa[e] = __floats2bfloat162_rn(gelu(v0), gelu(v1));
        }
        if (p.z) {
          reinterpret_cast<uint4*>(p.z + o)[0] = reinterpret_cast<const uint4*>(zz)[0];
          reinterpret_cast<uint4*>(p.z + o)[1] = reinterpret_cast<const uint4*>(zz)[1];
        }
        if (p.a) {
          reinterpret_cast<uint4*>(p.a + o)[0] = reinterpret_cast<const uint4*>(aa)[0];
          reinterpret_cast<uint4*>(p.a + o)[1] = reinterpret_cast<const uint4*>(aa)[1];
        }
      }
    }
  } else if (lane == 0) {
    // MMA issuer
    constexpr uint32_t idesc = umma_idesc<BN>();
    for (int ks = 0; ks < nk; ++ks) {
      const int s = ks % S;
      bad |= !tma::mbar_wait(&full[s], uint32_t((ks / S) & 1));
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(smem + s * TT::STAGE);
      const uint32_t b0 = a0 + TT::A_BYTES;
#pragma unroll
      for (int kk = 0; kk < TC_BK / 16; ++kk)
        umma_bf16(tmem, umma_desc(a0 + kk * 256), umma_desc(b0 + kk * 256), idesc,
                  (ks > 0 || kk > 0) ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    umma_commit(done);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 4)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TT::COLS));
  if (bad) atomicExch(err, 1);
}

// device flag set by a tcgen05 CTA that gave up on a wait (allocated once)
int* tc_error_flag() {
  static int* e = [] {
    int* f = nullptr;
    if (cudaMalloc(&f, sizeof(int)) != cudaSuccess) return static_cast<int*>(nullptr);
    cudaMemset(f, 0, sizeof(int));
    return f;
  }();
  return e;
}

}  // namespace conv
}  // namespace sp

extern "C" int sp_conv_tc_status(int* gave_up) {
  int* err = sp::conv::tc_error_flag();
  if (!err || !gave_up) return SP_EINVAL;
  if (cudaDeviceSynchronize() != cudaSuccess) return SP_ECUDA;
  if (cudaMemcpy(gave_up, err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    return SP_ECUDA;
  return cudaMemset(err, 0, sizeof(int)) == cudaSuccess ? SP_OK : SP_ECUDA;
}

namespace sp {
namespace conv {
template <int BN>
int launch_fwd_tc(const FwdParams& p, int* err, cudaStream_t s) {
  static const cudaError_t attr = cudaFuncSetAttribute(
      k_conv3x3_fwd_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcTile<BN>::SMEM);
  if (attr != cudaSuccess) return SP_ECUDA;
  const long long npix = (long long)p.n * p.h * p.wid;
  k_conv3x3_fwd_tc<BN><<<dim3(unsigned((npix + TC_BM - 1) / TC_BM), unsigned(p.cout / BN)), 160,
                         TcTile<BN>::SMEM, s>>>(p, err);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ECUDA;
}
}  // namespace conv
}  // namespace sp

extern "C" int sp_conv3x3_fwd_tc(const void* x, const void* w, const float* bias, const void* res,
                                 void* z, void* a, int n, int h, int w_, int cin, int cout,
                                 void* stream) {
  using namespace sp::conv;
  if (!x || !w || (!z && !a) || n < 1 || h < 1 || w_ < 1 || cin % 8 != 0 || cin < 8 ||
      !(cout == 32 || cout % 64 == 0))
    return SP_EINVAL;
  int* err = tc_error_flag();
  if (!err) return SP_ENOMEM;
  FwdParams p{static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(w), bias,
              static_cast<const __nv_bfloat16*>(res), static_cast<__nv_bfloat16*>(z),
              static_cast<__nv_bfloat16*>(a), n, h, w_, cin, cout};
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cout == 32) return launch_fwd_tc<32>(p, err, s);
  if (cout % 128 == 0) return launch_fwd_tc<128>(p, err, s);
  return launch_fwd_tc<64>(p, err, s);
}

// ---------------------------------------------------------------------------
// The forward convolution on tcgen05 with every input pixel gathered once.
//
// The input is staged as a strip of the PADDED position space: position
// Q = (n (H + 2) + y + 1) (W + 2) + x + 1 holds pixel (n, y mod H, x mod W)
// (circular padding), so a 3x3 tap (dy, dx) is the constant offset
// dy (W + 2) + dx between positions.  In shared memory the strip is
// chunk-major: for each 8-channel chunk, one 16-byte row per position.  In the
// K-major canonical layout without swizzle that is a stack of 8-row x 16-byte
// core matrices, 128 B apart along M (SBO) and P x 16 B apart along K (LBO,
// P = positions in the strip); the A operand of tap t is then the same strip
// with its start address moved by 16 x offset(t) bytes.  Each input value is
// copied into shared memory once per channel block instead of nine times.
//
// A CTA owns MT = 4 M-tiles of 128 consecutive padded positions (halo
// positions compute values nobody stores) and BN output channels; its fp32
// accumulators (MT x BN columns) sit in tensor memory.  K runs over channel
// blocks of CB input channels (stages): per stage the producers (warps 0-7)
// gather the strip with 16-byte cp.async, one of them loads the stage's
// pre-tiled weights with one bulk copy; one thread of warp 8 issues the
// 9 x CB/16 x MT MMAs (M 128, N BN, K 16) and commits them to the stage's
// empty barrier.  After the last stage warps 0-7 read the accumulators back
// (tcgen05.ld) for the bias / residual / GELU epilogue.
// ---------------------------------------------------------------------------
namespace sp {
namespace conv {

struct StripParams {
  const __nv_bfloat16* x;    // [N][H][W][Cin]
  const __nv_bfloat16* wt;   // weights tiled for the stages (k_tile_weights)
  const float* bias;         // [Cout] or null
  const __nv_bfloat16* res;  // [N][H][W][Cout] or null
  __nv_bfloat16* z;          // pre-activation out, or null
  __nv_bfloat16* a;          // gelu(z) out, or null
  int n, h, wid, cin, cout;
  int P;                     // positions of the strip (multiple of 8)
  int S;                     // stages in the ring
  int up;                    // 1: x is [N][H/2][W/2][Cin], read nearest-up-sampled
};

constexpr int ST_NPROD = 256, ST_NT = ST_NPROD + 32;
constexpr int ST_NPI = 8;  // strip positions per producer thread, at most

// BN output channels x MT 128-position M-tiles per CTA, CB input channels per
// K block
template <int BN, int CB, int MT>
struct StripTile {
  static constexpr int CH = CB / 8;
  static constexpr int B_BYTES = BN * 9 * CB * 2;
  static constexpr int M = MT * 128;       // output positions per CTA
  static constexpr int COLS = MT * BN;     // tensor-memory columns: a power of two
  static_assert(COLS == 64 || COLS == 128 || COLS == 256 || COLS == 512, "tensor memory columns");
  static_assert(CB % 16 == 0 && BN % 16 == 0 && BN <= 128, "tile");
  static_assert(MT == 2 || MT == 4, "two or four M-tiles: the epilogue's warps take every other one");
};

// wt, per (output block of BN channels, input block of CB channels), in the
// K-major canonical layout the MMA reads: [n group of 8 channels][K chunk
// (tap-major, 8 input channels)][8 rows x 16 B]
__global__ void k_tile_weights(const __nv_bfloat16* w, __nv_bfloat16* wt, int cin, int cout,
                               int bn, int cb) {
  const long long total = 9LL * cin * cout;
  const int nkb = cin / cb, kch = 9 * cb / 8;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
       id += (long long)gridDim.x * blockDim.x) {
    const int ci = int(id % cin), t = int((id / cin) % 9), co = int(id / (9LL * cin));
    const int cob = co / bn, g = (co % bn) / 8, r = co % 8;
    const int kb = ci / cb, j = (ci % cb) / 8, e = ci % 8;
    const int kc = t * (cb / 8) + j;
    const long long blk = (long long)(cob * nkb + kb) * bn * 9 * cb;
    wt[blk + ((long long)g * kch + kc) * 64 + r * 8 + e] = w[id];
  }
}

__device__ __forceinline__ uint64_t umma_desc_k(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  // K-major, no swizzle: start, leading (K) and stride (M/N) byte offsets, >> 4
  return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46);
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

template <int BN, int CB, int MT>
__global__ void __launch_bounds__(ST_NT) k_conv3x3_strip(const StripParams p, int* err) {
  using TT = StripTile<BN, CB, MT>;
  constexpr int ST_MT = MT, ST_M = TT::M;
  constexpr int CH = TT::CH;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int S = p.S, P = p.P;
  const int A_BYTES = CH * P * 16;
  const int STAGE = A_BYTES + TT::B_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * STAGE);
  uint64_t* empty = full + S;
  uint64_t* done = empty + S;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int W2 = p.wid + 2, H2 = p.h + 2;
  const long long HW2 = (long long)W2 * H2, QN = HW2 * p.n;
  const uint32_t W2u = uint32_t(W2), HW2u = uint32_t(HW2);
  const long long Q0 = (long long)blockIdx.x * ST_M;  // first output position
  const long long S0 = Q0 - (W2 + 1);                 // first strip position
  const int co0 = blockIdx.y * BN;
  const int nk = p.cin / CB;

  if (warp == 8) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TT::COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      tma::mbar_init(&full[s], ST_NPROD + 1);
      tma::mbar_init(&empty[s], 1);
    }
    tma::mbar_init(done, 1);
    tma::fence_barrier_init();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  bool bad = false;

  if (warp < 8) {
    // producer: strip positions tid + 256 i; the element offset of each
    // position's pixel (channel 0), or -1 for zeros (outside the batch)
    int off[ST_NPI];
#pragma unroll
    for (int i = 0; i < ST_NPI; ++i) {
      const int pos = tid + ST_NPROD * i;
      const long long q = S0 + pos;
      off[i] = -2;  // no such strip position
      if (pos < P) {
        off[i] = -1;
        if (q >= 0 && q < QN) {
          // 32-bit division (the host keeps every position below 2^31)
          const uint32_t qu = uint32_t(q), nn = qu / HW2u, r = qu - nn * HW2u, yq = r / W2u;
          int yy = int(yq) - 1, xx = int(r - yq * W2u) - 1;
          yy += yy < 0 ? p.h : 0;
          yy -= yy >= p.h ? p.h : 0;
          xx += xx < 0 ? p.wid : 0;
          xx -= xx >= p.wid ? p.wid : 0;
          off[i] = p.up ? ((int(nn) * (p.h >> 1) + (yy >> 1)) * (p.wid >> 1) + (xx >> 1)) * p.cin
                        : ((int(nn) * p.h + yy) * p.wid + xx) * p.cin;
        }
      }
    }
    for (int ks = 0; ks < nk && !bad; ++ks) {
      const int s = ks % S;
      if (ks >= S && !tma::mbar_wait(&empty[s], uint32_t((ks / S - 1) & 1))) {
        bad = true;
        break;
      }
      unsigned char* sa = smem + s * STAGE;
      if (tid == 0) {
        tma::mbar_arrive_expect_tx(&full[s], uint32_t(TT::B_BYTES));
        bulk_load(sa + A_BYTES,
                  p.wt + (long long)(blockIdx.y * nk + ks) * (TT::B_BYTES / 2),
                  uint32_t(TT::B_BYTES), &full[s]);
      }
      const int c0 = ks * CB;
#pragma unroll
      for (int i = 0; i < ST_NPI; ++i) {
        if (off[i] == -2) continue;
        const int pos = tid + ST_NPROD * i;
        const __nv_bfloat16* src = p.x + (off[i] >= 0 ? off[i] + c0 : 0);
#pragma unroll
        for (int j = 0; j < CH; ++j)
          cp_async16(sa + (j * P + pos) * 16, src + j * 8, off[i] >= 0);
      }
      asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(
                       smem_u32(&full[s]))
                   : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");

    // epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 of the
    // M-tiles m = w / 4, w / 4 + 2
    bad |= !tma::mbar_wait(done, 0);
    __syncwarp();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int lq = 32 * (warp & 3);
    for (int m = warp >> 2; m < ST_MT; m += 2) {
      const long long q = Q0 + m * 128 + lq + lane;
      const uint32_t qu = uint32_t(q), nn = qu / HW2u, r = qu - nn * HW2u, yq = r / W2u;
      const int yp = int(yq), xp = int(r - yq * W2u);
      const bool store = !bad && q < QN && yp >= 1 && yp <= p.h && xp >= 1 && xp <= p.wid;
      const long long pix = ((long long)nn * p.h + (yp - 1)) * p.wid + (xp - 1);
#pragma unroll
      for (int c16 = 0; c16 < BN / 16; ++c16) {
        uint32_t v[16];
        tmem_ld16(tmem + (uint32_t(lq) << 16) + uint32_t(m * BN + c16 * 16), v);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (store) {
          const int cob = co0 + c16 * 16;
          const long long o = pix * p.cout + cob;
          __align__(16) __nv_bfloat162 zz[8], aa[8];
          __align__(16) float bs[16];
          if (p.bias) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
              reinterpret_cast<float4*>(bs)[j] = __ldg(reinterpret_cast<const float4*>(p.bias + cob) + j);
          }
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            float v0 = __uint_as_float(v[2 * e]), v1 = __uint_as_float(v[2 * e + 1]);
            if (p.bias) {
              v0 += bs[2 * e];
              v1 += bs[2 * e + 1];
            }
            if (p.res) {
              const __nv_bfloat162 rr =
                  *reinterpret_cast<const __nv_bfloat162*>(p.res + o + 2 * e);
              v0 += __bfloat162float(rr.x);
              v1 += __bfloat162float(rr.y);
            }
            zz[e] = __floats2bfloat162_rn(v0, v1);
            if (p.a) aa[e] = __floats2bfloat162_rn(gelu(v0), gelu(v1));
          }
          if (p.z) {
            reinterpret_cast<uint4*>(p.z + o)[0] = reinterpret_cast<const uint4*>(zz)[0];
            reinterpret_cast<uint4*>(p.z + o)[1] = reinterpret_cast<const uint4*>(zz)[1];
          }
          if (p.a) {
            reinterpret_cast<uint4*>(p.a + o)[0] = reinterpret_cast<const uint4*>(aa)[0];
            reinterpret_cast<uint4*>(p.a + o)[1] = reinterpret_cast<const uint4*>(aa)[1];
          }
        }
      }
    }
  } else if (lane == 0) {
    // MMA issuer: per stage, for every tap and K step of 16 channels, one MMA
    // per M-tile
    constexpr uint32_t idesc = umma_idesc<BN>();
    const uint32_t lbo = uint32_t(P * 16), sbo_b = uint32_t(9 * CB / 8 * 128);
    for (int ks = 0; ks < nk; ++ks) {
      const int s = ks % S;
      if (!tma::mbar_wait(&full[s], uint32_t((ks / S) & 1))) {
        bad = true;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(smem + s * STAGE);
      const uint32_t b0 = a0 + uint32_t(A_BYTES);
#pragma unroll 1
      for (int t = 0; t < 9; ++t) {
        const int offp = (t / 3 - 1) * W2 + (t % 3 - 1) + (W2 + 1);  // strip row of M row 0
#pragma unroll
        for (int kk = 0; kk < CB / 16; ++kk) {
          const uint64_t bd = umma_desc_k(b0 + uint32_t((t * CH + 2 * kk) * 128), 128u, sbo_b);
#pragma unroll
          for (int m = 0; m < ST_MT; ++m) {
            const uint64_t ad =
                umma_desc_k(a0 + uint32_t((2 * kk * P + offp + m * 128) * 16), lbo, 128u);
            umma_bf16(tmem + uint32_t(m * BN), ad, bd, idesc,
                      (ks > 0 || t > 0 || kk > 0) ? 1u : 0u);
          }
        }
      }
      umma_commit(&empty[s]);
    }
    umma_commit(done);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 8)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TT::COLS));
  if (bad) atomicExch(err, 1);
}

template <int BN, int CB, int MT>
int launch_strip(StripParams p, int* err, cudaStream_t s, int smax) {
  using TT = StripTile<BN, CB, MT>;
  constexpr int ST_M = TT::M;
  const int W2 = p.wid + 2;
  p.P = ((ST_M + 2 * (W2 + 1)) + 7) / 8 * 8;
  if (p.P > ST_NPROD * ST_NPI) return SP_EINVAL;  // rows wider than the producers cover
  const int stage = TT::CH * p.P * 16 + TT::B_BYTES;
  const int nk = p.cin / CB;
  const int budget = 227 * 1024 - 1024;
  int S = budget / stage;
  if (S < 1) return SP_EINVAL;
  S = S < nk ? S : nk;
  S = S < smax ? S : smax;
  p.S = S;
  int smem = S * stage + (2 * S + 1) * 8 + 16;
  // no more CTAs on an SM than its 512 tensor-memory columns hold: ask for
  // enough shared memory (228 KB per SM, 1 KB reserved per CTA) that no
  // further one is resident
  const int fit = 512 / TT::COLS;
  const int floor_smem = 228 * 1024 / (fit + 1) + 1;
  if (fit < 7 && smem < floor_smem) smem = floor_smem;
  const cudaError_t attr = cudaFuncSetAttribute(
      k_conv3x3_strip<BN, CB, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (attr != cudaSuccess) return SP_ECUDA;
  const long long QN = (long long)(p.h + 2) * W2 * p.n;
  k_conv3x3_strip<BN, CB, MT><<<dim3(unsigned((QN + ST_M - 1) / ST_M), unsigned(p.cout / BN)),
                                ST_NT, smem, s>>>(p, err);
  return cudaGetLastError() == cudaSuccess ? SP_OK : SP_ECUDA;
}

}  // namespace conv
}  // namespace sp

namespace {
int strip_fwd(const void* x, const void* w, void* wt, const float* bias, const void* res, void* z,
              void* a, int n, int h, int w_, int cin, int cout, void* stream, int up) {
  using namespace sp::conv;
  if (!x || !w || !wt || (!z && !a) || n < 1 || h < 1 || w_ < 1 || cin % 16 != 0 ||
      !(cout == 32 || cout == 64 || cout % 128 == 0))
    return SP_EINVAL;
  // the epilogue reads the bias 16 channels (64 bytes) at a time
  if (bias && reinterpret_cast<uintptr_t>(bias) % 16 != 0) return SP_EINVAL;
  // rows the producers cover with four M-tiles per CTA, whatever shape runs
  if (w_ > 764) return SP_EINVAL;
  // (n (h + 2) + h + 1) (w + 2) + ... stays an int offset per pixel, and
  // every padded position (with a strip's reach past the end) below 2^31
  if ((long long)n * h * w_ * cin >= (1LL << 31)) return SP_EINVAL;
  if ((long long)n * (h + 2) * (w_ + 2) + 4LL * (w_ + 3) + 4096 >= (1LL << 31)) return SP_EINVAL;
  int* err = tc_error_flag();
  if (!err) return SP_ENOMEM;
  const int bn = cout == 32 ? 32 : cout == 64 ? 64 : 128;
  // CTA shape by layer class, from timing every shape on the jump network's
  // layers (256 samples, 256^2 .. 32^2): narrow outputs gain from more,
  // smaller CTAs (four or two M-tiles, one stage, so that more CTAs share an
  // SM and one CTA's gather overlaps another's MMAs and epilogue); wide
  // inputs and outputs keep the four-stage ring of 32-channel K blocks
  int cb = 16, mt = 4, smax = 1;
  if (cout == 64) {
    mt = 2;
    cb = cin >= 128 && cin % 32 == 0 ? 32 : 16;
  } else if (cout >= 128) {
    if (cin >= 128 && cin % 32 == 0) {
      cb = 32;
      smax = 4;
    } else {
      mt = 2;
    }
  }
  // SP_STRIP_SHAPE="mt,cb,stages": M-tiles per CTA (2 or 4), input channels
  // per K block (16 or 32) and the most ring stages, for timing shapes
  if (const char* e = getenv("SP_STRIP_SHAPE")) {
    int a = 0, b = 0, c = 0;
    if (sscanf(e, "%d,%d,%d", &a, &b, &c) == 3 && (a == 2 || a == 4) && (b == 16 || b == 32) &&
        c >= 1 && c <= 4 && cin % b == 0) {
      mt = a;
      cb = b;
      smax = c;
    }
  }
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_tile_weights<<<256, 256, 0, s>>>(static_cast<const __nv_bfloat16*>(w),
                                      static_cast<__nv_bfloat16*>(wt), cin, cout, bn, cb);
  if (cudaGetLastError() != cudaSuccess) return SP_ECUDA;
  StripParams p{static_cast<const __nv_bfloat16*>(x), static_cast<const __nv_bfloat16*>(wt),
                bias, static_cast<const __nv_bfloat16*>(res), static_cast<__nv_bfloat16*>(z),
                static_cast<__nv_bfloat16*>(a), n, h, w_, cin, cout, 0, 0, up};
  auto go = [&](auto bn_c, auto cb_c) {
    constexpr int BN = decltype(bn_c)::value, CB = decltype(cb_c)::value;
    return mt == 2 ? launch_strip<BN, CB, 2>(p, err, s, smax)
                   : launch_strip<BN, CB, 4>(p, err, s, smax);
  };
  using I32 = std::integral_constant<int, 32>;
  using I16 = std::integral_constant<int, 16>;
  using I64 = std::integral_constant<int, 64>;
  using I128 = std::integral_constant<int, 128>;
  if (bn == 32) return cb == 32 ? go(I32{}, I32{}) : go(I32{}, I16{});
  if (bn == 64) return cb == 32 ? go(I64{}, I32{}) : go(I64{}, I16{});
  return cb == 32 ? go(I128{}, I32{}) : go(I128{}, I16{});
}
}  // namespace

extern "C" int sp_conv3x3_fwd_strip(const void* x, const void* w, void* wt, const float* bias,
                                    const void* res, void* z, void* a, int n, int h, int w_,
                                    int cin, int cout, void* stream) {
  return strip_fwd(x, w, wt, bias, res, z, a, n, h, w_, cin, cout, stream, 0);
}

extern "C" int sp_conv3x3_fwd_strip_up2(const void* x, const void* w, void* wt, const float* bias,
                                        const void* res, void* z, void* a, int n, int h, int w_,
                                        int cin, int cout, void* stream) {
  if (h < 2 || w_ < 2 || h % 2 != 0 || w_ % 2 != 0) return SP_EINVAL;
  return strip_fwd(x, w, wt, bias, res, z, a, n, h, w_, cin, cout, stream, 1);
}
