/*
 * sp_common.cuh -- small device helpers shared by the step and auxiliary
 * kernels: integer helpers, the W-wide value type of the vectorised
 * evaluator, the shared-memory evaluation context and block reductions.
 */
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sp {

constexpr int ceil_to(int a, int b) { return (a + b - 1) / b * b; }
constexpr int imax(int a, int b) { return a > b ? a : b; }
constexpr int floordiv(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

enum : int { KERR_NONE = 0, KERR_TMA_TIMEOUT = 1 };

// ---------------------------------------------------------------------------
// Vec<T, W>: W consecutive x-sites evaluated together.  Every operation is
// elementwise, so an expression evaluated on Vec rounds exactly like W scalar
// evaluations (the FP64 exact form stays bit-identical to the CPU solver),
// while shared-memory traffic moves as 8- or 16-byte words.
// ---------------------------------------------------------------------------
template <class T, int W>
struct alignas(sizeof(T) * W) Vec {
  T v[W];
  Vec() = default;
  template <class S>
  __host__ __device__ __forceinline__ explicit Vec(S s) {
#pragma unroll
    for (int j = 0; j < W; ++j) v[j] = T(s);
  }
};

#define SP_VEC_BINOP(OP)                                                           \
  template <class T, int W>                                                        \
  __device__ __forceinline__ Vec<T, W> operator OP(const Vec<T, W>& a, const Vec<T, W>& b) { \
    Vec<T, W> r;                                                                   \
    _Pragma("unroll") for (int j = 0; j < W; ++j) r.v[j] = a.v[j] OP b.v[j];       \
    return r;                                                                      \
  }
SP_VEC_BINOP(+)
SP_VEC_BINOP(-)
SP_VEC_BINOP(*)
SP_VEC_BINOP(/)
#undef SP_VEC_BINOP

template <class T, int W>
__device__ __forceinline__ Vec<T, W> operator-(const Vec<T, W>& a) {
  Vec<T, W> r;
#pragma unroll
  for (int j = 0; j < W; ++j) r.v[j] = -a.v[j];
  return r;
}

// Two FP32 lanes map onto Blackwell's packed FP32x2 instructions
// (__fadd2_rn / __fmul2_rn / __ffma2_rn, sm_100): one instruction per two
// sites, each lane rounded exactly as the scalar operation (a - b is
// a + (-b), which is exact).
__device__ __forceinline__ float2 f2(const Vec<float, 2>& a) { return make_float2(a.v[0], a.v[1]); }
__device__ __forceinline__ Vec<float, 2> v2(float2 a) {
  Vec<float, 2> r;
  r.v[0] = a.x;
  r.v[1] = a.y;
  return r;
}
__device__ __forceinline__ Vec<float, 2> operator+(const Vec<float, 2>& a, const Vec<float, 2>& b) {
  return v2(__fadd2_rn(f2(a), f2(b)));
}
__device__ __forceinline__ Vec<float, 2> operator-(const Vec<float, 2>& a, const Vec<float, 2>& b) {
  return v2(__fadd2_rn(f2(a), make_float2(-b.v[0], -b.v[1])));
}
__device__ __forceinline__ Vec<float, 2> operator*(const Vec<float, 2>& a, const Vec<float, 2>& b) {
  return v2(__fmul2_rn(f2(a), f2(b)));
}
__device__ __forceinline__ Vec<float, 2> fma_op(const Vec<float, 2>& a, const Vec<float, 2>& b,
                                                 const Vec<float, 2>& c) {
  return v2(__ffma2_rn(f2(a), f2(b), f2(c)));
}
// four FP32 lanes: two packed instructions, lanes (0, 1) and (2, 3)
__device__ __forceinline__ float2 lo2(const Vec<float, 4>& a) { return make_float2(a.v[0], a.v[1]); }
__device__ __forceinline__ float2 hi2(const Vec<float, 4>& a) { return make_float2(a.v[2], a.v[3]); }
__device__ __forceinline__ Vec<float, 4> v4(float2 l, float2 h) {
  Vec<float, 4> r;
  r.v[0] = l.x;
  r.v[1] = l.y;
  r.v[2] = h.x;
  r.v[3] = h.y;
  return r;
}
__device__ __forceinline__ Vec<float, 4> operator+(const Vec<float, 4>& a, const Vec<float, 4>& b) {
  return v4(__fadd2_rn(lo2(a), lo2(b)), __fadd2_rn(hi2(a), hi2(b)));
}
__device__ __forceinline__ Vec<float, 4> operator-(const Vec<float, 4>& a, const Vec<float, 4>& b) {
  return v4(__fadd2_rn(lo2(a), make_float2(-b.v[0], -b.v[1])),
            __fadd2_rn(hi2(a), make_float2(-b.v[2], -b.v[3])));
}
__device__ __forceinline__ Vec<float, 4> operator*(const Vec<float, 4>& a, const Vec<float, 4>& b) {
  return v4(__fmul2_rn(lo2(a), lo2(b)), __fmul2_rn(hi2(a), hi2(b)));
}
__device__ __forceinline__ Vec<float, 4> fma_op(const Vec<float, 4>& a, const Vec<float, 4>& b,
                                                 const Vec<float, 4>& c) {
  return v4(__ffma2_rn(lo2(a), lo2(b), lo2(c)), __ffma2_rn(hi2(a), hi2(b), hi2(c)));
}
__device__ __forceinline__ float fma_op(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_op(double a, double b, double c) { return __fma_rn(a, b, c); }
template <class T, int W>
__device__ __forceinline__ Vec<T, W> fma_op(const Vec<T, W>& a, const Vec<T, W>& b,
                                            const Vec<T, W>& c) {
  Vec<T, W> r;
#pragma unroll
  for (int j = 0; j < W; ++j) r.v[j] = fma_op(a.v[j], b.v[j], c.v[j]);
  return r;
}

// a * b + c: one rounding (FMA) when CONTRACT, else a rounded product and then
// a rounded sum, as the exact form requires
template <bool CONTRACT, class V>
__device__ __forceinline__ V fmadd(const V& a, const V& b, const V& c) {
  if constexpr (CONTRACT) {
    return fma_op(a, b, c);
  } else {
    const V p = a * b;
    return p + c;
  }
}

template <class T, int W>
struct VecOf {
  using type = Vec<T, W>;
};
template <class T>
struct VecOf<T, 1> {
  using type = T;
};
template <class T, int W>
using vec_t = typename VecOf<T, W>::type;

template <class T>
__device__ __forceinline__ T lane(const T& x, int) {
  return x;
}
template <class T, int W>
__device__ __forceinline__ T lane(const Vec<T, W>& x, int j) {
  return x.v[j];
}
template <class T>
__device__ __forceinline__ void set_lane(T& x, int, T s) {
  x = s;
}
template <class T, int W>
__device__ __forceinline__ void set_lane(Vec<T, W>& x, int j, T s) {
  x.v[j] = s;
}

// value at offset X (elements) from a W-aligned pointer p, as a W-wide vector
// built from at most two aligned vector loads (offsets are compile-time)
template <class T, int W, int X>
__device__ __forceinline__ vec_t<T, W> load_at(const T* p) {
  if constexpr (W == 1) {
    return p[X];
  } else {
    constexpr int c0 = floordiv(X, W);
    constexpr int l0 = X - c0 * W;
    const Vec<T, W> a = *reinterpret_cast<const Vec<T, W>*>(p + c0 * W);
    if constexpr (l0 == 0) {
      return a;
    } else {
      const Vec<T, W> b = *reinterpret_cast<const Vec<T, W>*>(p + (c0 + 1) * W);
      Vec<T, W> r;
#pragma unroll
      for (int j = 0; j < W; ++j) r.v[j] = (l0 + j < W) ? a.v[l0 + j] : b.v[l0 + j - W];
      return r;
    }
  }
}

// Evaluation context of one W-wide site group: shared-memory pointers to the
// group's site in the field planes (NZ planes centred at ZR) and in the
// staged-operand planes; PW and SW are the row pitches of the field and stage
// tiles.  Holding pointers (not offsets from a base) makes every stencil
// point a compile-time displacement of one of them, i.e. a load immediate.
template <class T, int W, bool CONTRACT, int DIM, int LP, int GP, int BP, int NF, int NZ, int ZR,
          int PW, int NS, int NSZ, int SZR, int SW>
struct Ctx {
  using scalar_type = T;
  using value_type = vec_t<T, W>;
  static constexpr bool contract = CONTRACT;  // a*b + c may round once
  static constexpr int dim = DIM, lap_points = LP, gradlap_points = GP, bilap_points = BP;
  const T* fo[NF][NZ];
  const T* so[NS > 0 ? NS : 1][NSZ > 0 ? NSZ : 1];
  value_type divh2, divh3, divh4;
  const T* cf;
  template <int I, int X, int Y, int Z>
  __device__ __forceinline__ value_type var() const {
    static_assert(I >= 1 && I <= NF, "field index");
    static_assert(Z + ZR >= 0 && Z + ZR < NZ, "z reach beyond the loaded planes");
    static_assert(DIM == 3 || Z == 0, "z offset in 2D");
    return load_at<T, W, X>(fo[I - 1][Z + ZR] + Y * PW);
  }
  template <int K, int X, int Y, int Z>
  __device__ __forceinline__ value_type stg() const {
    static_assert(K >= 0 && K < NS, "stage index");
    static_assert(Z + SZR >= 0 && Z + SZR < NSZ, "z reach beyond the staged planes");
    return load_at<T, W, X>(so[K][Z + SZR] + Y * SW);
  }
  __device__ __forceinline__ value_type coef(int i) const { return value_type(cf[i - 1]); }
};

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane_id = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane_id == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < NT / 32; ++i) s += red[i];
  return s;
}

// Programmatic dependent launch: every step kernel is launched with
// programmatic stream serialization, so its grid may start while the previous
// grid in the stream drains.  Every thread calls this before its first global
// access: it waits until the previous grid has completed and its writes are
// visible, then lets the next grid be launched (whose CTAs only take the
// slots this grid frees: they start after all of this grid's CTAs have).
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace sp
