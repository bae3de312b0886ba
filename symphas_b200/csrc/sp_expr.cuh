/*
 * sp_expr.cuh -- compile-time expression trees for EVOLUTION right-hand sides
 * and their device-side evaluation.
 *
 * A SymPhas MODEL writes each field's evolution as an expression of the fields
 * op(i), coefficients c(i), literals, +, -, *, power<N>, and the derivatives
 * lap / bilap / gradlap (sol/inc/modelmacros.h:1086-1263).  Here the same tree
 * is a C++ type; evaluating it at a grid site is a chain of inlined device
 * calls whose neighbour offsets are template arguments, so a whole right-hand
 * side becomes straight-line code reading shared memory at base + immediate.
 *
 * Semantics kept from the reference:
 *   - a sum evaluates left operand then right operand exactly as written; the
 *     built-in models are written as right folds to match OpAdd's fold
 *     e0 + (e1 + (e2 + ...)) (sym/inc/expressions.h:2032-2040);
 *   - power<N>(x) is the right-fold product x*(x*(x...)) for N <= 6
 *     (lib/inc/spslibmath.h:255-268);
 *   - a derivative of a non-variable operand applies the stencil to the
 *     operand evaluated at each stencil point, which equals SymPhas's
 *     temporary grid filled over the halo (sym/inc/expressionderivatives.h:
 *     1546-1588) value for value;
 *   - Stage<K>: an operand the kernel materialises once per site in shared
 *     memory (the fused form), instead of re-evaluating it per stencil point.
 */
#pragma once

#include <type_traits>

#include "sp_common.cuh"
#include "sp_stencils.cuh"

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace sp {
namespace ex {

struct node {};
template <class E>
constexpr bool is_node_v = std::is_base_of<node, E>::value;

template <int I>
struct Var : node {};  // op(I), 1-based field index
template <int I>
struct Coef : node {};  // c(I), 1-based coefficient index
template <int K>
struct StageRef : node {};  // value of staged operand K (0-based)
struct Lit : node {
  double v;
  __host__ __device__ constexpr Lit(double x = 0) : v(x) {}
};
template <class A, class B>
struct Add : node {
  A a;
  B b;
  __host__ __device__ constexpr Add(A x, B y) : a(x), b(y) {}
};
template <class A, class B>
struct Sub : node {
  A a;
  B b;
  __host__ __device__ constexpr Sub(A x, B y) : a(x), b(y) {}
};
template <class A, class B>
struct Mul : node {
  A a;
  B b;
  __host__ __device__ constexpr Mul(A x, B y) : a(x), b(y) {}
};
template <class A>
struct Neg : node {
  A a;
  __host__ __device__ constexpr explicit Neg(A x) : a(x) {}
};
template <int N, class A>
struct Pow : node {
  A a;
  __host__ __device__ constexpr explicit Pow(A x) : a(x) {}
};
template <class A>
struct Lap : node {
  A a;
  __host__ __device__ constexpr explicit Lap(A x) : a(x) {}
};
template <class A>
struct Bilap : node {
  A a;
  __host__ __device__ constexpr explicit Bilap(A x) : a(x) {}
};
template <class A>
struct Gradlap : node {  // x component, as the reference's point functors return
  A a;
  __host__ __device__ constexpr explicit Gradlap(A x) : a(x) {}
};

template <class E>
__host__ __device__ constexpr auto lift(E e) {
  if constexpr (is_node_v<E>)
    return e;
  else
    return Lit(double(e));
}
template <class E>
using lift_t = decltype(lift(std::declval<E>()));

template <class A, class B, class = std::enable_if_t<is_node_v<A> || is_node_v<B>>>
__host__ __device__ constexpr auto operator+(A a, B b) {
  return Add<lift_t<A>, lift_t<B>>(lift(a), lift(b));
}
template <class A, class B, class = std::enable_if_t<is_node_v<A> || is_node_v<B>>>
__host__ __device__ constexpr auto operator-(A a, B b) {
  return Sub<lift_t<A>, lift_t<B>>(lift(a), lift(b));
}
template <class A, class B, class = std::enable_if_t<is_node_v<A> || is_node_v<B>>>
__host__ __device__ constexpr auto operator*(A a, B b) {
  return Mul<lift_t<A>, lift_t<B>>(lift(a), lift(b));
}
template <class A, class = std::enable_if_t<is_node_v<A>>>
__host__ __device__ constexpr auto operator-(A a) {
  return Neg<A>(a);
}
template <class A>
__host__ __device__ constexpr auto lap(A a) {
  return Lap<lift_t<A>>(lift(a));
}
template <class A>
__host__ __device__ constexpr auto bilap(A a) {
  return Bilap<lift_t<A>>(lift(a));
}
template <class A>
__host__ __device__ constexpr auto gradlap(A a) {
  return Gradlap<lift_t<A>>(lift(a));
}
template <int N, class A>
__host__ __device__ constexpr auto power(A a) {
  static_assert(N >= 1 && N <= 6, "power<N> is supported for 1 <= N <= 6");
  return Pow<N, lift_t<A>>(lift(a));
}
template <int I>
__host__ __device__ constexpr Var<I> op() {
  return {};
}
template <int I>
__host__ __device__ constexpr Coef<I> c() {
  return {};
}
template <int K>
__host__ __device__ constexpr StageRef<K> stage() {
  return {};
}

// ---------------------------------------------------------------------------
// reach: how far (Chebyshev radius) an expression reads into fields and into
// staged operands; -1 = does not read them at all.
// ---------------------------------------------------------------------------
constexpr int rmax(int a, int b) { return a > b ? a : b; }
constexpr int rplus(int a, int d) { return a < 0 ? -1 : a + d; }

// ACC: order of accuracy of the stencils (2: Stencil2d2h / Stencil3d2h, whose
// Laplacians reach 1 and bilaplacians and gradlaplacians 2; 4: Stencil2d4h,
// reaching 2, 3 and 3)
template <class E, int ACC = 2>
struct Reach {
  static constexpr int field = -1, stage = -1, max_var = 0, max_stage = -1;
};
template <int I, int ACC>
struct Reach<Var<I>, ACC> {
  static constexpr int field = 0, stage = -1, max_var = I, max_stage = -1;
};
template <int K, int ACC>
struct Reach<StageRef<K>, ACC> {
  static constexpr int field = -1, stage = 0, max_var = 0, max_stage = K;
};
template <class A, class B, int ACC>
struct Reach2 {
  static constexpr int field = rmax(Reach<A, ACC>::field, Reach<B, ACC>::field);
  static constexpr int stage = rmax(Reach<A, ACC>::stage, Reach<B, ACC>::stage);
  static constexpr int max_var = rmax(Reach<A, ACC>::max_var, Reach<B, ACC>::max_var);
  static constexpr int max_stage = rmax(Reach<A, ACC>::max_stage, Reach<B, ACC>::max_stage);
};
template <class A, class B, int ACC>
struct Reach<Add<A, B>, ACC> : Reach2<A, B, ACC> {};
template <class A, class B, int ACC>
struct Reach<Sub<A, B>, ACC> : Reach2<A, B, ACC> {};
template <class A, class B, int ACC>
struct Reach<Mul<A, B>, ACC> : Reach2<A, B, ACC> {};
template <class A, int ACC>
struct Reach<Neg<A>, ACC> : Reach<A, ACC> {};
template <int N, class A, int ACC>
struct Reach<Pow<N, A>, ACC> : Reach<A, ACC> {};
template <class A, int D, int ACC>
struct ReachD {
  static constexpr int field = rplus(Reach<A, ACC>::field, D);
  static constexpr int stage = rplus(Reach<A, ACC>::stage, D);
  static constexpr int max_var = Reach<A, ACC>::max_var, max_stage = Reach<A, ACC>::max_stage;
};
template <class A, int ACC>
struct Reach<Lap<A>, ACC> : ReachD<A, ACC == 4 ? 2 : 1, ACC> {};
template <class A, int ACC>
struct Reach<Bilap<A>, ACC> : ReachD<A, ACC == 4 ? 3 : 2, ACC> {};
template <class A, int ACC>
struct Reach<Gradlap<A>, ACC> : ReachD<A, ACC == 4 ? 3 : 2, ACC> {};

// ---------------------------------------------------------------------------
// evaluation at offset (X,Y,Z) from the site a context points at.
// A context C provides: value_type, dim, lap_points, gradlap_points,
// bilap_points, divh2/divh3/divh4, coef(i), var<I,X,Y,Z>(), stg<K,X,Y,Z>().
// ---------------------------------------------------------------------------
template <class E>
struct Ev;

template <class A, int X, int Y, int Z, class C>
struct Shifted {
  const A& e;
  const C& c;
  template <int i, int j, int k>
  __device__ __forceinline__ typename C::value_type at() const {
    return Ev<A>::template at<X + i, Y + j, Z + k>(e, c);
  }
};

template <int I>
struct Ev<Var<I>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Var<I>&, const C& c) {
    return c.template var<I, X, Y, Z>();
  }
};
template <int K>
struct Ev<StageRef<K>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const StageRef<K>&, const C& c) {
    return c.template stg<K, X, Y, Z>();
  }
};
template <int I>
struct Ev<Coef<I>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Coef<I>&, const C& c) {
    return c.coef(I);
  }
};
template <>
struct Ev<Lit> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Lit& e, const C&) {
    return typename C::value_type(e.v);
  }
};
template <class A, class B>
struct Ev<Add<A, B>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Add<A, B>& e, const C& c) {
    return Ev<A>::template at<X, Y, Z>(e.a, c) + Ev<B>::template at<X, Y, Z>(e.b, c);
  }
};
template <class A, class B>
struct Ev<Sub<A, B>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Sub<A, B>& e, const C& c) {
    return Ev<A>::template at<X, Y, Z>(e.a, c) - Ev<B>::template at<X, Y, Z>(e.b, c);
  }
};
template <class A, class B>
struct Ev<Mul<A, B>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Mul<A, B>& e, const C& c) {
    return Ev<A>::template at<X, Y, Z>(e.a, c) * Ev<B>::template at<X, Y, Z>(e.b, c);
  }
};
// a*b + c and its relatives: one FMA when the context may contract; in the
// exact form the same rounded product and rounded sum as the plain nodes
// (c + p = p + c and c - p = (-a)*b + c bit for bit)
template <class A, class B, class C2>
struct Ev<Add<Mul<A, B>, C2>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Add<Mul<A, B>, C2>& e,
                                                              const C& c) {
    return fmadd<C::contract>(Ev<A>::template at<X, Y, Z>(e.a.a, c),
                              Ev<B>::template at<X, Y, Z>(e.a.b, c),
                              Ev<C2>::template at<X, Y, Z>(e.b, c));
  }
};
template <class C2, class A, class B>
struct Ev<Add<C2, Mul<A, B>>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Add<C2, Mul<A, B>>& e,
                                                              const C& c) {
    return fmadd<C::contract>(Ev<A>::template at<X, Y, Z>(e.b.a, c),
                              Ev<B>::template at<X, Y, Z>(e.b.b, c),
                              Ev<C2>::template at<X, Y, Z>(e.a, c));
  }
};
template <class A, class B, class A2, class B2>
struct Ev<Add<Mul<A, B>, Mul<A2, B2>>> {  // left product first, as written
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(
      const Add<Mul<A, B>, Mul<A2, B2>>& e, const C& c) {
    return fmadd<C::contract>(Ev<A2>::template at<X, Y, Z>(e.b.a, c),
                              Ev<B2>::template at<X, Y, Z>(e.b.b, c),
                              Ev<Mul<A, B>>::template at<X, Y, Z>(e.a, c));
  }
};
template <class C2, class A, class B>
struct Ev<Sub<C2, Mul<A, B>>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Sub<C2, Mul<A, B>>& e,
                                                              const C& c) {
    return fmadd<C::contract>(-Ev<A>::template at<X, Y, Z>(e.b.a, c),
                              Ev<B>::template at<X, Y, Z>(e.b.b, c),
                              Ev<C2>::template at<X, Y, Z>(e.a, c));
  }
};
template <class A, class B, class C2>
struct Ev<Sub<Mul<A, B>, C2>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Sub<Mul<A, B>, C2>& e,
                                                              const C& c) {
    return fmadd<C::contract>(Ev<A>::template at<X, Y, Z>(e.a.a, c),
                              Ev<B>::template at<X, Y, Z>(e.a.b, c),
                              -Ev<C2>::template at<X, Y, Z>(e.b, c));
  }
};
template <class A, class B, class A2, class B2>
struct Ev<Sub<Mul<A, B>, Mul<A2, B2>>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(
      const Sub<Mul<A, B>, Mul<A2, B2>>& e, const C& c) {
    return fmadd<C::contract>(-Ev<A2>::template at<X, Y, Z>(e.b.a, c),
                              Ev<B2>::template at<X, Y, Z>(e.b.b, c),
                              Ev<Mul<A, B>>::template at<X, Y, Z>(e.a, c));
  }
};

template <class A>
struct Ev<Neg<A>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Neg<A>& e, const C& c) {
    return -Ev<A>::template at<X, Y, Z>(e.a, c);
  }
};
template <int N, class T>
__device__ __forceinline__ T rpow(T x) {
  if constexpr (N == 1)
    return x;
  else
    return x * rpow<N - 1>(x);
}
template <int N, class A>
struct Ev<Pow<N, A>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Pow<N, A>& e, const C& c) {
    return rpow<N>(Ev<A>::template at<X, Y, Z>(e.a, c));
  }
};
template <class A>
struct IsLeaf {
  static constexpr bool value = false;
};
template <int I>
struct IsLeaf<Var<I>> {
  static constexpr bool value = true;
};
template <int K>
struct IsLeaf<StageRef<K>> {
  static constexpr bool value = true;
};

// (value at x-1) + (value at x+1) at every lane of a W-group shifted by X.
// For a field or staged operand the lanes are summed one by one from the
// aligned groups at X-W, X and X+W (scalar adds, rounded as the vector add
// would round each lane), so no register shuffles build the shifted groups.
template <int X, int Y, int Z, class A, class C>
__device__ __forceinline__ typename C::value_type xpair(const A& a, const C& c) {
  using V = typename C::value_type;
  constexpr int W = int(sizeof(V) / sizeof(typename C::scalar_type));
  if constexpr (IsLeaf<A>::value && W > 1 && X % W == 0) {
    const V lo = Ev<A>::template at<X - W, Y, Z>(a, c);
    const V mid = Ev<A>::template at<X, Y, Z>(a, c);
    const V hi = Ev<A>::template at<X + W, Y, Z>(a, c);
    V r;
#pragma unroll
    for (int j = 0; j < W; ++j)
      r.v[j] = ((j == 0) ? lo.v[W - 1] : mid.v[j - 1]) + ((j == W - 1) ? hi.v[0] : mid.v[j + 1]);
    return r;
  } else {
    return Ev<A>::template at<X - 1, Y, Z>(a, c) + Ev<A>::template at<X + 1, Y, Z>(a, c);
  }
}

// Laplacian in a context that may contract and reassociate (the fused form):
// the 5- and 7-point sums become a balanced tree ending in one FMA, which
// shortens the dependency chain; other point sets, and the exact form, keep
// the reference's summation order.
template <class A>
struct Ev<Lap<A>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Lap<A>& e, const C& c) {
    using T = typename C::value_type;
    Shifted<A, X, Y, Z, C> s{e.a, c};
    if constexpr (C::contract && C::dim == 2 && C::lap_points == 5) {
      const T sx = xpair<X, Y, Z>(e.a, c);
      const T sy = s.template at<0, -1, 0>() + s.template at<0, 1, 0>();
      return fmadd<true>(T(-4.0) * c.divh2, s.template at<0, 0, 0>(), (sx + sy) * c.divh2);
    } else if constexpr (C::contract && C::dim == 3 && C::lap_points == 7) {
      const T sx = xpair<X, Y, Z>(e.a, c);
      const T sy = s.template at<0, -1, 0>() + s.template at<0, 1, 0>();
      const T sz = s.template at<0, 0, -1>() + s.template at<0, 0, 1>();
      return fmadd<true>(T(-6.0) * c.divh2, s.template at<0, 0, 0>(), ((sx + sy) + sz) * c.divh2);
    } else {
      if constexpr (C::lap_points >= 1000)  // Stencil2d4h: scale divh3, as the reference
        return st::lap4_pts<C::lap_points - 1000>::template apply<T>(s, c.divh3);
      else
        return st::lap_pts<C::dim, C::lap_points>::template apply<T>(s, c.divh2);
    }
  }
};
template <class A>
struct Ev<Bilap<A>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Bilap<A>& e, const C& c) {
    using T = typename C::value_type;
    Shifted<A, X, Y, Z, C> s{e.a, c};
    if constexpr (C::bilap_points >= 1000)  // Stencil2d4h: scale divh3, as the reference
      return st::bilap4_pts<C::bilap_points - 1000>::template apply<T>(s, c.divh3);
    else
      return st::bilap_pts<C::dim, C::bilap_points>::template apply<T>(s, c.divh4);
  }
};
template <class A>
struct Ev<Gradlap<A>> {
  template <int X, int Y, int Z, class C>
  __device__ __forceinline__ static typename C::value_type at(const Gradlap<A>& e, const C& c) {
    using T = typename C::value_type;
    Shifted<A, X, Y, Z, C> s{e.a, c};
    if constexpr (C::gradlap_points >= 1000)
      return st::gradlap4_pts<C::gradlap_points - 1000>::template apply<T>(s, c.divh3);
    else
      return st::gradlap_pts<C::dim, C::gradlap_points>::template apply<T>(s, c.divh3);
  }
};

template <class E, class C>
__device__ __forceinline__ typename C::value_type eval(const E& e, const C& c) {
  return Ev<E>::template at<0, 0, 0>(e, c);
}

// ---------------------------------------------------------------------------
// a lowered model: NF field right-hand sides and NS staged operands
// ---------------------------------------------------------------------------
template <int NF, int NS, class R0, class R1 = Lit, class S0 = Lit, class S1 = Lit>
struct ModelDef {
  static_assert(NF >= 1 && NF <= 2, "one or two fields");
  static_assert(NS >= 0 && NS <= 2, "at most two staged operands");
  R0 r0;
  R1 r1;
  S0 s0;
  S1 s1;
  static constexpr int nf = NF, ns = NS;
  // reach of the right-hand sides into the fields directly
  static constexpr int r_direct = rmax(Reach<R0>::field, NF > 1 ? Reach<R1>::field : -1);
  // reach of the right-hand sides into the staged operands
  static constexpr int RS =
      NS > 0 ? rmax(rmax(Reach<R0>::stage, NF > 1 ? Reach<R1>::stage : -1), 0) : 0;
  // reach of the staged operands into the fields
  static constexpr int r_stage = rmax(NS > 0 ? Reach<S0>::field : -1, NS > 1 ? Reach<S1>::field : -1);
  // halo radius a kernel must load around its tile
  static constexpr int R = rmax(rmax(r_direct, NS > 0 ? RS + rmax(r_stage, 0) : 0), 0);
  static_assert(Reach<R0>::max_var <= NF && Reach<R1>::max_var <= NF, "op(i) beyond the field count");
  static_assert(Reach<S0>::max_stage < 0 && Reach<S1>::max_stage < 0, "a staged operand may not use stages");
  static_assert(Reach<R0>::max_stage < NS && (NF < 2 || Reach<R1>::max_stage < NS), "stage index beyond NS");
  // the same reaches for stencils of order of accuracy ACC
  template <int ACC>
  struct reach_at {
    static constexpr int r_direct =
        rmax(Reach<R0, ACC>::field, NF > 1 ? Reach<R1, ACC>::field : -1);
    static constexpr int RS =
        NS > 0 ? rmax(rmax(Reach<R0, ACC>::stage, NF > 1 ? Reach<R1, ACC>::stage : -1), 0) : 0;
    static constexpr int r_stage =
        rmax(NS > 0 ? Reach<S0, ACC>::field : -1, NS > 1 ? Reach<S1, ACC>::field : -1);
    static constexpr int R = rmax(rmax(r_direct, NS > 0 ? RS + rmax(r_stage, 0) : 0), 0);
  };
};

// A lowered model evaluated with stencils of order of accuracy ACC: the same
// expressions, with the halo reaches of those stencils (the kernels read
// R, RS, r_direct and r_stage from their model type)
template <class M, int ACC>
struct ModelAcc : M {
  using RA = typename M::template reach_at<ACC>;
  static constexpr int r_direct = RA::r_direct, RS = RA::RS, r_stage = RA::r_stage, R = RA::R;
};

template <int NF, int NS, class R0, class R1 = Lit, class S0 = Lit, class S1 = Lit>
__host__ __device__ constexpr auto make_model(R0 r0, R1 r1 = Lit(), S0 s0 = Lit(), S1 s1 = Lit()) {
  return ModelDef<NF, NS, R0, R1, S0, S1>{r0, r1, s0, s1};
}

}  // namespace ex
}  // namespace sp
