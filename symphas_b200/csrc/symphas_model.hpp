/*
 * symphas_model.hpp -- C++ front end: write a model's EVOLUTION in C++, get
 * one fused sm_100a kernel per step for it.
 *
 * The SymPhas surface it mirrors (paths inside the SymPhas tree):
 *
 *   MODEL(MA, (SCALAR), EVOLUTION(dop(1) = lap(op(1)) + ...))
 *       (sol/inc/modelmacros.h:597-626)                       SP_MODEL(MA, 1, lap(op<1>()) + ...)
 *   model_MA_t<2, SolverFT<Stencil2d2h<5, 6, 13>>> m{coeff, n, params}
 *       (sol/inc/model.h:100-128)                             model_t<MA, SolverFT<Stencil2d2h<5, 6, 13>>, 2>
 *   symphas::find_solution(m, dt, steps) (modules-io.h:747-753)  find_solution(m, dt, steps)
 *   m.get_field<0>(), m.get_index(), m.get_time()             same
 *   SolverSystemFDwSD (sol/inc/solversystem.h:62-77)          regional_model_t<...>
 *
 * The expression is the C++ type of sp_expr.cuh (op<I>() = op(I), c<I>() =
 * c(I), lap / bilap / gradlap / power<N>, and stage<K>() for operands staged
 * once per site, see make_model); it is lowered at compile time into the
 * kernels of sp_kernels.cuh, registered with the runtime (sp_api.cu) under a
 * model id of its own, and run through the C ABI of symphas_b200.h.  Compile
 * the model's translation unit with the runtime sources:
 *
 *   nvcc -std=c++17 -O3 -gencode arch=compute_100a,code=sm_100a \
 *        --expt-relaxed-constexpr -I include -I symphas_b200/csrc \
 *        my_model.cu symphas_b200/csrc/sp_api.cu symphas_b200/csrc/sp_noalloc.cu \
 *        symphas_b200/csrc/sp_regional.cu -lcuda
 *
 * With SolverFT<..., true> (exact) and -fmad=false, FP64 results are
 * bit-identical to SymPhas's CPU solver when the expression is written in the
 * order of SymPhas's printed scheme.
 */
#pragma once

#include <atomic>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "sp_launch.cuh"
#include "symphas_b200.h"

namespace symphas_b200 {

using namespace sp::ex;

template <int L = 9, int G = 6, int B = 13>
struct Stencil2d2h {
  static constexpr int dim = 2, lp = L, gp = G, bp = B, acc = 2;
};
template <int L = 15, int G = 10, int B = 25>
struct Stencil3d2h {
  static constexpr int dim = 3, lp = L, gp = G, bp = B, acc = 2;
};
// 4th order of accuracy (sol/inc/stencilh4.h, defaults sol/inc/stencilincludes.h:774-779);
// every operator scaled by 1/h^3, as the reference does
template <int L = 9, int G = 14, int B = 21>
struct Stencil2d4h {
  static constexpr int dim = 2, lp = L, gp = G, bp = B, acc = 4;
};

// SolverFT<Stencil, Exact>: Exact = evaluate without FMA contraction (compile
// the translation unit with -fmad=false for bit-identical FP64)
template <class Sp, bool Exact = false>
struct SolverFT {
  using stencil = Sp;
  static constexpr bool exact = Exact;
};

// Problem parameters: interior points per axis (x first), spacing, boundaries
// per side (SP_PERIODIC or SP_DIRICHLET, LEFT RIGHT TOP BOTTOM FRONT BACK)
template <int D>
struct ProblemParameters {
  int n[3] = {1, 1, 1};
  double h = 1.0;
  int boundary[6] = {SP_PERIODIC, SP_PERIODIC, SP_PERIODIC,
                     SP_PERIODIC, SP_PERIODIC, SP_PERIODIC};
  double boundary_value[6] = {0, 0, 0, 0, 0, 0};
  ProblemParameters(std::initializer_list<int> dims, double spacing) : h(spacing) {
    int a = 0;
    for (int v : dims)
      if (a < 3) n[a++] = v;
  }
};

// var(N) of PROVISIONAL_DEF (sol/inc/modelmacros.h:682, :1102): a provisional
// variable is evaluated at every site (and its halo) before the equation and
// read under derivatives, which is what a staged operand is; declare the
// provisional expressions as the staged operands of SP_MODEL_STAGED, e.g.
// SymPhas's MBB (examples/models/modeldefinitions.h:150-155):
//   SP_MODEL_STAGED(MBB, 1, 1, -bilap(op<1>()) + lap(var<1>()), Lit(),
//                   -(c<1>() - Lit(4.0) * c<2>() * op<1>() * op<1>()) * op<1>())
template <int N>
__host__ __device__ constexpr auto var() {
  return stage<N - 1>();
}

namespace detail {
inline int next_model_id() {
  static std::atomic<int> id{1000};  // ids of user models, above the built-in ones
  return id++;
}
template <class MF, class Solver, int D, class T>
int registered_id() {
  // one registration per (model, solver, dimension, dtype), at first use
  static const int id = [] {
    using Sp = typename Solver::stencil;
    static_assert(Sp::dim == D, "stencil dimension differs from the model's");
    const int mid = next_model_id();
    const int dt = sizeof(T) == 8 ? SP_F64 : SP_F32;
    // 4th-order point sets are keyed (and evaluated) as SP_PTS4 + points
    constexpr int off = Sp::acc == 4 ? sp::SP_PTS4 : 0;
    const sp::KernelKey key{mid, Solver::exact ? SP_FORM_EXACT : SP_FORM_FUSED, D, dt,
                            off + Sp::lp, off + Sp::gp, off + Sp::bp};
    if constexpr (D == 3) {
      sp::register_kernel(key, sp::Entry3<MF, T, Sp::lp, Sp::gp, Sp::bp,
                                          typename sp::Tiles<T>::D3, Solver::exact>::info());
    } else {
      using MFA = sp::MFAcc<MF, Sp::acc>;  // the halo reach of the stencils
      sp::register_kernel(key, sp::Entry2<MFA, MFA, T, off + Sp::lp, off + Sp::gp, off + Sp::bp,
                                          typename sp::Tiles<T>::D2, Solver::exact>::info());
    }
    return mid;
  }();
  return id;
}
inline void check(int rc, const sp_handle* h) {
  if (rc != SP_OK)
    throw std::runtime_error(std::string("symphas_b200: ") +
                             (h ? sp_last_error(h) : sp_create_error()));
}
}  // namespace detail

// A device-resident model: fields live in HBM between steps.
template <class MF, class Solver, int D, class T = double>
class model_t {
 public:
  static constexpr int nfields = sp::model_of<MF>::nf;

  model_t(const double* coeff, size_t ncoeff, const ProblemParameters<D>& p) : n_(1) {
    using Sp = typename Solver::stencil;
    sp_desc d{};
    d.dim = D;
    for (int a = 0; a < 3; ++a) d.n[a] = a < D ? p.n[a] : 1;
    d.dtype = sizeof(T) == 8 ? SP_F64 : SP_F32;
    d.model = detail::registered_id<MF, Solver, D, T>();
    d.form = Solver::exact ? SP_FORM_EXACT : SP_FORM_FUSED;
    d.lap_pts = Sp::lp;
    d.gradlap_pts = Sp::gp;
    d.bilap_pts = Sp::bp;
    d.accuracy = Sp::acc;
    for (int s = 0; s < 6; ++s) {
      d.boundary[s] = p.boundary[s];
      d.boundary_value[s] = p.boundary_value[s];
    }
    d.h = p.h;
    for (int i = 0; i < 8; ++i) d.coeff[i] = i < int(ncoeff) ? coeff[i] : 1.0;  // c(i) = 1
    d.ncoeff = int(ncoeff);
    d.batch = 1;
    for (int a = 0; a < D; ++a) n_ *= size_t(p.n[a]);
    detail::check(sp_create(&d, &h_), nullptr);
  }
  explicit model_t(const ProblemParameters<D>& p) : model_t(nullptr, 0, p) {}
  model_t(const model_t&) = delete;
  model_t& operator=(const model_t&) = delete;
  ~model_t() { sp_destroy(h_); }

  // interior values, x fastest
  void set_field(int field, const std::vector<T>& v) {
    detail::check(sp_upload(h_, 0, field, v.data(), v.size() * sizeof(T)), h_);
  }
  std::vector<T> get_field(int field = 0) const {
    std::vector<T> v(n_);
    detail::check(sp_download(h_, 0, field, v.data(), v.size() * sizeof(T)), h_);
    return v;
  }
  template <size_t I>
  std::vector<T> get_field() const {
    return get_field(int(I));
  }
  void fill_uniform(int field, uint64_t seed, double lo, double hi) {
    detail::check(sp_fill_uniform(h_, 0, field, seed, lo, hi), h_);
  }

  // SolverFT: equation() and the halo update are fused into step()
  void update(double = 0) {}
  void equation() {}
  void step(double dt, int n = 1) {
    if (dt != dt_) {
      detail::check(sp_set_dt(h_, dt), h_);
      dt_ = dt;
    }
    detail::check(sp_step(h_, n), h_);
    index_ += n;
    time_ += n * dt;
  }
  int get_index() const { return index_; }
  double get_time() const { return time_; }
  sp_handle* handle() { return h_; }

 private:
  sp_handle* h_ = nullptr;
  size_t n_;
  double dt_ = 0.0, time_ = 0.0;
  int index_ = 0;
};

// Parameters of a regional system, SymPhas's command-line defaults
// (regional-resize-time, -factor, -eps, -fixed; sol/src/boundarysystem.cpp:24-27).
struct RegionalParameters {
  double resize_delta = 3.0;
  double padding_factor = 2.0;
  double cutoff_eps = 1e-6;
  bool fixed = true;
};

// A single-field model whose system is regional (SolverSystemFDwSD,
// sol/inc/solversystem.h:62-77): only a window of the domain is stored and
// stepped, and it follows the field (sp_regional_* in symphas_b200.h).  The
// domain must be periodic; fields in and out are whole-domain interiors.
// Compile sp_regional.cu with the runtime sources to use it.
template <class MF, class Solver, int D, class T = double>
class regional_model_t {
 public:
  static_assert(sp::model_of<MF>::nf == 1, "a regional system holds a single-field model");
  static constexpr int nfields = 1;

  regional_model_t(const double* coeff, size_t ncoeff, const ProblemParameters<D>& p,
                   const RegionalParameters& rp = RegionalParameters())
      : n_(1) {
    using Sp = typename Solver::stencil;
    sp_desc d{};
    d.dim = D;
    for (int a = 0; a < 3; ++a) d.n[a] = a < D ? p.n[a] : 1;
    d.dtype = sizeof(T) == 8 ? SP_F64 : SP_F32;
    d.model = detail::registered_id<MF, Solver, D, T>();
    d.form = Solver::exact ? SP_FORM_EXACT : SP_FORM_FUSED;
    d.lap_pts = Sp::lp;
    d.gradlap_pts = Sp::gp;
    d.bilap_pts = Sp::bp;
    d.accuracy = Sp::acc;
    for (int s = 0; s < 6; ++s) {
      d.boundary[s] = p.boundary[s];
      d.boundary_value[s] = p.boundary_value[s];
    }
    d.h = p.h;
    for (int i = 0; i < 8; ++i) d.coeff[i] = i < int(ncoeff) ? coeff[i] : 1.0;
    d.ncoeff = int(ncoeff);
    d.batch = 1;
    for (int a = 0; a < D; ++a) n_ *= size_t(p.n[a]);
    const sp_regional_params q{rp.resize_delta, rp.padding_factor, rp.cutoff_eps,
                               rp.fixed ? 1 : 0};
    if (sp_regional_create(&d, &q, &r_) != SP_OK)
      throw std::runtime_error(std::string("symphas_b200: ") + sp_regional_error(nullptr));
  }
  regional_model_t(const regional_model_t&) = delete;
  regional_model_t& operator=(const regional_model_t&) = delete;
  ~regional_model_t() { sp_regional_destroy(r_); }

  // whole-domain interior values, x fastest (`empty` outside the window)
  void set_field(int field, const std::vector<T>& v) {
    check(field == 0 ? sp_regional_upload(r_, v.data(), v.size() * sizeof(T)) : SP_EINVAL);
  }
  std::vector<T> get_field(int field = 0) const {
    std::vector<T> v(n_);
    check(field == 0 ? sp_regional_download(r_, v.data(), v.size() * sizeof(T)) : SP_EINVAL);
    return v;
  }
  template <size_t I>
  std::vector<T> get_field() const {
    return get_field(int(I));
  }

  // update(time) -- the window check -- runs inside step, before each iteration
  void update(double = 0) {}
  void equation() {}
  void step(double dt, int n = 1) {
    if (dt != dt_) {
      check(sp_regional_set_dt(r_, dt));
      dt_ = dt;
    }
    check(sp_regional_step(r_, n));
    index_ += n;
  }
  int get_index() const { return index_; }
  double get_time() const {
    double st[4];
    sp_regional_window(r_, nullptr, nullptr, st);
    return st[2];
  }
  // window origin and dims (storage coordinates, rim included)
  void window(int origin[3], int dims[3]) const { sp_regional_window(r_, origin, dims, nullptr); }
  sp_regional* handle() { return r_; }

 private:
  void check(int rc) const {
    if (rc != SP_OK)
      throw std::runtime_error(std::string("symphas_b200: ") + sp_regional_error(r_));
  }
  sp_regional* r_ = nullptr;
  size_t n_;
  double dt_ = 0.0;
  int index_ = 0;
};

template <class M>
M& find_solution(M& model, double dt, int steps) {
  model.update(model.get_time());
  model.step(dt, steps);
  return model;
}

}  // namespace symphas_b200

// MODEL(NAME, (types), EVOLUTION(...)): NAME is a factory of the lowered
// right-hand sides, one expression per field (op<1>(), op<2>() are fields 1, 2)
#define SP_MODEL(NAME, NF, ...)                                    \
  struct NAME {                                                    \
    constexpr auto operator()() const {                            \
      return ::sp::ex::make_model<NF, 0>(__VA_ARGS__);             \
    }                                                              \
  }

// The same with NS operands staged once per site in shared memory (the fused
// form): arguments are the right-hand side of field 1, of field 2 (or
// ::sp::ex::Lit()), then staged operands 0 and 1, referred to in the
// right-hand sides as stage<0>() and stage<1>() -- e.g. Cahn-Hilliard as
// SP_MODEL_STAGED(CH, 1, 1, lap(stage<0>()), Lit(),
//                 power<3>(op<1>()) - op<1>() - lap(op<1>()))
#define SP_MODEL_STAGED(NAME, NF, NS, ...)                         \
  struct NAME {                                                    \
    constexpr auto operator()() const {                            \
      return ::sp::ex::make_model<NF, NS>(__VA_ARGS__);            \
    }                                                              \
  }
