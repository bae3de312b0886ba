/*
 * solverftb200.h -- SymPhas's forward-Euler finite-difference solver on a
 * B200, for SymPhas's own models.
 *
 * Include it in a SymPhas program after the solver headers
 * (examples/solvers/solverft.h) and link libsymphas_b200.so.  It adds, through
 * SymPhas's own extension points:
 *
 *   SolverFTB200<Stencil...>   a solver declared like SolverFT
 *                              (START_NEW_SOLVER_WITH_STENCIL, sol/inc/solver.h:385);
 *   SolverSystemFDB200<T, D>   its solver system (ASSOCIATE_SOLVER_SYSTEM_TYPE,
 *                              sol/inc/solver.h:312-321): a SolverSystemFD whose
 *                              fields live on the GPU between steps.
 *
 * so that a model written for SolverFT runs unchanged on the GPU:
 *
 *   MODEL(MB, (SCALAR), EVOLUTION(dpsi = -bilap(psi) - lap((c(1) - c(2) * psi * psi) * psi)))
 *   model_MB_t<3, SolverFTB200<Stencil3d2h<7, 10, 25>>> model{coeff, 2, params};
 *   for (...) { model.update(t); model.equation(); model.step(dt); }   // model_iteration
 *   symphas_b200::binding::sync_to_host(model);                        // before reading values
 *
 * How it works.  SymPhas hands the solver each field's optimised equation
 * (SolverFT::form_expr_one, examples/solvers/solverft.h:112-119, the same
 * here).  On the first equation() call the equation is read back, at run
 * time, into terms c * D^k(psi^a eta^b) (k = 0, 2, 4: the value, lap, bilap;
 * OpAdd, OpDerivative and OpTerms nodes, sym/inc/expressions.h,
 * expressionderivatives.h, expressionaggregates.h); the terms of all fields
 * are matched against the models the B200 library has kernels for, and the
 * library's handle is created with SymPhas's dimensions, spacing, boundaries
 * (periodic, or DEFAULT with a CONSTANT value), stencil point set and
 * coefficients, and the fields' interiors are uploaded.  From then on
 * equation() does nothing (the fused step evaluates the equations) and step()
 * of the model's first system runs one fused step of every field on the GPU
 * (the others return: the fields are stepped together, after all equations,
 * as Model::step does, sol/inc/model.h:932-936).  The systems' update() does
 * not touch the host halo: the GPU keeps its own.  sync_to_host() copies the
 * fields back into each system's `values` (interior).
 *
 * Recognised (any coefficients; the terms in any order SymPhas prints them):
 *   model A    lap(psi) + a psi + b psi^3                   (MA, modeldefinitions.h:26-28)
 *   AMK        k lap(psi) + a psi - a psi^3
 *   model B    -bilap(psi) + a lap(psi) + b lap(psi^3)      (MB, modeldefinitions.h:31-33)
 *   BMK        -k bilap(psi) - m lap(psi) + m lap(psi^3)
 *   model C    psi: -bilap(psi) - lap(psi) + lap(psi^3) + lap(g psi eta^2),
 *              eta: lap(eta) + eta - eta^3 - g psi^2 eta    (the gamma form, g = 2 gamma)
 * Anything else (other terms, provisional variables, vector fields, other
 * solver variations) is refused at the first equation() with a message.
 *
 * Precision: by default the fields are FP64 and the step evaluates the
 * equations in SymPhas's term order (bit-identical to SymPhas's CPU solver
 * for unit coefficients); options().dtype / options().form select the FP32
 * fused step before the first equation() instead.
 */
#pragma once

#include <array>
#include <cmath>
#include <cstdio>
#include <tuple>
#include <utility>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "solver.h"
#include "solversystem.h"
#include "stencilincludes.h"
#include "symphas_b200.h"

namespace symphas_b200 {
namespace binding {

//! Precision and evaluation order of the handles created from now on.
struct settings {
  int dtype = SP_F64;         //!< SP_F64 or SP_F32
  int form = SP_FORM_EXACT;   //!< SP_FORM_EXACT (SymPhas's term order) or SP_FORM_FUSED
};
inline settings& options() {
  static settings s;
  return s;
}

//! One term of an equation: c * D^order(psi^pw[0] eta^pw[1]).
struct term {
  int order;
  int pw[2];
  double c;
};

//! Where reading an equation failed, or "" when it did not.
struct reader {
  std::vector<term> terms;
  std::string err;
  // the grid of every field the equation names (index = field)
  std::vector<const void*> grids;

  void fail(const std::string& s) {
    if (err.empty()) err = s;
  }
};

template <typename V>
double coeff_value(V const& v) {
  return double(expr::eval(v));
}

// one field factor of a monomial: its index and integer power
template <size_t I, typename BG, expr::exp_key_t X>
void factor(Term<Variable<I, NamedData<std::reference_wrapper<BG>>>, X> const& t, int (&pw)[2],
            reader& rd) {
  using key = expr::_Xk_t<X>;
  if (key::D != 1 || key::sign || key::N < 1 || key::N > 6) {
    rd.fail("a field is raised to a power other than 1..6");
    return;
  }
  if (I > 1) {
    rd.fail("more than two fields");
    return;
  }
  pw[I] += int(key::N);
  if (rd.grids.size() <= I) rd.grids.resize(I + 1, nullptr);
  rd.grids[I] = &static_cast<std::reference_wrapper<BG> const&>(t).get();
}
template <typename G, expr::exp_key_t X>
void factor(Term<G, X> const&, int (&)[2], reader& rd) {
  rd.fail("a term names data that is not a field of the model");
}

inline void factors(OpTermsList<> const&, int (&)[2], reader&) {}
template <typename T0, typename... Ts>
void factors(OpTermsList<T0, Ts...> const& l, int (&pw)[2], reader& rd) {
  factor(l.term, pw, rd);
  factors(static_cast<OpTermsList<Ts...> const&>(l), pw, rd);
}

// the terms of an expression, each scaled by `scale`, under `order`
template <typename V, typename... Gs, expr::exp_key_t... Xs>
void read(OpTerms<V, Term<Gs, Xs>...> const& e, double scale, int order, reader& rd) {
  term t{order, {0, 0}, scale * coeff_value(e.term)};
  factors(static_cast<OpTermsList<Term<Gs, Xs>...> const&>(e), t.pw, rd);
  rd.terms.push_back(t);
}
inline void read_list(OpAddList<> const&, double, int, reader&) {}
template <typename E0, typename... Es>
void read_list(OpAddList<E0, Es...> const& l, double scale, int order, reader& rd);
template <typename... Es>
void read(OpAdd<Es...> const& e, double scale, int order, reader& rd) {
  read_list(static_cast<OpAddList<Es...> const&>(e), scale, order, rd);
}
template <typename Dd, typename V, typename E, typename Sp>
void read(OpDerivative<Dd, V, E, Sp> const& d, double scale, int order, reader& rd) {
  using D = OpDerivative<Dd, V, E, Sp>;
  if (order != 0 || D::is_directional || D::axis != Axis::X || (D::order != 2 && D::order != 4)) {
    rd.fail("a derivative other than lap or bilap of a polynomial");
    return;
  }
  read(expr::get_enclosed_expression(d), scale * coeff_value(d.value), int(D::order), rd);
}
template <typename E>
void read(E const&, double, int, reader& rd) {
  rd.fail("an expression node other than sums, products of fields and lap/bilap");
}
template <typename E0, typename... Es>
void read_list(OpAddList<E0, Es...> const& l, double scale, int order, reader& rd) {
  read(l.term, scale, order, rd);
  read_list(static_cast<OpAddList<Es...> const&>(l), scale, order, rd);
}

//! The model the B200 library runs for the equations of every field, and its
//! coefficients; `why` says what did not match.
struct match_result {
  int model = -1;
  double coeff[8] = {1, 1, 1, 1, 1, 1, 1, 1};
  std::string why;
};

// coefficient of D^order(psi^a eta^b) in a list of terms (summed), and whether
// every term of the list is one of `allowed`
inline double coef(const std::vector<term>& ts, int order, int a, int b) {
  double c = 0.0;
  for (const term& t : ts)
    if (t.order == order && t.pw[0] == a && t.pw[1] == b) c += t.c;
  return c;
}
inline bool only(const std::vector<term>& ts, std::initializer_list<std::array<int, 3>> allowed) {
  for (const term& t : ts) {
    bool ok = false;
    for (const auto& a : allowed) ok |= t.order == a[0] && t.pw[0] == a[1] && t.pw[1] == a[2];
    if (!ok) return false;
  }
  return true;
}
inline bool same(double a, double b) { return std::fabs(a - b) <= 1e-12 * std::fmax(1.0, std::fabs(b)); }

inline match_result match(const std::vector<std::vector<term>>& eqs) {
  match_result r;
  if (eqs.size() == 1) {
    const auto& e = eqs[0];
    if (only(e, {{2, 1, 0}, {0, 1, 0}, {0, 3, 0}}) && coef(e, 2, 1, 0) != 0.0) {
      const double k = coef(e, 2, 1, 0), a = coef(e, 0, 1, 0), b = coef(e, 0, 3, 0);
      if (k == 1.0) {  // lap(psi) + c1 psi - c2 psi^3
        r.model = SP_MODEL_A;
        r.coeff[0] = a;
        r.coeff[1] = -b;
      } else if (same(b, -a) && a != 0.0) {  // M kappa lap(psi) + M psi - M psi^3
        r.model = SP_MODEL_AMK;
        r.coeff[0] = a;
        r.coeff[1] = k / a;
      } else {
        r.why = "lap, psi and psi^3 terms that are neither model A nor AMK";
      }
      return r;
    }
    if (only(e, {{4, 1, 0}, {2, 1, 0}, {2, 3, 0}}) && coef(e, 4, 1, 0) != 0.0) {
      const double k = coef(e, 4, 1, 0), a = coef(e, 2, 1, 0), b = coef(e, 2, 3, 0);
      if (k == -1.0) {  // -bilap(psi) - c1 lap(psi) + c2 lap(psi^3)
        r.model = SP_MODEL_B;
        r.coeff[0] = -a;
        r.coeff[1] = b;
      } else if (same(a, -b) && b != 0.0) {  // M (-kappa bilap + lap(psi^3) - lap(psi))
        r.model = SP_MODEL_BMK;
        r.coeff[0] = b;
        r.coeff[1] = -k / b;
      } else {
        r.why = "bilap, lap(psi) and lap(psi^3) terms that are neither model B nor BMK";
      }
      return r;
    }
    r.why = "terms outside models A, AMK, B and BMK";
    return r;
  }
  if (eqs.size() == 2) {
    const auto& p = eqs[0];
    const auto& q = eqs[1];
    if (only(p, {{4, 1, 0}, {2, 1, 0}, {2, 3, 0}, {2, 1, 2}}) &&
        only(q, {{2, 0, 1}, {0, 0, 1}, {0, 0, 3}, {0, 2, 1}})) {
      const double g = coef(p, 2, 1, 2);
      if (coef(p, 4, 1, 0) == -1.0 && coef(p, 2, 1, 0) == -1.0 && coef(p, 2, 3, 0) == 1.0 &&
          coef(q, 2, 0, 1) == 1.0 && coef(q, 0, 0, 1) == 1.0 && coef(q, 0, 0, 3) == -1.0 &&
          same(coef(q, 0, 2, 1), -g)) {
        r.model = SP_MODEL_C;
        r.coeff[0] = g / 2.0;  // gamma
        return r;
      }
    }
    r.why = "two fields that are not model C in the gamma form";
    return r;
  }
  r.why = "more than two fields";
  return r;
}

// stencil point sets of SymPhas's stencil types
template <typename Sp>
struct stencil_info {
  static constexpr bool ok = false;
};
template <size_t L, size_t G, size_t B>
struct stencil_info<Stencil2d2h<L, G, B>> {
  static constexpr bool ok = true;
  static constexpr int dim = 2, acc = 2, lp = int(L), gp = int(G), bp = int(B);
};
template <size_t L, size_t G, size_t B>
struct stencil_info<Stencil3d2h<L, G, B>> {
  static constexpr bool ok = true;
  static constexpr int dim = 3, acc = 2, lp = int(L), gp = int(G), bp = int(B);
};
template <size_t L, size_t G, size_t B>
struct stencil_info<Stencil2d4h<L, G, B>> {
  static constexpr bool ok = true;
  static constexpr int dim = 2, acc = 4, lp = int(L), gp = int(G), bp = int(B);
};

//! The GPU side of one model, shared by its systems.
struct device_model {
  sp_handle* h = nullptr;
  int nf = 0;
  std::vector<std::vector<term>> eqs;  // per field, read at the first equation()
  std::vector<bool> read_done;
  std::vector<void*> systems;          // SolverSystemFDB200<T, D>* per field
  double dt = std::nan("");
  match_result m;
  ~device_model() {
    if (h) sp_destroy(h);
  }
};

inline void check(int rc, sp_handle* h, const char* what) {
  if (rc != SP_OK) {
    std::string msg = std::string("symphas_b200: ") + what + ": " +
                      (h ? sp_last_error(h) : sp_create_error());
    throw std::runtime_error(msg);
  }
}

}  // namespace binding
}  // namespace symphas_b200

//! SymPhas's finite-difference solver system with its fields on the GPU: a
//! SolverSystemFD (host `values`, `dframe`, boundaries) plus the device side
//! of its model.
template <typename T, size_t D>
struct SolverSystemFDB200 : SolverSystemFD<T, D> {
  using SolverSystemFD<T, D>::SolverSystemFD;
  using field_type = T;
  static constexpr size_t field_dimension = D;
  std::shared_ptr<symphas_b200::binding::device_model> dev;

  //! The halo of the host copy is not maintained: the GPU keeps its own.
  void update(iter_type, double) {}

  //! Copy field `id` of the GPU into the interior of `values`.
  void download() {
    if (!dev || !dev->h) return;
    const int field = int(this->id);
    std::vector<T> in;
    const long long cnt = interior();
    std::vector<char> buf(size_t(cnt) * esz());
    symphas_b200::binding::check(sp_download(dev->h, 0, field, buf.data(), buf.size()), dev->h,
                                 "sp_download");
    for_interior([&](long long i, long long n) { this->values[n] = value_at(buf, i); });
  }
  //! Copy the interior of `values` to field `id` of the GPU.
  void upload() {
    const int field = int(this->id);
    const long long cnt = interior();
    std::vector<char> buf(size_t(cnt) * esz());
    for_interior([&](long long i, long long n) { store_at(buf, i, this->values[n]); });
    symphas_b200::binding::check(sp_upload(dev->h, 0, field, buf.data(), buf.size()), dev->h,
                                 "sp_upload");
  }

  long long interior() const {
    long long c = 1;
    for (size_t a = 0; a < D; ++a) c *= this->dims[a] - 2 * BOUNDARY_DEPTH;
    return c;
  }

 private:
  static size_t esz() { return symphas_b200::binding::options().dtype == SP_F32 ? 4 : 8; }
  static T value_at(const std::vector<char>& b, long long i) {
    if (esz() == 4) return T(reinterpret_cast<const float*>(b.data())[i]);
    return T(reinterpret_cast<const double*>(b.data())[i]);
  }
  static void store_at(std::vector<char>& b, long long i, T v) {
    if (esz() == 4)
      reinterpret_cast<float*>(b.data())[i] = float(v);
    else
      reinterpret_cast<double*>(b.data())[i] = double(v);
  }
  // f(compact index, storage index) over the interior, x fastest
  template <typename F>
  void for_interior(F f) const {
    const long long B = BOUNDARY_DEPTH;
    const long long lx = this->dims[0], ly = D > 1 ? this->dims[1] : 1;
    const long long nx = lx - 2 * B, ny = D > 1 ? ly - 2 * B : 1,
                    nz = D > 2 ? this->dims[2] - 2 * B : 1;
    long long i = 0;
    for (long long k = 0; k < nz; ++k)
      for (long long j = 0; j < ny; ++j)
        for (long long x = 0; x < nx; ++x, ++i)
          f(i, (x + B) + (D > 1 ? (j + B) * lx : 0) + (D > 2 ? (k + B) * lx * ly : 0));
  }
};

START_NEW_SOLVER_WITH_STENCIL(SolverFTB200)

double h_ = 1.0;  //!< grid spacing of the problem (the first system's x axis)

/*
 * one fused GPU step of every field of the model, from its first system (the
 * other systems' steps return: their fields were stepped with it)
 */
template <typename S>
void step(S& sys) const {
  auto& dm = *sys.dev;
  if (sys.id != 0) return;
  if (!(dm.dt == dt)) {
    symphas_b200::binding::check(sp_set_dt(dm.h, dt), dm.h, "sp_set_dt");
    dm.dt = dt;
  }
  symphas_b200::binding::check(sp_step(dm.h, 1), dm.h, "sp_step");
}

/*
 * the first call of each field reads its equation; once every field's is
 * read, the model is matched and the GPU handle created; later calls do
 * nothing (the fused step evaluates the equations)
 */
template <typename S, typename E>
inline void equation(std::pair<S, E>& r) const {
  auto& sys = r.first.get();
  using sys_t = std::decay_t<decltype(sys)>;
  if (sys.dev && sys.dev->h) return;
  symphas_b200::binding::reader rd;
  symphas_b200::binding::read(r.second, 1.0, 0, rd);
  if (!rd.err.empty())
    throw std::runtime_error("symphas_b200: the equation of field " + std::to_string(sys.id) +
                             " has " + rd.err);
  // every field the equation names shares one device model
  std::shared_ptr<symphas_b200::binding::device_model> dm = sys.dev;
  std::vector<sys_t*> named(rd.grids.size(), nullptr);
  for (size_t i = 0; i < rd.grids.size(); ++i)
    if (rd.grids[i]) {
      // the grid a field term names is the system itself (SymPhas's systems
      // are their grids, sol/inc/systemlib.h:228)
      using grid_t = BoundaryGrid<typename sys_t::field_type, sys_t::field_dimension>;
      named[i] = static_cast<sys_t*>(
          const_cast<grid_t*>(static_cast<const grid_t*>(rd.grids[i])));
      if (!dm) dm = named[i]->dev;
    }
  if (!dm) dm = std::make_shared<symphas_b200::binding::device_model>();
  const size_t nf = std::max(rd.grids.size(), size_t(sys.id) + 1);
  if (dm->eqs.size() < nf) {
    dm->eqs.resize(nf);
    dm->read_done.resize(nf, false);
    dm->systems.resize(nf, nullptr);
  }
  sys.dev = dm;
  dm->systems[sys.id] = &sys;
  for (size_t i = 0; i < named.size(); ++i)
    if (named[i]) {
      named[i]->dev = dm;
      dm->systems[i] = named[i];
    }
  dm->eqs[sys.id] = rd.terms;
  dm->read_done[sys.id] = true;
  for (size_t i = 0; i < nf; ++i)
    if (!dm->read_done[i]) return;  // the other fields' equations come next
  create(*dm, static_cast<sys_t*>(nullptr));
}

template <typename S, typename E>
inline void equation(std::pair<S, E>* r, len_type len) const {
  for (iter_type i = 0; i < len; ++i) equation(r[i]);
}

template <typename sys_t>
void create(symphas_b200::binding::device_model& dm, sys_t*) const {
  using info = symphas_b200::binding::stencil_info<stencil_t>;
  static_assert(info::ok, "SolverFTB200 takes Stencil2d2h, Stencil3d2h or Stencil2d4h");
  dm.nf = int(dm.eqs.size());
  dm.m = symphas_b200::binding::match(dm.eqs);
  if (dm.m.model < 0)
    throw std::runtime_error("symphas_b200: the model's equations are not built for the GPU: " +
                             dm.m.why);
  auto& s0 = *static_cast<sys_t*>(dm.systems[0]);
  constexpr size_t D = sys_t::field_dimension;
  sp_desc d{};
  d.dim = int(D);
  for (int a = 0; a < 3; ++a)
    d.n[a] = a < int(D) ? int(s0.dims[a] - 2 * BOUNDARY_DEPTH) : 1;
  d.dtype = symphas_b200::binding::options().dtype;
  d.model = dm.m.model;
  d.form = symphas_b200::binding::options().form;
  d.lap_pts = info::lp;
  d.gradlap_pts = info::gp;
  d.bilap_pts = info::bp;
  d.accuracy = info::acc;
  for (int s = 0; s < 2 * int(D); ++s) {
    const BoundaryType t = s0.types[s];
    if (t == BoundaryType::PERIODIC || t == BoundaryType::PERIODIC0 ||
        t == BoundaryType::PERIODIC3XY || t == BoundaryType::PERIODIC3XZ ||
        t == BoundaryType::PERIODIC3YZ) {
      d.boundary[s] = SP_PERIODIC;
    } else if (t == BoundaryType::DEFAULT && s0.boundaries[s]) {
      const symphas::b_element_type b = s0.boundaries[s]->get_parameters();
      if (b.tag[0] != BoundaryTag::CONSTANT)
        throw std::runtime_error("symphas_b200: only periodic and constant boundaries");
      d.boundary[s] = SP_DIRICHLET;
      d.boundary_value[s] = b.argc > 0 ? b.params[0] : 0.0;
    } else {
      throw std::runtime_error("symphas_b200: only periodic and constant boundaries");
    }
  }
  d.h = h_;
  d.dt = dt;
  for (int i = 0; i < 8; ++i) d.coeff[i] = dm.m.coeff[i];
  d.ncoeff = 8;
  d.batch = 1;
  symphas_b200::binding::check(sp_create(&d, &dm.h), nullptr, "sp_create");
  dm.dt = dt;
  for (int f = 0; f < dm.nf; ++f) static_cast<sys_t*>(dm.systems[f])->upload();
}

// the forward-Euler scheme of SolverFT: the equation as given, optimised
// (SolverFT::form_expr_one, examples/solvers/solverft.h:112-119)
template <size_t En, typename SS, typename S, typename E>
auto form_expr_one(SS&&, std::pair<S, E> const& e) const {
  auto [sys, equation] = e;
  auto eq_ft = expr::transform::optimize(expr::apply_operators(equation));
  expr::prune::update(eq_ft);
  return std::make_pair(sys, eq_ft);
}

static auto make_solver(symphas::problem_parameters_type const& parameters) {
  if (parameters.length()) {
    const double h = parameters.get_interval_data()[0].at(Axis::X).width();
    const size_t dim = parameters.get_dimension();
    std::vector<len_type> dims(dim);
    for (size_t i = 0; i < dim; ++i)
      dims[i] = parameters.get_interval_data()[0].at(symphas::index_to_axis(i)).get_count() +
                2 * BOUNDARY_DEPTH;
    auto s = this_type{dims.data(), h};
    s.h_ = h;
    return s;
  }
  return this_type{grid::dim_list(nullptr, 3), grid::h_list(nullptr, 3)};
}

template <typename G, typename E>
void evaluate_one(std::pair<G, E>&) const {
  throw std::runtime_error("symphas_b200: provisional variables are not built for the GPU");
}
template <typename G, typename E>
void evaluate_one(std::pair<G, E>&&) const {
  throw std::runtime_error("symphas_b200: provisional variables are not built for the GPU");
}
END_SOLVER

ASSOCIATE_SOLVER_SYSTEM_TYPE(SolverFTB200, SolverSystemFDB200)
SYMPHAS_SOLVER_SUPPORTED_TYPE(SolverFTB200, scalar_t)

namespace symphas_b200 {
namespace binding {

//! The matched model of a SolverFTB200 model, read from its equations without
//! touching the GPU (for checking what a MODEL maps to).
template <typename M>
match_result describe(M& model) {
  std::vector<std::vector<term>> eqs;
  std::string err;
  std::apply(
      [&](auto&... pairs) {
        ((
             [&] {
               reader rd;
               read(pairs.second, 1.0, 0, rd);
               if (!rd.err.empty() && err.empty()) err = rd.err;
               eqs.push_back(rd.terms);
             }()),
         ...);
      },
      model.equations);
  if (!err.empty()) {
    match_result r;
    r.why = "an equation has " + err;
    return r;
  }
  return match(eqs);
}

template <typename M, size_t... Is>
void sync_each(M& model, std::index_sequence<Is...>) {
  (model.template system<Is>().download(), ...);
}

//! Copy every field of a SolverFTB200 model from the GPU into its systems'
//! `values` (interior).
template <typename M>
void sync_to_host(M& model) {
  constexpr size_t n = std::tuple_size<std::decay_t<decltype(model.systems_tuple())>>::value;
  sync_each(model, std::make_index_sequence<n>{});
}

}  // namespace binding
}  // namespace symphas_b200
