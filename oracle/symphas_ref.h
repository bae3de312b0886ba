/*
 * symphas_ref.h -- SymPhas's own CPU SolverFT behind a C ABI, for pinning
 * the oracle (spo.c).
 *
 * TEST INFRASTRUCTURE ONLY.  This header and the ref_*.cpp files are compiled by oracle/ref.mk against
 * the SymPhas headers and sources where they lie (nothing of SymPhas is
 * copied into this repository); the result, oracle/_ref/libsymphas_ref.so, is
 * called by tests/ and by bench.py's reference arm, and never by the product.
 *
 * Every model below is a SymPhas MODEL(...) definition and runs through
 * SymPhas's own types end to end: model_NAME_t<D, SolverFT<Stencil...>>
 * (sol/inc/modelmacros.h:597-626), its coefficient constructor
 * (sol/inc/model.h:100-128), and the loop of model_iteration
 * (modules-models.h:435-467: update(time), equation(), step(dt)).  The
 * operator checks evaluate SymPhas's stencil functors directly
 * (Stencil<Sp>::laplacian / bilaplacian / gradlaplacian with the strides of
 * applied_*, sol/inc/stencil.h:130-159) over a field whose halo SymPhas's
 * own boundary update filled.
 *
 * Layout of the descriptor: the oracle's spo_desc (oracle/spo.c), so the
 * tests hand both the same inputs.  Field arrays are the interior only,
 * x-fastest, fields back to back; the driver copies them into SymPhas's
 * storage at (k + 3) Lx Ly + (j + 3) Lx + (i + 3) (BOUNDARY_DEPTH 3,
 * datatypes/inc/gridinfo.h:46).  Each axis is given n + 6 points with
 * params::extend_boundary left at its default (false, lib/src/params.cpp:90),
 * so the halo counts toward the points (sol/inc/boundarysystem.h:198-207)
 * and the interior has exactly n.  With extend_boundary set instead, SymPhas
 * sizes the temporaries of derivatives of expressions (OpDerivative::allocate,
 * sym/inc/expressionderivatives.h:1557-1563) by the interval's point count,
 * the interior, while it fills and reads them over the storage: a heap
 * overflow (found under AddressSanitizer on model B with coefficients).
 */
#include <cstdio>
#include <cstring>
#include <exception>
#include <type_traits>
#include <utility>
#include <vector>

#include "solverft.h"
#include "modelmacros.h"

extern "C" {
typedef struct symref_desc {
  int dim;
  int n[3];
  int model;
  int lap_pts, gradlap_pts, bilap_pts;
  double h, dt;
  double c[8];
  int bc[6];
  double bcv[6];
  int acc;
} symref_desc;
}

// model ids: those of the oracle (spo.c)
enum {
  REF_MODEL_A = 0,
  REF_MODEL_B = 1,
  REF_MODEL_C = 2,
  REF_MODEL_AMK = 3,
  REF_MODEL_BMK = 4,
  REF_MODEL_MBB = 5,
  REF_OP_LAP = 10,
  REF_OP_BILAP = 11,
  REF_OP_GRADLAP = 12,
  REF_OP_LAPCUBE = 13,
};

#define psi op(1)
#define dpsi dop(1)
#define eta op(2)
#define deta dop(2)

// SymPhas's models A and B as examples/models/modeldefinitions.h:26-33 define them
MODEL(REFMA, (SCALAR), EVOLUTION(dpsi = lap(psi) + (c(1) - c(2) * psi * psi) * psi))
MODEL(REFMB, (SCALAR),
      EVOLUTION(dpsi = -bilap(psi) - lap((c(1) - c(2) * psi * psi) * psi)))
// model C in the gamma form of the ensemble configurations:
// d psi = lap(-psi + psi^3 + 2 gamma psi eta^2 - lap psi),
// d eta = eta - eta^3 - 2 gamma psi^2 eta + lap eta, gamma = c(1)
MODEL(REFMC, (SCALARS(2)),
      EVOLUTION(dpsi = lap(-psi + psi * psi * psi + 2_n * c(1) * psi * eta * eta - lap(psi)),
                deta = eta - eta * eta * eta - 2_n * c(1) * psi * psi * eta + lap(eta)))
// models A and B with a mobility M = c(1) and a gradient coefficient kappa = c(2)
MODEL(REFAMK, (SCALAR), EVOLUTION(dpsi = c(1) * (c(2) * lap(psi) - psi * psi * psi + psi)))
MODEL(REFBMK, (SCALAR),
      EVOLUTION(dpsi = c(1) * lap(psi * psi * psi - psi - c(2) * lap(psi))))
// SymPhas's MBB (examples/models/modeldefinitions.h:152-156): a provisional variable
MODEL(REFMBB, (SCALAR),
      PROVISIONAL_DEF((SCALAR), var(1) <= -(c(1) - lit(4.) * c(2) * psi * psi) * psi)
          EVOLUTION(dpsi = -bilap(psi) + lap(var(1))))
// operator checks
MODEL(REFOPLAP, (SCALAR), EVOLUTION(dpsi = lap(psi)))
MODEL(REFOPBILAP, (SCALAR), EVOLUTION(dpsi = bilap(psi)))
MODEL(REFOPLAPCUBE, (SCALAR), EVOLUTION(dpsi = lap(psi * psi * psi)))

#undef psi
#undef dpsi
#undef eta
#undef deta

namespace symref {

constexpr int BD = 3;

struct system_base;
using models_fn = int (*)(const symref_desc&, const double*, double*, int);
using ops_fn = int (*)(const symref_desc&, const double*, double*);
using create_fn = system_base* (*)(const symref_desc&, const double*);
struct entry {
  int e_dim, e_acc, e_lap, e_gradlap, e_bilap;
  models_fn e_models;
  ops_fn e_ops;
  create_fn e_create;
};
// every stencil a translation unit instantiated, filled at load time
std::vector<entry>& registry();
struct reg {
  reg(int dim, int acc, int l, int g, int b, models_fn m, ops_fn o, create_fn c) {
    registry().push_back(entry{dim, acc, l, g, b, m, o, c});
  }
};

inline long interior_count(const symref_desc& d) {
  return long(d.n[0]) * d.n[1] * (d.dim == 3 ? d.n[2] : 1);
}

// problem parameters: n + 6 points of spacing h per axis, the oracle's boundary
// per side (LEFT RIGHT TOP BOTTOM FRONT BACK), a constant zero initial field
// (replaced by the caller's values before the first step)
inline symphas::problem_parameters_type make_params(const symref_desc& d, size_t nf) {
  symphas::problem_parameters_type pp{nf};
  symphas::interval_data_type vdata(d.dim);
  for (int a = 0; a < d.dim; ++a) {
    symphas::interval_element_type iv(0.0, (d.n[a] + 2 * BD - 1) * d.h, d.h);
    vdata[symphas::index_to_axis(a)] = iv;
  }
  // each side copy-constructed into the map: b_element_type's assignment and
  // move lose the parameter count (its swap exchanges first.argc with itself,
  // datatypes/inc/boundary.h:288-294), and the shorthand
  // BoundaryTag::CONSTANT << value never copies the value into the
  // boundary_info it builds (datatypes/inc/boundary.h:139-142), so a constant
  // side set by `bdata[side] = BoundaryTag::CONSTANT << v` holds 0
  symphas::b_data_type bdata;
  const Side sides[6] = {Side::LEFT, Side::RIGHT, Side::TOP, Side::BOTTOM, Side::FRONT, Side::BACK};
  for (int s = 0; s < 2 * d.dim; ++s) {
    const symphas::b_element_type side =
        d.bc[s] == 1 ? symphas::b_element_type(BoundaryType::DEFAULT,
                                               {BoundaryTag::CONSTANT, BoundaryTag::NONE},
                                               &d.bcv[s], 1)
                     : symphas::b_element_type(BoundaryType::PERIODIC,
                                               {BoundaryTag::NONE, BoundaryTag::NONE}, nullptr, 0);
    bdata.emplace(std::piecewise_construct, std::forward_as_tuple(sides[s]),
                  std::forward_as_tuple(side));
  }
  symphas::init_data_type tdata(Inside::CONSTANT, {0.0});
  std::vector<symphas::b_data_type> bv(nf, bdata);
  std::vector<symphas::interval_data_type> vv(nf, vdata);
  std::vector<symphas::init_data_type> tv(nf, tdata);
  pp.set_boundary_data(bv.data(), nf);
  pp.set_interval_data(vv.data(), nf);
  pp.set_initial_data(tv.data(), nf);
  pp.set_time_step(d.dt);
  return pp;
}

template <typename Sys>
bool dims_match(const symref_desc& d, Sys const& sys) {
  for (int a = 0; a < d.dim; ++a)
    if (sys.dims[a] != d.n[a] + 2 * BD) return false;
  return true;
}

template <typename Sys>
long storage_index(const symref_desc& d, Sys const& sys, long i, long j, long k) {
  const long lx = sys.dims[0], ly = sys.dims[1];
  return (i + BD) + (j + BD) * lx + (d.dim == 3 ? (k + BD) * lx * ly : 0);
}

template <typename Sys>
void copy_in(const symref_desc& d, Sys& sys, const double* src) {
  const long nz = d.dim == 3 ? d.n[2] : 1;
  for (long k = 0; k < nz; ++k)
    for (long j = 0; j < d.n[1]; ++j)
      for (long i = 0; i < d.n[0]; ++i)
        sys.values[storage_index(d, sys, i, j, k)] = src[(k * d.n[1] + j) * d.n[0] + i];
}

template <typename Arr, typename Sys>
void copy_out(const symref_desc& d, Sys const& sys, Arr const& from, double* dst) {
  const long nz = d.dim == 3 ? d.n[2] : 1;
  for (long k = 0; k < nz; ++k)
    for (long j = 0; j < d.n[1]; ++j)
      for (long i = 0; i < d.n[0]; ++i)
        dst[(k * d.n[1] + j) * d.n[0] + i] = from[iter_type(storage_index(d, sys, i, j, k))];
}

template <size_t NF, typename M, size_t... Is>
bool load_fields(const symref_desc& d, M& model, const double* fields, std::index_sequence<Is...>) {
  const long cnt = interior_count(d);
  bool ok = (dims_match(d, model.template system<Is>()) && ...);
  if (ok) (copy_in(d, model.template system<Is>(), fields + Is * cnt), ...);
  return ok;
}

template <typename M, size_t... Is>
void store_fields(const symref_desc& d, M& model, double* fields, bool dframe,
                  std::index_sequence<Is...>) {
  const long cnt = interior_count(d);
  if (dframe)
    (copy_out(d, model.template system<Is>(), model.template system<Is>().dframe,
              fields + Is * cnt),
     ...);
  else
    (copy_out(d, model.template system<Is>(), model.template system<Is>().values,
              fields + Is * cnt),
     ...);
}

// A SymPhas model held between calls (bench.py's reference arm times its
// steps without the construction): one MODEL type on one stencil, its fields
// loaded from the caller's interior arrays.
struct system_base {
  virtual ~system_base() = default;
  // advance by n SolverFT iterations (the loop of model_iteration)
  virtual void step(int n) = 0;
  // the fields (interior, back to back) after a last update(), as
  // find_solution leaves them
  virtual void get(double* out) = 0;
  // update() and equation() once; each system's dframe into out
  virtual void rhs(double* out) = 0;
};

inline symphas::problem_parameters_type default_params(const symref_desc& d, size_t nf) {
  params::extend_boundary = false;
  return make_params(d, nf);
}

template <template <size_t, typename> class MT, size_t D, typename Sp, size_t NF>
struct system : system_base {
  using model_type = MT<D, SolverFT<Sp>>;
  symref_desc d;
  symphas::problem_parameters_type pp;
  model_type model;
  double t = 0.0;
  bool ok;

  system(const symref_desc& d0, const double* in)
      : d(d0), pp(default_params(d0, NF)), model(d0.c, 8, pp) {
    ok = load_fields<NF>(d, model, in, std::make_index_sequence<NF>{});
  }
  void step(int n) override {
    for (int s = 0; s < n; ++s) {
      model.update(t);
      model.equation();
      model.step(d.dt);
      t += d.dt;
    }
  }
  void get(double* out) override {
    model.update(t);
    store_fields(d, model, out, false, std::make_index_sequence<NF>{});
  }
  void rhs(double* out) override {
    model.update(t);
    model.equation();
    store_fields(d, model, out, true, std::make_index_sequence<NF>{});
  }
};

template <template <size_t, typename> class MT, size_t D, typename Sp, size_t NF>
system_base* make_system(const symref_desc& d, const double* in) {
  auto* s = new system<MT, D, Sp, NF>(d, in);
  if (!s->ok) {
    delete s;
    return nullptr;
  }
  return s;
}

// steps > 0: advance the fields by that many SolverFT iterations.  steps ==
// 0: one update() and equation(), then the right-hand side (each system's
// dframe) is written to out.
template <template <size_t, typename> class MT, size_t D, typename Sp, size_t NF>
int run(const symref_desc& d, const double* in, double* out, int steps) {
  system<MT, D, Sp, NF> s(d, in);
  if (!s.ok) return 2;
  if (steps == 0) {
    s.rhs(out);
  } else {
    s.step(steps);
    s.get(out);
  }
  return 0;
}

// the x component of gradlap: SymPhas's functor at every interior site of a
// field whose halo SymPhas's boundary update filled (the strides of
// applied_gradlaplacian<Axis::X>, sol/inc/stencil.h:150-156)
template <typename R>
double first_component(R const& r) {
  if constexpr (std::is_arithmetic_v<R>)
    return r;
  else
    return r[0];
}

template <size_t D, typename Sp>
int gradlap_x(const symref_desc& d, const double* in, double* out) {
  params::extend_boundary = false;
  auto pp = make_params(d, 1);
  model_REFOPLAP_t<D, SolverFT<Sp>> model(d.c, 8, pp);
  auto& sys = model.template system<0>();
  if (!dims_match(d, sys)) return 2;
  copy_in(d, sys, in);
  model.update(0.0);
  len_type dims[D];
  for (size_t a = 0; a < D; ++a) dims[a] = sys.dims[a];
  Sp st(dims, d.h);
  len_type stride[D];
  grid::get_stride<Axis::X>(stride, dims);
  const long nz = d.dim == 3 ? d.n[2] : 1;
  for (long k = 0; k < nz; ++k)
    for (long j = 0; j < d.n[1]; ++j)
      for (long i = 0; i < d.n[0]; ++i) {
        const long n = storage_index(d, sys, i, j, k);
        out[(k * d.n[1] + j) * d.n[0] + i] =
            first_component(st.gradlaplacian(sys.values + n, stride));
      }
  return 0;
}

template <size_t D, typename Sp>
system_base* create_model(const symref_desc& d, const double* in) {
  switch (d.model) {
    case REF_MODEL_A: return make_system<model_REFMA_t, D, Sp, 1>(d, in);
    case REF_MODEL_B: return make_system<model_REFMB_t, D, Sp, 1>(d, in);
    case REF_MODEL_C: return make_system<model_REFMC_t, D, Sp, 2>(d, in);
    case REF_MODEL_AMK: return make_system<model_REFAMK_t, D, Sp, 1>(d, in);
    case REF_MODEL_BMK: return make_system<model_REFBMK_t, D, Sp, 1>(d, in);
    case REF_MODEL_MBB: return make_system<model_REFMBB_t, D, Sp, 1>(d, in);
    default: return nullptr;
  }
}

template <size_t D, typename Sp>
int dispatch_model(const symref_desc& d, const double* in, double* out, int steps) {
  switch (d.model) {
    case REF_MODEL_A: return run<model_REFMA_t, D, Sp, 1>(d, in, out, steps);
    case REF_MODEL_B: return run<model_REFMB_t, D, Sp, 1>(d, in, out, steps);
    case REF_MODEL_C: return run<model_REFMC_t, D, Sp, 2>(d, in, out, steps);
    case REF_MODEL_AMK: return run<model_REFAMK_t, D, Sp, 1>(d, in, out, steps);
    case REF_MODEL_BMK: return run<model_REFBMK_t, D, Sp, 1>(d, in, out, steps);
    case REF_MODEL_MBB: return run<model_REFMBB_t, D, Sp, 1>(d, in, out, steps);
    default: return 1;
  }
}

template <size_t D, typename Sp>
int models(const symref_desc& d, const double* in, double* out, int steps) {
  return dispatch_model<D, Sp>(d, in, out, steps);
}
template <size_t D, typename Sp>
int ops(const symref_desc& d, const double* in, double* out) {
  switch (d.model) {
    case REF_OP_LAP: return run<model_REFOPLAP_t, D, Sp, 1>(d, in, out, 0);
    case REF_OP_BILAP: return run<model_REFOPBILAP_t, D, Sp, 1>(d, in, out, 0);
    case REF_OP_LAPCUBE: return run<model_REFOPLAPCUBE_t, D, Sp, 1>(d, in, out, 0);
    case REF_OP_GRADLAP: return gradlap_x<D, Sp>(d, in, out);
    default: return 1;
  }
}

}  // namespace symref

// register SymPhas's models (M = 1) and/or the operator checks (O = 1) on one
// stencil type, e.g. SYMREF_REGISTER(r0, 2, 2, Stencil2d2h, 5, 6, 13, 1, 1)
#define SYMREF_REGISTER(NAME, D, ACC, SP, L, G, B, M, O)                                   \
  static symref::reg NAME(D, ACC, L, G, B, (M) ? &symref::models<D, SP<L, G, B>> : nullptr, \
                          (O) ? &symref::ops<D, SP<L, G, B>> : nullptr,                     \
                          (M) ? &symref::create_model<D, SP<L, G, B>> : nullptr);
