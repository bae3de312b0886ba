/*
 * symphas_binding.cpp -- SymPhas's own models on the B200 through the
 * SymPhas-side binding (symphas_b200/binding/solverftb200.h), checked against
 * SymPhas's own CPU SolverFT.  Built by oracle/ref.mk against the SymPhas
 * sources (test infrastructure); tests/test_symphas_binding.py runs it.
 *
 *   symphas_binding match    which B200 model every MODEL below maps to (no GPU)
 *   symphas_binding run      the models through model_iteration's loop on the
 *                            GPU and on SymPhas's CPU solver; exit 0 when they agree
 */
#include <cstdio>
#include <cstring>
#include <vector>

#include "solverft.h"
#include "modelmacros.h"
#include "../../symphas_b200/binding/solverftb200.h"

#define psi op(1)
#define dpsi dop(1)
#define eta op(2)
#define deta dop(2)

// SymPhas's models A and B as examples/models/modeldefinitions.h:26-33 write them
MODEL(MA, (SCALAR), EVOLUTION(dpsi = lap(psi) + (c(1) - c(2) * psi * psi) * psi))
MODEL(MB, (SCALAR), EVOLUTION(dpsi = -bilap(psi) - lap((c(1) - c(2) * psi * psi) * psi)))
// model C in the gamma form, gamma = c(1)
MODEL(MCG, (SCALARS(2)),
      EVOLUTION(dpsi = lap(-psi + psi * psi * psi + 2_n * c(1) * psi * eta * eta - lap(psi)),
                deta = eta - eta * eta * eta - 2_n * c(1) * psi * psi * eta + lap(eta)))
MODEL(AMK, (SCALAR), EVOLUTION(dpsi = c(1) * (c(2) * lap(psi) - psi * psi * psi + psi)))
MODEL(BMK, (SCALAR), EVOLUTION(dpsi = c(1) * lap(psi * psi * psi - psi - c(2) * lap(psi))))
// a model the GPU library has no kernel for (a psi^2 term)
MODEL(QUAD, (SCALAR), EVOLUTION(dpsi = lap(psi) + c(1) * psi * psi))

#undef psi
#undef dpsi
#undef eta
#undef deta

// SymPhas's initial-expression registry lives in its modules library, which
// is not built here; no model below names an initial expression
template <size_t D, typename T>
bool match_init_expr(const char*, Axis, T*, grid::region_interval<D> const&,
                     symphas::interval_data_type const&, double const*, size_t) {
  return false;
}
template bool match_init_expr<2, double>(const char*, Axis, double*,
                                         grid::region_interval<2> const&,
                                         symphas::interval_data_type const&, double const*,
                                         size_t);
template bool match_init_expr<3, double>(const char*, Axis, double*,
                                         grid::region_interval<3> const&,
                                         symphas::interval_data_type const&, double const*,
                                         size_t);

namespace {

constexpr int BD = BOUNDARY_DEPTH;

// n + 6 points of spacing h per axis (the halo counts toward the points with
// SymPhas's default params::extend_boundary = false), periodic sides, a
// constant zero initial field (the seeded field is written in afterwards)
symphas::problem_parameters_type make_params(int dim, const int* n, double h, size_t nf) {
  symphas::problem_parameters_type pp{nf};
  symphas::interval_data_type vdata(dim);
  for (int a = 0; a < dim; ++a)
    vdata[symphas::index_to_axis(a)] = symphas::interval_element_type(0.0, (n[a] + 2 * BD - 1) * h, h);
  symphas::b_data_type bdata(dim, BoundaryType::PERIODIC);
  symphas::init_data_type tdata(Inside::CONSTANT, {0.0});
  std::vector<symphas::b_data_type> bv(nf, bdata);
  std::vector<symphas::interval_data_type> vv(nf, vdata);
  std::vector<symphas::init_data_type> tv(nf, tdata);
  pp.set_boundary_data(bv.data(), nf);
  pp.set_interval_data(vv.data(), nf);
  pp.set_initial_data(tv.data(), nf);
  return pp;
}

// SplitMix64 counter stream, value(i) = lo + (hi - lo) u53 (the project's seeded init)
double seeded(uint64_t seed, long long i, double lo, double hi) {
  uint64_t z = seed + uint64_t(i + 1) * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  return lo + (hi - lo) * (double(z >> 11) * (1.0 / 9007199254740992.0));
}

template <typename Sys>
void fill(Sys& sys, int dim, uint64_t seed, double lo, double hi) {
  const long long lx = sys.dims[0], ly = sys.dims[1];
  const long long nx = lx - 2 * BD, ny = ly - 2 * BD, nz = dim == 3 ? sys.dims[2] - 2 * BD : 1;
  long long i = 0;
  for (long long k = 0; k < nz; ++k)
    for (long long j = 0; j < ny; ++j)
      for (long long x = 0; x < nx; ++x, ++i)
        sys.values[(x + BD) + (j + BD) * lx + (dim == 3 ? (k + BD) * lx * ly : 0)] =
            seeded(seed, i, lo, hi);
}

// model_iteration's loop (modules-models.h:435-467): update, equation, step
template <typename M>
void iterate(M& m, double dt, int steps) {
  double t = 0.0;
  for (int s = 0; s < steps; ++s) {
    m.update(t);
    m.equation();
    m.step(dt);
    t += dt;
  }
}

template <typename SysA, typename SysB>
double compare(SysA const& a, SysB const& b, int dim, double& scale) {
  const long long lx = a.dims[0], ly = a.dims[1];
  const long long nx = lx - 2 * BD, ny = ly - 2 * BD, nz = dim == 3 ? a.dims[2] - 2 * BD : 1;
  double worst = 0.0;
  for (long long k = 0; k < nz; ++k)
    for (long long j = 0; j < ny; ++j)
      for (long long x = 0; x < nx; ++x) {
        const long long n = (x + BD) + (j + BD) * lx + (dim == 3 ? (k + BD) * lx * ly : 0);
        worst = std::max(worst, std::fabs(a.values[n] - b.values[n]));
        scale = std::max(scale, std::fabs(b.values[n]));
      }
  return worst;
}

template <typename M, size_t... Is>
void seed_all(M& m, int dim, std::index_sequence<Is...>) {
  (fill(m.template system<Is>(), dim, 1000 + Is, -0.1 + 0.05 * Is, 0.1), ...);
}

template <typename MA, typename MB, size_t... Is>
double compare_all(MA& a, MB& b, int dim, double& scale, std::index_sequence<Is...>) {
  double worst = 0.0;
  ((worst = std::max(worst, compare(a.template system<Is>(), b.template system<Is>(), dim, scale))),
   ...);
  return worst;
}

// one model on both solvers: the same initial field, `steps` iterations, and
// the largest difference relative to the largest value
template <template <size_t, typename> class MT, size_t D, typename Sp, size_t NF>
int run_case(const char* name, const int* n, double h, double dt, int steps,
             std::vector<double> coeff, double tol) {
  auto pp = make_params(int(D), n, h, NF);
  MT<D, SolverFT<Sp>> cpu(coeff.data(), coeff.size(), pp);
  MT<D, SolverFTB200<Sp>> gpu(coeff.data(), coeff.size(), pp);
  int rc = 0;
  double worst = 0.0, scale = 0.0;
  seed_all(cpu, int(D), std::make_index_sequence<NF>{});
  seed_all(gpu, int(D), std::make_index_sequence<NF>{});
  iterate(cpu, dt, steps);
  iterate(gpu, dt, steps);
  symphas_b200::binding::sync_to_host(gpu);
  worst = compare_all(gpu, cpu, int(D), scale, std::make_index_sequence<NF>{});
  const double rel = worst / (scale > 0 ? scale : 1.0);
  const bool ok = rel <= tol;
  std::printf("%-28s %d steps: max |gpu - symphas| / max |symphas| = %.3g (bound %.0e) %s\n",
              name, steps, rel, tol, ok ? "ok" : "FAIL");
  if (!ok) rc = 1;
  return rc;
}

template <typename M>
void print_match(const char* name, M& m) {
  const auto r = symphas_b200::binding::describe(m);
  if (r.model < 0) {
    std::printf("%s: refused (%s)\n", name, r.why.c_str());
    return;
  }
  std::printf("%s: model %d coeff %.17g %.17g\n", name, r.model, r.coeff[0], r.coeff[1]);
}

}  // namespace

int main(int argc, char** argv) {
  const char* mode = argc > 1 ? argv[1] : "match";
  const int n2[3] = {48, 40, 1}, n3[3] = {20, 16, 12};
  if (!std::strcmp(mode, "match")) {
    std::vector<double> c = {0.7, 1.3};
    auto p2 = make_params(2, n2, 1.0, 1), p22 = make_params(2, n2, 1.0, 2);
    model_MA_t<2, SolverFTB200<Stencil2d2h<5, 6, 13>>> ma(c.data(), 2, p2);
    print_match("MA", ma);
    model_MB_t<2, SolverFTB200<Stencil2d2h<5, 6, 13>>> mb(c.data(), 2, p2);
    print_match("MB", mb);
    std::vector<double> g = {0.5};
    model_MCG_t<2, SolverFTB200<Stencil2d2h<5, 6, 13>>> mc(g.data(), 1, p22);
    print_match("MCG", mc);
    std::vector<double> mk = {1.7, 0.6};
    model_AMK_t<2, SolverFTB200<Stencil2d2h<5, 6, 13>>> amk(mk.data(), 2, p2);
    print_match("AMK", amk);
    model_BMK_t<2, SolverFTB200<Stencil2d2h<5, 6, 13>>> bmk(mk.data(), 2, p2);
    print_match("BMK", bmk);
    model_QUAD_t<2, SolverFTB200<Stencil2d2h<5, 6, 13>>> quad(c.data(), 1, p2);
    print_match("QUAD", quad);
    return 0;
  }
  // SymPhas's configurations and models through the binding, FP64 in
  // SymPhas's term order: bit-identical for unit coefficients (model A, B
  // and the configurations), within 1e-12 where SymPhas folds coefficients
  int rc = 0;
  const int n64[3] = {64, 64, 1}, n32[3] = {32, 32, 32};
  rc |= run_case<model_MA_t, 2, Stencil2d2h<5, 6, 13>, 1>("model A 2D 64^2 (config)", n64, 0.5,
                                                          0.01, 1000, {1.0, 1.0}, 0.0);
  rc |= run_case<model_MB_t, 3, Stencil3d2h<7, 10, 25>, 1>("model B 3D 32^3", n32, 1.0, 0.005,
                                                           200, {1.0, 1.0}, 0.0);
  rc |= run_case<model_MA_t, 2, Stencil2d2h<5, 6, 13>, 1>("model A coefficients", n2, 0.5, 0.01,
                                                          200, {0.7, 1.3}, 0.0);
  rc |= run_case<model_MB_t, 2, Stencil2d2h<5, 6, 13>, 1>("model B coefficients", n2, 1.0,
                                                          0.005, 200, {0.7, 1.3}, 1e-12);
  rc |= run_case<model_AMK_t, 3, Stencil3d2h<7, 10, 25>, 1>("AMK 3D", n3, 1.0, 0.01, 100,
                                                            {1.7, 0.6}, 1e-12);
  rc |= run_case<model_BMK_t, 2, Stencil2d2h<5, 6, 13>, 1>("BMK 2D", n2, 1.0, 0.005, 100,
                                                           {1.7, 0.6}, 1e-12);
  rc |= run_case<model_MCG_t, 3, Stencil3d2h<7, 10, 25>, 2>("model C 3D", n3, 1.0, 0.005, 100,
                                                            {0.5}, 1e-12);
  rc |= run_case<model_MB_t, 2, Stencil2d4h<9, 14, 21>, 1>("model B Stencil2d4h", n2, 1.0,
                                                           0.002, 100, {1.0, 1.0}, 0.0);
  return rc;
}
