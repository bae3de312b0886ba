/*
 * symphas_ref.cpp -- the C entry points of oracle/_ref/libsymphas_ref.so:
 * SymPhas's own CPU SolverFT (see symphas_ref.h).  TEST INFRASTRUCTURE ONLY:
 * tests/ and bench.py's reference arm call it, the product never does.
 */
#include "symphas_ref.h"

#include <thread>

// The initial-expression registry lives in SymPhas's modules library, which
// is not built here; no model below names an initial expression.
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

namespace symref {
std::vector<entry>& registry() {
  static std::vector<entry> r;
  return r;
}
}  // namespace symref

namespace {
const symref::entry* find(const symref_desc* d, bool models) {
  const int acc = d->acc == 4 ? 4 : 2;
  for (const auto& e : symref::registry())
    if (e.e_dim == d->dim && e.e_acc == acc && e.e_lap == d->lap_pts && e.e_gradlap == d->gradlap_pts &&
        e.e_bilap == d->bilap_pts && (models ? e.e_models != nullptr : e.e_ops != nullptr))
      return &e;
  return nullptr;
}
bool is_op(int model) { return model >= REF_OP_LAP && model <= REF_OP_LAPCUBE; }
}  // namespace

extern "C" {

// 1 when the library holds the combination of model (or operator) and
// stencil that *d names, else 0
int symref_available(const symref_desc* d) {
  return find(d, !is_op(d->model)) != nullptr ? 1 : 0;
}

// fields of the model (interior, x-fastest, back to back) advanced in place
// by nsteps SolverFT iterations; 0 on success, 1 for a combination not built,
// 2 when SymPhas's storage does not have the requested interior, 3 on a C++
// exception
int symref_run(const symref_desc* d, double* fields, int nsteps) {
  if (is_op(d->model) || nsteps < 1) return 1;
  const symref::entry* e = find(d, true);
  if (!e) return 1;
  try {
    std::vector<double> in(fields, fields + (d->model == REF_MODEL_C ? 2 : 1) *
                                                 symref::interior_count(*d));
    return e->e_models(*d, in.data(), fields, nsteps);
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "symref_run: %s\n", ex.what());
    return 3;
  }
}

// the right-hand side once (update(), equation(): each system's dframe) of a
// model, or an operator over the field; same status codes as symref_run
int symref_rhs(const symref_desc* d, const double* fields, double* rhs) {
  const symref::entry* e = find(d, !is_op(d->model));
  if (!e) return 1;
  try {
    return is_op(d->model) ? e->e_ops(*d, fields, rhs) : e->e_models(*d, fields, rhs, 0);
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "symref_rhs: %s\n", ex.what());
    return 3;
  }
}

// a model held between calls, built from the fields (interior, back to back):
// NULL for a combination not built or a storage of other extents
void* symref_create(const symref_desc* d, const double* fields) {
  if (is_op(d->model)) return nullptr;
  const symref::entry* e = find(d, true);
  if (!e) return nullptr;
  try {
    return e->e_create(*d, fields);
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "symref_create: %s\n", ex.what());
    return nullptr;
  }
}

void symref_step(void* h, int nsteps) { static_cast<symref::system_base*>(h)->step(nsteps); }

void symref_get(void* h, double* fields) { static_cast<symref::system_base*>(h)->get(fields); }

void symref_destroy(void* h) { delete static_cast<symref::system_base*>(h); }

// nsteps iterations of each of `count` independent models, the models spread
// over `threads` host threads (each model on one thread, as SymPhas runs one
// model)
void symref_step_many(void** hs, int count, int nsteps, int threads) {
  if (threads < 1) threads = 1;
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([=] {
      for (int i = t; i < count; i += threads) symref_step(hs[i], nsteps);
    });
  for (auto& th : pool) th.join();
}
}

