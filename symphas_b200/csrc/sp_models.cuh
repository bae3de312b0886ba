/*
 * sp_models.cuh -- the built-in models, each in two forms.
 *
 * EXACT form: the term order SymPhas prints for the model's optimised scheme
 * (SolverFT::form_expr_one, examples/solvers/solverft.h:112-119), as a right
 * fold; compiled without FMA contraction it reproduces the CPU solver bit for
 * bit in FP64.
 *
 * FUSED form: the same right-hand side rewritten with exact identities of the
 * discrete operators so that one kernel pass does less work:
 *   bilap = lap o lap for the point pairs (5,13) in 2D and (7,25) in 3D,
 *   lap(a) + lap(b) = lap(a + b),
 * and the operand of the outer lap is staged once per site in shared memory.
 * It differs from the exact form only by rounding.
 *
 * Model definitions follow examples/models/modeldefinitions.h (MA :43-46,
 * MB :48-51); model C has the coupling 2*gamma*psi*eta^2 instead of the
 * reference's MC (:61-68); AMK/BMK carry a mobility M = c(1) and gradient
 * coefficient kappa = c(2).
 */
#pragma once

#include "sp_expr.cuh"

namespace sp {
namespace models {

using namespace sp::ex;

constexpr Var<1> psi{};
constexpr Var<2> eta{};

// --- model A: dpsi = lap(psi) + (c1 - c2 psi^2) psi; scheme V^2(psi) - psi^3 + psi
inline constexpr auto a_exact() {
  return make_model<1, 0>(lap(psi) + (-(c<2>() * power<3>(psi)) + c<1>() * psi));
}
inline constexpr auto a_fused() {
  return make_model<1, 0>(lap(psi) + (c<1>() * psi - c<2>() * power<3>(psi)));
}

// --- model B: dpsi = -bilap(psi) - lap((c1 - c2 psi^2) psi);
//     scheme -V^4(psi) + V^2(psi^3) - V^2(psi)
inline constexpr auto b_exact() {
  return make_model<1, 0>(-bilap(psi) + (c<2>() * lap(power<3>(psi)) + -(c<1>() * lap(psi))));
}
inline constexpr auto b_fused() {
  // lap(mu), mu = c2 psi^3 - c1 psi - lap(psi)
  return make_model<1, 1>(lap(stage<0>()), Lit(),
                          c<2>() * power<3>(psi) - c<1>() * psi - lap(psi));
}

// --- model C: g = 2 gamma = 2 c1
//     dpsi = -bilap(psi) + lap(psi^3) - lap(psi) + lap(g psi eta^2)
//     deta = lap(eta) + eta - eta^3 - g psi^2 eta
inline constexpr auto c_exact() {
  return make_model<2, 0>(
      -bilap(psi) +
          (lap(power<3>(psi)) + (-lap(psi) + lap((Lit(2.0) * c<1>()) * (psi * (eta * eta))))),
      lap(eta) + (eta + (-power<3>(eta) + -((Lit(2.0) * c<1>()) * ((psi * psi) * eta)))));
}
inline constexpr auto c_fused() {
  return make_model<2, 1>(
      lap(stage<0>()),
      lap(eta) + eta - power<3>(eta) - (Lit(2.0) * c<1>()) * (psi * psi) * eta,
      power<3>(psi) - psi + (Lit(2.0) * c<1>()) * psi * (eta * eta) - lap(psi));
}

// --- AMK: dpsi = M (kappa lap(psi) - psi^3 + psi)
inline constexpr auto amk_exact() {
  return make_model<1, 0>(c<1>() * (c<2>() * lap(psi) + (-power<3>(psi) + psi)));
}
inline constexpr auto amk_fused() {
  return make_model<1, 0>(c<1>() * (c<2>() * lap(psi) + psi - power<3>(psi)));
}

// --- BMK: dpsi = M lap(psi^3 - psi - kappa lap psi)
inline constexpr auto bmk_exact() {
  return make_model<1, 0>(
      c<1>() * (-(c<2>() * bilap(psi)) + (lap(power<3>(psi)) + -lap(psi))));
}
inline constexpr auto bmk_fused() {
  return make_model<1, 1>(c<1>() * lap(stage<0>()), Lit(),
                          power<3>(psi) - psi - c<2>() * lap(psi));
}

// --- single operators, to check each stencil point set on its own
inline constexpr auto op_lap() { return make_model<1, 0>(lap(psi)); }
inline constexpr auto op_bilap() { return make_model<1, 0>(bilap(psi)); }
inline constexpr auto op_gradlap() { return make_model<1, 0>(gradlap(psi)); }
inline constexpr auto op_lapcube() { return make_model<1, 0>(lap(power<3>(psi))); }

}  // namespace models
}  // namespace sp
