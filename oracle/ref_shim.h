/*
 * ref_shim.h -- force-included (g++ -include) before every SymPhas source the
 * oracle's pin compiles (oracle/ref.mk).  TEST INFRASTRUCTURE ONLY.
 *
 * It lets GCC 13 compile SymPhas's sources as they are, without editing them:
 * - sol/inc/boundarysystem.h:385,390 name `symphas::lib::abs` in a
 *   using-declaration, a name SymPhas never declares (GCC rejects the
 *   declaration at definition time); std::abs is what those lines reach for;
 * - sol/inc/modelarray.h:568-569 define the alias ArrayModel = Model<...>
 *   before the declaration of Model at :571-572; declaring the template
 *   first, with the same signature, is what the alias needs.
 */
#pragma once
#include <cmath>
#include <cstddef>

namespace symphas {
namespace lib {
using std::abs;
}
}  // namespace symphas

template <size_t D, typename Sp, typename... S>
struct Model;
