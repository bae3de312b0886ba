// A user-written model through the C++ front end (symphas_model.hpp): Allen-Cahn
// (SymPhas's MA, examples/models/modeldefinitions.h:43-46) in the order of
// SymPhas's printed scheme V^2(psi) - psi^3 + psi, FP64, exact form, run with
// find_solution; the final field is written to the file named on the command
// line (raw doubles, x fastest) for the test to compare with the CPU oracle.
//
//   user_model <out> <n> <h> <dt> <steps> <seed> <lo> <hi>
#include <cstdio>
#include <cstdlib>

#include "symphas_model.hpp"

using namespace symphas_b200;

SP_MODEL(MA, 1, lap(op<1>()) + (-(c<2>() * power<3>(op<1>())) + c<1>() * op<1>()));

int main(int argc, char** argv) {
  if (argc != 9) {
    std::fprintf(stderr, "usage: %s out n h dt steps seed lo hi\n", argv[0]);
    return 2;
  }
  const int n = std::atoi(argv[2]), steps = std::atoi(argv[5]);
  const double h = std::atof(argv[3]), dt = std::atof(argv[4]);
  const double lo = std::atof(argv[7]), hi = std::atof(argv[8]);
  const unsigned long long seed = std::strtoull(argv[6], nullptr, 10);
  const double coeff[2] = {1.0, 1.0};
  model_t<MA, SolverFT<Stencil2d2h<5, 6, 13>, true>, 2> m(coeff, 2, ProblemParameters<2>{{n, n}, h});
  m.fill_uniform(0, seed, lo, hi);
  find_solution(m, dt, steps);
  const std::vector<double> psi = m.get_field<0>();
  FILE* f = std::fopen(argv[1], "wb");
  if (!f || std::fwrite(psi.data(), sizeof(double), psi.size(), f) != psi.size()) return 1;
  std::fclose(f);
  std::printf("index %d time %.6f\n", m.get_index(), m.get_time());
  return 0;
}
