// User-written models through the C++ front end (symphas_model.hpp), FP64, run
// with find_solution; the final field is written to the file named on the
// command line (raw doubles, x fastest) for the tests to compare with the CPU
// oracle.
//   ma:  Allen-Cahn (SymPhas's MA, examples/models/modeldefinitions.h:43-46) in
//        the order of SymPhas's printed scheme V^2(psi) - psi^3 + psi, exact form
//   mbb: SymPhas's MBB (modeldefinitions.h:150-155), model B through a
//        provisional variable var(1) = -(c1 - 4 c2 psi^2) psi, fused form
//   ma4: the same MA with SymPhas's 4th-order stencils Stencil2d4h<>, exact
//   mareg: the same MA on a regional system (regional_model_t, window checks
//        every 0.05 of time), from a disc of +1 (radius n/5 at (n/3, n/2)) in
//        -1; seed, lo and hi unused
//
//   user_model <ma|mbb|ma4|mareg> <out> <n> <h> <dt> <steps> <seed> <lo> <hi>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "symphas_model.hpp"

using namespace symphas_b200;

SP_MODEL(MA, 1, lap(op<1>()) + (-(c<2>() * power<3>(op<1>())) + c<1>() * op<1>()));
SP_MODEL_STAGED(MBB, 1, 1, -bilap(op<1>()) + lap(var<1>()), Lit(),
                -(c<1>() - Lit(4.0) * c<2>() * op<1>() * op<1>()) * op<1>());

template <class M>
int run(M& m, const char* out, unsigned long long seed, double lo, double hi, double dt,
        int steps) {
  m.fill_uniform(0, seed, lo, hi);
  find_solution(m, dt, steps);
  const std::vector<double> psi = m.template get_field<0>();
  FILE* f = std::fopen(out, "wb");
  if (!f || std::fwrite(psi.data(), sizeof(double), psi.size(), f) != psi.size()) return 1;
  std::fclose(f);
  std::printf("index %d time %.6f\n", m.get_index(), m.get_time());
  return 0;
}

int main(int argc, char** argv) {
  if (argc != 10) {
    std::fprintf(stderr, "usage: %s ma|mbb|ma4|mareg out n h dt steps seed lo hi\n", argv[0]);
    return 2;
  }
  const std::string which = argv[1];
  const int n = std::atoi(argv[3]), steps = std::atoi(argv[6]);
  const double h = std::atof(argv[4]), dt = std::atof(argv[5]);
  const double lo = std::atof(argv[8]), hi = std::atof(argv[9]);
  const unsigned long long seed = std::strtoull(argv[7], nullptr, 10);
  const ProblemParameters<2> params{{n, n}, h};
  if (which == "ma") {
    const double coeff[2] = {1.0, 1.0};
    model_t<MA, SolverFT<Stencil2d2h<5, 6, 13>, true>, 2> m(coeff, 2, params);
    return run(m, argv[2], seed, lo, hi, dt, steps);
  }
  if (which == "ma4") {
    const double coeff[2] = {1.0, 1.0};
    model_t<MA, SolverFT<Stencil2d4h<>, true>, 2> m(coeff, 2, params);
    return run(m, argv[2], seed, lo, hi, dt, steps);
  }
  if (which == "mareg") {
    const double coeff[2] = {1.0, 1.0};
    RegionalParameters rp;
    rp.resize_delta = 0.05;
    regional_model_t<MA, SolverFT<Stencil2d2h<5, 6, 13>, true>, 2> m(coeff, 2, params, rp);
    std::vector<double> psi0(size_t(n) * n);
    const double r = n / 5.0, cx = n / 3, cy = n / 2;
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x)
        psi0[size_t(y) * n + x] = (x - cx) * (x - cx) + (y - cy) * (y - cy) < r * r ? 1.0 : -1.0;
    m.set_field(0, psi0);
    find_solution(m, dt, steps);
    const std::vector<double> psi = m.get_field<0>();
    FILE* f = std::fopen(argv[2], "wb");
    if (!f || std::fwrite(psi.data(), sizeof(double), psi.size(), f) != psi.size()) return 1;
    std::fclose(f);
    int o[3], d[3];
    m.window(o, d);
    std::printf("index %d time %.6f window %d %d %d %d\n", m.get_index(), m.get_time(), o[0], o[1],
                d[0], d[1]);
    return 0;
  }
  if (which == "mbb") {
    const double coeff[2] = {1.0, 0.25};  // var(1) = psi^3 - psi: model B
    model_t<MBB, SolverFT<Stencil2d2h<5, 6, 13>, false>, 2> m(coeff, 2, params);
    return run(m, argv[2], seed, lo, hi, dt, steps);
  }
  return 2;
}
