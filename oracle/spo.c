/*
 * spo.c -- CPU oracle for the explicit finite-difference path of SymPhas.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the symphas_b200
 * package, its CUDA library or the C++ front end) may include, link or run
 * this file; only tests/, the smoke check and the CPU-baseline leg of
 * bench.py use it, and only as the checker.
 *
 * What it restates (paths are inside the SymPhas source tree):
 *   - storage: x-fastest, BOUNDARY_DEPTH = 3 halo cells on every side
 *     (datatypes/inc/gridinfo.h:46, grid::get_stride datatypes/inc/grid.h:536-580)
 *   - halo refresh before every evaluation: periodic copies of the opposite
 *     interior (datatypes/inc/boundaryupdate.h:154-356, :650-690) and the
 *     constant DEFAULT/CONSTANT boundary (datatypes/inc/boundaryupdate.h:1148-1526)
 *   - stencils of 2nd-order accuracy, every point variant, with their
 *     summation order (sol/inc/stencilh2.h:87-507) and the divh powers
 *     divh2 = divh*divh, divh3 = divh*divh2, divh4 = divh2*divh2
 *     (sol/inc/stencilincludes.h:100-107)
 *   - derivatives of non-variable expressions are materialised first over the
 *     whole storage, halo included, then the stencil runs on the temporary
 *     (sym/inc/expressionderivatives.h:1546-1588)
 *   - sums of terms are a right fold e0 + (e1 + (e2 + ...))
 *     (sym/inc/expressions.h:2032-2040); power<N> for N <= 6 is the right-fold
 *     product x*(x*x) (lib/inc/spslibmath.h:255-268)
 *   - equations of all fields are evaluated before any field is stepped
 *     (sol/inc/modelspecialized.h:377-385, sol/inc/model.h:932-936), and the
 *     step is psi + dt*dframe over the interior (examples/solvers/solverft.h:46-50)
 *
 * Parity status: pinned to SymPhas itself.  oracle/ref.mk compiles
 * SymPhas's own CPU SolverFT from its sources (oracle/_ref/libsymphas_ref.so,
 * wrapped by oracle/symref.py), and tests/test_ref_pin.py runs both on the
 * same seeded inputs: bit-identical for the configurations, every stencil
 * point set, unit-coefficient models A and B and the Dirichlet mixes SymPhas
 * treats alike; within 1e-12 (about 5e-16) where SymPhas's optimiser folds
 * non-unit coefficients into the terms in another order.
 *
 * Build: oracle/Makefile (gcc -O3 -ffp-contract=off -fopenmp -shared).
 * Floating-point contraction is disabled so every product and sum rounds on
 * its own, as in the reference's plain C++ expression evaluation.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define BD 3 /* BOUNDARY_DEPTH */

enum {
  SPO_MODEL_A = 0,      /* dpsi = lap(psi) + (c1 - c2 psi^2) psi          */
  SPO_MODEL_B = 1,      /* dpsi = -bilap(psi) - lap((c1 - c2 psi^2) psi)  */
  SPO_MODEL_C = 2,      /* two fields, coupling 2*gamma*psi*eta^2         */
  SPO_MODEL_AMK = 3,    /* dpsi = M (kappa lap psi - psi^3 + psi)         */
  SPO_MODEL_BMK = 4,    /* dpsi = M lap(psi^3 - psi - kappa lap psi)      */
  SPO_OP_LAP = 10,      /* dframe = lap(psi)         (operator checks)    */
  SPO_OP_BILAP = 11,    /* dframe = bilap(psi)                            */
  SPO_OP_GRADLAP = 12,  /* dframe = x-component of gradlap(psi)           */
  SPO_OP_LAPCUBE = 13,  /* dframe = lap(psi^3)                            */
};

enum { SPO_PERIODIC = 0, SPO_DIRICHLET = 1 };

typedef struct spo_desc {
  int dim;          /* 2 or 3 */
  int n[3];         /* interior extents x, y, z (z ignored in 2D) */
  int model;
  int lap_pts, gradlap_pts, bilap_pts;
  double h, dt;
  double c[8];      /* c(1)..c(8) */
  int bc[6];        /* sides in the order LEFT RIGHT TOP BOTTOM FRONT BACK */
  double bcv[6];    /* constant value of a DIRICHLET side */
  int acc;          /* order of accuracy: 2 (or 0) Stencil2d2h/3d2h, 4 Stencil2d4h */
} spo_desc;

/* ------------------------------------------------------------------ */
/* seeded initial values: SplitMix64 counter stream                    */
/* ------------------------------------------------------------------ */

static uint64_t spo_mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

/* value i of stream `seed`: lo + (hi - lo) * u, u = top 53 bits / 2^53 */
void spo_seed_uniform(uint64_t seed, double lo, double hi, long long count,
                      long long first, double* out) {
  const double inv = 1.0 / 9007199254740992.0; /* 2^-53 */
  for (long long i = 0; i < count; ++i) {
    uint64_t z = seed + (uint64_t)(first + i + 1) * 0x9E3779B97F4A7C15ULL;
    double u = (double)(spo_mix(z) >> 11) * inv;
    out[i] = lo + (hi - lo) * u;
  }
}

/* ------------------------------------------------------------------ */
/* grids                                                               */
/* ------------------------------------------------------------------ */

typedef struct {
  int dim;
  long L[3];      /* storage extents incl. halo */
  long s[3];      /* strides {1, Lx, Lx*Ly} */
  long size;
} spo_geom;

static spo_geom spo_make_geom(const spo_desc* d) {
  spo_geom g;
  g.dim = d->dim;
  g.L[0] = d->n[0] + 2 * BD;
  g.L[1] = d->n[1] + 2 * BD;
  g.L[2] = (d->dim == 3) ? d->n[2] + 2 * BD : 1;
  g.s[0] = 1;
  g.s[1] = g.L[0];
  g.s[2] = g.L[0] * g.L[1];
  g.size = g.L[0] * g.L[1] * g.L[2];
  return g;
}

/* Fill the halo.  A halo cell outside the domain along a DIRICHLET axis takes
 * that side's value (later sides in LEFT..BACK order win); a cell outside only
 * along periodic axes takes the value of its periodic image. */
static void spo_halo_cell(const spo_desc* d, const spo_geom* g, double* v, long i, long j,
                          long k) {
  const int D = d->dim;
  long c[3] = {i - BD, j - BD, (D == 3) ? k - BD : 0};
  int dir = -1;
  double dval = 0;
  for (int a = 0; a < D; ++a) {
    if (c[a] < 0 && d->bc[2 * a] == SPO_DIRICHLET) { dir = 2 * a; dval = d->bcv[2 * a]; }
    if (c[a] >= d->n[a] && d->bc[2 * a + 1] == SPO_DIRICHLET) { dir = 2 * a + 1; dval = d->bcv[2 * a + 1]; }
  }
  long idx = i + j * g->s[1] + k * g->s[2];
  if (dir >= 0) {
    v[idx] = dval;
    return;
  }
  long w[3];
  for (int a = 0; a < 3; ++a) {
    long n = (a < D) ? d->n[a] : 1;
    long x = c[a];
    if (a < D) {
      while (x < 0) x += n;
      while (x >= n) x -= n;
    }
    w[a] = x + ((a < D) ? BD : 0);
  }
  v[idx] = v[w[0] + w[1] * g->s[1] + w[2] * g->s[2]];
}

static void spo_update_halo(const spo_desc* d, const spo_geom* g, double* v) {
  const int D = d->dim;
  for (long k = 0; k < g->L[2]; ++k)
    for (long j = 0; j < g->L[1]; ++j) {
      int row_out = (j < BD || j >= BD + d->n[1]) ||
                    (D == 3 && (k < BD || k >= BD + d->n[2]));
      if (row_out) {
        for (long i = 0; i < g->L[0]; ++i) spo_halo_cell(d, g, v, i, j, k);
      } else {
        for (long i = 0; i < BD; ++i) spo_halo_cell(d, g, v, i, j, k);
        for (long i = BD + d->n[0]; i < g->L[0]; ++i) spo_halo_cell(d, g, v, i, j, k);
      }
    }
}

/* ------------------------------------------------------------------ */
/* stencils (sol/inc/stencilh2.h), neighbour names as in sol/inc/stencil.h */
/* ------------------------------------------------------------------ */

#define P(i, j, k) v[(i) * sx + (j) * sy + (k) * sz]
#define v0 P(0, 0, 0)
#define vx P(1, 0, 0)
#define vx_ P(-1, 0, 0)
#define vy P(0, 1, 0)
#define vy_ P(0, -1, 0)
#define vz P(0, 0, 1)
#define vz_ P(0, 0, -1)
#define vx2 P(2, 0, 0)
#define vx2_ P(-2, 0, 0)
#define vy2 P(0, 2, 0)
#define vy2_ P(0, -2, 0)
#define vz2 P(0, 0, 2)
#define vz2_ P(0, 0, -2)
#define vxy P(1, 1, 0)
#define vxy_ P(1, -1, 0)
#define vx_y P(-1, 1, 0)
#define vx_y_ P(-1, -1, 0)
#define vx2y P(2, 1, 0)
#define vx2y_ P(2, -1, 0)
#define vx2_y P(-2, 1, 0)
#define vx2_y_ P(-2, -1, 0)
#define vxy2 P(1, 2, 0)
#define vxy2_ P(1, -2, 0)
#define vx_y2 P(-1, 2, 0)
#define vx_y2_ P(-1, -2, 0)
#define vx2y2 P(2, 2, 0)
#define vx2y2_ P(2, -2, 0)
#define vx2_y2 P(-2, 2, 0)
#define vx2_y2_ P(-2, -2, 0)
#define vxz P(1, 0, 1)
#define vxz_ P(1, 0, -1)
#define vx_z P(-1, 0, 1)
#define vx_z_ P(-1, 0, -1)
#define vx2z P(2, 0, 1)
#define vx2z_ P(2, 0, -1)
#define vx2_z P(-2, 0, 1)
#define vx2_z_ P(-2, 0, -1)
#define vxz2 P(1, 0, 2)
#define vxz2_ P(1, 0, -2)
#define vx_z2 P(-1, 0, 2)
#define vx_z2_ P(-1, 0, -2)
#define vx2z2 P(2, 0, 2)
#define vx2z2_ P(2, 0, -2)
#define vx2_z2 P(-2, 0, 2)
#define vx2_z2_ P(-2, 0, -2)
#define vyz P(0, 1, 1)
#define vyz_ P(0, 1, -1)
#define vy_z P(0, -1, 1)
#define vy_z_ P(0, -1, -1)
#define vyz2 P(0, 1, 2)
#define vyz2_ P(0, 1, -2)
#define vy_z2 P(0, -1, 2)
#define vy_z2_ P(0, -1, -2)
#define vy2z P(0, 2, 1)
#define vy2z_ P(0, 2, -1)
#define vy2_z P(0, -2, 1)
#define vy2_z_ P(0, -2, -1)
#define vy2z2 P(0, 2, 2)
#define vy2z2_ P(0, 2, -2)
#define vy2_z2 P(0, -2, 2)
#define vy2_z2_ P(0, -2, -2)
#define vxyz P(1, 1, 1)
#define vxyz_ P(1, 1, -1)
#define vxy_z P(1, -1, 1)
#define vxy_z_ P(1, -1, -1)
#define vx_yz P(-1, 1, 1)
#define vx_yz_ P(-1, 1, -1)
#define vx_y_z P(-1, -1, 1)
#define vx_y_z_ P(-1, -1, -1)
#define vx2yz P(2, 1, 1)
#define vx2yz_ P(2, 1, -1)
#define vx2y_z P(2, -1, 1)
#define vx2y_z_ P(2, -1, -1)
#define vx2_yz P(-2, 1, 1)
#define vx2_yz_ P(-2, 1, -1)
#define vx2_y_z P(-2, -1, 1)
#define vx2_y_z_ P(-2, -1, -1)
#define vxy2z P(1, 2, 1)
#define vxy2z_ P(1, 2, -1)
#define vxy2_z P(1, -2, 1)
#define vxy2_z_ P(1, -2, -1)
#define vx_y2z P(-1, 2, 1)
#define vx_y2z_ P(-1, 2, -1)
#define vx_y2_z P(-1, -2, 1)
#define vx_y2_z_ P(-1, -2, -1)
#define vxyz2 P(1, 1, 2)
#define vxyz2_ P(1, 1, -2)
#define vxy_z2 P(1, -1, 2)
#define vxy_z2_ P(1, -1, -2)
#define vx_yz2 P(-1, 1, 2)
#define vx_yz2_ P(-1, 1, -2)
#define vx_y_z2 P(-1, -1, 2)
#define vx_y_z2_ P(-1, -1, -2)
#define vx2y2z2 P(2, 2, 2)
#define vx2y2z2_ P(2, 2, -2)
#define vx2y2_z2 P(2, -2, 2)
#define vx2y2_z2_ P(2, -2, -2)
#define vx2_y2z2 P(-2, 2, 2)
#define vx2_y2z2_ P(-2, 2, -2)
#define vx2_y2_z2 P(-2, -2, 2)
#define vx2_y2_z2_ P(-2, -2, -2)

#define vx3 P(3, 0, 0)
#define vx3_ P(-3, 0, 0)
#define vy3 P(0, 3, 0)
#define vy3_ P(0, -3, 0)
#define vx3y P(3, 1, 0)
#define vx3y_ P(3, -1, 0)
#define vx3_y P(-3, 1, 0)
#define vx3_y_ P(-3, -1, 0)
#define vxy3 P(1, 3, 0)
#define vxy3_ P(1, -3, 0)
#define vx_y3 P(-1, 3, 0)
#define vx_y3_ P(-1, -3, 0)
#define vx3y3 P(3, 3, 0)
#define vx3y3_ P(3, -3, 0)
#define vx3_y3 P(-3, 3, 0)
#define vx3_y3_ P(-3, -3, 0)

typedef struct {
  long sx, sy, sz;
  double divh2, divh3, divh4;
  int lap, grad, bilap, dim, acc;
} spo_stencil;

/* Stencil2d4h, sol/inc/stencilh4.h:44-216.  The reference hands every
 * operator divh3 as its scale (sol/inc/stencilincludes.h:446, :453, :460),
 * so s = divh3 below for the Laplacian and the bilaplacian too. */
static double spo_lap4(const spo_stencil* st, const double* v) {
  const long sx = st->sx, sy = st->sy, sz = 0;
  const double s = st->divh3;
  switch (st->lap) {
    case 9:
      return (-vx2_ - vx2 - vy2 - vy2_ + 16. * (vx_ + vx + vy + vy_) - 60. * v0) * s * (1.0 / 12);
    case 17:
      return (-(vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_) - 8. * (vx2 + vx2_ + vy2 + vy2_) +
              16. * (vxy + vx_y + vxy_ + vx_y_) + 128. * (vx + vx_ + vy + vy_) - 540. * v0) *
             s * (1.0 / 120);
    case 21:
      return (-2. * (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_) -
              (vx2 + vx2_ + vy2 + vy2_) + 16. * (vxy + vx_y + vxy_ + vx_y_) +
              52. * (vx + vx_ + vy + vy_) - 252. * v0) *
             s * (1.0 / 60);
  }
  abort();
}

static double spo_bilap4(const spo_stencil* st, const double* v) {
  const long sx = st->sx, sy = st->sy, sz = 0;
  const double s = st->divh3;
  switch (st->bilap) {
    case 21:
      return (-4. * (vx3 + vx3_ + vy3 + vy3_) - (vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_) +
              50. * (vx2 + vx2_ + vy2 + vy2_) + 64. * (vxy + vx_y + vxy_ + vx_y_) -
              284. * (vx + vx_ + vy + vy_) + 700. * v0) *
             s * (1.0 / 24);
    case 25:
      return (-(vx3 + vx3_ + vy3 + vy3_) -
              (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_) +
              14. * (vx2 + vx2_ + vy2 + vy2_) + 20. * (vxy + vx_y + vxy_ + vx_y_) -
              77. * (vx + vx_ + vy + vy_) + 184. * v0) *
             s * (1.0 / 6);
    case 33:
      return (-17. * (vx3y3 + vx3_y3 + vx3y3_ + vx3_y3_) - 236. * (vx3 + vx3_ + vy3 + vy3_) +
              351. * (vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_) -
              756. * (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_) +
              4050. * (vx2 + vx2_ + vy2 + vy2_) + 5049. * (vxy + vx_y + vxy_ + vx_y_) -
              19116. * (vx + vx_ + vy + vy_) + 45724. * v0) *
             s * (1.0 / 1620);
    case 37:
      return (-17. * (vx3y + vx3_y + vx3y_ + vx3_y_ + vxy3 + vx_y3 + vxy3_ + vx_y3_) +
              4. * (vx3 + vx3_ + vy3 + vy3_) - 29. * (vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_) +
              188. * (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_) +
              42. * (vx2 + vx2_ + vy2 + vy2_) - 374. * (vxy + vx_y + vxy_ + vx_y_) -
              764. * (vx + vx_ + vy + vy_) + 3116. * v0) *
             s * (1.0 / 180);
  }
  abort();
}

static double spo_gradlap4_x(const spo_stencil* st, const double* v) {
  const long sx = st->sx, sy = st->sy, sz = 0;
  const double s = st->divh3;
  switch (st->grad) {
    case 14:
      return (-6. * (vx3 - vx3_) - (vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_) + 50. * (vx2 - vx2_) +
              32. * (vxy - vx_y + vxy_ - vx_y_) - 142. * (vx - vx_)) *
             s * (1.0 / 48);
    case 18:
      return (-3. * (vx3) - 2. * (vx2y - vx2_y + vx2y_ - vx2_y_) + 28. * (vx2) -
              (vxy2 - vx_y2 + vxy2_ - vx_y2_) + 20. * (vxy - vx_y + vxy_ - vx_y_) - 77. * (vx)) *
             s * (1.0 / 24);
    case 26: /* the reference divides by 2160 divh3 here (stencilh4.h:184-195) */
      return (-17. * (vx3y3 - vx3_y3 + vx3y3_ - vx3_y3_) - 236. * (vx3) +
              234. * (vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_) - 504. * (vx2y - vx2_y + vx2y_ - vx2_y_) +
              2700. * (vx2) - 252. * (vxy2 - vx_y2 + vxy2_ - vx_y2_) +
              1683. * (vxy - vx_y + vxy_ - vx_y_) - 6372. * (vx)) /
             (2160. * s);
    case 30:
      return (-51. * (vx3y - vx3_y + vx3y_ - vx3_y_) + 12. * (vx3) -
              58. * (vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_) + 376. * (vx2y - vx2_y + vx2y_ - vx2_y_) +
              84. * (vx2) - 17. * (vxy3 - vx_y3 + vxy3_ - vx_y3_) +
              188. * (vxy2 - vx_y2 + vxy2_ - vx_y2_) - 374. * (vxy - vx_y + vxy_ - vx_y_) -
              764. * (vx)) *
             s * (1.0 / 720);
  }
  abort();
}

/* sol/inc/stencilh2.h:87-107 (2D) and :235-327 (3D) */
static double spo_lap(const spo_stencil* st, const double* v) {
  if (st->acc == 4) return spo_lap4(st, v);
  const long sx = st->sx, sy = st->sy, sz = st->sz;
  const double divh2 = st->divh2;
  if (st->dim == 2) {
    switch (st->lap) {
      case 5: return (vx_ + vx + vy + vy_ - 4. * v0) * divh2;
      case 9:
        return (vx_y + vxy_ + vxy + vx_y_ + 4. * vx + 4. * vy + 4. * vy_ + 4. * vx_ - 20. * v0) *
               divh2 * (1.0 / 6);
    }
  } else {
    switch (st->lap) {
      case 7: return (vx_ + vx + vy + vy_ + vz + vz_ - 6. * v0) * divh2;
      case 15:
        return (vx_y_z_ + vxy_z_ + vx_yz_ + vxyz_ + vx_y_z + vxy_z + vx_yz + vxyz +
                8. * (vx_ + vx + vy + vy_ + vz + vz_ - 7. * v0)) *
               divh2 * (1.0 / 12);
      case 19: /* the reference reads vz twice here (stencilh2.h:273) */
        return (vx_y_ + vxy_ + vx_y + vxy + vx_z_ + vxz_ + vx_z + vxz + vy_z_ + vyz_ + vy_z +
                vyz + 2. * (vx_ + vx + vy + vy_ + vz + vz) - 24. * v0) *
               divh2 * (1.0 / 6);
      case 21:
        return (-(vx_y_z_ + vxy_z_ + vx_yz_ + vxyz_ + vx_y_z + vxy_z + vx_yz + vxyz) +
                4. * (vx_y_ + vxy_ + vx_y + vxy + vx_z_ + vxz_ + vx_z + vxz + vy_z_ + vyz_ +
                      vy_z + vyz) +
                -40. * v0) *
               divh2 * (1.0 / 12);
      case 27:
        return (vx_y_z_ + vxy_z_ + vx_yz_ + vxyz_ + vx_y_z + vxy_z + vx_yz + vxyz +
                3. * (vx_y_ + vxy_ + vx_y + vxy + vx_z_ + vxz_ + vx_z + vxz + vy_z_ + vyz_ +
                      vy_z + vyz) +
                14. * (vx_ + vx + vy + vy_ + vz + vz_) - 128. * v0) *
               divh2 * (1.0 / 30);
    }
  }
  abort();
}

/* sol/inc/stencilh2.h:112-156 (2D) and :329-412 (3D) */
static double spo_bilap(const spo_stencil* st, const double* v) {
  if (st->acc == 4) return spo_bilap4(st, v);
  const long sx = st->sx, sy = st->sy, sz = st->sz;
  const double divh4 = st->divh4;
  if (st->dim == 2) {
    switch (st->bilap) {
      case 13:
        return (vy2_ + vy2 + vx2_ + vx2 + 2. * (vx_y_ + vxy_ + vx_y + vxy) -
                8. * (vx_ + vx + vy_ + vy) + 20. * v0) *
               divh4;
      case 17:
        return ((vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_) + 10. * (vx2 + vx2_ + vy2 + vy2_) +
                8. * (vxy + vx_y + vxy_ + vx_y_) - 64. * (vx + vx_ + vy + vy_) + 180. * v0) *
               divh4 * (1.0 / 12);
      case 21:
        return ((vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_) +
                (vx2 + vx2_ + vy2 + vy2_) - 2. * (vxy + vx_y + vxy_ + vx_y_) -
                10. * (vx + vx_ + vy + vy_) + 36. * v0) *
               divh4 * (1.0 / 12);
    }
  } else {
    switch (st->bilap) {
      case 21:
        return ((vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_ + vx2z2_ + vx2_z2_ + vx2z2 + vx2_z2 + vy2z2_ +
                 vy2z2 + vy2_z2_ + vy2_z2) -
                4. * (vxyz + vx_yz + vxy_z + vx_y_z + vxyz_ + vx_yz_ + vxy_z_ + vx_y_z_) +
                20. * v0) *
               divh4 * (1.0 / 4);
      case 25:
        return (2. * (vxy + vx_y + vxy_ + vx_y_ + vxz_ + vx_z_ + vxz + vx_z + vyz_ + vyz +
                      vy_z_ + vy_z) +
                (vx2 + vx2_ + vy2 + vy2_ + vz2 + vz2_) -
                12. * (vx + vx_ + vy + vy_ + vz + vz_) + 42. * v0) *
               divh4;
      case 41:
        return ((vx2y2z2 + vx2_y2z2 + vx2y2_z2 + vx2_y2_z2 + vx2y2z2_ + vx2_y2z2_ + vx2y2_z2_ +
                 vx2_y2_z2_) -
                40. * (vxyz + vx_yz + vxy_z + vx_y_z + vxyz_ + vx_yz_ + vxy_z_ + vx_y_z_) +
                96. * (vxy + vx_y + vxy_ + vx_y_ + vxz_ + vx_z_ + vxz + vx_z + vyz_ + vyz +
                       vy_z_ + vy_z) +
                20. * (vx2 + vx2_ + vy2 + vy2_ + vz2 + vz2_) -
                320. * (vx + vx_ + vy + vy_ + vz + vz_) + 960. * v0) *
               divh4 * (1.0 / 24);
      case 52:
        return (-(vx2y2z2 + vx2_y2z2 + vx2y2_z2 + vx2_y2_z2 + vx2y2z2_ + vx2_y2z2_ + vx2y2_z2_ +
                  vx2_y2_z2_) +
                10. * (vxyz2 + vx_yz2 + vxy_z2 + vx_y_z2 + vxyz2_ + vx_yz2_ + vxy_z2_ +
                       vx_y_z2_ + vxy2z + vx_y2z + vxy2_z + vx_y2_z + vxy2z_ + vx_y2z_ +
                       vxy2_z_ + vx_y2_z_ + vx2yz + vx2_yz + vx2y_z + vx2_y_z + vx2yz_ +
                       vx2_yz_ + vx2y_z_ + vx2_y_z_) -
                20. * (vxyz + vx_yz + vxy_z + vx_y_z + vxyz_ + vx_yz_ + vxy_z_ + vx_y_z_) -
                36. * (vxy + vx_y + vxy_ + vx_y_ + vxz_ + vx_z_ + vxz + vx_z + vyz_ + vyz +
                       vy_z_ + vy_z) +
                360. * v0) *
               divh4 * (1.0 / 36);
      case 57:
        return ((vyz2 + vy_z2 + vyz2_ + vy_z2_ + vy2z + vy2_z + vy2z_ + vy2_z_ + vx2z + vx2_z +
                 vx2z_ + vx2_z_ + vxz2 + vx_z2 + vxz2_ + vx_z2_ + vxy2 + vx_y2 + vxy2_ +
                 vx_y2_ + vx2y + vx2_y + vx2y_ + vx2_y_) +
                3. * (vxyz + vx_yz + vxy_z + vx_y_z + vxyz_ + vx_yz_ + vxy_z_ + vx_y_z_) -
                8. * (vxy + vx_y + vxy_ + vx_y_ + vxz_ + vx_z_ + vxz + vx_z + vyz_ + vyz +
                      vy_z_ + vy_z) -
                (vx2 + vx2_ + vy2 + vy2_ + vz2 + vz2_) +
                4. * (vx + vx_ + vy + vy_ + vz + vz_) + 30. * v0) *
               divh4 * (1.0 / 3);
    }
  }
  abort();
}

/* x component of the gradlaplacian, sol/inc/stencilh2.h:161-221, :417-507 */
static double spo_gradlap_x(const spo_stencil* st, const double* v) {
  if (st->acc == 4) return spo_gradlap4_x(st, v);
  const long sx = st->sx, sy = st->sy, sz = st->sz;
  const double divh3 = st->divh3;
  if (st->dim == 2) {
    switch (st->grad) {
      case 6:
        return ((vx2y - vx2_y + vx2y_ - vx2_y_) - 4. * (vx - vx_)) * divh3 * (1.0 / 4);
      case 8:
        return ((vx2 - vx2_) + (vxy - vx_y + vxy_ - vx_y_) - 4. * (vx - vx_)) * divh3 *
               (1.0 / 2);
      case 12:
        return ((vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_) + 10. * (vx2 - vx2_) +
                4. * (vxy - vx_y + vxy_ - vx_y_) - 32. * (vx - vx_)) *
               divh3 * (1.0 / 24);
      case 16:
        return (2. * (vx2y - vx2_y + vx2y_ - vx2_y_) + 2. * (vx2 - vx2_) +
                (vxy2 - vx_y2 + vxy2_ - vx_y2_) - 2. * (vxy - vx_y + vxy_ - vx_y_) -
                10. * (vx - vx_)) *
               divh3 * (1.0 / 12);
    }
  } else {
    switch (st->grad) {
      case 10:
        return ((vx2yz - vx2_yz + vx2y_z - vx2_y_z + vx2yz_ - vx2_yz_ + vx2y_z_ - vx2_y_z_) -
                8. * (vx - vx_)) *
               divh3 * (1.0 / 8);
      case 12:
        return ((vx2 - vx2_) + (vxy - vx_y + vxy_ - vx_y_ + vxz_ - vx_z_ + vxz - vx_z) -
                6. * (vx - vx_)) *
               divh3 * (1.0 / 2);
      case 28:
        return ((vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_ + vx2z2_ - vx2_z2_ + vx2z2 - vx2_z2) +
                8. * (vx2 - vx2_) +
                6. * (vxyz - vx_yz + vxy_z - vx_y_z + vxyz_ - vx_yz_ + vxy_z_ - vx_y_z_) -
                8. * (vxy - vx_y + vxy_ - vx_y_ + vxz_ - vx_z_ + vxz - vx_z) -
                16. * (vx - vx_)) *
               divh3 * (1.0 / 24);
      case 36:
        return (2. * (vx2z - vx2_z + vx2z_ - vx2_z_ + vx2y - vx2_y + vx2y_ - vx2_y_) -
                2. * (vx2 - vx2_) +
                (vxz2 - vx_z2 + vxz2_ - vx_z2_ + vxy2 - vx_y2 + vxy2_ - vx_y2_) +
                3. * (vxyz - vx_yz + vxy_z - vx_y_z + vxyz_ - vx_yz_ + vxy_z_ - vx_y_z_) -
                8. * (vxy - vx_y + vxy_ - vx_y_ + vxz_ - vx_z_ + vxz - vx_z) +
                4. * (vx - vx_)) *
               divh3 * (1.0 / 12);
      case 40:
        return (16. * (vx2z - vx2_z + vx2z_ - vx2_z_ + vx2y - vx2_y + vx2y_ - vx2_y_) -
                16. * (vx2 - vx2_) +
                3. * (vxy2z - vx_y2z + vxy2_z - vx_y2_z + vxy2z_ - vx_y2z_ + vxy2_z_ -
                      vx_y2_z_ + vxyz2 - vx_yz2 + vxy_z2 - vx_y_z2 + vxyz2_ - vx_yz2_ +
                      vxy_z2_ - vx_y_z2_) +
                2. * (vxz2 - vx_z2 + vxz2_ - vx_z2_ + vxy2 - vx_y2 + vxy2_ - vx_y2_) -
                22. * (vxy - vx_y + vxy_ - vx_y_ + vxz_ - vx_z_ + vxz - vx_z) -
                40. * (vx - vx_)) *
               divh3 * (1.0 / 96);
    }
  }
  abort();
}

/* ------------------------------------------------------------------ */
/* models                                                              */
/* ------------------------------------------------------------------ */

static int spo_field_count(int model) { return model == SPO_MODEL_C ? 2 : 1; }

static double pow3(double x) { return x * (x * x); }

typedef struct {
  spo_desc d;
  spo_geom g;
  spo_stencil st;
  int nf;
  double* psi[2];    /* storage incl. halo */
  double* dframe[2];
  double* tmp[2];    /* materialised operands of derivatives */
  int threads;
} spo_sys;

static void spo_sys_init(spo_sys* s, const spo_desc* d, int threads) {
  memset(s, 0, sizeof(*s));
  s->d = *d;
  s->g = spo_make_geom(d);
  s->nf = spo_field_count(d->model);
  s->threads = threads > 0 ? threads : 1;
  double divh = 1.0 / d->h;
  s->st.divh2 = divh * divh;
  s->st.divh3 = divh * s->st.divh2;
  s->st.divh4 = s->st.divh2 * s->st.divh2;
  s->st.sx = 1;
  s->st.sy = s->g.s[1];
  s->st.sz = (d->dim == 3) ? s->g.s[2] : 0;
  s->st.lap = d->lap_pts;
  s->st.grad = d->gradlap_pts;
  s->st.bilap = d->bilap_pts;
  s->st.dim = d->dim;
  s->st.acc = d->acc == 4 ? 4 : 2;
  for (int f = 0; f < 2; ++f) {
    s->psi[f] = (double*)calloc(s->g.size, sizeof(double));
    s->dframe[f] = (double*)calloc(s->g.size, sizeof(double));
    s->tmp[f] = (double*)calloc(s->g.size, sizeof(double));
  }
}

static void spo_sys_free(spo_sys* s) {
  for (int f = 0; f < 2; ++f) {
    free(s->psi[f]);
    free(s->dframe[f]);
    free(s->tmp[f]);
  }
}

#define SPO_FOR_STORAGE(body)                                   \
  _Pragma("omp parallel for num_threads(s->threads) schedule(static)") \
  for (long n = 0; n < s->g.size; ++n) { body; }

#define SPO_FOR_INTERIOR(body)                                                        \
  {                                                                                   \
    const long K0 = (s->d.dim == 3) ? BD : 0, K1 = (s->d.dim == 3) ? BD + s->d.n[2] : 1; \
    const long plane = (long)s->d.n[1] * (K1 - K0);                                   \
    _Pragma("omp parallel for num_threads(s->threads) schedule(static)")             \
    for (long jk = 0; jk < plane; ++jk) {                                             \
      long k = K0 + jk / s->d.n[1], j = BD + jk % s->d.n[1];                          \
      for (long i = BD; i < BD + s->d.n[0]; ++i) {                                    \
        long n = i + j * s->g.s[1] + k * s->g.s[2];                                   \
        body;                                                                         \
      }                                                                               \
    }                                                                                 \
  }

/* One SolverFT iteration: halo refresh, all equations into dframe, then the
 * forward-Euler step of every field. */
static void spo_sys_step(spo_sys* s) {
  const double* c = s->d.c;
  const spo_stencil* st = &s->st;
  for (int f = 0; f < s->nf; ++f) spo_update_halo(&s->d, &s->g, s->psi[f]);
  double* p = s->psi[0];
  double* q = s->psi[1];
  double* t0 = s->tmp[0];
  double* t1 = s->tmp[1];
  double* d0 = s->dframe[0];
  double* d1 = s->dframe[1];
  switch (s->d.model) {
    case SPO_MODEL_A:
      /* printed scheme: V^2(psi) - psi^3 + psi  (c1 = c2 = 1) */
      SPO_FOR_INTERIOR(d0[n] = spo_lap(st, p + n) + (-(c[1] * pow3(p[n])) + c[0] * p[n]));
      break;
    case SPO_MODEL_B:
      /* printed scheme: -V^4(psi) + V^2(psi^3) - V^2(psi)  (c1 = c2 = 1) */
      SPO_FOR_STORAGE(t0[n] = pow3(p[n]));
      SPO_FOR_INTERIOR(d0[n] = -spo_bilap(st, p + n) +
                               (c[1] * spo_lap(st, t0 + n) + -(c[0] * spo_lap(st, p + n))));
      break;
    case SPO_MODEL_C: {
      /* psi: -V^4(psi) + V^2(psi^3) - V^2(psi) + V^2(g psi eta^2), g = 2 gamma = 2 c1
       * eta: V^2(eta) + eta - eta^3 - g psi^2 eta                                   */
      const double g = 2.0 * c[0];
      SPO_FOR_STORAGE(t0[n] = pow3(p[n]); t1[n] = g * (p[n] * (q[n] * q[n])));
      SPO_FOR_INTERIOR(
          d0[n] = -spo_bilap(st, p + n) +
                  (spo_lap(st, t0 + n) + (-spo_lap(st, p + n) + spo_lap(st, t1 + n)));
          d1[n] = spo_lap(st, q + n) + (q[n] + (-pow3(q[n]) + -(g * ((p[n] * p[n]) * q[n])))));
      break;
    }
    case SPO_MODEL_AMK:
      /* M (kappa V^2(psi) - psi^3 + psi), M = c1, kappa = c2 */
      SPO_FOR_INTERIOR(d0[n] = c[0] * (c[1] * spo_lap(st, p + n) + (-pow3(p[n]) + p[n])));
      break;
    case SPO_MODEL_BMK:
      /* M (-kappa V^4(psi) + V^2(psi^3) - V^2(psi)) */
      SPO_FOR_STORAGE(t0[n] = pow3(p[n]));
      SPO_FOR_INTERIOR(d0[n] = c[0] * (-(c[1] * spo_bilap(st, p + n)) +
                                       (spo_lap(st, t0 + n) + -spo_lap(st, p + n))));
      break;
    case SPO_OP_LAP: SPO_FOR_INTERIOR(d0[n] = spo_lap(st, p + n)); break;
    case SPO_OP_BILAP: SPO_FOR_INTERIOR(d0[n] = spo_bilap(st, p + n)); break;
    case SPO_OP_GRADLAP: SPO_FOR_INTERIOR(d0[n] = spo_gradlap_x(st, p + n)); break;
    case SPO_OP_LAPCUBE:
      SPO_FOR_STORAGE(t0[n] = pow3(p[n]));
      SPO_FOR_INTERIOR(d0[n] = spo_lap(st, t0 + n));
      break;
    default: abort();
  }
  const double dt = s->d.dt;
  for (int f = 0; f < s->nf; ++f) {
    double* pf = s->psi[f];
    double* df = s->dframe[f];
    SPO_FOR_INTERIOR(pf[n] = pf[n] + dt * df[n]);
  }
}

static void spo_copy_in(spo_sys* s, int f, const double* interior) {
  const spo_geom* g = &s->g;
  const long nz = (s->d.dim == 3) ? s->d.n[2] : 1;
  for (long k = 0; k < nz; ++k)
    for (long j = 0; j < s->d.n[1]; ++j)
      memcpy(s->psi[f] + BD + (j + BD) * g->s[1] + (k + (s->d.dim == 3 ? BD : 0)) * g->s[2],
             interior + (k * s->d.n[1] + j) * s->d.n[0], sizeof(double) * s->d.n[0]);
}

static void spo_copy_out(const spo_sys* s, double* const* src, int f, double* interior) {
  const spo_geom* g = &s->g;
  const long nz = (s->d.dim == 3) ? s->d.n[2] : 1;
  for (long k = 0; k < nz; ++k)
    for (long j = 0; j < s->d.n[1]; ++j)
      memcpy(interior + (k * s->d.n[1] + j) * s->d.n[0],
             src[f] + BD + (j + BD) * g->s[1] + (k + (s->d.dim == 3 ? BD : 0)) * g->s[2],
             sizeof(double) * s->d.n[0]);
}

/* ------------------------------------------------------------------ */
/* exported entry points                                               */
/* ------------------------------------------------------------------ */

int spo_fields(int model) { return spo_field_count(model); }

/* A persistent system, for timing loops: create, upload, step, download. */
void* spo_create(const spo_desc* d, int threads) {
  spo_sys* s = (spo_sys*)malloc(sizeof(spo_sys));
  spo_sys_init(s, d, threads);
  return s;
}
void spo_set(void* h, int f, const double* interior) { spo_copy_in((spo_sys*)h, f, interior); }
void spo_get(void* h, int f, double* interior) {
  spo_sys* s = (spo_sys*)h;
  spo_copy_out(s, s->psi, f, interior);
}
void spo_step(void* h, int nsteps) {
  for (int i = 0; i < nsteps; ++i) spo_sys_step((spo_sys*)h);
}
void spo_destroy(void* h) {
  spo_sys_free((spo_sys*)h);
  free(h);
}

/* Advance `fields` (nf interior arrays laid out back to back, x-fastest) by
 * `nsteps` SolverFT iterations using `threads` OpenMP threads.  Returns 0. */
int spo_run(const spo_desc* d, double* fields, int nsteps, int threads) {
  spo_sys s;
  spo_sys_init(&s, d, threads);
  long cnt = (long)d->n[0] * d->n[1] * (d->dim == 3 ? d->n[2] : 1);
  for (int f = 0; f < s.nf; ++f) spo_copy_in(&s, f, fields + f * cnt);
  for (int it = 0; it < nsteps; ++it) spo_sys_step(&s);
  for (int f = 0; f < s.nf; ++f) spo_copy_out(&s, s.psi, f, fields + f * cnt);
  spo_sys_free(&s);
  return 0;
}

/* Evaluate the right-hand side once (no step): dframe of every field. */
int spo_rhs(const spo_desc* d, const double* fields, double* rhs) {
  spo_sys s;
  spo_sys_init(&s, d, 1);
  long cnt = (long)d->n[0] * d->n[1] * (d->dim == 3 ? d->n[2] : 1);
  for (int f = 0; f < s.nf; ++f) spo_copy_in(&s, f, fields + f * cnt);
  spo_desc dd = *d;
  dd.dt = 0.0; /* psi + 0*dframe leaves psi unchanged; dframe is what we want */
  s.d = dd;
  spo_sys_step(&s);
  for (int f = 0; f < s.nf; ++f) spo_copy_out(&s, s.dframe, f, rhs + f * cnt);
  spo_sys_free(&s);
  return 0;
}

/* Run many independent systems (e.g. an ensemble) in parallel, one system per
 * thread; descs[i] and field pointers ptrs[i] describe system i. */
int spo_run_batch(const spo_desc* descs, double** ptrs, int count, const int* nsteps,
                  int threads) {
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(dynamic, 1)
  for (int i = 0; i < count; ++i) spo_run(&descs[i], ptrs[i], nsteps[i], 1);
  return 0;
}

/* Sum of the interior values (Kahan-free plain double sum, x-fastest order). */
double spo_mass(const double* interior, long long count) {
  double m = 0.0;
  for (long long i = 0; i < count; ++i) m += interior[i];
  return m;
}

int spo_omp_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* regional systems: the moving window of SolverSystemFDwSD            */
/* ------------------------------------------------------------------ */
/*
 * A RegionalGrid (datatypes/inc/grid.h:2038-2158) stores only a window of the
 * domain: select_region origin o and dims d in storage coordinates, each
 * including a BD-deep rim (grid.h:1222-1261), with its d0*d1*d2 values
 * x-fastest; a position outside the window's interior reads `empty`
 * (grid.h:1264-1277).  The solver evaluates the window's interior only
 * (get_iterable_domain, datatypes/inc/dataiterator.h:2454-2470) with the
 * window's own strides (sol/inc/stencil.h:209-240).  Here the window is an
 * spo_sys whose storage is that buffer, its halo being the rim: along an axis
 * the window spans from origin 0 the rim takes periodic images
 * (regional_update_boundary, datatypes/inc/boundaryupdatedata.h:1397-1431);
 * along any other axis it keeps what the last move wrote there (empty).
 *
 * The window follows the field (update_regional_system,
 * sol/inc/boundarysystem.h:438-471): at the first update the cutoff becomes
 * min + eps and `empty` the minimum (grid::min_value, boundarysystem.h:372-376),
 * and the window is resized around the values >= cutoff; afterwards, every
 * resize_delta of time, it is re-centred (fixed size) or resized again.
 * The searches and moves restate datatypes/inc/gridfunctions.h:
 *   get_view                   :1962-1986  (re-centre, size kept)
 *   get_view_resized           :1873-1913  (bounding box; the reference runs it
 *                                            under an OpenMP lock, in no fixed
 *                                            order: here the serial order)
 *   get_view_resized_periodic  :1988-2163  (box grown from the first value
 *                                            >= cutoff, wrapping periodically)
 *   adjust_region              :2166-2176, resize_adjust_region :2194-2238
 *   adjust_region_to_from      :1662-1683  (new buffer of `empty`, interior
 *                                            copied modulo the domain)
 *   adjust_origin_to_from      :1770-1852  (shift in place; whether a cell
 *                                            becomes empty is decided by the
 *                                            last axis alone, and other cells
 *                                            take the buffer value at
 *                                            index + offset, rim included.
 *                                            Here a gather from the old buffer,
 *                                            so the overlaps of the in-place
 *                                            order are not reproduced; a source
 *                                            outside the buffer reads empty)
 */

typedef struct {
  int D;
  int G[3];  /* storage dims of the domain, n + 2 BD */
  int o[3];  /* window origin (storage coordinates, rim included) */
  int d[3];  /* window dims, rim included */
  const double* v;  /* window buffer, d0*d1*d2 x-fastest (null when empty) */
  double cut;
} spo_rview;

static long spo_rv_stride(const spo_rview* r, int a) {
  long s = 1;
  for (int i = 0; i < a; ++i) s *= r->d[i];
  return s;
}

static long spo_rv_interior(const spo_rview* r, long c[3]) {
  long len = 1;
  for (int a = 0; a < r->D; ++a) {
    c[a] = r->d[a] - 2 * BD;
    if (c[a] <= 0) len = 0;
    len *= (c[a] > 0 ? c[a] : 0);
  }
  return r->v ? len : 0;
}

/* get_view: buffer entries 0 .. len(interior)-1 (rim cells among them) at
 * positions (n / stride) % interior_dims */
static void spo_view_fixed(const spo_rview* r, int origin[3]) {
  long c[3], iv[3][2], st[3];
  const long len = spo_rv_interior(r, c);
  for (int a = 0; a < r->D; ++a) {
    iv[a][0] = c[a];
    iv[a][1] = 0;
    st[a] = spo_rv_stride(r, a);
  }
  for (long n = 0; n < len; ++n)
    if (r->v[n] >= r->cut)
      for (int a = 0; a < r->D; ++a) {
        const long p = (n / st[a]) % c[a];
        if (p < iv[a][0]) iv[a][0] = p;
        if (p > iv[a][1]) iv[a][1] = p;
      }
  for (int a = 0; a < r->D; ++a) {
    const long dims = iv[a][1] - iv[a][0] + 1 + 2 * BD;
    const long delta = r->d[a] - dims;
    origin[a] = (int)(r->o[a] + (iv[a][0] - delta / 2));
  }
}

/* get_view_resized: bounding box of the interior values >= cutoff, serial order */
static void spo_view_resized(const spo_rview* r, int origin[3], int dims[3]) {
  long c[3], iv[3][2], st[3];
  const long len = spo_rv_interior(r, c);
  for (int a = 0; a < r->D; ++a) {
    iv[a][0] = r->d[a];
    iv[a][1] = 0;
    st[a] = spo_rv_stride(r, a);
  }
  for (long n = 0; n < len; ++n) {
    long pos[3], rem = n, idx = 0;
    for (int a = 0; a < r->D; ++a) {
      pos[a] = rem % c[a] + BD;
      rem /= c[a];
      idx += pos[a] * st[a];
    }
    if (!(r->v[idx] >= r->cut)) continue;
    int inside = 1;
    for (int a = 0; a < r->D; ++a) inside &= (pos[a] >= iv[a][0] && pos[a] < iv[a][1]);
    if (inside) continue;
    for (int a = 0; a < r->D; ++a) {
      if (pos[a] >= iv[a][0]) {
        if (pos[a] > iv[a][1]) iv[a][1] = pos[a];
      } else if (pos[a] < iv[a][0]) {
        iv[a][0] = pos[a];
      }
    }
  }
  for (int a = 0; a < r->D; ++a) {
    origin[a] = (int)(iv[a][0] - BD + r->o[a]);
    const long w = iv[a][1] - iv[a][0] + 1 + 2 * BD;
    dims[a] = (int)(w > 0 ? w : 0);
  }
}

static int spo_rv_at(const spo_rview* r, const long pos[3], const long st[3]) {
  long idx = 0;
  for (int a = 0; a < r->D; ++a) idx += (pos[a] + BD) * st[a];
  return r->v[idx] >= r->cut;
}

/* get_view_resized_periodic: the window is the whole domain; grow a box from
 * the first interior value >= cutoff, one slice at a time on each side of each
 * axis, wrapping, until a pass changes nothing */
static void spo_view_periodic(const spo_rview* r, int origin[3], int dims_out[3]) {
  const int D = r->D;
  long c[3], st[3];
  const long len = spo_rv_interior(r, c);
  for (int a = 0; a < D; ++a) st[a] = spo_rv_stride(r, a);
  long start = -1;
  for (long n = 0; n < len && start < 0; ++n) {
    long pos[3], rem = n;
    for (int a = 0; a < D; ++a) {
      pos[a] = rem % c[a];
      rem /= c[a];
    }
    if (spo_rv_at(r, pos, st)) start = n;
  }
  if (start < 0) {
    for (int a = 0; a < D; ++a) dims_out[a] = 0;
    return;
  }
  long iv[3][2], iu[3][2];
  {
    long rem = start;
    for (int a = 0; a < D; ++a) {
      iu[a][0] = iu[a][1] = rem % c[a];
      rem /= c[a];
    }
  }
  int grown;
  do {
    for (int a = 0; a < D; ++a) {
      iv[a][0] = iu[a][0];
      iv[a][1] = iu[a][1];
    }
    for (int i = 0; i < D; ++i) {
      int right = 1;
      long pos[3];
      for (int j = 0; j < D; ++j) {
        pos[j] = (j == i) ? iu[j][1] + 1 : iu[j][0];
        /* the reference wraps a negative entry with the extent of axis i */
        pos[j] = (pos[j] >= c[j]) ? pos[j] - c[j] : (pos[j] < 0) ? c[i] + pos[j] : pos[j];
      }
      long sd[2] = {1, 1};
      int ns = 0;
      for (int j = 0; j < D; ++j)
        if (j != i) sd[ns++] = iu[j][1] - iu[j][0] + 1;
      long slen = 1;
      for (int q = 0; q < ns; ++q) slen *= sd[q];
      const long steps = c[i] - (iu[i][1] - iu[i][0] + 1);
      int found[2] = {1, 0};
      long last[2] = {iu[i][0], iu[i][1]};
      for (long n = 0; n < steps; ++n) {
        for (long m = 0; m < slen && !found[right ? 1 : 0]; ++m) {
          long sp[2] = {m % sd[0], ns > 1 ? m / sd[0] : 0};
          int q = 0;
          for (int j = 0; j < D; ++j) {
            if (j == i) continue;
            long p = sp[q++] + iu[j][0];
            pos[j] = (p < 0) ? p + c[j] : (p >= c[j]) ? p - c[j] : p;
          }
          if (spo_rv_at(r, pos, st)) found[right ? 1 : 0] = 1;
        }
        if (right) {
          if (found[1]) {
            iu[i][1] = (pos[i] < iu[i][1]) ? pos[i] + c[i] : pos[i];
            ++last[1];
          }
          pos[i] = (last[0] <= 0) ? c[i] + last[0] - 1 : last[0] - 1;
          found[0] = 0;
          right = 0;
        } else {
          if (found[0]) {
            iu[i][0] = (pos[i] > iu[i][0]) ? pos[i] - c[i] : pos[i];
            --last[0];
          }
          pos[i] = (last[1] >= c[i] - 1) ? last[1] + 1 - c[i] : last[1] + 1;
          found[1] = 0;
          right = 1;
        }
      }
    }
    grown = 0;
    for (int a = 0; a < D; ++a) grown |= !(iv[a][0] <= iu[a][0] && iv[a][1] >= iu[a][1]);
  } while (grown);
  for (int a = 0; a < D; ++a) {
    origin[a] = (int)(iu[a][0] + r->o[a]);
    const long w = iu[a][1] - iu[a][0] + 1 + 2 * BD;
    dims_out[a] = (int)(w > 0 ? w : 0);
  }
}

/* The window the next move goes to.  mode 0: adjust_region (re-centred, dims
 * kept, origin wrapped into the domain); mode 1: resize_adjust_region with
 * padding factor `factor` and relative-dims tolerance `rel_eps`. */
static void spo_view_target(const spo_rview* r, int mode, double factor, double rel_eps,
                            int no[3], int nd[3]) {
  const int D = r->D;
  for (int a = 0; a < 3; ++a) {
    no[a] = r->o[a];
    nd[a] = r->d[a];
  }
  if (mode == 0) {
    int origin[3] = {0, 0, 0};
    spo_view_fixed(r, origin);
    for (int a = 0; a < D; ++a) {
      const int delta = r->G[a] - 2 * BD;
      no[a] = origin[a] + ((origin[a] < 0) ? delta : (origin[a] >= delta) ? -delta : 0);
    }
    return;
  }
  int origin[3] = {0, 0, 0}, dims[3] = {0, 0, 0};
  int whole = 1;
  for (int a = 0; a < D; ++a) whole &= (r->G[a] == r->d[a]);
  if (whole)
    spo_view_periodic(r, origin, dims);
  else
    spo_view_resized(r, origin, dims);
  int same = 1;
  for (int a = 0; a < D; ++a) {
    int scaled = (int)(dims[a] * factor);
    const int dim0 = r->G[a] < scaled ? r->G[a] : scaled;
    no[a] = origin[a] - (dim0 - dims[a]) / 2;
    no[a] += (no[a] < 0) ? (r->G[a] - 2 * BD) : 0;
    nd[a] = dim0;
    if (abs(nd[a] - r->d[a]) / (double)r->d[a] > rel_eps) same = 0;
  }
  if (same) {
    for (int a = 0; a < D; ++a) {
      no[a] = origin[a] - (r->d[a] - dims[a]) / 2;
      no[a] += (no[a] < 0) ? (r->G[a] - 2 * BD) : 0;
      nd[a] = r->d[a];
    }
  }
}

/* exported for the host-logic tests: the target window of a buffer of values */
int spo_reg_search(int dim, const int G[3], const int o[3], const int d[3], const double* buf,
                   double cutoff, int mode, double factor, double rel_eps, int no[3], int nd[3]) {
  spo_rview r;
  memset(&r, 0, sizeof(r));
  r.D = dim;
  for (int a = 0; a < 3; ++a) {
    r.G[a] = a < dim ? G[a] : 1;
    r.o[a] = a < dim ? o[a] : 0;
    r.d[a] = a < dim ? d[a] : 1;
  }
  r.v = buf;
  r.cut = cutoff;
  spo_view_target(&r, mode, factor, rel_eps, no, nd);
  return 0;
}

typedef struct {
  spo_desc gd;  /* the whole system (n = domain interior) */
  int D;
  int G[3], o[3], d[3];
  double empty, cutoff, time;
  int next_resize;
  double delta, factor, eps;
  int fixed, threads, has;
  spo_sys sys;  /* the window (valid when has) */
} spo_reg;

static long spo_mod(long a, long n) {
  long r = a % n;
  return r < 0 ? r + n : r;
}

static void spo_reg_build(spo_reg* r) {
  spo_desc w = r->gd;
  r->has = 1;
  for (int a = 0; a < r->D; ++a) {
    w.n[a] = r->d[a] - 2 * BD;
    if (w.n[a] <= 0) r->has = 0;
    const int whole = (r->o[a] == 0 && r->d[a] == r->G[a]);
    w.bc[2 * a] = w.bc[2 * a + 1] = whole ? SPO_PERIODIC : SPO_DIRICHLET;
    w.bcv[2 * a] = w.bcv[2 * a + 1] = r->empty;
  }
  if (!r->has) return;
  spo_sys_init(&r->sys, &w, r->threads);
  for (long i = 0; i < r->sys.g.size; ++i) r->sys.psi[0][i] = r->empty;
}

static void spo_reg_view(const spo_reg* r, spo_rview* v) {
  memset(v, 0, sizeof(*v));
  v->D = r->D;
  for (int a = 0; a < 3; ++a) {
    v->G[a] = r->G[a];
    v->o[a] = r->o[a];
    v->d[a] = r->d[a];
  }
  v->v = r->has ? r->sys.psi[0] : NULL;
  v->cut = r->cutoff;
}

/* adjust_region_to_from / adjust_origin_to_from_replace: a new buffer of
 * `empty`, interior cells copied from the old window modulo the domain */
static void spo_reg_replace(spo_reg* r, const int no[3], const int nd[3]) {
  spo_reg old = *r;
  for (int a = 0; a < 3; ++a) {
    r->o[a] = no[a];
    r->d[a] = nd[a];
  }
  spo_reg_build(r);
  if (r->has && old.has) {
    long cn[3] = {1, 1, 1}, co[3] = {1, 1, 1}, delta[3] = {0, 0, 0};
    for (int a = 0; a < r->D; ++a) {
      const long wrap = r->G[a] - 2 * BD;
      cn[a] = nd[a] - 2 * BD;
      co[a] = old.d[a] - 2 * BD;
      const long on = old.o[a] - wrap * lround((double)old.o[a] / wrap);
      const long nn = no[a] - wrap * lround((double)no[a] / wrap);
      delta[a] = nn - on;
    }
    const long len = cn[0] * cn[1] * cn[2];
    for (long n = 0; n < len; ++n) {
      long p[3] = {n % cn[0], (n / cn[0]) % cn[1], n / (cn[0] * cn[1])};
      long q[3];
      int in = 1;
      for (int a = 0; a < 3; ++a) {
        if (a < r->D) {
          const long wrap = r->G[a] - 2 * BD;
          q[a] = p[a] + delta[a];
          q[a] = (q[a] < 0) ? q[a] + wrap : (q[a] >= wrap) ? q[a] - wrap : q[a];
          in &= (q[a] >= 0 && q[a] < co[a]);
        } else {
          q[a] = 0;
        }
      }
      if (!in) continue;
      const long dz = (r->D == 3) ? BD : 0;
      const long ni = (p[0] + BD) + (p[1] + BD) * r->sys.g.s[1] + (p[2] + dz) * r->sys.g.s[2];
      const long oi = (q[0] + BD) + (q[1] + BD) * old.sys.g.s[1] + (q[2] + dz) * old.sys.g.s[2];
      r->sys.psi[0][ni] = old.sys.psi[0][oi];
    }
  }
  if (old.has) spo_sys_free(&old.sys);
}

/* adjust_origin_to_from: the window keeps its dims */
static void spo_reg_shift(spo_reg* r, const int no[3]) {
  int skip = 1, replace = 0, dir[3] = {1, 1, 1};
  for (int a = 0; a < r->D; ++a) {
    const int delta = no[a] - r->o[a];
    dir[a] = delta >= 0 ? 1 : -1;
    skip &= (delta == 0);
  }
  if (skip) return;
  for (int a = 0; a < r->D; ++a) replace |= (abs(no[a] - r->o[a]) + r->d[a] > r->G[a]);
  if (replace || !r->has) {
    spo_reg_replace(r, no, r->d);
    return;
  }
  const long size = r->sys.g.size;
  double* old = (double*)malloc(sizeof(double) * size);
  memcpy(old, r->sys.psi[0], sizeof(double) * size);
  long c[3] = {1, 1, 1}, ov[3] = {0, 0, 0}, off = 0, bo = 0;
  for (int a = 0; a < r->D; ++a) {
    c[a] = r->d[a] - 2 * BD;
    const long sh = no[a] - r->o[a];
    ov[a] = c[a] - (sh < 0 ? -sh : sh);
    off += sh * r->sys.g.s[a];
    bo += BD * r->sys.g.s[a];
  }
  const int L = r->D - 1;
  const long len = c[0] * c[1] * c[2];
  for (long n = 0; n < len; ++n) {
    long p[3] = {n % c[0], (n / c[0]) % c[1], n / (c[0] * c[1])};
    long idx = 0;
    for (int a = 0; a < r->D; ++a) idx += p[a] * r->sys.g.s[a];
    const int set_empty = dir[L] > 0 ? (p[L] >= ov[L]) : (p[L] < c[L] - ov[L]);
    const long src = idx + off + bo;
    r->sys.psi[0][idx + bo] =
        (set_empty || src < 0 || src >= size) ? r->empty : old[src];
  }
  free(old);
  for (int a = 0; a < 3; ++a) r->o[a] = no[a];
}

/* RegionalGrid::adjust(select_region) (grid.h:2118-2128) */
static void spo_reg_move(spo_reg* r, const int no[3], const int nd[3]) {
  int same_d = 1, same_o = 1;
  for (int a = 0; a < r->D; ++a) {
    same_d &= (nd[a] == r->d[a]);
    same_o &= (no[a] == r->o[a]);
  }
  if (same_d && same_o) return;
  if (same_d)
    spo_reg_shift(r, no);
  else
    spo_reg_replace(r, no, nd);
}

/* grid::min_value of a RegionalGrid: the whole buffer, then empty */
static double spo_reg_min(const spo_reg* r) {
  double m = r->empty;
  if (r->has) {
    double e = r->sys.psi[0][0];
    for (long i = 1; i < r->sys.g.size; ++i)
      if (r->sys.psi[0][i] < e) e = r->sys.psi[0][i];
    m = (r->empty < e) ? r->empty : e;
  }
  return m;
}

static void spo_reg_update(spo_reg* r) {
  spo_rview v;
  int no[3], nd[3];
  if (r->next_resize == 0) {
    const double m0 = spo_reg_min(r);
    r->cutoff = m0 + r->eps;
    r->empty = m0; /* windows made from now on fill with it; the present
                      window's rim keeps what its last move wrote there */
    spo_reg_view(r, &v);
    spo_view_target(&v, 1, r->factor, 0.0, no, nd);
    spo_reg_move(r, no, nd);
    ++r->next_resize;
  } else if (r->next_resize > 0) {
    const int cur = (int)(r->time / r->delta);
    if (cur >= r->next_resize) {
      spo_reg_view(r, &v);
      spo_view_target(&v, r->fixed ? 0 : 1, r->factor, 0.05, no, nd);
      spo_reg_move(r, no, nd);
      r->next_resize = cur + 1;
    }
  }
}

void* spo_reg_create(const spo_desc* d, double resize_delta, double factor, double eps, int fixed,
                     int threads) {
  spo_reg* r = (spo_reg*)calloc(1, sizeof(spo_reg));
  r->gd = *d;
  r->D = d->dim;
  for (int a = 0; a < 3; ++a) {
    r->G[a] = a < d->dim ? d->n[a] + 2 * BD : 1;
    r->o[a] = 0;
    r->d[a] = r->G[a];
  }
  r->empty = 0.0; /* REGIONAL_GRID_OUTER_VALUE, datatypes/inc/grid.h:2022 */
  r->delta = resize_delta;
  r->factor = factor;
  r->eps = eps;
  r->fixed = fixed;
  r->threads = threads > 0 ? threads : 1;
  spo_reg_build(r);
  return r;
}

/* whole-domain interior values in (x-fastest); the window takes its cells */
void spo_reg_set(void* h, const double* global) {
  spo_reg* r = (spo_reg*)h;
  if (!r->has) return;
  const long c0 = r->d[0] - 2 * BD, c1 = r->d[1] - 2 * BD, c2 = r->D == 3 ? r->d[2] - 2 * BD : 1;
  const long n0 = r->gd.n[0], n1 = r->gd.n[1], n2 = r->D == 3 ? r->gd.n[2] : 1;
  const long dz = (r->D == 3) ? BD : 0;
  for (long k = 0; k < c2; ++k)
    for (long j = 0; j < c1; ++j)
      for (long i = 0; i < c0; ++i) {
        const long gx = spo_mod(r->o[0] + i, n0), gy = spo_mod(r->o[1] + j, n1);
        const long gz = r->D == 3 ? spo_mod(r->o[2] + k, n2) : 0;
        r->sys.psi[0][(i + BD) + (j + BD) * r->sys.g.s[1] + (k + dz) * r->sys.g.s[2]] =
            global[gx + n0 * (gy + n1 * gz)];
      }
  spo_update_halo(&r->sys.d, &r->sys.g, r->sys.psi[0]);
}

/* whole-domain interior values out: empty outside the window's interior */
void spo_reg_get(void* h, double* global) {
  spo_reg* r = (spo_reg*)h;
  const long n0 = r->gd.n[0], n1 = r->gd.n[1], n2 = r->D == 3 ? r->gd.n[2] : 1;
  for (long i = 0; i < n0 * n1 * n2; ++i) global[i] = r->empty;
  if (!r->has) return;
  const long c0 = r->d[0] - 2 * BD, c1 = r->d[1] - 2 * BD, c2 = r->D == 3 ? r->d[2] - 2 * BD : 1;
  const long dz = (r->D == 3) ? BD : 0;
  for (long k = 0; k < c2; ++k)
    for (long j = 0; j < c1; ++j)
      for (long i = 0; i < c0; ++i) {
        const long gx = spo_mod(r->o[0] + i, n0), gy = spo_mod(r->o[1] + j, n1);
        const long gz = r->D == 3 ? spo_mod(r->o[2] + k, n2) : 0;
        global[gx + n0 * (gy + n1 * gz)] =
            r->sys.psi[0][(i + BD) + (j + BD) * r->sys.g.s[1] + (k + dz) * r->sys.g.s[2]];
      }
}

/* n iterations of run_model: update(time), equation, step, time += dt */
void spo_reg_step(void* h, int nsteps) {
  spo_reg* r = (spo_reg*)h;
  for (int i = 0; i < nsteps; ++i) {
    spo_reg_update(r);
    if (r->has) spo_sys_step(&r->sys);
    r->time += r->gd.dt;
  }
}

void spo_reg_adjust(void* h, const int o[3], const int d[3]) {
  spo_reg* r = (spo_reg*)h;
  int no[3] = {0, 0, 0}, nd[3] = {1, 1, 1};
  for (int a = 0; a < r->D; ++a) {
    no[a] = o[a];
    nd[a] = d[a];
  }
  spo_reg_move(r, no, nd);
}

/* window origin and dims; state = {empty, cutoff, time, next_resize} */
void spo_reg_window(void* h, int o[3], int d[3], double state[4]) {
  spo_reg* r = (spo_reg*)h;
  for (int a = 0; a < 3; ++a) {
    o[a] = r->o[a];
    d[a] = r->d[a];
  }
  state[0] = r->empty;
  state[1] = r->cutoff;
  state[2] = r->time;
  state[3] = r->next_resize;
}

void spo_reg_destroy(void* h) {
  spo_reg* r = (spo_reg*)h;
  if (r->has) spo_sys_free(&r->sys);
  free(r);
}
