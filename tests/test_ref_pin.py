"""The oracle (oracle/spo.c) against SymPhas itself: SymPhas's own CPU
SolverFT compiled from its sources (oracle/ref.mk -> oracle/_ref/
libsymphas_ref.so), run on the same seeded inputs through its MODEL types,
its coefficient constructor and the update / equation / step loop of
model_iteration (modules-models.h:435-467).

Bit-identical (array equality) wherever SymPhas's evaluation order is the
oracle's: the configurations (model A 2D 64^2 dx 0.5 dt 0.01 x 1000 steps;
model B 3D 32^3 x 200 steps at mean 0 and -0.2), models A and B at unit
coefficients on every stencil family, every operator point set of
Stencil2d2h / Stencil3d2h / Stencil2d4h, and Dirichlet sides in every 2D mix
and in the 3D mixes SymPhas's halo update treats alike (see
test_dirichlet_3d).  For non-unit coefficients SymPhas's optimiser folds the
coefficients into the terms (BMK prints as -c1 c2 V^4(psi) + c1 V^2(psi^3) -
c1 V^2(psi)), so the roundings differ: those runs are held to the 1e-12
relative L-infinity bound of the FP64 parity contract (they agree to ~5e-16).
"""
import numpy as np
import pytest

import spo
import symref

pytestmark = pytest.mark.skipif(symref.loaded() is None,
                                reason="SymPhas's solver is not built (oracle/ref.mk)")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def noise(seed, dims, nf=1, mean=0.0, lo=-0.1, hi=0.1):
    cnt = int(np.prod(dims))
    a = mean + spo.seed_uniform(seed, lo, hi, nf * cnt)
    shape = tuple(reversed(dims))
    return a.reshape((nf,) + shape) if nf > 1 else a.reshape(shape)


def test_config_model_a_2d_64():
    n = 64
    x0 = noise(7, (n, n))
    d = spo.make_desc(2, (n, n), spo.MODEL_A, 0.5, 0.01)
    assert np.array_equal(spo.run(d, x0, 1000), symref.run(d, x0, 1000))


@pytest.mark.parametrize("mean", [0.0, -0.2])
def test_config_model_b_3d_32(mean):
    n = 32
    x0 = noise(11, (n, n, n), mean=mean)
    d = spo.make_desc(3, (n, n, n), spo.MODEL_B, 1.0, 0.005)
    got = symref.run(d, x0, 200)
    assert np.array_equal(spo.run(d, x0, 200), got)
    # conserved: the mass after 200 steps (FP64 sums) equals the initial one
    assert abs(got.sum() - x0.sum()) <= 1e-10 * abs(x0.sum())


OPS2 = ([("lap", (p, 6, 13)) for p in (5, 9)] + [("bilap", (5, 6, p)) for p in (13, 17, 21)] +
        [("gradlap", (5, p, 13)) for p in (6, 8, 12, 16)] + [("lapcube", (5, 6, 13))])
OPS3 = ([("lap", (p, 10, 25)) for p in (7, 15, 19, 21, 27)] +
        [("bilap", (7, 10, p)) for p in (21, 25, 41, 52, 57)] +
        [("gradlap", (7, p, 25)) for p in (10, 12, 28, 36, 40)] + [("lapcube", (7, 10, 25))])
OPS4 = ([("lap", (p, 14, 21)) for p in (9, 17, 21)] + [("bilap", (9, 14, p)) for p in (21, 25, 33, 37)] +
        [("gradlap", (9, p, 21)) for p in (14, 18, 26, 30)] + [("lapcube", (9, 14, 21))])
OPID = {"lap": spo.OP_LAP, "bilap": spo.OP_BILAP, "gradlap": spo.OP_GRADLAP,
        "lapcube": spo.OP_LAPCUBE}


@pytest.mark.parametrize("dim,acc,op,pts", [(2, 2) + c for c in OPS2] + [(3, 2) + c for c in OPS3] +
                         [(2, 4) + c for c in OPS4])
@pytest.mark.parametrize("h", [1.0, 0.7])
def test_every_point_set(dim, acc, op, pts, h):
    dims = (23, 19) if dim == 2 else (13, 11, 9)
    x0 = noise(3, dims, lo=-1.0, hi=1.0)
    d = spo.make_desc(dim, dims, OPID[op], h, 0.0, stencil=pts, acc=acc)
    assert symref.available(d)
    assert np.array_equal(spo.rhs(d, x0), symref.rhs(d, x0))


# (name, dim, dims, model, coefficients, stencil, accuracy, h, dt, fields)
MODELS = [
    ("A", 2, (33, 29), spo.MODEL_A, (0.7, 1.3), (5, 6, 13), 2, 0.5, 0.01, 1),
    ("A default Stencil2d2h<>", 2, (33, 29), spo.MODEL_A, (1.0, 1.0), (9, 6, 13), 2, 0.5, 0.01, 1),
    ("A 3D", 3, (17, 13, 11), spo.MODEL_A, (0.7, 1.3), (7, 10, 25), 2, 1.0, 0.01, 1),
    ("A 4h", 2, (33, 29), spo.MODEL_A, (1.0, 1.0), (9, 14, 21), 4, 1.0, 0.01, 1),
    ("B 2D", 2, (33, 29), spo.MODEL_B, (1.0, 1.0), (5, 6, 13), 2, 1.0, 0.005, 1),
    ("B default Stencil3d2h<>", 3, (17, 13, 11), spo.MODEL_B, (1.0, 1.0), (15, 10, 25), 2, 1.0,
     0.002, 1),
    ("B 4h", 2, (33, 29), spo.MODEL_B, (1.0, 1.0), (9, 14, 21), 4, 1.0, 0.002, 1),
]
FOLDED = [
    ("B coefficients 2D", 2, (33, 29), spo.MODEL_B, (0.7, 1.3), (5, 6, 13), 2, 1.0, 0.005, 1),
    ("B coefficients 3D", 3, (17, 13, 11), spo.MODEL_B, (0.7, 1.3), (7, 10, 25), 2, 1.0, 0.005, 1),
    ("AMK 2D", 2, (33, 29), spo.MODEL_AMK, (1.7, 0.6), (5, 6, 13), 2, 1.0, 0.01, 1),
    ("BMK 2D", 2, (33, 29), spo.MODEL_BMK, (1.7, 0.6), (5, 6, 13), 2, 1.0, 0.005, 1),
    ("AMK 3D", 3, (17, 13, 11), spo.MODEL_AMK, (1.7, 0.6), (7, 10, 25), 2, 1.0, 0.01, 1),
    ("BMK 3D", 3, (17, 13, 11), spo.MODEL_BMK, (1.7, 0.6), (7, 10, 25), 2, 1.0, 0.005, 1),
    ("C 2D", 2, (33, 29), spo.MODEL_C, (0.5,), (5, 6, 13), 2, 1.0, 0.005, 2),
    ("C 3D", 3, (17, 13, 11), spo.MODEL_C, (0.5,), (7, 10, 25), 2, 1.0, 0.005, 2),
    ("C 4h", 2, (33, 29), spo.MODEL_C, (0.5,), (9, 14, 21), 4, 1.0, 0.002, 2),
    ("AMK 4h", 2, (33, 29), spo.MODEL_AMK, (1.7, 0.6), (9, 14, 21), 4, 0.8, 0.005, 1),
    ("BMK 4h", 2, (33, 29), spo.MODEL_BMK, (1.7, 0.6), (9, 14, 21), 4, 1.0, 0.002, 1),
]


def _run_both(case, steps):
    name, dim, dims, model, coef, st, acc, h, dt, nf = case
    x0 = noise(5, dims, nf=nf, mean=0.1)
    d = spo.make_desc(dim, dims, model, h, dt, coeff=coef, stencil=st, acc=acc)
    return spo.run(d, x0, steps), symref.run(d, x0, steps), spo.rhs(d, x0), symref.rhs(d, x0)


@pytest.mark.parametrize("case", MODELS, ids=[c[0] for c in MODELS])
def test_models_bit_identical(case):
    a, b, ra, rb = _run_both(case, 50)
    assert np.array_equal(ra, rb)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("case", FOLDED, ids=[c[0] for c in FOLDED])
def test_models_folded_coefficients(case):
    a, b, ra, rb = _run_both(case, 50)
    assert rel(ra, rb) <= 1e-12
    assert rel(a, b) <= 1e-12


def test_provisional_variable_mbb_is_model_b():
    """SymPhas's MBB (examples/models/modeldefinitions.h:152-156) with c1 = 1,
    c2 = 1/4 has var(1) = psi^3 - psi: model B, through a provisional system.

    In SymPhas's CPU-only build the provisional variable has no halo update:
    SolverFT associates its boundary-managed provisional system only under
    USING_CUDA (examples/solvers/solverft.h:228-235), so var(1)'s halo stays 0
    and lap(var(1)) differs from model B on the first ring of sites.  The
    rest of the grid is model B to rounding (var is evaluated as
    -(c1 - 4 c2 psi^2) psi).  This project fills the halo, as the CUDA build
    of SymPhas does."""
    dims = (24, 20)
    x0 = noise(13, dims, mean=-0.1)
    d = spo.make_desc(2, dims, symref.MODEL_MBB, 1.0, 0.005, coeff=(1.0, 0.25))
    db = spo.make_desc(2, dims, spo.MODEL_B, 1.0, 0.005)
    got, want = symref.rhs(d, x0), spo.rhs(db, x0)
    inner = (slice(1, -1), slice(1, -1))
    assert rel(got[inner], want[inner]) <= 1e-12
    ring = np.ones(got.shape, bool)
    ring[inner] = False
    assert np.max(np.abs(got - want)[ring]) > 1e-3  # the zero halo shows on the ring


SIDES = [spo.DIRICHLET] * 6
VALUES = [0.1, -0.1, 0.3, -0.2, 0.05, 0.15]


def _bc(axes):
    return [spo.DIRICHLET if (a // 2) in axes else spo.PERIODIC for a in range(6)]


@pytest.mark.parametrize("axes", [(0,), (1,), (0, 1)])
@pytest.mark.parametrize("model", [spo.MODEL_A, spo.MODEL_B])
def test_dirichlet_2d(axes, model):
    dims = (33, 29)
    x0 = noise(9, dims)
    d = spo.make_desc(2, dims, model, 1.0, 0.005, bc=_bc(axes), bcv=VALUES)
    assert np.array_equal(spo.run(d, x0, 40), symref.run(d, x0, 40))


@pytest.mark.parametrize("axes", [(0,), (0, 1), (0, 2), (1, 2), (0, 1, 2), (1,), (2,)])
@pytest.mark.parametrize("model", [spo.MODEL_A, spo.MODEL_B])
def test_dirichlet_3d(axes, model):
    """With exactly one Dirichlet axis of y or z in 3D, SymPhas's halo update
    (validate_periodic_boundaries picks one PERIODIC3 variant for one pair of
    sides, sol/inc/boundarygroup.h:200-243) leaves some edge cells of the halo
    off the boundary condition: with y Dirichlet the y-z edges hold periodic
    images (as if y were periodic), with z Dirichlet the x-y edges are never
    written.  Only stencils with diagonal points read those cells, so model A
    (7-point Laplacian) stays bit-identical there and model B (bilaplacian<25>)
    is compared only on the other mixes."""
    if model == spo.MODEL_B and axes in ((1,), (2,)):
        pytest.skip("SymPhas's edge cells are off the boundary condition for this mix")
    dims = (17, 13, 11)
    x0 = noise(9, dims)
    d = spo.make_desc(3, dims, model, 1.0, 0.005, bc=_bc(axes), bcv=VALUES)
    assert np.array_equal(spo.run(d, x0, 30), symref.run(d, x0, 30))
