"""Known-answer tests pinning the CPU oracle (oracle/spo.c), which runs without
a GPU: published SplitMix64 outputs, analytic derivatives of smooth periodic
fields (second-order convergence of every stencil point set), an independent
numpy restatement, conservation, the Dirichlet halo rule, and the committed
golden trajectories, the oracle's own and SymPhas's (the SymPhas solver itself
is compared case by case in test_ref_pin.py)."""
import os

import numpy as np
import pytest

import spo

HERE = os.path.dirname(os.path.abspath(__file__))

# first outputs of SplitMix64 seeded with 0 (published reference sequence)
SPLITMIX64_SEED0 = [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F,
                    0xF88BB8A8724C81EC]


def test_splitmix64_published_sequence():
    got = spo.seed_uniform(0, 0.0, 1.0, 4)
    want = np.array([(z >> 11) / 2.0 ** 53 for z in SPLITMIX64_SEED0])
    assert np.array_equal(got, want)
    # lo + (hi - lo) * u, counter stream offsets
    assert np.array_equal(spo.seed_uniform(0, -1.0, 3.0, 4), -1.0 + 4.0 * want)
    assert np.array_equal(spo.seed_uniform(0, 0.0, 1.0, 2, first=2), want[2:])


def smooth(dim, n):
    """Periodic test field on [0, 2pi)^dim with its analytic derivatives."""
    h = 2 * np.pi / n
    c = np.arange(n) * h
    if dim == 2:
        y, x = np.meshgrid(c, c, indexing="ij")
        f = np.sin(x) * np.cos(2 * y)
        k2 = 1 + 4
        fx = np.cos(x) * np.cos(2 * y)
    else:
        z, y, x = np.meshgrid(c, c, c, indexing="ij")
        f = np.sin(x) * np.cos(2 * y) * np.sin(z)
        k2 = 1 + 4 + 1
        fx = np.cos(x) * np.cos(2 * y) * np.sin(z)
    return h, f, {"lap": -k2 * f, "bilap": k2 * k2 * f, "gradlap": -k2 * fx}


OPID = {"lap": spo.OP_LAP, "bilap": spo.OP_BILAP, "gradlap": spo.OP_GRADLAP}
CASES = ([(2, "lap", (p, 6, 13)) for p in (5, 9)] +
         [(2, "bilap", (5, 6, p)) for p in (13, 17)] +
         [(2, "gradlap", (5, p, 13)) for p in (6, 8, 12, 16)] +
         [(3, "lap", (p, 10, 25)) for p in (7, 15, 21, 27)] +
         [(3, "bilap", (7, 10, p)) for p in (21, 25, 41, 52, 57)] +
         [(3, "gradlap", (7, p, 25)) for p in (10, 12, 28, 36, 40)])


def err_at(dim, op, pts, n):
    h, f, exact = smooth(dim, n)
    d = spo.make_desc(dim, (n,) * dim, OPID[op], h, 0.0, stencil=pts)
    return np.max(np.abs(spo.rhs(d, f) - exact[op])) / np.max(np.abs(exact[op]))


@pytest.mark.parametrize("dim,op,pts", CASES)
def test_every_point_set_is_second_order(dim, op, pts):
    n = 16 if dim == 3 else 32
    e1, e2 = err_at(dim, op, pts, n), err_at(dim, op, pts, 2 * n)
    assert e2 < 0.07
    assert 3.3 < e1 / e2 < 4.7, (e1, e2)


def test_bilap21_2d_keeps_the_reference_scaling():
    """Stencil2d2h bilap<21> (stencilh2.h:144-156) weighs its points so that it
    converges to a quarter of the bilaplacian; the oracle (and the kernels)
    keep that, so it tends to 0.25 * bilap(f) at second order."""
    for n in (32, 64):
        h, f, exact = smooth(2, n)
        d = spo.make_desc(2, (n, n), spo.OP_BILAP, h, 0.0, stencil=(5, 6, 21))
        r = spo.rhs(d, f)
        assert np.max(np.abs(r - 0.25 * exact["bilap"])) < 0.05 * np.max(np.abs(exact["bilap"]))


def test_lap19_keeps_the_reference_quirk():
    """Stencil3d2h lap<19> adds vz twice instead of vz + vz_ (stencilh2.h:273):
    exact on fields constant in z, inconsistent once the field varies in z."""
    n = 16
    h = 2 * np.pi / n
    c = np.arange(n) * h
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    fxy = np.sin(x) * np.cos(2 * y)
    d = spo.make_desc(3, (n,) * 3, spo.OP_LAP, h, 0.0, stencil=(19, 10, 25))
    e_flat = np.max(np.abs(spo.rhs(d, fxy) + 5 * fxy)) / 5
    e_z = np.max(np.abs(spo.rhs(d, fxy * np.sin(z)) + 6 * fxy * np.sin(z))) / 6
    assert e_flat < 0.1 and e_z > 0.2


def test_numpy_restatement_bit_identical():
    """Model A and model B right-hand sides restated with numpy rolls, in the
    printed-scheme order, agree with the C oracle bit for bit."""
    n, h = 24, 0.5
    x = spo.seed_uniform(5, -0.5, 0.5, n * n).reshape(n, n)
    divh = 1.0 / h
    divh2 = divh * divh
    divh4 = divh2 * divh2

    def lap5(v):
        vx_, vx = np.roll(v, 1, 1), np.roll(v, -1, 1)
        vy_, vy = np.roll(v, 1, 0), np.roll(v, -1, 0)
        return (vx_ + vx + vy + vy_ - 4.0 * v) * divh2

    def bilap13(v):
        r = lambda a, b: np.roll(np.roll(v, -a, 1), -b, 0)  # value at (x+a, y+b)
        return (r(0, -2) + r(0, 2) + r(-2, 0) + r(2, 0) +
                2.0 * (r(-1, -1) + r(1, -1) + r(-1, 1) + r(1, 1)) -
                8.0 * (r(-1, 0) + r(1, 0) + r(0, -1) + r(0, 1)) + 20.0 * v) * divh4

    cube = x * (x * x)
    a = spo.rhs(spo.make_desc(2, (n, n), spo.MODEL_A, h, 0.0), x)
    assert np.array_equal(a, lap5(x) + (-(1.0 * cube) + 1.0 * x))
    b = spo.rhs(spo.make_desc(2, (n, n), spo.MODEL_B, h, 0.0), x)
    assert np.array_equal(b, -bilap13(x) + (1.0 * lap5(cube) + -(1.0 * lap5(x))))


def test_model_b_conserves_mass_and_lowers_energy():
    n = 16
    d = spo.make_desc(3, (n, n, n), spo.MODEL_B, 1.0, 0.005)
    x0 = spo.seed_uniform(9, -0.3, -0.1, n ** 3).reshape(n, n, n)
    x1 = spo.run(d, x0, 300)
    assert abs(x1.sum() - x0.sum()) <= 1e-12 * abs(x0.sum())

    def energy(v):
        g2 = sum((np.roll(v, -1, a) - v) ** 2 for a in range(3))
        return np.sum(-0.5 * v * v + 0.25 * v ** 4 + 0.5 * g2)

    assert energy(x1) < energy(x0)


def test_dirichlet_halo_rule():
    """A zero field with constant boundary c: the 5-point Laplacian sees c at
    each missing neighbour (c per side, 2c at a corner, h = 1)."""
    n, c = 8, 0.25
    d = spo.make_desc(2, (n, n), spo.OP_LAP, 1.0, 0.0, bc=spo.DIRICHLET, bcv=c)
    r = spo.rhs(d, np.zeros((n, n)))
    assert r[0, 0] == 2 * c and r[0, n // 2] == c and r[n // 2, n // 2] == 0.0


def test_oracle_reproduces_golden_fixtures():
    g = np.load(os.path.join(HERE, "golden", "oracle_golden.npz"))
    cases = {
        "model_a_2d": (2, (16, 12), spo.MODEL_A, 0.5, 0.01, 100, ()),
        "model_b_3d": (3, (8, 8, 6), spo.MODEL_B, 1.0, 0.005, 50, ()),
        "model_c_3d": (3, (8, 6, 8), spo.MODEL_C, 1.0, 0.005, 30, (0.5,)),
        "model_bmk_2d": (2, (12, 16), spo.MODEL_BMK, 1.0, 0.004, 40, (1.5, 0.6)),
    }
    for name, (dim, dims, model, h, dt, steps, coeff) in cases.items():
        d = spo.make_desc(dim, dims, model, h, dt, coeff=coeff)
        out = spo.run(d, g[name + "_init"], steps)
        assert np.array_equal(out, g[name + "_final"]), name
    assert np.array_equal(g["splitmix_seed0_u01"], spo.seed_uniform(0, 0.0, 1.0, 8))


def test_oracle_equals_symphas_golden_trajectories():
    """Trajectories of SymPhas's own CPU SolverFT (written by
    tests/golden/make_golden.py through oracle/ref.mk's build of SymPhas):
    the first configuration (model A 2D 64^2, dx 0.5, dt 0.01, 1000 steps),
    model B 3D 16^3 x 100 steps, model B on SymPhas's default
    Stencil3d2h<15,10,25>.  The oracle reproduces every one bit for bit."""
    g = np.load(os.path.join(HERE, "golden", "symphas_golden.npz"))
    cases = {
        "config_model_a_2d_64": (2, (64, 64), spo.MODEL_A, 0.5, 0.01, 1000, None),
        "model_b_3d_16": (3, (16, 16, 16), spo.MODEL_B, 1.0, 0.005, 100, None),
        "model_b_3d_default_stencil": (3, (12, 10, 8), spo.MODEL_B, 1.0, 0.002, 50, (15, 10, 25)),
    }
    for name, (dim, dims, model, h, dt, steps, st) in cases.items():
        d = spo.make_desc(dim, dims, model, h, dt, stencil=st)
        assert np.array_equal(spo.run(d, g[name + "_init"], steps), g[name + "_final"]), name
