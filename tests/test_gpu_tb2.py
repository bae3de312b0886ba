"""The temporally blocked 2D step (sp_tb2.cuh): up to k steps per launch,
each tile loaded once with a margin of k * R sites wrapped around the
periodic faces, the steps run in shared memory.

Every site of every step is evaluated by the expression code of the one-step
kernel in the same order, so:
- in the exact form (FP64) it is bit-identical to the CPU oracle after any
  number of steps, including counts that are not multiples of k (the last
  launch then runs fewer steps) and counts long enough for graph replay;
- in the fused form (FP32) it is bit-identical to the one-step kernel;
- ensembles of members of different sizes, models and coefficients give each
  member the bits of the one-step ensemble kernel;
- the right-hand side evaluation and the fused mass of the last step match;
- grids it cannot run (Dirichlet sides, x extents not a multiple of 16 bytes)
  fall back to the one-step kernel.
"""
import numpy as np
import pytest

import spo
import symphas_b200 as sp

pytestmark = pytest.mark.gpu

S2 = sp.Stencil2d2h(5, 6, 13)
CLS = {"A": sp.model_MA_t, "B": sp.model_MB_t, "C": sp.model_MC_t,
       "AMK": sp.model_MAMK_t, "BMK": sp.model_MBMK_t}
ORACLE = {"A": spo.MODEL_A, "B": spo.MODEL_B, "C": spo.MODEL_C, "AMK": spo.MODEL_AMK,
          "BMK": spo.MODEL_BMK}
COEFF = {"A": (), "B": (), "C": (0.5,), "AMK": (1.3, 0.7), "BMK": (0.8, 1.4)}
DT = {"A": 0.02, "B": 0.004, "C": 0.004, "AMK": 0.02, "BMK": 0.004}


def make(name, dims, form, dtype, tile=None, monkeypatch=None, bc=None):
    if tile is not None:
        monkeypatch.setenv("SP_TILE", str(tile))
    params = sp.ProblemParameters(dims, h=1.0) if bc is None else \
        sp.ProblemParameters(dims, h=1.0, boundary=bc, boundary_value=0.2)
    m = CLS[name](2, sp.SolverFT(S2, form=form), params, coeff=COEFF[name], dtype=dtype)
    if tile is not None:
        monkeypatch.delenv("SP_TILE")
    for f in range(m.nfields):
        m.fill_uniform(f, 31 + f, -0.3, 0.3)
    return m


def blocked_variants(name, form, dtype, monkeypatch, dims=(128, 64)):
    """Indices of the temporally blocked variants of this kernel key."""
    base = make(name, dims, form, dtype)
    nv = base.kernel_info()["variants"]
    base.close()
    out = []
    for v in range(nv):
        m = make(name, dims, form, dtype, v, monkeypatch)
        info = m.kernel_info()
        if info["variant"] == v and info["steps_per_launch"] > 1:
            out.append((v, info["steps_per_launch"]))
        m.close()
    return out


def fields(m):
    return np.stack([m.get_field(f) for f in range(m.nfields)])


@pytest.mark.parametrize("name", ["A", "B", "C"])
@pytest.mark.parametrize("dims", [(100, 70), (64, 36), (130, 98)])
@pytest.mark.parametrize("steps", [1, 2, 5, 70])
def test_exact_fp64_bit_identical_to_oracle(name, dims, steps, monkeypatch):
    tb = blocked_variants(name, "exact", "f64", monkeypatch)
    assert tb, "no temporally blocked FP64 kernel for model " + name
    for v, kt in tb:
        m = make(name, dims, "exact", "f64", v, monkeypatch)
        assert m.kernel_info()["steps_per_launch"] == kt
        x0 = np.stack([spo.seed_uniform(31 + f, -0.3, 0.3, dims[0] * dims[1]).reshape(dims[1], dims[0])
                       for f in range(m.nfields)])
        assert np.array_equal(fields(m), x0)
        launches = m.launch_count()
        m.step(DT[name], steps)
        assert m.launch_count() - launches <= -(-steps // kt) + 1
        d = spo.make_desc(2, dims, ORACLE[name], 1.0, DT[name], coeff=COEFF[name])
        want = spo.run(d, x0 if m.nfields > 1 else x0[0], steps)
        got = fields(m)
        assert np.array_equal(got if m.nfields > 1 else got[0], want), (v, kt)
        m.close()


@pytest.mark.parametrize("name", ["A", "B", "C", "AMK", "BMK"])
@pytest.mark.parametrize("dims", [(256, 96), (132, 76), (64, 64), (16, 24)])
def test_fused_fp32_same_bits_as_one_step_kernel(name, dims, monkeypatch):
    tb = blocked_variants(name, "fused", "f32", monkeypatch)
    assert len(tb) >= 2, tb
    steps = 37
    ref = make(name, dims, "fused", "f32", 0, monkeypatch)
    ref.step(DT[name], steps)
    want = fields(ref)
    ref.close()
    for v, kt in tb:
        m = make(name, dims, "fused", "f32", v, monkeypatch)
        m.step(DT[name], steps)
        assert np.array_equal(fields(m), want), (name, dims, v, kt)
        m.close()


def test_graph_replay_and_remainders(monkeypatch):
    """Long step counts go through the captured graph of launches of k steps;
    the remainder through shorter launches: the same bits as one-step launches."""
    name, dims = "B", (128, 96)
    ref = make(name, dims, "fused", "f32", 0, monkeypatch)
    for v, kt in blocked_variants(name, "fused", "f32", monkeypatch):
        m = make(name, dims, "fused", "f32", v, monkeypatch)
        r = make(name, dims, "fused", "f32", 0, monkeypatch)
        for n in (3, 64 * kt + 1, 129):
            m.step(DT[name], n)
            r.step(DT[name], n)
            assert np.array_equal(fields(m), fields(r)), (v, n)
        m.close()
        r.close()
    ref.close()


@pytest.mark.parametrize("name", ["B", "C", "AMK"])
def test_rhs_and_fused_mass(name, monkeypatch):
    dims = (128, 68)
    ref = make(name, dims, "fused", "f32", 0, monkeypatch)
    r0 = [ref.eval_rhs(f) for f in range(ref.nfields)]
    m0 = ref.step_mass(DT[name], 9)
    want = fields(ref)
    ref.close()
    for v, kt in blocked_variants(name, "fused", "f32", monkeypatch):
        m = make(name, dims, "fused", "f32", v, monkeypatch)
        for f in range(m.nfields):
            assert np.array_equal(m.eval_rhs(f), r0[f]), (v, f)
        masses = m.step_mass(DT[name], 9)
        assert np.array_equal(fields(m), want)
        assert abs(masses[0] - m0[0]) <= 1e-12 * max(abs(m0[0]), 1.0)
        m.close()


def test_not_applicable_falls_back(monkeypatch):
    """Dirichlet sides, or an x extent that is not a whole number of 16-byte
    copies: the temporally blocked shape is refused and the default runs."""
    tb = blocked_variants("B", "fused", "f32", monkeypatch)
    P, D = sp.BoundaryType.PERIODIC, sp.BoundaryType.DEFAULT
    for v, _ in tb:
        m = make("B", (128, 64), "fused", "f32", v, monkeypatch, bc=[D, D, P, P, P, P])
        assert m.kernel_info()["variant"] == 0 and m.kernel_info()["steps_per_launch"] == 1
        m.close()
        m = make("B", (130, 64), "fused", "f32", v, monkeypatch)
        assert m.kernel_info()["variant"] == 0
        m.close()


MEMBERS = [
    {"dims": (16, 16), "model": "AMK", "coeff": (1.0, 1.0)},
    {"dims": (40, 24), "model": "BMK", "coeff": (0.7, 1.3)},
    {"dims": (132, 34), "model": "AMK", "coeff": (1.9, 0.6)},
    {"dims": (36, 70), "model": "BMK", "coeff": (1.2, 0.5)},
    {"dims": (256, 200), "model": "BMK", "coeff": (0.5, 2.0)},
    {"dims": (64, 96), "model": "AMK", "coeff": (0.8, 1.7)},
]


def with_dt(members, safety=0.4):
    out = []
    for m in members:
        M, kappa = m["coeff"]
        lim = (2.0 / (M * (8.0 * kappa + 2.0)) if m["model"] == "AMK"
               else 2.0 / (M * (64.0 * kappa + 16.0)))
        out.append(dict(m, dt=safety * lim))
    return out


@pytest.mark.parametrize("form,dtype", [("fused", "f32"), ("exact", "f64")])
def test_ensemble_members_same_bits(form, dtype, monkeypatch):
    members = with_dt(MEMBERS)

    def run(v):
        monkeypatch.setenv("SP_TILE", str(v))
        ens = sp.Ensemble(sp.SolverFT(S2, form=form), members, dtype=dtype)
        monkeypatch.delenv("SP_TILE")
        info = ens.kernel_info()
        for i in range(len(members)):
            ens.fill_uniform(0, 500 + i, -0.3, 0.3, inst=i)
        ens.step(41)
        out = [ens.get_field(0, inst=i) for i in range(len(members))]
        ens.close()
        return info, out

    info0, ref = run(0)
    blocked = 0
    for v in range(1, info0["variants"]):
        info, out = run(v)
        if info["variant"] != v:
            continue
        for i, (a, b) in enumerate(zip(out, ref)):
            assert np.array_equal(a, b), (v, i)
        blocked += info["steps_per_launch"] > 1
    assert blocked >= 1
    if dtype == "f64":  # and the exact form is the oracle's
        for i, mb in enumerate(members):
            nx, ny = mb["dims"]
            d = spo.make_desc(2, mb["dims"], ORACLE[mb["model"]], 1.0, mb["dt"], coeff=mb["coeff"])
            x0 = spo.seed_uniform(500 + i, -0.3, 0.3, nx * ny).reshape(ny, nx)
            assert np.array_equal(ref[i], spo.run(d, x0, 41)), i


def test_autotune_leaves_the_state_and_reports_its_depth():
    """The autotuner times the blocked shapes by launches into the buffer that
    is not current: the fields are unchanged, and the choice (with its depth)
    is what the next system of the same kernel and size starts with."""
    def mk():
        m = sp.model_MA_t(2, sp.SolverFT(S2, form="fused"), sp.ProblemParameters((1024, 512), h=1.0),
                          dtype="f32")
        m.fill_uniform(0, 3, -0.1, 0.1)
        return m

    m = mk()
    x0 = m.get_field(0)
    info = m.autotune(5)
    assert np.array_equal(m.get_field(0), x0)
    assert info["steps_per_launch"] >= 1
    m2 = mk()
    assert m2.kernel_info()["variant"] == info["variant"]
    m.step(0.02, 23)
    m2.step(0.02, 23)
    assert np.array_equal(m.get_field(0), m2.get_field(0))
    m.close()
    m2.close()
