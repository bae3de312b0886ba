"""Ensembles of independent 2D systems (sp_create_ensemble): members of
different extents, models (model_MAMK_t / model_MBMK_t), coefficients and time
steps advanced by one persistent kernel launch per step.

Each member must evolve exactly as the same system run alone: in the exact
form and FP64 bit-identical to the CPU oracle, in the fused form within 1e-10
relative L-infinity of the oracle (FP64) and 2e-5 (FP32, against the FP64
oracle, 40 steps of fields of magnitude ~0.3)."""
import numpy as np
import pytest

import spo
import symphas_b200 as sp
from symphas_b200 import _capi as C

pytestmark = pytest.mark.gpu

S2 = sp.Stencil2d2h(5, 6, 13)
ORACLE_MODEL = {"AMK": spo.MODEL_AMK, "BMK": spo.MODEL_BMK}

# ragged on purpose: extents that are not multiples of the tile, odd x
# extents (scalar store path), a member smaller than one tile and one that
# spans several tiles in both directions
MEMBERS = [
    {"dims": (16, 16), "model": "AMK", "coeff": (1.0, 1.0)},
    {"dims": (40, 24), "model": "BMK", "coeff": (0.7, 1.3)},
    {"dims": (130, 34), "model": "AMK", "coeff": (1.9, 0.6)},
    {"dims": (33, 70), "model": "BMK", "coeff": (1.2, 0.5)},
    {"dims": (64, 64), "model": "BMK", "coeff": (0.5, 2.0)},
    {"dims": (27, 19), "model": "AMK", "coeff": (0.8, 1.7)},
]


def with_dt(members, h=1.0, safety=0.4):
    out = []
    for m in members:
        M, kappa = m["coeff"]
        if m["model"] == "AMK":
            lim = 2.0 / (M * (8.0 * kappa / h ** 2 + 2.0))
        else:
            lim = 2.0 / (M * (64.0 * kappa / h ** 4 + 16.0 / h ** 2))
        out.append(dict(m, dt=safety * lim))
    return out


def oracle_member(m, x0, steps, h=1.0):
    d = spo.make_desc(2, m["dims"], ORACLE_MODEL[m["model"]], h, m["dt"], coeff=m["coeff"])
    return spo.run(d, x0, steps)


def rel_linf(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def seeded(ens, members):
    inits = []
    for i, m in enumerate(members):
        ens.fill_uniform(0, 100 + i, -0.3, 0.3, inst=i)
        nx, ny = m["dims"]
        inits.append(spo.seed_uniform(100 + i, -0.3, 0.3, nx * ny).reshape(ny, nx))
    return inits


@pytest.mark.parametrize("form,dtype,tol", [("exact", "f64", 0.0), ("fused", "f64", 1e-10),
                                            ("fused", "f32", 2e-5)])
def test_ensemble_members_match_the_oracle(form, dtype, tol):
    members = with_dt(MEMBERS)
    steps = 40
    ens = sp.Ensemble(sp.SolverFT(S2, form=form), members, dtype=dtype)
    inits = seeded(ens, members)
    for i, m in enumerate(members):
        got = ens.get_field(0, inst=i)
        assert got.shape == inits[i].shape
        assert np.array_equal(got, inits[i].astype(ens.np_dtype))
    ens.step(steps)
    for i, m in enumerate(members):
        ref = oracle_member(m, inits[i], steps)
        got = ens.get_field(0, inst=i).astype(np.float64)
        err = rel_linf(got, ref)
        if tol == 0.0:
            assert np.array_equal(got, ref), (i, m, err)
        else:
            assert err <= tol, (i, m, err)
    ens.close()


def test_ensemble_member_equals_the_same_system_alone():
    """FP32 fused: the ensemble kernel (both models in one launch) and the
    single-model kernel compute every site with the same operations."""
    members = with_dt(MEMBERS)
    steps = 25
    ens = sp.Ensemble(sp.SolverFT(S2, form="fused"), members, dtype="f32")
    seeded(ens, members)
    ens.step(steps)
    for i, m in enumerate(members):
        cls = sp.model_MAMK_t if m["model"] == "AMK" else sp.model_MBMK_t
        alone = cls(2, sp.SolverFT(S2, form="fused"), sp.ProblemParameters(m["dims"]),
                    coeff=m["coeff"], dtype="f32")
        alone.fill_uniform(0, 100 + i, -0.3, 0.3)
        alone.step(m["dt"], steps)
        a, b = ens.get_field(0, inst=i), alone.get_field(0)
        assert rel_linf(a.astype(np.float64), b.astype(np.float64)) <= 1e-6, i
        alone.close()
    ens.close()


def test_ensemble_uploads_reductions_and_graphs():
    """Per-member upload/download of differing shapes, FP64 mass of each
    member (conserved for BMK members), graph-replayed steps (64 = two graph
    chunks) equal to single launches, and sp_set_dt refused."""
    members = with_dt(MEMBERS)
    a = sp.Ensemble(sp.SolverFT(S2, form="fused"), members, dtype="f64")
    b = sp.Ensemble(sp.SolverFT(S2, form="fused"), members, dtype="f64")
    rng = np.random.default_rng(3)
    fields = [rng.uniform(-0.4, 0.2, size=(m["dims"][1], m["dims"][0])) for m in members]
    for i, f in enumerate(fields):
        a.set_field(0, f, inst=i)
        b.set_field(0, f, inst=i)
        assert np.array_equal(a.get_field(0, inst=i), f)
    a.step(64)
    for _ in range(64):
        b.step(1)
    for i, m in enumerate(members):
        fa = a.get_field(0, inst=i)
        assert np.array_equal(fa, b.get_field(0, inst=i)), i
        mass, _ = a.reduce(0, inst=i)
        assert abs(mass - fa.sum()) <= 1e-12 * max(1.0, abs(fa.sum()))
        if m["model"] == "BMK":
            assert abs(mass - fields[i].sum()) <= 1e-10 * fields[i].size
    assert C.lib().sp_set_dt(a._h, 0.01) == C.SP_EINVAL
    assert b"own dt" in C.lib().sp_last_error(a._h)
    a.close()
    b.close()


def test_ensemble_of_one_model_uses_its_kernel():
    members = with_dt([m for m in MEMBERS if m["model"] == "BMK"])
    ens = sp.Ensemble(sp.SolverFT(S2, form="fused"), members, dtype="f32")
    inits = seeded(ens, members)
    ens.step(10)
    for i, m in enumerate(members):
        ref = oracle_member(m, inits[i], 10)
        assert rel_linf(ens.get_field(0, inst=i).astype(np.float64), ref) <= 2e-5
    ens.close()


def test_generated_sweep_runs_and_stays_bounded():
    """The sweep generator's members (sides 64..1024, M and kappa in
    U[0.5, 2], dt 40% of each member's stability limit) stay finite and
    bounded over 200 steps; every BMK member conserves its mass."""
    members = sp.ensemble_members(24, seed=1, sides=(64, 96, 128, 256))
    ens = sp.Ensemble(sp.SolverFT(S2, form="fused"), members, dtype="f32")
    for i in range(len(members)):
        ens.fill_uniform(0, 500 + i, -0.2, 0.2, inst=i)
    m0 = [ens.reduce(0, inst=i)[0] for i in range(len(members))]
    ens.step(200)
    for i, m in enumerate(members):
        f = ens.get_field(0, inst=i)
        assert np.isfinite(f).all() and np.max(np.abs(f)) < 1.5, i
        if m["model"] == "BMK":
            assert abs(ens.reduce(0, inst=i)[0] - m0[i]) <= 1e-3 * f.size ** 0.5
    ens.close()


def test_every_tile_shape_gives_the_same_members(monkeypatch):
    """The autotuner may pick any tile shape of the ensemble kernel (2 or 4
    sites per thread): each gives the same bits, ragged members included."""
    members = with_dt(MEMBERS)
    ref, nv = None, None
    for v in range(64):
        monkeypatch.setenv("SP_TILE", str(v))
        ens = sp.Ensemble(sp.SolverFT(S2, form="fused"), members, dtype="f32")
        info = ens.kernel_info()
        nv = info["variants"]
        if info["variant"] != v:
            ens.close()
            if v >= nv:
                break
            continue
        seeded(ens, members)
        ens.step(30)
        out = [ens.get_field(0, inst=i) for i in range(len(members))]
        ens.close()
        if ref is None:
            ref = out
        else:
            for a, b in zip(out, ref):
                assert np.array_equal(a, b), v
    monkeypatch.delenv("SP_TILE")
    assert nv and nv > 1


def test_large_ensemble_members_equal_the_systems_alone():
    """72 members of 1024^2 (~37 K tiles): enough work per CTA that the
    kernel takes its work items in batches, requested ahead.  Members must
    still evolve exactly as the same systems run alone."""
    base = {"dims": (1024, 1024), "model": "BMK", "coeff": (1.0, 1.0)}
    members = with_dt([dict(base, model="AMK" if i % 2 else "BMK", coeff=(1.0 + 0.01 * i, 1.0))
                       for i in range(72)])
    ens = sp.Ensemble(sp.SolverFT(S2, form="fused"), members, dtype="f32")
    for i in range(len(members)):
        ens.fill_uniform(0, 500 + i, -0.3, 0.3, inst=i)
    ens.step(3)
    for i in (0, 35, 71):
        m = members[i]
        cls = sp.model_MAMK_t if m["model"] == "AMK" else sp.model_MBMK_t
        alone = cls(2, sp.SolverFT(S2, form="fused"), sp.ProblemParameters(m["dims"]),
                    coeff=m["coeff"], dtype="f32")
        alone.fill_uniform(0, 500 + i, -0.3, 0.3)
        alone.step(m["dt"], 3)
        assert np.array_equal(ens.get_field(0, inst=i), alone.get_field(0)), i
        alone.close()
    ens.close()
