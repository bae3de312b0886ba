"""The configurations at their stated sizes, against the oracle (FP64, all
host threads) and, where it is affordable, against SymPhas's own solver:

- model B 3D 256^3 (dx 1, dt 0.005, Stencil3d2h<7,10,25>, psi_bar -0.2 +-
  0.1): the FP64 exact step bit-identical after 10 steps; the FP32 fused step
  (the autotuned kernel the benchmark times) within 1e-5 relative L-infinity
  of FP64 after 1, 10 and 100 steps;
- the ensemble of 1024 2D members (sides 64..1024, AMK/BMK, M and kappa in
  [0.5, 2], dt 40 % of each stability limit): all 1024 advanced together for
  200 steps; a stratified sample -- every side with both models, and the
  members of smallest and largest M and kappa -- checked member by member,
  FP64 exact bit-identical and FP32 fused within 2e-4;
- model C, 8 instances of 256^3 (gamma 0.5, psi 0.1 +- 0.1, eta +- 0.1):
  the FP32 fused batch within 1e-5 of FP64 after 5 steps (first and last
  instance), the FP64 exact batch bit-identical for one instance.
"""
import os

import numpy as np
import pytest

import spo
import symphas_b200 as sp
import symref

pytestmark = pytest.mark.gpu

S3 = sp.Stencil3d2h(7, 10, 25)
S2 = sp.Stencil2d2h(5, 6, 13)
THREADS = os.cpu_count() or 1
ORACLE_MODEL = {"AMK": spo.MODEL_AMK, "BMK": spo.MODEL_BMK}


def rel_linf(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def b256_init():
    n = 256
    return spo.seed_uniform(20261203, -0.3, -0.1, n ** 3).reshape(n, n, n)


def b256(form, dtype):
    n = 256
    m = sp.model_MB_t(3, sp.SolverFT(S3, form=form), sp.ProblemParameters((n, n, n), h=1.0),
                      dtype=dtype)
    m.fill_uniform(0, 20261203, -0.3, -0.1)
    return m


def test_model_b_256_fp64_exact_bit_identical():
    n, steps = 256, 10
    m = b256("exact", "f64")
    x0 = b256_init()
    assert np.array_equal(m.get_field(0), x0)
    m.step(0.005, steps)
    got = m.get_field(0)
    m.close()
    d = spo.make_desc(3, (n, n, n), spo.MODEL_B, 1.0, 0.005)
    assert np.array_equal(got, spo.run(d, x0, steps, threads=THREADS))
    if symref.loaded() is not None:  # SymPhas itself, on one core: 3 steps
        m = b256("exact", "f64")
        m.step(0.005, 3)
        assert np.array_equal(m.get_field(0), symref.run(d, x0, 3))
        m.close()


def test_model_b_256_fp32_fused_within_1e_5_of_fp64():
    n = 256
    m = b256("fused", "f32")
    m.autotune(3)
    x = b256_init()
    d = spo.make_desc(3, (n, n, n), spo.MODEL_B, 1.0, 0.005)
    done = 0
    for steps in (1, 10, 100):
        m.step(0.005, steps - done)
        x = spo.run(d, x, steps - done, threads=THREADS)
        done = steps
        err = rel_linf(m.get_field(0).astype(np.float64), x)
        assert err <= 1e-5, (steps, err)
    m.close()


def stratified(members):
    """Every side with both models, and the members of smallest and largest M
    and kappa."""
    pick = {}
    for i, mb in enumerate(members):
        pick.setdefault((mb["dims"][0], mb["model"]), i)
    idx = set(pick.values())
    for c in (0, 1):
        vals = [mb["coeff"][c] for mb in members]
        idx.add(int(np.argmin(vals)))
        idx.add(int(np.argmax(vals)))
    return sorted(idx)


@pytest.mark.parametrize("form,dtype,tol", [("exact", "f64", 0.0), ("fused", "f32", 2e-4)])
def test_ensemble_1024_members_stratified_sample(form, dtype, tol):
    seed, steps = 20261203, 200
    members = sp.ensemble_members(1024, seed=seed)
    ens = sp.Ensemble(sp.SolverFT(S2, form=form), members, dtype=dtype)
    for i in range(len(members)):
        ens.fill_uniform(0, seed + i, -0.1, 0.1, inst=i)
    if form == "fused":
        ens.autotune(3)
    ens.step(steps)
    sample = stratified(members)
    assert len({(members[i]["dims"][0], members[i]["model"]) for i in sample}) == 16
    descs, fields = [], []
    for i in sample:
        mb = members[i]
        descs.append(spo.make_desc(2, mb["dims"], ORACLE_MODEL[mb["model"]], 1.0, mb["dt"],
                                   coeff=mb["coeff"]))
        fields.append(spo.seed_uniform(seed + i, -0.1, 0.1, mb["dims"][0] * mb["dims"][1]))
    spo.run_batch(descs, fields, [steps] * len(sample), THREADS)
    worst = 0.0
    for i, ref in zip(sample, fields):
        nx, ny = members[i]["dims"]
        got = ens.get_field(0, inst=i).astype(np.float64)
        ref = ref.reshape(ny, nx)
        if tol == 0.0:
            assert np.array_equal(got, ref), i
        else:
            worst = max(worst, rel_linf(got, ref))
    ens.close()
    assert worst <= tol, worst


@pytest.mark.parametrize("form,dtype", [("exact", "f64"), ("fused", "f32")])
def test_ensemble_1024_members_5000_steps(form, dtype):
    """The configuration's full length: all 1024 members advanced 5000 steps
    of their own dt in one launch per step (graph-replayed), then the
    stratified sample checked against the FP64 oracle, member by member: the
    exact form bit-identical, the fused FP32 form within 5e-3 relative
    L-infinity (printed per member: the figure the configuration asks for)."""
    seed, steps = 20261203, 5000
    members = sp.ensemble_members(1024, seed=seed)
    ens = sp.Ensemble(sp.SolverFT(S2, form=form), members, dtype=dtype)
    for i in range(len(members)):
        ens.fill_uniform(0, seed + i, -0.1, 0.1, inst=i)
    if form == "fused":
        ens.autotune(3)
    ens.step(steps)
    sample = stratified(members)
    descs, fields = [], []
    for i in sample:
        mb = members[i]
        descs.append(spo.make_desc(2, mb["dims"], ORACLE_MODEL[mb["model"]], 1.0, mb["dt"],
                                   coeff=mb["coeff"]))
        fields.append(spo.seed_uniform(seed + i, -0.1, 0.1, mb["dims"][0] * mb["dims"][1]))
    spo.run_batch(descs, fields, [steps] * len(sample), THREADS)
    worst = 0.0
    for i, ref in zip(sample, fields):
        nx, ny = members[i]["dims"]
        got = ens.get_field(0, inst=i).astype(np.float64)
        ref = ref.reshape(ny, nx)
        if dtype == "f64":
            assert np.array_equal(got, ref), i
        else:
            e = rel_linf(got, ref)
            print("member %d (%s %dx%d, M %.3f, kappa %.3f): FP32 vs FP64 rel L-inf %.3e"
                  % (i, members[i]["model"], nx, ny, members[i]["coeff"][0],
                     members[i]["coeff"][1], e))
            worst = max(worst, e)
    ens.close()
    assert worst <= 5e-3, worst


def test_model_c_8x256_batch():
    n, batch, steps = 256, 8, 5
    coeff = (0.5,)

    def init(i):
        return np.stack([spo.seed_uniform(7000 + 2 * i, 0.0, 0.2, n ** 3),
                         spo.seed_uniform(7001 + 2 * i, -0.1, 0.1, n ** 3)]).reshape(2, n, n, n)

    d = spo.make_desc(3, (n, n, n), spo.MODEL_C, 1.0, 0.005, coeff=coeff)
    for form, dtype, check in (("fused", "f32", (0, batch - 1)), ("exact", "f64", (3,))):
        m = sp.model_MC_t(3, sp.SolverFT(S3, form=form), sp.ProblemParameters((n, n, n), h=1.0),
                          coeff=coeff, dtype=dtype, batch=batch)
        for i in range(batch):
            m.fill_uniform(0, 7000 + 2 * i, 0.0, 0.2, inst=i)
            m.fill_uniform(1, 7001 + 2 * i, -0.1, 0.1, inst=i)
        m.step(0.005, steps)
        for i in check:
            got = np.stack([m.get_field(f, inst=i) for f in range(2)]).astype(np.float64)
            ref = spo.run(d, init(i), steps, threads=THREADS)
            if dtype == "f64":
                assert np.array_equal(got, ref), i
            else:
                assert rel_linf(got, ref) <= 1e-5, (i, rel_linf(got, ref))
        m.close()
