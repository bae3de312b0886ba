"""GPU parity: the fused sm_100a kernels (through the C ABI) against the CPU
oracle on the same seeded fields.

Tolerances: FP64 exact form -- bit-identical (and therefore <= 1e-12 relative
L-infinity); FP64 fused form -- 1e-10 relative; FP32 -- stated per case
against the FP64 oracle.
"""
import numpy as np
import pytest

import spo
import symphas_b200 as sp

pytestmark = pytest.mark.gpu

S2 = sp.Stencil2d2h(5, 6, 13)
S3 = sp.Stencil3d2h(7, 10, 25)


def rel_linf(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def oracle_init(seed, lo, hi, shape):
    return spo.seed_uniform(seed, lo, hi, int(np.prod(shape))).reshape(shape)


def model_of(cls, dim, dims, h, form="exact", dtype="f64", stencil=None, coeff=(), **kw):
    st = stencil or (S2 if dim == 2 else S3)
    return cls(dim, sp.SolverFT(st, form=form), sp.ProblemParameters(dims, h=h, **kw),
               coeff=coeff, dtype=dtype)


@pytest.mark.parametrize("dim,dims", [(2, (64, 48)), (3, (24, 20, 16))])
def test_fill_uniform_matches_oracle_bits(dim, dims):
    m = model_of(sp.model_MA_t, dim, dims, 1.0)
    m.fill_uniform(0, 1234, -0.3, 0.1)
    got = m.get_field(0)
    ref = oracle_init(1234, -0.3, 0.1, m.shape)
    assert np.array_equal(got, ref)
    m32 = model_of(sp.model_MA_t, dim, dims, 1.0, dtype="f32")
    m32.fill_uniform(0, 1234, -0.3, 0.1)
    assert np.array_equal(m32.get_field(0), ref.astype(np.float32))


def test_model_a_2d_config_bit_identical():
    """Allen-Cahn 64x64 periodic, dx 0.5, dt 0.01, 1000 steps, Stencil2d2h<5,6,13>."""
    n, h, dt, steps = 64, 0.5, 0.01, 1000
    m = model_of(sp.model_MA_t, 2, (n, n), h)
    m.fill_uniform(0, 11, -0.1, 0.1)
    sp.find_solution(m, dt, steps)
    got = m.get_field(0)
    ref = spo.run(spo.make_desc(2, (n, n), spo.MODEL_A, h, dt), oracle_init(11, -0.1, 0.1, (n, n)),
                  steps)
    assert rel_linf(got, ref) <= 1e-12
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("mean", [0.0, -0.2])
def test_model_b_3d_bit_identical(mean):
    """Cahn-Hilliard 3D, dx 1, dt 0.005, Stencil3d2h<7,10,25>, 32^3, 200 steps."""
    n, h, dt, steps = 32, 1.0, 0.005, 200
    m = model_of(sp.model_MB_t, 3, (n, n, n), h)
    m.fill_uniform(0, 5, mean - 0.1, mean + 0.1)
    sp.find_solution(m, dt, steps)
    got = m.get_field(0)
    ref = spo.run(spo.make_desc(3, (n, n, n), spo.MODEL_B, h, dt),
                  oracle_init(5, mean - 0.1, mean + 0.1, (n, n, n)), steps)
    assert rel_linf(got, ref) <= 1e-12
    assert np.array_equal(got, ref)


OPS2 = [("lap", (5, 6, 13)), ("lap", (9, 6, 13)), ("bilap", (5, 6, 13)), ("bilap", (5, 6, 17)),
        ("bilap", (5, 6, 21)), ("gradlap", (5, 6, 13)), ("gradlap", (5, 8, 13)),
        ("gradlap", (5, 12, 13)), ("gradlap", (5, 16, 13)), ("lapcube", (5, 6, 13))]
OPS3 = [("lap", (7, 10, 25)), ("lap", (15, 10, 25)), ("lap", (19, 10, 25)), ("lap", (21, 10, 25)),
        ("lap", (27, 10, 25)), ("bilap", (7, 10, 21)), ("bilap", (7, 10, 25)),
        ("bilap", (7, 10, 41)), ("bilap", (7, 10, 52)), ("bilap", (7, 10, 57)),
        ("gradlap", (7, 10, 25)), ("gradlap", (7, 12, 25)), ("gradlap", (7, 28, 25)),
        ("gradlap", (7, 36, 25)), ("gradlap", (7, 40, 25)), ("lapcube", (7, 10, 25))]
OPID = {"lap": spo.OP_LAP, "bilap": spo.OP_BILAP, "gradlap": spo.OP_GRADLAP,
        "lapcube": spo.OP_LAPCUBE}


@pytest.mark.parametrize("op,pts", OPS2)
def test_operator_2d_every_point_set(op, pts):
    dims, h = (40, 36), 0.7
    st = sp.Stencil2d2h(*pts)
    m = sp.model_OP_t(op, 2, sp.SolverFT(st, form="exact"), sp.ProblemParameters(dims, h=h))
    m.fill_uniform(0, 99, -1.0, 1.0)
    got = m.eval_rhs(0)
    x = oracle_init(99, -1.0, 1.0, m.shape)
    ref = spo.rhs(spo.make_desc(2, dims, OPID[op], h, 0.0, stencil=pts), x)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("op,pts", OPS3)
def test_operator_3d_every_point_set(op, pts):
    dims, h = (20, 18, 16), 0.9
    st = sp.Stencil3d2h(*pts)
    m = sp.model_OP_t(op, 3, sp.SolverFT(st, form="exact"), sp.ProblemParameters(dims, h=h))
    m.fill_uniform(0, 77, -1.0, 1.0)
    got = m.eval_rhs(0)
    x = oracle_init(77, -1.0, 1.0, m.shape)
    ref = spo.rhs(spo.make_desc(3, dims, OPID[op], h, 0.0, stencil=pts), x)
    assert np.array_equal(got, ref)


def test_model_c_3d_bit_identical():
    n, h, dt, steps, gamma = 16, 1.0, 0.005, 60, 0.5
    m = model_of(sp.model_MC_t, 3, (n, n, n), h, coeff=(gamma,))
    m.fill_uniform(0, 1, 0.0, 0.2)
    m.fill_uniform(1, 2, -0.1, 0.1)
    sp.find_solution(m, dt, steps)
    got = np.stack([m.get_field(0), m.get_field(1)])
    x = np.stack([oracle_init(1, 0.0, 0.2, (n, n, n)), oracle_init(2, -0.1, 0.1, (n, n, n))])
    ref = spo.run(spo.make_desc(3, (n, n, n), spo.MODEL_C, h, dt, coeff=(gamma,)), x, steps)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("cls,oid", [(sp.model_MAMK_t, spo.MODEL_AMK), (sp.model_MBMK_t, spo.MODEL_BMK)])
def test_mobility_kappa_models_2d_bit_identical(cls, oid):
    dims, h, dt, steps, coeff = (48, 40), 1.0, 0.01, 150, (1.3, 0.7)
    m = model_of(cls, 2, dims, h, coeff=coeff)
    m.fill_uniform(0, 3, -0.1, 0.1)
    sp.find_solution(m, dt, steps)
    ref = spo.run(spo.make_desc(2, dims, oid, h, dt, coeff=coeff), oracle_init(3, -0.1, 0.1, m.shape),
                  steps)
    assert np.array_equal(m.get_field(0), ref)


@pytest.mark.parametrize("dim,dims", [(2, (37, 45)), (3, (21, 13, 11))])
def test_ragged_sizes_bit_identical(dim, dims):
    h, dt, steps = 1.0, 0.002, 40
    m = model_of(sp.model_MB_t, dim, dims, h)
    m.fill_uniform(0, 8, -0.3, 0.3)
    sp.find_solution(m, dt, steps)
    ref = spo.run(spo.make_desc(dim, dims, spo.MODEL_B, h, dt), oracle_init(8, -0.3, 0.3, m.shape),
                  steps)
    assert np.array_equal(m.get_field(0), ref)


@pytest.mark.parametrize("dim,dims,cls,oid", [(2, (40, 32), sp.model_MA_t, spo.MODEL_A),
                                              (3, (16, 16, 12), sp.model_MB_t, spo.MODEL_B)])
def test_dirichlet_bit_identical(dim, dims, cls, oid):
    h, dt, steps, val = 1.0, 0.004, 50, 0.3
    m = model_of(cls, dim, dims, h, boundary=sp.BoundaryType.DEFAULT, boundary_value=val)
    m.fill_uniform(0, 4, -0.5, 0.5)
    sp.find_solution(m, dt, steps)
    ref = spo.run(spo.make_desc(dim, dims, oid, h, dt, bc=spo.DIRICHLET, bcv=val),
                  oracle_init(4, -0.5, 0.5, m.shape), steps)
    assert np.array_equal(m.get_field(0), ref)


def test_fused_f64_close_to_oracle():
    n, h, dt, steps = 32, 1.0, 0.005, 200
    m = model_of(sp.model_MB_t, 3, (n, n, n), h, form="fused")
    m.fill_uniform(0, 5, -0.3, -0.1)
    sp.find_solution(m, dt, steps)
    ref = spo.run(spo.make_desc(3, (n, n, n), spo.MODEL_B, h, dt), oracle_init(5, -0.3, -0.1, m.shape),
                  steps)
    assert rel_linf(m.get_field(0), ref) <= 1e-10


@pytest.mark.parametrize("dim,dims,cls,oid,h,dt,steps,tol", [
    (2, (64, 64), sp.model_MA_t, spo.MODEL_A, 0.5, 0.01, 1000, 1e-4),
    (3, (32, 32, 32), sp.model_MB_t, spo.MODEL_B, 1.0, 0.005, 200, 1e-5),
])
def test_f32_fused_against_f64_oracle(dim, dims, cls, oid, h, dt, steps, tol):
    m = model_of(cls, dim, dims, h, form="fused", dtype="f32")
    m.fill_uniform(0, 21, -0.3, -0.1)
    sp.find_solution(m, dt, steps)
    ref = spo.run(spo.make_desc(dim, dims, oid, h, dt), oracle_init(21, -0.3, -0.1, m.shape), steps)
    assert rel_linf(m.get_field(0).astype(np.float64), ref) <= tol


def test_batch_instances_match_single_runs():
    n, dt, steps = 16, 0.005, 30
    params = sp.ProblemParameters((n, n, n), h=1.0)
    mb = sp.model_MB_t(3, sp.SolverFT(S3, form="exact"), params, batch=3)
    for i in range(3):
        mb.fill_uniform(0, 100 + i, -0.2, 0.2, inst=i)
    sp.find_solution(mb, dt, steps)
    for i in range(3):
        ref = spo.run(spo.make_desc(3, (n, n, n), spo.MODEL_B, 1.0, dt),
                      oracle_init(100 + i, -0.2, 0.2, (n, n, n)), steps)
        assert np.array_equal(mb.get_field(0, inst=i), ref)


def test_graph_replay_equals_direct_launches():
    n, dt = 24, 0.005
    a = model_of(sp.model_MB_t, 3, (n, n, n), 1.0, form="fused", dtype="f32")
    b = model_of(sp.model_MB_t, 3, (n, n, n), 1.0, form="fused", dtype="f32")
    for m in (a, b):
        m.fill_uniform(0, 9, -0.2, 0.2)
    a.step(dt, 70)  # 2 graph replays of 32 steps + 6 launches
    for _ in range(70):
        b.step(dt, 1)
    assert np.array_equal(a.get_field(0), b.get_field(0))
    assert a.launch_count() == 70 and b.launch_count() == 70


def test_mass_conservation_and_fused_reduction():
    n, dt = 48, 0.005
    m = model_of(sp.model_MB_t, 3, (n, n, n), 1.0, form="fused", dtype="f64")
    m.fill_uniform(0, 13, -0.3, -0.1)
    m0, e0 = m.reduce(0)
    masses = m.step_mass(dt, 500)
    m1, e1 = m.reduce(0)
    assert abs(m1 - m0) <= 1e-10 * abs(m0)
    assert abs(masses[0] - m1) <= 1e-12 * abs(m1)
    assert e1 < e0  # Cahn-Hilliard free energy decreases


def test_f32_mass_drift_with_fp64_reduction():
    n, dt = 64, 0.005
    m = model_of(sp.model_MB_t, 3, (n, n, n), 1.0, form="fused", dtype="f32")
    m.fill_uniform(0, 13, -0.3, -0.1)
    m0, _ = m.reduce(0)
    m.step(dt, 1000)
    m1, _ = m.reduce(0)
    assert abs(m1 - m0) <= 1e-4 * abs(m0)


@pytest.mark.parametrize("dim,n,cls", [(3, 40, sp.model_MB_t), (3, 42, sp.model_MB_t),
                                       (3, 24, sp.model_MC_t),
                                       (2, 200, sp.model_MB_t), (2, 202, sp.model_MB_t),
                                       (2, 136, sp.model_MA_t)])
def test_every_tile_shape_gives_the_same_fields(dim, n, cls, monkeypatch):
    """The autotuner may pick any tile shape: each must give the same bits."""
    st = S2 if dim == 2 else S3
    dims = (n,) * dim
    coeff = (0.5,) if cls is sp.model_MC_t else ()
    base = cls(dim, sp.SolverFT(st, form="fused"), sp.ProblemParameters(dims, h=1.0),
               coeff=coeff, dtype="f32")
    nv = base.kernel_info()["variants"]
    ref = None
    for v in range(nv):
        monkeypatch.setenv("SP_TILE", str(v))
        m = cls(dim, sp.SolverFT(st, form="fused"), sp.ProblemParameters(dims, h=1.0),
                coeff=coeff, dtype="f32")
        if m.kernel_info()["variant"] != v:  # a row kernel of another x extent
            assert v > 0 and m.kernel_info()["variant"] == 0
            m.close()
            continue
        for f in range(cls.nfields):
            m.fill_uniform(f, 60 + f, -0.3, 0.1)
        m.step(0.004, 25)
        out = np.stack([m.get_field(f) for f in range(cls.nfields)])
        if ref is None:
            ref = out
        else:
            assert np.array_equal(out, ref), v
        m.close()
    monkeypatch.delenv("SP_TILE")
    base.autotune(3)
    assert 0 <= base.kernel_info()["variant"] < nv


@pytest.mark.parametrize("dims,ybc", [((128, 40, 24), "periodic"), ((256, 36, 20), "periodic"),
                                      ((128, 34, 18), "dirichlet")])
@pytest.mark.parametrize("classes", [(sp.model_MB_t, sp.model_MBMK_t), (sp.model_MA_t,),
                                     (sp.model_MC_t,)])
def test_row_kernels_give_the_same_fields(dims, ybc, classes, monkeypatch):
    """The row kernels (whole x rows per CTA, x neighbours by warp shuffles:
    the conserved-pattern kernel for models B and BMK, the generic one for
    every fused 7-point model) run on grids of x extent 128 or 256, periodic
    in x; on such grids they must give the bits of every other tile shape --
    here with ragged y tiles, and with Dirichlet y sides."""
    P, D = sp.BoundaryType.PERIODIC, sp.BoundaryType.DEFAULT
    bc = [P, P] + ([P, P] if ybc == "periodic" else [D, D]) + [P, P]

    def make(cls):
        return cls(3, sp.SolverFT(S3, form="fused"),
                   sp.ProblemParameters(dims, h=1.0, boundary=bc, boundary_value=0.25),
                   coeff=(0.5,) if cls is sp.model_MC_t else (), dtype="f32")

    for cls in classes:
        nv = make(cls).kernel_info()["variants"]
        ref, rows = None, 0
        for v in range(nv):
            monkeypatch.setenv("SP_TILE", str(v))
            m = make(cls)
            info = m.kernel_info()
            if info["variant"] != v:
                m.close()
                continue
            rows += info["tile_x"] == dims[0]
            for f in range(cls.nfields):
                m.fill_uniform(f, 77 + f, -0.35, -0.05)
            masses = m.step_mass(0.004, 30)
            out = np.stack([m.get_field(f) for f in range(cls.nfields)])
            if ref is None:
                ref, ref_mass = out, masses[0]
            else:
                assert np.array_equal(out, ref), (cls.__name__, v)
                assert abs(masses[0] - ref_mass) <= 1e-12 * abs(ref_mass)
            m.close()
        monkeypatch.delenv("SP_TILE")
        assert rows >= 1, cls.__name__
        # the autotuner's timing launches (right-hand sides only, the row
        # kernels among them) leave the model's state as it was
        m = make(cls)
        for f in range(cls.nfields):
            m.fill_uniform(f, 77 + f, -0.35, -0.05)
        m.autotune(2)
        m.step_mass(0.004, 30)
        assert np.array_equal(np.stack([m.get_field(f) for f in range(cls.nfields)]), ref)
        m.close()


# ---------------------------------------------------------------------------
# Stencil2d4h (4th order, 2D): every point set of each operator, and the
# models with the default point sets, against the oracle in FP64 (exact form)
# ---------------------------------------------------------------------------
OPS2_4 = [("lap", (9, 14, 21)), ("lap", (17, 14, 21)), ("lap", (21, 14, 21)),
          ("bilap", (9, 14, 21)), ("bilap", (9, 14, 25)), ("bilap", (9, 14, 33)),
          ("bilap", (9, 14, 37)), ("gradlap", (9, 14, 21)), ("gradlap", (9, 18, 21)),
          ("gradlap", (9, 26, 21)), ("gradlap", (9, 30, 21))]


@pytest.mark.parametrize("op,pts", OPS2_4)
def test_operator_2d4h_every_point_set(op, pts):
    dims, h = (40, 36), 0.7
    m = sp.model_OP_t(op, 2, sp.SolverFT(sp.Stencil2d4h(*pts), form="exact"),
                      sp.ProblemParameters(dims, h=h))
    m.fill_uniform(0, 98, -1.0, 1.0)
    got = m.eval_rhs(0)
    x = oracle_init(98, -1.0, 1.0, m.shape)
    ref = spo.rhs(spo.make_desc(2, dims, OPID[op], h, 0.0, stencil=pts, acc=4), x)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("cls,oid,coeff", [(sp.model_MA_t, spo.MODEL_A, ()),
                                           (sp.model_MB_t, spo.MODEL_B, ()),
                                           (sp.model_MAMK_t, spo.MODEL_AMK, (1.3, 0.7)),
                                           (sp.model_MBMK_t, spo.MODEL_BMK, (1.3, 0.7))])
@pytest.mark.parametrize("h,bc", [(1.0, sp.BoundaryType.PERIODIC), (0.8, sp.BoundaryType.DEFAULT)])
def test_models_2d4h_bit_identical(cls, oid, coeff, h, bc):
    dims, dt, steps, val = (46, 38), 0.002, 60, 0.05
    m = cls(2, sp.SolverFT(sp.Stencil2d4h(), form="exact"),
            sp.ProblemParameters(dims, h=h, boundary=bc, boundary_value=val), coeff=coeff,
            dtype="f64")
    m.fill_uniform(0, 8, -0.2, 0.2)
    sp.find_solution(m, dt, steps)
    obc = spo.PERIODIC if bc == sp.BoundaryType.PERIODIC else spo.DIRICHLET
    ref = spo.run(spo.make_desc(2, dims, oid, h, dt, coeff=coeff, stencil=(9, 14, 21), bc=obc,
                                bcv=val, acc=4), oracle_init(8, -0.2, 0.2, m.shape), steps)
    assert np.array_equal(m.get_field(0), ref)


def test_model_c_2d4h_bit_identical():
    dims, h, dt, steps, gamma = (36, 40), 1.0, 0.002, 50, 0.5
    m = sp.model_MC_t(2, sp.SolverFT(sp.Stencil2d4h(), form="exact"),
                      sp.ProblemParameters(dims, h=h), coeff=(gamma,), dtype="f64")
    m.fill_uniform(0, 1, 0.0, 0.2)
    m.fill_uniform(1, 2, -0.1, 0.1)
    sp.find_solution(m, dt, steps)
    got = np.stack([m.get_field(0), m.get_field(1)])
    x = np.stack([oracle_init(1, 0.0, 0.2, m.shape), oracle_init(2, -0.1, 0.1, m.shape)])
    ref = spo.run(spo.make_desc(2, dims, spo.MODEL_C, h, dt, coeff=(gamma,), stencil=(9, 14, 21),
                                acc=4), x, steps)
    assert np.array_equal(got, ref)


def test_f32_2d4h_against_f64_oracle():
    """The FP32 fused key of Stencil2d4h (the reference's term order with
    FMA contraction): within FP32 rounding of the FP64 oracle."""
    dims, h, dt, steps = (64, 48), 1.0, 0.002, 200
    m = sp.model_MB_t(2, sp.SolverFT(sp.Stencil2d4h(), form="fused"), sp.ProblemParameters(dims, h=h),
                      dtype="f32")
    m.fill_uniform(0, 4, -0.3, 0.1)
    x = m.get_field(0).astype(np.float64)
    sp.find_solution(m, dt, steps)
    ref = spo.run(spo.make_desc(2, dims, spo.MODEL_B, h, dt, stencil=(9, 14, 21), acc=4), x, steps)
    assert rel_linf(m.get_field(0).astype(np.float64), ref) < 2e-5


@pytest.mark.parametrize("cls", [sp.model_MB_t, sp.model_MC_t])
def test_row_kernels_on_a_batch_of_instances(cls, monkeypatch):
    """A batch of instances (one launch, instance = grid z index) on the row
    kernels gives, instance by instance, the bits of the tile kernel."""
    dims, batch = (128, 20, 12), 3
    coeff = (0.5,) if cls is sp.model_MC_t else ()

    def run(v):
        monkeypatch.setenv("SP_TILE", str(v))
        m = cls(3, sp.SolverFT(S3, form="fused"), sp.ProblemParameters(dims, h=1.0),
                coeff=coeff, dtype="f32", batch=batch)
        got_v = m.kernel_info()["variant"]
        for i in range(batch):
            for f in range(cls.nfields):
                m.fill_uniform(f, 100 * i + f, -0.3, 0.1, inst=i)
        m.step(0.004, 20)
        out = np.stack([m.get_field(f, inst=i) for i in range(batch) for f in range(cls.nfields)])
        m.close()
        return got_v, out

    _, ref = run(0)
    nv = cls(3, sp.SolverFT(S3, form="fused"), sp.ProblemParameters(dims, h=1.0), coeff=coeff,
             dtype="f32").kernel_info()["variants"]
    rows = 0
    for v in range(1, nv):
        got_v, out = run(v)
        if got_v != v:
            continue
        assert np.array_equal(out, ref), v
        rows += 1
    monkeypatch.delenv("SP_TILE")
    assert rows >= 1
