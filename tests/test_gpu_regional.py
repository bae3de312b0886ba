"""GPU parity of regional systems: the moving window stepped by the fused
sm_100a kernels (through sp_regional_*) against the oracle's regional
system, window by window and field by field.

Tolerances: FP64 exact form -- bit-identical whole-domain fields and the same
window after every chunk of steps; FP32 fused -- 2e-5 relative L-infinity
against the FP64 oracle, same windows.
"""
import numpy as np
import pytest

import spo
import symphas_b200 as sp

pytestmark = pytest.mark.gpu

S2 = sp.Stencil2d2h(5, 6, 13)
S3 = sp.Stencil3d2h(7, 10, 25)
MODELS = {"A": (sp.model_MA_t, spo.MODEL_A), "B": (sp.model_MB_t, spo.MODEL_B),
          "AMK": (sp.model_MAMK_t, spo.MODEL_AMK), "BMK": (sp.model_MBMK_t, spo.MODEL_BMK)}


def blob_field(dims, centres, radius, seed=3):
    """-1 outside, +1 inside discs/balls, plus seeded noise of 1e-3 inside."""
    shape = tuple(reversed(dims))
    idx = np.indices(shape).astype(np.float64)
    f = -np.ones(shape)
    for c in centres:
        r2 = 0.0
        for a, ca in enumerate(reversed(c)):
            dd = np.abs(idx[a] - ca)
            dd = np.minimum(dd, shape[a] - dd)  # periodic distance
            r2 = r2 + dd * dd
        f[r2 < radius * radius] = 1.0
    noise = spo.seed_uniform(seed, -1e-3, 1e-3, f.size).reshape(shape)
    return np.where(f > 0, f + noise, f)


def pair(model, dim, dims, field, dt=0.01, delta=0.05, fixed=True, dtype="f64", form="exact",
         coeff=(1.0, 1.0), factor=2.0, eps=1e-6):
    cls, oid = MODELS[model]
    st = S2 if dim == 2 else S3
    g = sp.RegionalModel(cls, dim, sp.SolverFT(st, form=form), sp.ProblemParameters(dims, h=1.0),
                         coeff=coeff, dtype=dtype, dt=dt, resize_delta=delta, fixed=fixed,
                         padding_factor=factor, cutoff_eps=eps)
    g.set_field(field)
    r = spo.Regional(spo.make_desc(dim, dims, oid, 1.0, dt, coeff=coeff), field,
                     resize_delta=delta, fixed=fixed, factor=factor, eps=eps)
    return g, r


def check_same(g, r, exact=True, tol=0.0):
    o, d, empty, cutoff, t, nxt = r.window()
    assert g.window() == (o, d)
    ge, gc, gt, gn = g.state()
    assert gn == nxt and gt == t
    got, ref = g.get_field(), r.get()
    if exact:
        assert ge == empty and gc == cutoff
        assert np.array_equal(got, ref)
    else:
        assert abs(ge - empty) <= 1e-6
        err = float(np.max(np.abs(got.astype(np.float64) - ref)) / np.max(np.abs(ref)))
        assert err <= tol, err


@pytest.mark.parametrize("model", ["A", "B", "BMK"])
@pytest.mark.parametrize("fixed", [True, False])
def test_regional_2d_windows_and_fields_bit_identical(model, fixed):
    dims = (96, 80)
    f = blob_field(dims, [(30, 40)], 9)
    g, r = pair(model, 2, dims, f, fixed=fixed, coeff=(1.0, 1.0) if model != "BMK" else (0.7, 1.3))
    for _ in range(4):
        g.step(9)
        r.step(9)
        check_same(g, r)
    assert g.launch_count() > 0


def test_regional_window_wraps_across_the_periodic_edge():
    dims = (64, 64)
    f = blob_field(dims, [(1, 62)], 8)
    g, r = pair("A", 2, dims, f)
    g.step(1)
    r.step(1)
    o, d = g.window()
    assert o[0] + d[0] > dims[0] + 6 or o[1] + d[1] > dims[1] + 6  # the window wraps
    check_same(g, r)
    for _ in range(3):
        g.step(7)
        r.step(7)
        check_same(g, r)


@pytest.mark.parametrize("model", ["A", "B"])
def test_regional_3d_bit_identical(model):
    dims = (32, 28, 24)
    f = blob_field(dims, [(12, 14, 11)], 5)
    g, r = pair(model, 3, dims, f, delta=0.04)
    for _ in range(3):
        g.step(6)
        r.step(6)
        check_same(g, r)


def test_regional_window_as_wide_as_the_domain():
    # a blob wider than half the domain: the padded window spans the whole
    # axis, off origin 0, so its rim cuts the periodic axis as SymPhas's does
    dims = (40, 40)
    f = blob_field(dims, [(20, 20)], 13)
    g, r = pair("A", 2, dims, f)
    g.step(5)
    r.step(5)
    check_same(g, r)
    g.step(10)
    r.step(10)
    check_same(g, r)


def test_regional_moves_by_hand_match_the_oracle():
    # adjust_region_to_from (new dims), then in-place shifts along x (the
    # cells at the row ends take the rim and the next row's values) and y
    dims = (48, 40)
    f = blob_field(dims, [(20, 18)], 6)
    g, r = pair("A", 2, dims, f)
    for o, d in [((6, 5), (30, 28)), ((11, 5), (30, 28)), ((11, 2), (30, 28)),
                 ((40, 30), (30, 28)), ((0, 0), (54, 46))]:
        g.adjust(o, d)
        r.adjust(o, d)
        check_same(g, r)
        g.step(3)
        r.step(3)
        check_same(g, r)


def test_regional_f32_fused_follows_the_oracle():
    dims = (128, 96)
    f = blob_field(dims, [(40, 50), (90, 30)], 10)
    # a cutoff well above the minimum, where FP32 and FP64 fields cannot
    # straddle it, so both choose the same windows
    g, r = pair("B", 2, dims, f, dtype="f32", form="fused", delta=0.1, eps=0.05)
    for _ in range(3):
        g.step(10)
        r.step(10)
        check_same(g, r, exact=False, tol=2e-5)


def test_regional_rejects_what_it_does_not_cover():
    with pytest.raises(sp.SymPhasError):
        sp.RegionalModel(sp.model_MC_t, 2, sp.SolverFT(S2), sp.ProblemParameters((32, 32)))
    with pytest.raises(sp.SymPhasError):
        sp.RegionalModel(sp.model_MA_t, 2, sp.SolverFT(S2),
                         sp.ProblemParameters((32, 32), boundary=sp.BoundaryType.DEFAULT))
    g = sp.RegionalModel(sp.model_MA_t, 2, sp.SolverFT(S2), sp.ProblemParameters((32, 32)), dt=0.01)
    with pytest.raises(sp.SymPhasError):
        g.adjust((0, 0), (8, 20))  # interior of 2 cells along x
    with pytest.raises(sp.SymPhasError):
        g.adjust((0, 0), (50, 20))  # wider than the domain's storage


@pytest.mark.parametrize("model,fixed", [("BMK", False), ("AMK", True), ("A", False)])
def test_regional_3d_other_models_and_modes(model, fixed):
    dims = (30, 26, 28)
    f = blob_field(dims, [(10, 16, 9)], 5, seed=9)
    coeff = (0.8, 1.2) if model in ("AMK", "BMK") else (1.0, 1.0)
    g, r = pair(model, 3, dims, f, delta=0.03, fixed=fixed, coeff=coeff)
    for _ in range(3):
        g.step(5)
        r.step(5)
        check_same(g, r)


def test_regional_two_droplets_resize_f64_fused():
    # the fused form in FP64 against the oracle's printed scheme: within the
    # fused form's tolerance, and the same windows (no value near the cutoff)
    dims = (80, 72)
    f = blob_field(dims, [(20, 20), (55, 48)], 7, seed=5)
    g, r = pair("B", 2, dims, f, form="fused", fixed=False, eps=0.05)
    for _ in range(3):
        g.step(8)
        r.step(8)
        check_same(g, r, exact=False, tol=1e-10)


def test_regional_fourth_order_stencils():
    # Stencil2d4h<> reaches 3 cells (bilap): exactly the window's rim
    dims = (72, 64)
    f = blob_field(dims, [(30, 28)], 8, seed=12)
    st = sp.Stencil2d4h()
    g = sp.RegionalModel(sp.model_MA_t, 2, sp.SolverFT(st, form="exact"),
                         sp.ProblemParameters(dims, h=1.0), coeff=(1.0, 1.0), dtype="f64",
                         dt=0.01, resize_delta=0.05)
    g.set_field(f)
    r = spo.Regional(spo.make_desc(2, dims, spo.MODEL_A, 1.0, 0.01, coeff=(1.0, 1.0),
                                   stencil=st.points, acc=4), f, resize_delta=0.05)
    for _ in range(3):
        g.step(8)
        r.step(8)
        check_same(g, r)


def test_regional_3d_f32_fused():
    dims = (40, 36, 32)
    f = blob_field(dims, [(20, 18, 16)], 7, seed=4)
    g, r = pair("B", 3, dims, f, dtype="f32", form="fused", delta=0.05, eps=0.05, dt=0.005)
    for _ in range(3):
        g.step(10)
        r.step(10)
        check_same(g, r, exact=False, tol=2e-5)


def test_regional_hand_set_window_keeps_its_rim():
    # a window set by hand before the first step, which the first check keeps:
    # `empty` becomes the minimum (-1) there, but the window's rim keeps the 0
    # its move wrote (SymPhas rewrites a rim only when the window moves)
    dims = (64, 56)
    f = blob_field(dims, [(30, 26)], 7, seed=6)
    probe = spo.Regional(spo.make_desc(2, dims, spo.MODEL_A, 1.0, 0.01, coeff=(1.0, 1.0)), f,
                         resize_delta=0.05)
    probe.step(1)
    o, d = probe.window()[:2]
    g, r = pair("A", 2, dims, f)
    g.adjust(o, d)
    r.adjust(o, d)
    g.step(1)
    r.step(1)
    assert g.window() == (o, d) and g.state()[0] == -1.0  # kept by the first check
    check_same(g, r)
    for _ in range(3):
        g.step(6)
        r.step(6)
        check_same(g, r)


def test_regional_on_a_caller_stream_across_window_replacements():
    # a resizing window makes new window handles; each takes the caller's
    # stream, and the results stay those of the oracle
    torch = pytest.importorskip("torch")
    dims = (96, 80)
    f = blob_field(dims, [(40, 36)], 9, seed=8)
    g, r = pair("B", 2, dims, f, fixed=False)
    s = torch.cuda.Stream()
    g.set_stream(s.cuda_stream)
    handles = set()
    for _ in range(4):
        g.step(9)
        r.step(9)
        handles.add(g.handle())
        check_same(g, r)
    assert len(handles) > 1  # the window was replaced at least once
