"""The C++ front end (symphas_b200/csrc/symphas_model.hpp): models written by
the user as EVOLUTION expressions in C++, compiled with the runtime sources
(tests/cpp/user_model.cu, built by __graft_entry__.build), run through
model_t / find_solution: model A matches the CPU oracle bit for bit in FP64
(SymPhas's model A config, 64^2, dx 0.5, dt 0.01, 1000 steps), and a model
with a provisional variable matches the oracle's equivalent model."""
import os
import subprocess

import numpy as np
import pytest

import spo

pytestmark = pytest.mark.gpu

EXE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpp", "user_model")


def test_user_model_matches_the_oracle(tmp_path):
    if not os.path.exists(EXE):
        pytest.fail("tests/cpp/user_model is not built (run __graft_entry__.build())")
    n, h, dt, steps, seed, lo, hi = 64, 0.5, 0.01, 1000, 11, -0.1, 0.1
    out = tmp_path / "psi.bin"
    r = subprocess.run([EXE, "ma", str(out), str(n), str(h), str(dt), str(steps), str(seed),
                        str(lo), str(hi)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "index %d" % steps in r.stdout
    got = np.fromfile(out, dtype=np.float64).reshape(n, n)
    ref = spo.run(spo.make_desc(2, (n, n), spo.MODEL_A, h, dt),
                  spo.seed_uniform(seed, lo, hi, n * n).reshape(n, n), steps)
    assert np.array_equal(got, ref)


def test_provisional_variable_model(tmp_path):
    """SymPhas's MBB (a provisional variable var(1) = -(c1 - 4 c2 psi^2) psi,
    dpsi = -bilap(psi) + lap(var(1))), with c1 = 1 and c2 = 1/4 model B, run
    with the provisional variable as a staged operand: within 1e-10 of the
    oracle's model B (the same scheme in another rounding order)."""
    n, h, dt, steps, seed, lo, hi = 48, 1.0, 0.005, 300, 21, -0.4, 0.2
    out = tmp_path / "psi.bin"
    r = subprocess.run([EXE, "mbb", str(out), str(n), str(h), str(dt), str(steps), str(seed),
                        str(lo), str(hi)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=np.float64).reshape(n, n)
    ref = spo.run(spo.make_desc(2, (n, n), spo.MODEL_B, h, dt),
                  spo.seed_uniform(seed, lo, hi, n * n).reshape(n, n), steps)
    assert float(np.max(np.abs(got - ref)) / np.max(np.abs(ref))) <= 1e-10


def test_user_model_with_fourth_order_stencils(tmp_path):
    """The same user-written MA with Stencil2d4h<> (4th order): bit-identical
    to the oracle's model A with those stencils."""
    n, h, dt, steps, seed, lo, hi = 48, 1.0, 0.01, 400, 13, -0.1, 0.1
    out = tmp_path / "psi.bin"
    r = subprocess.run([EXE, "ma4", str(out), str(n), str(h), str(dt), str(steps), str(seed),
                        str(lo), str(hi)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=np.float64).reshape(n, n)
    ref = spo.run(spo.make_desc(2, (n, n), spo.MODEL_A, h, dt, stencil=(9, 14, 21), acc=4),
                  spo.seed_uniform(seed, lo, hi, n * n).reshape(n, n), steps)
    assert np.array_equal(got, ref)


def test_user_model_on_a_regional_system(tmp_path):
    """The user-written MA on regional_model_t (SolverSystemFDwSD): the same
    windows and whole-domain field as the oracle's regional system, bit for
    bit in FP64."""
    n, h, dt, steps = 80, 1.0, 0.01, 40
    out = tmp_path / "psi.bin"
    r = subprocess.run([EXE, "mareg", str(out), str(n), str(h), str(dt), str(steps), "0", "0", "0"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=np.float64).reshape(n, n)
    y, x = np.mgrid[0:n, 0:n]
    rad, cx, cy = n / 5.0, n // 3, n // 2
    f0 = np.where((x - cx) ** 2 + (y - cy) ** 2 < rad * rad, 1.0, -1.0)
    ref = spo.Regional(spo.make_desc(2, (n, n), spo.MODEL_A, h, dt), f0, resize_delta=0.05)
    ref.step(steps)
    o, d = ref.window()[:2]
    assert "window %d %d %d %d" % (o[0], o[1], d[0], d[1]) in r.stdout
    assert d[0] < n + 6  # the window is smaller than the domain
    assert np.array_equal(got, ref.get())
