"""The C++ front end (symphas_b200/csrc/symphas_model.hpp): a model written by
the user as an EVOLUTION expression in C++, compiled with the runtime sources
(tests/cpp/user_model.cu, built by __graft_entry__.build), runs through
model_t / find_solution and matches the CPU oracle bit for bit in FP64 --
SymPhas's model A config, 64^2, dx 0.5, dt 0.01, 1000 steps."""
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
    r = subprocess.run([EXE, str(out), str(n), str(h), str(dt), str(steps), str(seed), str(lo),
                        str(hi)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "index %d" % steps in r.stdout
    got = np.fromfile(out, dtype=np.float64).reshape(n, n)
    ref = spo.run(spo.make_desc(2, (n, n), spo.MODEL_A, h, dt),
                  spo.seed_uniform(seed, lo, hi, n * n).reshape(n, n), steps)
    assert np.array_equal(got, ref)
