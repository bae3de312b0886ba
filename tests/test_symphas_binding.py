"""SymPhas's own MODEL definitions through the SymPhas-side binding of the
B200 library (symphas_b200/binding/solverftb200.h): SolverFTB200, a solver
declared with SymPhas's own macros, and SolverSystemFDB200, its solver system
(ASSOCIATE_SOLVER_SYSTEM_TYPE, sol/inc/solver.h:312-321).

The test program (tests/cpp/symphas_binding.cpp) is compiled against
SymPhas's headers and sources by oracle/ref.mk.  On the CPU it checks which
B200 model each MODEL maps to, read back from SymPhas's optimised equations;
on the GPU it runs the models through model_iteration's loop
(modules-models.h:435-467: update, equation, step) beside SymPhas's own CPU
SolverFT and compares the fields.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "symphas_binding")

pytestmark = pytest.mark.skipif(not os.path.exists(BIN),
                                reason="the SymPhas binding test is not built (oracle/ref.mk)")


def test_symphas_models_map_to_the_b200_kernels():
    out = subprocess.run([BIN, "match"], capture_output=True, text=True, timeout=120,
                         check=True).stdout
    got = dict(line.split(": ", 1) for line in out.strip().splitlines())
    # ids of include/symphas_b200.h: A 0, B 1, C 2, AMK 3, BMK 4
    assert got["MA"].startswith("model 0 coeff 0.69999999999999996 1.3")
    assert got["MB"].startswith("model 1 coeff 0.69999999999999996 1.3")
    assert got["MCG"].startswith("model 2 coeff 0.5 ")
    # SymPhas folds M kappa into one literal; M and kappa are read back
    assert got["AMK"].startswith("model 3 coeff 1.7 0.59999999999999998")
    assert got["BMK"].startswith("model 4 coeff 1.7 0.59999999999999998")
    assert got["QUAD"].startswith("refused")


@pytest.mark.gpu
def test_symphas_models_run_on_the_gpu_as_symphas_runs_them():
    r = subprocess.run([BIN, "run"], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [l for l in r.stdout.splitlines() if "steps:" in l]
    assert len(lines) == 8 and all(l.endswith("ok") for l in lines)
