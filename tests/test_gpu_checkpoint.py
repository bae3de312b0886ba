"""A run resumed from SymPhas's checkpoint file continues as the original one,
up to the ten digits the format keeps."""
import numpy as np
import pytest

import symphas_b200 as sp
from symphas_b200 import checkpoint as ck

pytestmark = pytest.mark.gpu


def test_resume_from_checkpoint(tmp_path):
    st = sp.SolverFT(sp.Stencil2d2h(5, 6, 13), form="fused")
    a = sp.model_MB_t(2, st, sp.ProblemParameters((48, 40)), dtype="f64")
    a.fill_uniform(0, 3, -0.3, 0.1)
    a.step(0.01, 200)
    path = ck.save(a, str(tmp_path), 200)
    assert path.endswith("checkpoint/data0_200")
    b = sp.model_MB_t(2, st, sp.ProblemParameters((48, 40)), dtype="f64")
    assert ck.load(b, path) == 200
    a.step(0.01, 300)
    b.step(0.01, 300)
    fa, fb = a.get_field(0), b.get_field(0)
    assert np.max(np.abs(fa - fb)) <= 1e-8 * np.max(np.abs(fa))
    a.close()
    b.close()
