"""FP32 mass conservation (sp_conserve_mass): the FP64 mass of a conserved
field returns to its target every k steps.  The restoring shift is rounded
stochastically (unbiased), so the restored mass sits within about
sqrt(|correction| * ulp(psi)) of the target -- far below the drift of the
unrestored run, and within 1e-10 relative here -- while the field stays within
FP32 rounding of the unrestored run."""
import numpy as np
import pytest

import symphas_b200 as sp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim,n,steps", [(3, 64, 3000), (2, 512, 3000)])
def test_fp32_mass_held(dim, n, steps):
    st = sp.Stencil2d2h(5, 6, 13) if dim == 2 else sp.Stencil3d2h(7, 10, 25)
    runs = []
    for every in (0, 100):
        m = sp.model_MB_t(dim, sp.SolverFT(st, form="fused"), sp.ProblemParameters((n,) * dim),
                          dtype="f32")
        m.fill_uniform(0, 5, -0.3, -0.1)
        m0, _ = m.reduce(0)
        if every:
            m.conserve_mass(every)
        m.step(0.005, steps)
        mass, _ = m.reduce(0)
        f = m.get_field(0)
        runs.append((abs(mass - m0), f.astype(np.float64)))
        m.close()
    (drift_plain, f_plain), (drift_held, f_held) = runs
    passes = steps // 100
    ulp = float(np.spacing(np.float32(np.max(np.abs(f_held)))))
    bound = max(1e-10 * abs(m0), 6 * np.sqrt(drift_plain / passes * ulp))
    assert drift_held <= bound, (drift_held, bound, drift_plain)
    assert drift_plain > 100 * drift_held, (drift_plain, drift_held)
    assert np.max(np.abs(f_held - f_plain)) <= 1e-3 * np.max(np.abs(f_plain))


def test_conserve_mass_needs_periodic_boundaries():
    m = sp.model_MB_t(2, sp.SolverFT(sp.Stencil2d2h(5, 6, 13)), sp.ProblemParameters(
        (32, 32), boundary=sp.BoundaryType.DEFAULT), dtype="f32")
    with pytest.raises(sp.SymPhasError):
        m.conserve_mass(10)
    m.close()
