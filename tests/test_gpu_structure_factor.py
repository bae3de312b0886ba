"""Device structure factor (sp_structure_factor) against a numpy restatement
of SymPhas's SF collector: threshold at 0, |FFT|^2 / sites, averaged over the
classes of wave vectors whose absolute integer components agree up to order
(dataprocesses/datasf.h:137-245, datatypes/inc/datalib.h:1120-1330)."""
import itertools

import numpy as np
import pytest

import symphas_b200 as sp

pytestmark = pytest.mark.gpu


def numpy_sf(field, threshold=True):
    f = (field > 0).astype(np.float64) if threshold else field.astype(np.float64)
    power = np.abs(np.fft.fftn(f)) ** 2 / f.size
    sums, counts = {}, {}
    for idx in itertools.product(*[range(n) for n in f.shape]):
        key = tuple(sorted(min(i, n - i) for i, n in zip(idx, f.shape)))
        sums[key] = sums.get(key, 0.0) + power[idx]
        counts[key] = counts.get(key, 0) + 1
    keys = sorted(sums, key=lambda t: (sum(v * v for v in t), t))
    k = np.array([np.sqrt(sum(v * v for v in t)) for t in keys])
    return k, np.array([sums[t] / counts[t] for t in keys])


@pytest.mark.parametrize("dim,n,dtype", [(2, 24, "f64"), (2, 17, "f32"), (3, 12, "f64"),
                                         (3, 10, "f32")])
@pytest.mark.parametrize("threshold", [True, False])
def test_structure_factor_matches_numpy(dim, n, dtype, threshold):
    st = sp.Stencil2d2h(5, 6, 13) if dim == 2 else sp.Stencil3d2h(7, 10, 25)
    m = sp.model_MB_t(dim, sp.SolverFT(st, form="fused"), sp.ProblemParameters((n,) * dim),
                      dtype=dtype)
    m.fill_uniform(0, 77, -0.5, 0.4)
    m.step(0.005, 20)
    field = m.get_field(0)
    k, s = m.structure_factor(threshold=threshold)
    kr, sr = numpy_sf(field, threshold)
    assert len(k) == len(kr)
    assert np.allclose(k, kr, rtol=0, atol=1e-12)
    assert np.allclose(s, sr, rtol=1e-9, atol=1e-12)
    m.close()


def test_structure_factor_of_a_plane_wave():
    """cos(2 pi 3 x / n) (no threshold): all power sits in the class (0, 0, 3)."""
    n = 16
    m = sp.model_MA_t(3, sp.SolverFT(sp.Stencil3d2h(7, 10, 25)), sp.ProblemParameters((n,) * 3))
    x = np.arange(n)
    field = np.broadcast_to(np.cos(2 * np.pi * 3 * x / n), (n, n, n)).copy()
    m.set_field(0, field)
    k, s = m.structure_factor(threshold=False)
    b = int(np.argmax(s))
    assert k[b] == 3.0
    # |F|^2 at +-3 along each axis: (n^3 / 2)^2 each; the class holds 6 points
    assert np.isclose(s[b], 2 * (n ** 3 / 2) ** 2 / n ** 3 / 6)
    m.close()
