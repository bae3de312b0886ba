"""Stream order of the step kernels under programmatic dependent launch.

A foreign kernel (a PyTorch in-place op) writes straight into the solver's
current field on the solver's stream between steps, with no host
synchronisation.  The step after it must see the write: the fields equal, bit
for bit, those of the same sequence run with a device synchronisation after
every operation.
"""
import ctypes

import numpy as np
import pytest

import symphas_b200 as sp
from symphas_b200 import _capi as C

pytestmark = pytest.mark.gpu


class _View:
    """__cuda_array_interface__ over a strided device region."""

    def __init__(self, ptr, shape, strides, typestr):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": shape,
                                         "strides": strides, "typestr": typestr,
                                         "version": 3}


def _interior(torch, m, esz, typestr):
    ptr, pitch, plane = ctypes.c_void_p(), ctypes.c_longlong(), ctypes.c_longlong()
    halo = (ctypes.c_int * 3)()
    C.check(C.lib().sp_field_geometry(m._h, 0, 0, ctypes.byref(ptr), ctypes.byref(pitch),
                                      ctypes.byref(plane), halo), m._h)
    n0, n1 = m.dims
    return torch.as_tensor(_View(ptr.value, (n1, n0), (pitch.value * esz, esz), typestr),
                           device="cuda")


def _run(torch, dim_model, dtype, sync):
    cls, form = dim_model
    esz, typestr = (4, "<f4") if dtype == "f32" else (8, "<f8")
    m = cls(2, sp.SolverFT(sp.Stencil2d2h(5, 6, 13), form=form),
            sp.ProblemParameters((256, 192), h=1.0), dtype=dtype)
    s = torch.cuda.Stream()
    m.set_stream(s.cuda_stream)
    m.fill_uniform(0, 77, -0.4, 0.4)
    m.synchronize()
    for k in range(24):
        m.step(0.01, 1 + k % 3)
        if sync:
            m.synchronize()
        view = _interior(torch, m, esz, typestr)
        with torch.cuda.stream(s):
            view.mul_(-1.0)  # a foreign kernel on the solver's stream
            view.add_(0.25)
        if sync:
            torch.cuda.synchronize()
    m.step(0.01, 40)  # graph-replayed steps right after the last foreign kernel
    out = m.get_field(0)
    m.close()
    return out


@pytest.mark.parametrize("dim_model,dtype", [((sp.model_MB_t, "fused"), "f32"),
                                              ((sp.model_MA_t, "exact"), "f64")])
def test_foreign_kernels_between_steps_are_ordered(dim_model, dtype):
    torch = pytest.importorskip("torch")
    a = _run(torch, dim_model, dtype, sync=False)
    b = _run(torch, dim_model, dtype, sync=True)
    assert np.isfinite(b).all()
    assert np.array_equal(a, b)
