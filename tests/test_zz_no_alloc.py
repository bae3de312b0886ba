"""The no-allocation reduction (sp_reduce_fields_noalloc) against sp_reduce.

sp_reduce_fields_noalloc exists for callers that cannot call cudaMalloc (an
application whose device memory belongs to another allocator, or a stepping
loop that must not stall on an allocation's device synchronisation).  It works
on fields the caller holds in device memory and writes its sums to caller
memory; its only scratch is a static device array.  Here it must give the same
(mass, energy) as the handle-based sp_reduce, within 1e-12 relative, on two
calls in a row (the second call reuses the static scratch after the fields
changed).  This file is collected last so a failing run has already run every
other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import symphas_b200 as sp
from symphas_b200 import _capi as C

pytestmark = pytest.mark.gpu

S3 = sp.Stencil3d2h(7, 10, 25)


def noalloc(fields_dev, dtype, dims, model, coeff, h, batch):
    out = torch.zeros(2 * batch, dtype=torch.float64, device="cuda")
    n = (ctypes.c_int * 3)(*(list(dims) + [1] * (3 - len(dims))))
    cs = list(coeff) + [1.0] * (8 - len(coeff))
    c = (ctypes.c_double * 8)(*cs)
    rc = C.lib().sp_reduce_fields_noalloc(
        ctypes.c_void_p(fields_dev.data_ptr()), dtype, len(dims), n, model, c, h, batch,
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == C.SP_OK, C.lib().sp_noalloc_error()
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(batch, 2)


def close(a, b, tol=1e-12):
    return abs(a - b) <= tol * max(abs(b), 1e-300)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_noalloc_matches_sp_reduce_twice(dtype):
    torch.cuda.set_device(0)
    n, h, dt = 32, 1.0, 0.005
    m = sp.model_MB_t(3, sp.SolverFT(S3, form="fused"), sp.ProblemParameters((n, n, n), h=h),
                      dtype=dtype)
    m.fill_uniform(0, 31, -0.3, -0.1)
    code = C.SP_F64 if dtype == "f64" else C.SP_F32
    tdt = torch.float64 if dtype == "f64" else torch.float32
    for _ in range(2):
        m.step(dt, 20)
        mass, energy = m.reduce(0)
        field = torch.from_numpy(m.get_field(0)).to(device="cuda", dtype=tdt).contiguous()
        got = noalloc(field, code, (n, n, n), C.SP_MODEL_B, (), h, 1)
        assert close(got[0, 0], mass) and close(got[0, 1], energy), (got, mass, energy)
    m.close()


def test_noalloc_batch_of_two_field_instances():
    torch.cuda.set_device(0)
    n, h, dt, gamma = 16, 1.0, 0.005, 0.5
    m = sp.model_MC_t(3, sp.SolverFT(S3, form="fused"), sp.ProblemParameters((n, n, n), h=h),
                      coeff=(gamma,), dtype="f64", batch=2)
    for i in range(2):
        m.fill_uniform(0, 40 + i, 0.0, 0.2, inst=i)
        m.fill_uniform(1, 50 + i, -0.1, 0.1, inst=i)
    for _ in range(2):
        m.step(dt, 10)
        host = np.stack([np.stack([m.get_field(f, inst=i) for f in range(2)]) for i in range(2)])
        fields = torch.from_numpy(host).to("cuda").contiguous()
        got = noalloc(fields, C.SP_F64, (n, n, n), C.SP_MODEL_C, (gamma,), h, 2)
        for i in range(2):
            mass, energy = m.reduce(0, inst=i)
            assert close(got[i, 0], mass) and close(got[i, 1], energy), (i, got[i], mass, energy)
    m.close()


def test_noalloc_rejects_batch_beyond_the_static_scratch():
    torch.cuda.set_device(0)
    field = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    n = (ctypes.c_int * 3)(2, 2, 2)
    rc = C.lib().sp_reduce_fields_noalloc(
        ctypes.c_void_p(field.data_ptr()), C.SP_F64, 3, n, C.SP_MODEL_B, None, 1.0,
        C.SP_NOALLOC_MAX_INSTANCES + 1,
        ctypes.c_void_p(out.data_ptr()), None)
    assert rc == C.SP_EINVAL
    assert b"batch" in C.lib().sp_noalloc_error()
