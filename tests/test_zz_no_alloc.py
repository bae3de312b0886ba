"""The no-allocation reduction (sp_reduce_fields_noalloc) against sp_reduce.

sp_reduce_fields_noalloc exists for callers that cannot call cudaMalloc (an
application whose device memory belongs to another allocator, or a stepping
loop that must not stall on an allocation's device synchronisation).  It works
on fields the caller holds in device memory and writes its sums to caller
memory; its only scratch is a static device array.  Here it must give the same
(mass, energy) as the handle-based sp_reduce, within 1e-12 relative, on two
calls in a row (the second call reuses the static scratch after the fields
changed), and both must equal an FP64 NumPy evaluation of the formula
(include/symphas_b200.h, sp_reduce) within 1e-10 relative (the sums run in
another order).  This file is collected last so a failing run has already run
every other test.
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


def landau_np(fields, model, coeff, h, dim):
    """(mass of field 0, energy) of one instance, in FP64 NumPy: `fields` is
    (nf, *shape) with x the last axis; forward differences, periodic."""
    c = list(coeff) + [1.0] * (8 - len(coeff))
    f = np.asarray(fields, dtype=np.float64)
    axes = [-1, -2, -3][:dim]
    energy = 0.0
    for v in f:
        g2 = sum(((np.roll(v, -1, axis=a) - v) / h) ** 2 for a in axes)
        v2 = v * v
        if model in (C.SP_MODEL_A, C.SP_MODEL_B):
            e = -0.5 * c[0] * v2 + 0.25 * c[1] * v2 * v2 + 0.5 * g2
        else:
            kappa = 1.0 if model == C.SP_MODEL_C else c[1]
            e = -0.5 * v2 + 0.25 * v2 * v2 + 0.5 * kappa * g2
        energy += float(e.sum())
    if model == C.SP_MODEL_C:
        energy += float((c[0] * f[0] * f[0] * f[1] * f[1]).sum())
    return float(f[0].sum()), energy * h ** dim


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


MODELS = {"A": (sp.model_MA_t, C.SP_MODEL_A), "B": (sp.model_MB_t, C.SP_MODEL_B),
          "AMK": (sp.model_MAMK_t, C.SP_MODEL_AMK), "BMK": (sp.model_MBMK_t, C.SP_MODEL_BMK)}
S2 = sp.Stencil2d2h(5, 6, 13)


@pytest.mark.parametrize("name,dim,coeff,dtype,batch,h", [
    ("A", 2, (0.7, 1.3), "f64", 1, 0.5),
    ("AMK", 2, (1.7, 0.6), "f64", 1, 1.0),
    ("BMK", 3, (1.2, 0.8), "f64", 1, 1.0),
    ("B", 2, (), "f32", 3, 1.0),
])
def test_noalloc_and_sp_reduce_against_numpy(name, dim, coeff, dtype, batch, h):
    torch.cuda.set_device(0)
    cls, code_model = MODELS[name]
    dims = (40, 24) if dim == 2 else (20, 12, 16)
    m = cls(dim, sp.SolverFT(S2 if dim == 2 else S3, form="fused"),
            sp.ProblemParameters(dims, h=h), coeff=coeff, dtype=dtype, batch=batch)
    for i in range(batch):
        m.fill_uniform(0, 70 + i, -0.35, -0.05, inst=i)
    code = C.SP_F64 if dtype == "f64" else C.SP_F32
    tdt = torch.float64 if dtype == "f64" else torch.float32
    for _ in range(2):
        m.step(0.002, 10)
        host = np.stack([m.get_field(0, inst=i) for i in range(batch)])
        fields = torch.from_numpy(host).to(device="cuda", dtype=tdt).contiguous()
        got = noalloc(fields, code, dims, code_model, coeff, h, batch)
        for i in range(batch):
            want = landau_np(host[i][None], code_model, coeff, h, dim)
            mass, energy = m.reduce(0, inst=i)
            assert close(mass, want[0], 1e-10) and close(energy, want[1], 1e-10), (mass, energy,
                                                                                   want)
            assert close(got[i, 0], mass) and close(got[i, 1], energy), (i, got[i], mass, energy)
            # SymPhas's collectors: Density is the sum, Energy the mean
            assert close(m.density(0, inst=i), want[0], 1e-10)
            assert close(m.energy(0, inst=i), want[0] / host[i].size, 1e-10)
    m.close()


def test_noalloc_model_c_against_numpy():
    torch.cuda.set_device(0)
    n, h, gamma = 12, 1.0, 0.5
    m = sp.model_MC_t(3, sp.SolverFT(S3, form="fused"), sp.ProblemParameters((n, n, n), h=h),
                      coeff=(gamma,), dtype="f64")
    m.fill_uniform(0, 90, 0.0, 0.2)
    m.fill_uniform(1, 91, -0.1, 0.1)
    m.step(0.005, 5)
    host = np.stack([m.get_field(f) for f in range(2)])
    want = landau_np(host, C.SP_MODEL_C, (gamma,), h, 3)
    got = noalloc(torch.from_numpy(host).to("cuda").contiguous(), C.SP_F64, (n, n, n),
                  C.SP_MODEL_C, (gamma,), h, 1)
    assert close(got[0, 0], want[0], 1e-10) and close(got[0, 1], want[1], 1e-10), (got, want)
    m.close()


@pytest.mark.parametrize("model,h,what", [(C.SP_OP_LAP, 1.0, b"model"), (99, 1.0, b"model"),
                                          (C.SP_MODEL_B, float("inf"), b"spacing"),
                                          (C.SP_MODEL_B, float("nan"), b"spacing")])
def test_noalloc_rejects_unknown_models_and_bad_spacing(model, h, what):
    torch.cuda.set_device(0)
    field = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    n = (ctypes.c_int * 3)(2, 2, 2)
    rc = C.lib().sp_reduce_fields_noalloc(
        ctypes.c_void_p(field.data_ptr()), C.SP_F64, 3, n, model, None, h, 1,
        ctypes.c_void_p(out.data_ptr()), None)
    assert rc == C.SP_EINVAL
    assert what in C.lib().sp_noalloc_error()
