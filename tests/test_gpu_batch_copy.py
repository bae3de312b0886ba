"""Batched device copies (sp_upload_batch_device / sp_download_batch_device):
one field of every instance to or from one dense device array.  They must
move the same values as the per-instance copies, and an upload must leave
the halos as the per-instance upload does (the steps after it give the same
bits), for periodic and Dirichlet sides, 2D and 3D, FP32 and FP64."""
import numpy as np
import pytest
import torch

import symphas_b200 as sp
from symphas_b200 import _capi as C

pytestmark = pytest.mark.gpu


def make(dim, n, dtype, batch, dirichlet=False):
    P, D = sp.BoundaryType.PERIODIC, sp.BoundaryType.DEFAULT
    bc = [D, D] + [P] * 4 if dirichlet else [P] * 6
    st = sp.Stencil2d2h(5, 6, 13) if dim == 2 else sp.Stencil3d2h(7, 10, 25)
    return sp.model_MB_t(dim, sp.SolverFT(st, form="fused"),
                         sp.ProblemParameters((n,) * dim, h=1.0, boundary=bc, boundary_value=0.3),
                         dtype=dtype, batch=batch)


@pytest.mark.parametrize("dim,n", [(2, 40), (3, 20)])
@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("dirichlet", [False, True])
def test_batch_copies_match_per_instance_copies(dim, n, dtype, dirichlet):
    torch.cuda.set_device(0)
    batch = 5
    tdt = torch.float32 if dtype == "f32" else torch.float64
    g = torch.Generator(device="cuda").manual_seed(3)
    x = (0.2 * torch.rand((batch,) + (n,) * dim, device="cuda", generator=g, dtype=tdt) - 0.1)
    a = make(dim, n, dtype, batch, dirichlet)
    b = make(dim, n, dtype, batch, dirichlet)
    esz = x.element_size()
    sites = n ** dim
    a.batch_from_device(0, x.data_ptr(), x.numel() * esz)
    for i in range(batch):
        b.field_from_device(0, x[i].data_ptr(), sites * esz, inst=i)
    torch.cuda.synchronize()
    for i in range(batch):
        assert np.array_equal(a.get_field(0, inst=i), x[i].cpu().numpy())
    a.step(0.002, 7)
    b.step(0.002, 7)
    out = torch.empty_like(x)
    a.batch_to_device(0, out.data_ptr(), out.numel() * esz)
    a.synchronize()
    for i in range(batch):
        got = b.get_field(0, inst=i)
        assert np.array_equal(a.get_field(0, inst=i), got), i
        assert np.array_equal(out[i].cpu().numpy(), got), i
    a.close()
    b.close()


def test_batch_copy_rejects_wrong_sizes():
    torch.cuda.set_device(0)
    m = make(2, 16, "f32", 3)
    x = torch.zeros(2, 16, 16, device="cuda")
    with pytest.raises(C.SymPhasError):
        m.batch_from_device(0, x.data_ptr(), x.numel() * 4)
    with pytest.raises(C.SymPhasError):
        m.batch_to_device(1, x.data_ptr(), 3 * 256 * 4)
    m.close()
