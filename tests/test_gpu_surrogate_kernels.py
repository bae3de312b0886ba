"""The surrogate's BF16 tensor-core kernels against plain PyTorch fp32
references on the same bf16-rounded operands: the circular 3x3 convolution
(bias, residual, GELU epilogue), its data gradient (flipped weights through
the forward kernel), its weight gradient (split-K atomics) and Adam.

Tolerances: the kernels accumulate in fp32 like the reference, so sums agree
to ~1e-6 relative before the bf16 rounding of the stored outputs (2^-8
relative); outputs are compared at 1.5e-2 relative to their scale, fp32
gradients at 1e-3."""
import ctypes

import pytest
import torch
import torch.nn.functional as F

from symphas_b200 import _capi as C

pytestmark = pytest.mark.gpu


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ref_conv(x, w, b=None):
    """x [N,H,W,Ci], w [Co,3,3,Ci] (fp32) -> [N,H,W,Co], circular padding."""
    xp = F.pad(x.permute(0, 3, 1, 2), (1, 1, 1, 1), mode="circular")
    return F.conv2d(xp, w.permute(0, 3, 1, 2), b).permute(0, 2, 3, 1)


def rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-30))


@pytest.mark.parametrize("n,h,w,ci,co", [(2, 16, 24, 32, 64), (1, 9, 7, 64, 32),
                                         (3, 32, 32, 32, 8), (1, 8, 8, 128, 256)])
def test_conv_forward_epilogue(n, h, w, ci, co):
    torch.manual_seed(0)
    x = torch.randn(n, h, w, ci, device="cuda").bfloat16()
    wt = (torch.randn(co, 3, 3, ci, device="cuda") / (3 * ci ** 0.5)).bfloat16()
    b = torch.randn(co, device="cuda") * 0.1
    res = torch.randn(n, h, w, co, device="cuda").bfloat16()
    z = torch.empty(n, h, w, co, device="cuda", dtype=torch.bfloat16)
    a = torch.empty_like(z)
    rc = C.lib().sp_conv3x3_fwd(ptr(x), ptr(wt), ptr(b), ptr(res), ptr(z), ptr(a), n, h, w, ci,
                                co, stream())
    assert rc == C.SP_OK
    torch.cuda.synchronize()
    zr = ref_conv(x.float(), wt.float(), b) + res.float()
    assert rel(z.float(), zr) < 1.5e-2
    assert rel(a.float(), F.gelu(zr, approximate="tanh")) < 1.5e-2


def test_conv_input_and_weight_gradients():
    torch.manual_seed(1)
    n, h, w, ci, co = 2, 20, 12, 32, 64
    x = torch.randn(n, h, w, ci, device="cuda").bfloat16()
    wt = (torch.randn(co, 3, 3, ci, device="cuda") / (3 * ci ** 0.5)).bfloat16()
    dy = torch.randn(n, h, w, co, device="cuda").bfloat16()
    xr = x.float().requires_grad_()
    wr = wt.float().requires_grad_()
    ref_conv(xr, wr).backward(dy.float())
    # data gradient: forward kernel with the flipped weights
    wf = torch.empty(ci, 3, 3, co, device="cuda", dtype=torch.bfloat16)
    assert C.lib().sp_conv3x3_flip(ptr(wt), ptr(wf), ci, co, stream()) == C.SP_OK
    dx = torch.empty(n, h, w, ci, device="cuda", dtype=torch.bfloat16)
    assert C.lib().sp_conv3x3_fwd(ptr(dy), ptr(wf), None, None, ptr(dx), None, n, h, w, co, ci,
                                  stream()) == C.SP_OK
    # weight gradient
    dw = torch.zeros(co, 3, 3, ci, device="cuda")
    assert C.lib().sp_conv3x3_wgrad(ptr(x), ptr(dy), ptr(dw), n, h, w, ci, co,
                                    stream()) == C.SP_OK
    torch.cuda.synchronize()
    assert rel(dx.float(), xr.grad) < 1.5e-2
    assert rel(dw, wr.grad) < 1e-3


def test_weight_gradient_many_chunks():
    """Enough pixels that the split-K grid has many chunks per tile."""
    torch.manual_seed(2)
    n, h, w, ci, co = 4, 64, 64, 64, 32
    x = torch.randn(n, h, w, ci, device="cuda").bfloat16()
    dy = torch.randn(n, h, w, co, device="cuda").bfloat16()
    wr = torch.zeros(co, 3, 3, ci, device="cuda", requires_grad=True)
    ref_conv(x.float(), wr).backward(dy.float())
    dw = torch.zeros(co, 3, 3, ci, device="cuda")
    assert C.lib().sp_conv3x3_wgrad(ptr(x), ptr(dy), ptr(dw), n, h, w, ci, co,
                                    stream()) == C.SP_OK
    torch.cuda.synchronize()
    assert rel(dw, wr.grad) < 1e-3


def test_adam_matches_the_update_rule():
    torch.manual_seed(3)
    nel = 10007
    w = torch.randn(nel, device="cuda")
    wb = torch.empty(nel, device="cuda", dtype=torch.bfloat16)
    m = torch.zeros(nel, device="cuda")
    v = torch.zeros(nel, device="cuda")
    ref_w, ref_m, ref_v = w.clone(), m.clone(), v.clone()
    lr, b1, b2, eps = 1e-3, 0.9, 0.999, 1e-8
    for step in range(1, 4):
        g = torch.randn(nel, device="cuda")
        assert C.lib().sp_adam_step(ptr(w), ptr(wb), ptr(g), ptr(m), ptr(v), nel, lr, b1, b2,
                                    eps, step, 0.0, stream()) == C.SP_OK
        ref_m = b1 * ref_m + (1 - b1) * g
        ref_v = b2 * ref_v + (1 - b2) * g * g
        ref_w = ref_w - lr * (ref_m / (1 - b1 ** step)) / ((ref_v / (1 - b2 ** step)).sqrt() + eps)
    torch.cuda.synchronize()
    assert torch.allclose(w, ref_w, rtol=1e-5, atol=1e-6)
    assert torch.equal(wb, w.bfloat16())
