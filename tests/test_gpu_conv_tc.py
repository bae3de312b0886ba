"""The tcgen05 forward convolution (fp32 accumulator in tensor memory) against
the plain PyTorch fp32 reference on the same bf16 operands, and against the
mma.sync kernel it can replace: the epilogue (bias, residual, GELU), ragged
pixel counts (not a multiple of the 128-pixel tile), a partial last K step
(cin = 8: K = 72), both output widths (cout 32 and multiples of 64), and the
bounded waits' flag left clear.

Tolerances: both kernels accumulate in fp32, so their sums agree to ~1e-6
relative before the bf16 rounding of the stored outputs; outputs are compared
with the reference at 1.5e-2 relative to their scale and with each other at
2^-7 relative (one bf16 rounding step either way)."""
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
    xp = F.pad(x.permute(0, 3, 1, 2), (1, 1, 1, 1), mode="circular")
    return F.conv2d(xp, w.permute(0, 3, 1, 2), b).permute(0, 2, 3, 1)


def rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-30))


def status():
    flag = ctypes.c_int(-1)
    assert C.lib().sp_conv_tc_status(ctypes.byref(flag)) == C.SP_OK
    return flag.value


@pytest.mark.parametrize("n,h,w,ci,co", [(2, 16, 24, 32, 64), (1, 9, 7, 64, 32),
                                         (1, 8, 8, 128, 256), (3, 33, 17, 32, 32),
                                         (1, 10, 10, 8, 64), (2, 64, 64, 64, 128)])
def test_tc_forward_matches_reference_and_mma_sync(n, h, w, ci, co):
    torch.manual_seed(0)
    x = torch.randn(n, h, w, ci, device="cuda").bfloat16()
    wt = (torch.randn(co, 3, 3, ci, device="cuda") / (3 * ci ** 0.5)).bfloat16()
    b = torch.randn(co, device="cuda") * 0.1
    res = torch.randn(n, h, w, co, device="cuda").bfloat16()
    z = torch.full((n, h, w, co), float("nan"), device="cuda", dtype=torch.bfloat16)
    a = torch.full_like(z, float("nan"))
    rc = C.lib().sp_conv3x3_fwd_tc(ptr(x), ptr(wt), ptr(b), ptr(res), ptr(z), ptr(a), n, h, w,
                                   ci, co, stream())
    assert rc == C.SP_OK
    assert status() == 0
    zr = ref_conv(x.float(), wt.float(), b) + res.float()
    assert not torch.isnan(z).any() and not torch.isnan(a).any()
    assert rel(z.float(), zr) < 1.5e-2
    assert rel(a.float(), F.gelu(zr, approximate="tanh")) < 1.5e-2
    if ci % 32 == 0:
        z2 = torch.empty_like(z)
        assert C.lib().sp_conv3x3_fwd(ptr(x), ptr(wt), ptr(b), ptr(res), ptr(z2), None, n, h, w,
                                      ci, co, stream()) == C.SP_OK
        torch.cuda.synchronize()
        assert rel(z.float(), z2.float()) < 2.0 ** -7


def test_tc_forward_single_output_and_no_epilogue_operands():
    torch.manual_seed(2)
    n, h, w, ci, co = 1, 12, 20, 32, 64
    x = torch.randn(n, h, w, ci, device="cuda").bfloat16()
    wt = (torch.randn(co, 3, 3, ci, device="cuda") / (3 * ci ** 0.5)).bfloat16()
    a = torch.empty(n, h, w, co, device="cuda", dtype=torch.bfloat16)
    assert C.lib().sp_conv3x3_fwd_tc(ptr(x), ptr(wt), None, None, None, ptr(a), n, h, w, ci, co,
                                     stream()) == C.SP_OK
    assert status() == 0
    zr = ref_conv(x.float(), wt.float())
    assert rel(a.float(), F.gelu(zr, approximate="tanh")) < 1.5e-2


def test_tc_forward_rejects_unsupported_shapes():
    x = torch.zeros(1, 4, 4, 32, device="cuda", dtype=torch.bfloat16)
    wt = torch.zeros(48, 3, 3, 32, device="cuda", dtype=torch.bfloat16)
    z = torch.zeros(1, 4, 4, 48, device="cuda", dtype=torch.bfloat16)
    assert C.lib().sp_conv3x3_fwd_tc(ptr(x), ptr(wt), None, None, ptr(z), None, 1, 4, 4, 32, 48,
                                     stream()) == C.SP_EINVAL
    assert C.lib().sp_conv3x3_fwd_tc(ptr(x), ptr(wt), None, None, ptr(z), None, 1, 4, 4, 12, 64,
                                     stream()) == C.SP_EINVAL


@pytest.mark.parametrize("kernel", ["tc", "strip"])
def test_surrogate_network_on_either_kernel(kernel):
    """The jump network gives the same prediction with its forward
    convolutions on tcgen05 or on mma.sync (bf16 activations: 2e-2)."""
    from symphas_b200 import surrogate as S

    torch.cuda.set_device(0)
    net = S.JumpNet((32, 64, 128))
    psi = torch.rand(2, 64, 64, device="cuda") - 0.5
    old = S.KERNEL
    try:
        with torch.no_grad():
            S.KERNEL = "mma"
            d0 = net(psi)
            S.KERNEL = kernel
            d1 = net(psi)
    finally:
        S.KERNEL = old
    assert status() == 0
    assert rel(d1, d0) < 2e-2


STRIP_SHAPES = [(2, 16, 24, 32, 64), (1, 9, 7, 64, 32), (1, 8, 8, 128, 256), (3, 33, 17, 32, 32),
                (1, 10, 10, 16, 128), (2, 64, 64, 64, 128), (1, 40, 256, 32, 32),
                (4, 32, 32, 256, 256)]


@pytest.mark.parametrize("tile", ["2,16,1", "2,32,4", "4,16,1", "2,16,4"])
@pytest.mark.parametrize("n,h,w,ci,co", [STRIP_SHAPES[i] for i in (0, 1, 2, 4, 6)])
def test_strip_tile_shapes(n, h, w, ci, co, tile, monkeypatch):
    """Every CTA shape of the strip kernel (SP_STRIP_SHAPE: 2 or 4 M-tiles,
    16 or 32 input channels per K block, 1 or up to 4 ring stages) gives the
    convolution: against the reference as the default shape is."""
    if ci % int(tile.split(",")[1]):
        pytest.skip("input channels not a multiple of the K block")
    monkeypatch.setenv("SP_STRIP_SHAPE", tile)
    test_strip_forward_matches_reference_and_mma_sync(n, h, w, ci, co)


@pytest.mark.parametrize("n,h,w,ci,co", STRIP_SHAPES)
def test_strip_forward_matches_reference_and_mma_sync(n, h, w, ci, co):
    """The gather-once kernel: padded-position strip, taps as operand offsets,
    pre-tiled weights by bulk copy -- ragged position counts, every channel
    block size (16 and 32 input channels per stage, 1 to 16 stages), every
    output block (32, 64, 128 channels), rows as wide as the network's 256."""
    torch.manual_seed(1)
    x = torch.randn(n, h, w, ci, device="cuda").bfloat16()
    wt = (torch.randn(co, 3, 3, ci, device="cuda") / (3 * ci ** 0.5)).bfloat16()
    b = torch.randn(co, device="cuda") * 0.1
    res = torch.randn(n, h, w, co, device="cuda").bfloat16()
    scratch = torch.empty(9 * ci * co, device="cuda", dtype=torch.bfloat16)
    z = torch.full((n, h, w, co), float("nan"), device="cuda", dtype=torch.bfloat16)
    a = torch.full_like(z, float("nan"))
    rc = C.lib().sp_conv3x3_fwd_strip(ptr(x), ptr(wt), ptr(scratch), ptr(b), ptr(res), ptr(z),
                                      ptr(a), n, h, w, ci, co, stream())
    assert rc == C.SP_OK
    assert status() == 0
    zr = ref_conv(x.float(), wt.float(), b) + res.float()
    assert not torch.isnan(z).any() and not torch.isnan(a).any()
    assert rel(z.float(), zr) < 1.5e-2
    assert rel(a.float(), F.gelu(zr, approximate="tanh")) < 1.5e-2
    if ci % 32 == 0:
        z2 = torch.empty_like(z)
        assert C.lib().sp_conv3x3_fwd(ptr(x), ptr(wt), ptr(b), ptr(res), ptr(z2), None, n, h, w,
                                      ci, co, stream()) == C.SP_OK
        torch.cuda.synchronize()
        assert rel(z.float(), z2.float()) < 2.0 ** -7


def test_strip_forward_rejects_unsupported_shapes():
    x = torch.zeros(1, 4, 800, 32, device="cuda", dtype=torch.bfloat16)
    wt = torch.zeros(64, 3, 3, 32, device="cuda", dtype=torch.bfloat16)
    s = torch.zeros(9 * 32 * 64, device="cuda", dtype=torch.bfloat16)
    z = torch.zeros(1, 4, 800, 64, device="cuda", dtype=torch.bfloat16)
    # too wide a row for the strip, an input channel count not a multiple of 16,
    # an output block the kernel does not build
    assert C.lib().sp_conv3x3_fwd_strip(ptr(x), ptr(wt), ptr(s), None, None, ptr(z), None, 1, 4,
                                        800, 32, 64, stream()) == C.SP_EINVAL
    assert C.lib().sp_conv3x3_fwd_strip(ptr(x), ptr(wt), ptr(s), None, None, ptr(z), None, 1, 4,
                                        4, 24, 64, stream()) == C.SP_EINVAL
    assert C.lib().sp_conv3x3_fwd_strip(ptr(x), ptr(wt), ptr(s), None, None, ptr(z), None, 1, 4,
                                        4, 32, 96, stream()) == C.SP_EINVAL


@pytest.mark.parametrize("n,h,w,ci,co", [(2, 16, 24, 64, 32), (1, 32, 32, 128, 64),
                                         (2, 8, 8, 256, 128), (1, 40, 256, 64, 32)])
def test_strip_up2_equals_strip_on_the_upsampled_input(n, h, w, ci, co):
    """The decoder's convolution of a 2x nearest up-sampling, with the
    up-sampling read in the gather: the bits of the strip kernel on the
    materialised up-sampled input."""
    torch.manual_seed(2)
    x = torch.randn(n, h // 2, w // 2, ci, device="cuda").bfloat16()
    up = x[:, :, None, :, None, :].expand(n, h // 2, 2, w // 2, 2, ci).reshape(n, h, w, ci).contiguous()
    wt = (torch.randn(co, 3, 3, ci, device="cuda") / (3 * ci ** 0.5)).bfloat16()
    b = torch.randn(co, device="cuda") * 0.1
    res = torch.randn(n, h, w, co, device="cuda").bfloat16()
    scratch = torch.empty(9 * ci * co, device="cuda", dtype=torch.bfloat16)
    a0 = torch.empty(n, h, w, co, device="cuda", dtype=torch.bfloat16)
    a1 = torch.full_like(a0, float("nan"))
    assert C.lib().sp_conv3x3_fwd_strip(ptr(up), ptr(wt), ptr(scratch), ptr(b), ptr(res), None,
                                        ptr(a0), n, h, w, ci, co, stream()) == C.SP_OK
    assert C.lib().sp_conv3x3_fwd_strip_up2(ptr(x), ptr(wt), ptr(scratch), ptr(b), ptr(res), None,
                                            ptr(a1), n, h, w, ci, co, stream()) == C.SP_OK
    torch.cuda.synchronize()
    assert status() == 0
    assert torch.equal(a0, a1)
    # odd output extents are refused
    assert C.lib().sp_conv3x3_fwd_strip_up2(ptr(x), ptr(wt), ptr(scratch), ptr(b), ptr(res), None,
                                            ptr(a1), n, h - 1, w, ci, co, stream()) == C.SP_EINVAL


@pytest.mark.parametrize("n,h,w,c", [(3, 16, 24, 32), (1, 256, 256, 64), (2, 8, 4, 256)])
def test_avgpool2_kernel_matches_torch_mean(n, h, w, c):
    """The inference pooling kernel: the 2x2 mean of torch within one bf16
    rounding; odd extents and channel counts that are not a multiple of 8 are
    refused."""
    torch.manual_seed(4)
    x = torch.randn(n, h, w, c, device="cuda").bfloat16()
    y = torch.full((n, h // 2, w // 2, c), float("nan"), device="cuda", dtype=torch.bfloat16)
    assert C.lib().sp_avgpool2_bf16(ptr(x), ptr(y), n, h, w, c, stream()) == C.SP_OK
    torch.cuda.synchronize()
    want = x.float().view(n, h // 2, 2, w // 2, 2, c).mean((2, 4))
    assert torch.allclose(y.float(), want, rtol=2.0 ** -7, atol=1e-6)
    assert C.lib().sp_avgpool2_bf16(ptr(x), ptr(y), n, h - 1, w, c, stream()) == C.SP_EINVAL
    assert C.lib().sp_avgpool2_bf16(ptr(x), ptr(y), n, h, w, 12, stream()) == C.SP_EINVAL


def test_embed_channel0_kernel():
    """The network's input: the field in channel 0 (rounded to bf16), zeros
    elsewhere, as torch builds it."""
    torch.manual_seed(5)
    psi = torch.randn(3, 40, 24, device="cuda")
    x = torch.full((3, 40, 24, 32), float("nan"), device="cuda", dtype=torch.bfloat16)
    assert C.lib().sp_embed_channel0_bf16(ptr(psi), ptr(x), psi.numel(), 32, stream()) == C.SP_OK
    torch.cuda.synchronize()
    want = torch.zeros_like(x)
    want[..., 0] = psi.bfloat16()
    assert torch.equal(x, want)
    assert C.lib().sp_embed_channel0_bf16(ptr(psi), ptr(x), psi.numel(), 12, stream()) == C.SP_EINVAL
