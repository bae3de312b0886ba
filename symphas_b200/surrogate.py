"""Learned k-step jump for 2D model B (Cahn-Hilliard), judged by the
finite-difference solver.  No counterpart in SymPhas.

A circular-padded convolutional encoder-decoder (levels of 32/64/128/256
channels at 256^2 / 128^2 / 64^2 / 32^2, 3x3 kernels, GELU, additive skips,
~1.9 M parameters) maps psi(t) to the change over `jump` solver steps; the
prediction is projected onto zero mean, so every jump conserves the mass of
psi exactly as model B does.  Convolutions, their gradients and the Adam
update run in this package's BF16 tensor-core kernels
(sp_conv3x3_fwd_tc on tcgen05 with the accumulator in tensor memory, or
sp_conv3x3_fwd on mma.sync; sp_conv3x3_wgrad / sp_conv3x3_flip /
sp_adam_step; fp32 accumulation, fp32 master weights); PyTorch holds the
tensors and does the element-wise glue (pooling, up-sampling, the loss, and
GELU under autograd -- at inference the convolution's epilogue applies it).

Training data are trajectories of this package's own fused FD kernel
(model_MB_t, batch of instances in one persistent launch).  At inference each
jump is followed by a few FD steps that judge it: when those FD steps move the
jumped field much faster than they moved the field before the jump (a jump off
the solution manifold relaxes fast under the stiff bilaplacian, while model B
only slows down as it coarsens), the batch falls back to plain FD for that
interval.
"""
import ctypes
import math
import time

import numpy as np
import torch
import torch.nn.functional as F

from . import _capi as C
from .model import ProblemParameters, SolverFT, Stencil2d2h, model_MB_t

CIN = 32  # channels of the network input (psi, zero-padded)


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _s():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ok(rc, what):
    if rc != C.SP_OK:
        raise C.SymPhasError(rc, what)


# The forward convolutions (and the data gradients, forward convolutions of
# the flipped weights) run on
#   "strip"  the tcgen05 kernel that stages each input pixel once and reads the
#            nine taps as operand offsets (sp_conv3x3_fwd_strip), where its
#            shapes allow (cin % 16 == 0, cout 32, 64 or a multiple of 128,
#            width <= 764), else on the next;
#   "tc"     the tcgen05 kernel with a per-tap gather (sp_conv3x3_fwd_tc);
#   "mma"    the mma.sync kernel (sp_conv3x3_fwd).
KERNEL = "strip"


def _strip_ok(ci, co, w):
    return ci % 16 == 0 and (co in (32, 64) or co % 128 == 0) and w <= 764


def _fwd(x, wb, bias, res, z, a, ci, co, scratch=None):
    n, h, w = x.shape[:3]
    if KERNEL == "strip" and scratch is not None and _strip_ok(ci, co, w):
        _ok(C.lib().sp_conv3x3_fwd_strip(_p(x), _p(wb), _p(scratch), _p(bias), _p(res), _p(z),
                                         _p(a), n, h, w, ci, co, _s()), "sp_conv3x3_fwd_strip")
    elif KERNEL in ("strip", "tc") and ci % 8 == 0 and (co == 32 or co % 64 == 0):
        _ok(C.lib().sp_conv3x3_fwd_tc(_p(x), _p(wb), _p(bias), _p(res), _p(z), _p(a), n, h, w,
                                      ci, co, _s()), "sp_conv3x3_fwd_tc")
    else:
        _ok(C.lib().sp_conv3x3_fwd(_p(x), _p(wb), _p(bias), _p(res), _p(z), _p(a), n, h, w, ci,
                                   co, _s()), "sp_conv3x3_fwd")


class ConvLayer:
    """A 3x3 circular convolution: fp32 master weights [cout][3][3][cin] and
    bias, a bf16 copy for the kernels, gradient buffers and Adam moments."""

    def __init__(self, cin, cout, gen, gain=1.0):
        std = gain * math.sqrt(2.0 / (9 * cin))
        self.cin, self.cout = cin, cout
        self.w = (torch.randn(cout, 3, 3, cin, generator=gen) * std).cuda()
        self.b = torch.zeros(cout, device="cuda")
        self.wb = self.w.bfloat16()
        self.wf = torch.empty(cin, 3, 3, cout, device="cuda", dtype=torch.bfloat16)
        # the weights (or the flipped weights) re-tiled for the strip kernel
        self.wt = torch.empty(9 * cin * cout, device="cuda", dtype=torch.bfloat16)
        self.gw = torch.zeros_like(self.w)
        self.gb = torch.zeros_like(self.b)
        self.m = [torch.zeros_like(self.w), torch.zeros_like(self.b)]
        self.v = [torch.zeros_like(self.w), torch.zeros_like(self.b)]
        # the weights live outside autograd (their gradients accumulate in gw,
        # gb); this empty tensor puts the layer on the graph
        self.anchor = torch.zeros(0, device="cuda", requires_grad=True)

    def nparams(self):
        return self.w.numel() + self.b.numel()

    def zero_grad(self):
        self.gw.zero_()
        self.gb.zero_()

    def adam(self, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
        _ok(C.lib().sp_adam_step(_p(self.w), _p(self.wb), _p(self.gw), _p(self.m[0]),
                                 _p(self.v[0]), self.w.numel(), lr, b1, b2, eps, step, wd, _s()),
            "sp_adam_step")
        _ok(C.lib().sp_adam_step(_p(self.b), None, _p(self.gb), _p(self.m[1]), _p(self.v[1]),
                                 self.b.numel(), lr, b1, b2, eps, step, 0.0, _s()),
            "sp_adam_step")


class _Conv(torch.autograd.Function):
    """z = conv3x3(x) + bias (+ res): forward and both gradients in the
    package's kernels; the weight and bias gradients accumulate in the layer."""

    @staticmethod
    def forward(ctx, x, anchor, layer, res):
        n, h, w, ci = x.shape
        z = torch.empty(n, h, w, layer.cout, device="cuda", dtype=torch.bfloat16)
        _fwd(x, layer.wb, layer.b, res, z, None, ci, layer.cout, layer.wt)
        ctx.save_for_backward(x)
        ctx.layer = layer
        ctx.has_res = res is not None
        return z

    @staticmethod
    def backward(ctx, dz):
        (x,) = ctx.saved_tensors
        L = ctx.layer
        dz = dz.contiguous().bfloat16()
        n, h, w, ci = x.shape
        _ok(C.lib().sp_conv3x3_wgrad(_p(x), _p(dz), _p(L.gw), n, h, w, ci, L.cout, _s()),
            "sp_conv3x3_wgrad")
        L.gb += dz.float().sum((0, 1, 2))
        dx = None
        if ctx.needs_input_grad[0]:
            _ok(C.lib().sp_conv3x3_flip(_p(L.wb), _p(L.wf), ci, L.cout, _s()), "sp_conv3x3_flip")
            dx = torch.empty_like(x)
            _fwd(dz, L.wf, None, None, dx, None, L.cout, ci, L.wt)
        return dx, None, None, (dz if ctx.has_res else None)


def conv(x, layer, res=None):
    return _Conv.apply(x, layer.anchor, layer, res)


def gelu(z):
    return F.gelu(z, approximate="tanh")


def conv_gelu(x, layer, res=None):
    """gelu(conv(x) + bias (+ res)); without autograd, one kernel writes the
    activation from its epilogue."""
    if torch.is_grad_enabled():
        return gelu(conv(x, layer, res))
    n, h, w, ci = x.shape
    a = torch.empty(n, h, w, layer.cout, device="cuda", dtype=torch.bfloat16)
    _fwd(x, layer.wb, layer.b, res, None, a, ci, layer.cout, layer.wt)
    return a


def conv_gelu_up(x, layer, res=None):
    """conv_gelu(up2(x), layer, res): without autograd, and where the strip
    kernel runs, one kernel reads the up-sampled input in its gather (no
    up-sampled copy is made)."""
    n, h, w, ci = x.shape
    if torch.is_grad_enabled() or KERNEL != "strip" or not _strip_ok(ci, layer.cout, 2 * w):
        return conv_gelu(up2(x), layer, res)
    a = torch.empty(n, 2 * h, 2 * w, layer.cout, device="cuda", dtype=torch.bfloat16)
    _ok(C.lib().sp_conv3x3_fwd_strip_up2(_p(x.contiguous()), _p(layer.wb), _p(layer.wt),
                                         _p(layer.b), _p(res), None, _p(a), n, 2 * h, 2 * w, ci,
                                         layer.cout, _s()), "sp_conv3x3_fwd_strip_up2")
    return a


def pool2(x):
    n, h, w, c = x.shape
    if not torch.is_grad_enabled() and x.is_contiguous() and c % 8 == 0:
        # inference: one vectorised kernel (the mean of the four in fp32)
        y = torch.empty(n, h // 2, w // 2, c, device="cuda", dtype=torch.bfloat16)
        _ok(C.lib().sp_avgpool2_bf16(_p(x), _p(y), n, h, w, c, _s()), "sp_avgpool2_bf16")
        return y
    return x.view(n, h // 2, 2, w // 2, 2, c).mean((2, 4))


def up2(x):
    n, h, w, c = x.shape
    return x[:, :, None, :, None, :].expand(n, h, 2, w, 2, c).reshape(n, 2 * h, 2 * w, c)


class JumpNet:
    """Encoder-decoder over `levels` resolutions with additive skips."""

    def __init__(self, channels=(32, 64, 128, 256), seed=0):
        g = torch.Generator().manual_seed(seed)
        self.ch = tuple(channels)
        self.enc, self.dec = [], []
        cin = CIN
        for c in self.ch:
            self.enc.append((ConvLayer(cin, c, g), ConvLayer(c, c, g)))
            cin = c
        for lvl in range(len(self.ch) - 2, -1, -1):
            c = self.ch[lvl]
            self.dec.append((ConvLayer(self.ch[lvl + 1], c, g), ConvLayer(c, c, g)))
        self.head = ConvLayer(self.ch[0], 32, g, gain=0.1)  # channel 0 is the output
        self.head.w[1:] = 0.0  # channels 1..31 pad the kernel's channel count
        self.head.wb.copy_(self.head.w.bfloat16())
        self.scale = 1.0  # target scale: the network predicts delta / scale

    def layers(self):
        out = []
        for a, b in self.enc + self.dec:
            out += [a, b]
        return out + [self.head]

    def nparams(self):
        # the head's output channels 1..31 are padding (zero, and no loss reaches them)
        return sum(l.nparams() for l in self.layers()) - 31 * (9 * self.ch[0] + 1)

    def __call__(self, psi):
        """psi [N, H, W] (fp32) -> predicted change over one jump, zero mean."""
        n, h, w = psi.shape
        x = torch.empty(n, h, w, CIN, device="cuda", dtype=torch.bfloat16)
        src = psi.contiguous().float()
        _ok(C.lib().sp_embed_channel0_bf16(_p(src), _p(x), n * h * w, CIN, _s()),
            "sp_embed_channel0_bf16")
        skips = []
        for lvl, (a, b) in enumerate(self.enc):
            x = conv_gelu(conv_gelu(x, a), b)
            if lvl < len(self.enc) - 1:
                skips.append(x)
                x = pool2(x)
        for (a, b), s in zip(self.dec, reversed(skips)):
            x = conv_gelu_up(x, a, res=s)
            x = conv_gelu(x, b)
        d = conv(x, self.head)[..., 0].float()
        d = d - d.mean((1, 2), keepdim=True)  # exact mass conservation
        return d * self.scale

    def flops(self, n):
        """Multiply-add FLOPs of one forward pass of one n x n sample."""
        total, size = 0, n
        for lvl, (a, b) in enumerate(self.enc):
            total += 18 * size * size * (a.cin * a.cout + b.cin * b.cout)
            if lvl < len(self.enc) - 1:
                size //= 2
        for a, b in self.dec:
            size *= 2
            total += 18 * size * size * (a.cin * a.cout + b.cin * b.cout)
        return total + 18 * n * n * self.head.cin * self.head.cout

    def state(self):
        return {"ch": self.ch, "scale": self.scale,
                "w": [l.w.cpu() for l in self.layers()], "b": [l.b.cpu() for l in self.layers()]}

    def load(self, st):
        for l, w, b in zip(self.layers(), st["w"], st["b"]):
            l.w.copy_(w.cuda())
            l.b.copy_(b.cuda())
            l.wb.copy_(l.w.bfloat16())
        self.scale = st["scale"]


# ---------------------------------------------------------------------------
# data: trajectories of the FD solver
# ---------------------------------------------------------------------------
def fd_model(n, batch, dt, dtype="f32"):
    m = model_MB_t(2, SolverFT(Stencil2d2h(5, 6, 13), form="fused"), ProblemParameters((n, n)),
                   dtype=dtype, batch=batch)
    m.set_stream(torch.cuda.current_stream().cuda_stream)
    m.step(dt, 0)  # sets dt
    return m


def seed_fields(m, batch, seed, mean_range=0.4, noise=0.1):
    """psi_bar ~ U[-mean_range, mean_range] per instance, plus U[-noise, noise]."""
    rng = np.random.default_rng(seed)
    for i in range(batch):
        pb = float(rng.uniform(-mean_range, mean_range))
        m.fill_uniform(0, seed * 100003 + i, pb - noise, pb + noise, inst=i)


def get_batch(m, batch, n, out=None):
    """The first `batch` instances' fields as [batch, n, n] (one copy kernel
    when the model holds exactly that many instances)."""
    out = torch.empty(batch, n, n, device="cuda") if out is None else out
    if m.batch == batch and out.is_contiguous():
        m.batch_to_device(0, out.data_ptr(), batch * n * n * 4)
        return out
    for i in range(batch):
        m.field_to_device(0, out[i].data_ptr(), n * n * 4, inst=i)
    return out


def put_batch(m, psi):
    n = psi.shape[-1]
    psi = psi.contiguous()
    if psi.shape[0] == m.batch:
        m.batch_from_device(0, psi.data_ptr(), psi.numel() * 4)
        return
    for i in range(psi.shape[0]):
        m.field_from_device(0, psi[i].data_ptr(), n * n * 4, inst=i)


def trajectories(ntraj, nsnap, jump=100, n=256, dt=0.01, seed=1, warm=0):
    """[ntraj, nsnap + 1, n, n] fp32 snapshots every `jump` steps (after `warm`
    steps), from seeded inits, by the package's fused FD step."""
    m = fd_model(n, ntraj, dt)
    seed_fields(m, ntraj, seed)
    if warm:
        m.step(dt, warm)
    snaps = torch.empty(ntraj, nsnap + 1, n, n, device="cuda")
    for s in range(nsnap + 1):
        snaps[:, s] = get_batch(m, ntraj, n)
        if s < nsnap:
            m.step(dt, jump)
    torch.cuda.synchronize()
    m.close()
    return snaps


# ---------------------------------------------------------------------------
# training
# ---------------------------------------------------------------------------
def train(net, snaps, steps=2000, batch=32, lr=1e-3, seed=0, log_every=200, log=print,
          warmup=0.05, clip=1.0):
    """Fit delta = psi(t + jump) - psi(t) over all snapshot pairs (MSE on the
    scaled change): Adam with a linear warm-up over the first `warmup`
    fraction of the steps, cosine decay after it, and the gradients clipped to
    a global norm of `clip` (an occasional large batch gradient otherwise
    throws the encoder-decoder off for good)."""
    ntraj, ns1, n, _ = snaps.shape
    pairs = ntraj * (ns1 - 1)
    d = snaps[:, 1:] - snaps[:, :-1]
    net.scale = float(d.std())
    gen = torch.Generator(device="cuda").manual_seed(seed)
    layers = net.layers()
    hist = []
    t0 = time.perf_counter()
    for step in range(1, steps + 1):
        idx = torch.randint(0, pairs, (batch,), device="cuda", generator=gen)
        ti, si = idx // (ns1 - 1), idx % (ns1 - 1)
        x, y = snaps[ti, si], snaps[ti, si + 1] - snaps[ti, si]
        for l in layers:
            l.zero_grad()
        pred = net(x)
        loss = ((pred - y) ** 2).mean() / (net.scale ** 2)
        loss.backward()
        if clip:
            # on the device: no host wait per step
            sq = torch.zeros((), device="cuda")
            for l in layers:
                sq = sq + (l.gw * l.gw).sum() + (l.gb * l.gb).sum()
            f = torch.clamp(clip / (sq.sqrt() + 1e-12), max=1.0)
            for l in layers:
                l.gw.mul_(f)
                l.gb.mul_(f)
        nw = max(1, int(warmup * steps))
        lr_t = (lr * step / nw if step <= nw else
                lr * 0.5 * (1 + math.cos(math.pi * (step - nw) / max(1, steps - nw))))
        for l in layers:
            l.adam(step, lr_t)
        if step % log_every == 0 or step == steps:
            hist.append((step, float(loss.detach())))
            log("step %d loss %.4e (%.1f s)" % (step, hist[-1][1], time.perf_counter() - t0))
    return hist


# ---------------------------------------------------------------------------
# inference: jumps judged by the FD solver
# ---------------------------------------------------------------------------
class FdPool:
    """FD models of 1, 2, 3, 4, 5, 6, 8, 10, 12, 16, ... instances (about 1.25x
    apart, up to `batch`), on which the intervals of the members the judge
    rejects are redone: each member of a batch is judged on its own, and only
    the rejected ones pay for plain FD (padded to the next pool size)."""

    def __init__(self, n, batch, dt):
        self.n, self.dt, self.batch = n, dt, batch
        self.models = {}
        sizes, s = [], 1
        while s < batch:
            sizes.append(s)
            s = max(s + 1, int(s * 1.25 + 0.5))
        self.sizes = sizes + [batch]

    def get(self, count):
        size = next((s for s in self.sizes if s >= count), count)
        if size not in self.models:
            self.models[size] = fd_model(self.n, size, self.dt)
        return self.models[size], size

    def warm(self, steps):
        """Create every size, let the autotuner pick each one's kernel shape
        (a redo of a few members is launch-bound, where a temporally blocked
        shape can pay) and run `steps` steps on each (graph capture)."""
        for size in self.sizes:
            m = self.get(size)[0]
            m.autotune(3)
            m.step(self.dt, steps)

    def close(self):
        for m in self.models.values():
            m.close()
        self.models = {}


@torch.no_grad()
def rollout(net, psi0, jumps, jump=100, judge_steps=4, dt=0.01, threshold=3.0, m=None,
            pool=None, stats=None):
    """Advance psi0 [B, n, n] by `jumps` intervals of jump + judge_steps FD
    steps each.  Per interval: one network jump, then judge_steps FD steps
    from the jumped field.  How far those FD steps move a member's field is
    its rate of relaxation; under model B it only slows down as domains
    coarsen, so a jump whose rate exceeds `threshold` times the member's rate
    before the jump (or is not finite) left the solution manifold, and that
    member's interval is redone by plain FD (on a pool model of the rejected
    members only).  Returns the final field and the number of intervals in
    which some member fell back; `stats` (a dict), if given, receives the
    number of member-intervals that fell back."""
    b, n, _ = psi0.shape
    own = m is None
    if own:
        m = fd_model(n, b, dt)
    own_pool = pool is None
    if own_pool:
        pool = FdPool(n, b, dt)

    def norm(x):
        return x.flatten(1).norm(dim=1)

    psi = psi0.clone()
    put_batch(m, psi)
    m.step(dt, judge_steps)
    rate = norm(get_batch(m, b, n) - psi)
    fallbacks, members, sizes = 0, 0, []
    timed = stats is not None
    ev = []

    def mark():
        if timed:
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            ev.append(e)

    for _ in range(jumps):
        mark()
        js = psi + net(psi)
        mark()
        put_batch(m, js)
        m.step(dt, judge_steps)
        judged = get_batch(m, b, n)
        moved = norm(judged - js)
        bad = ~torch.isfinite(moved) | (moved > threshold * rate)
        idx = bad.nonzero().flatten()
        mark()
        if idx.numel():
            fallbacks += 1
            members += idx.numel()
            sizes.append(int(idx.numel()))
            fm, size = pool.get(idx.numel())
            sub = torch.zeros(size, n, n, device="cuda")
            sub[: idx.numel()] = psi[idx]
            put_batch(fm, sub)
            fm.step(dt, jump)
            start = get_batch(fm, idx.numel(), n)
            fm.step(dt, judge_steps)
            redone = get_batch(fm, idx.numel(), n)
            judged[idx] = redone
            moved[idx] = norm(redone - start)
        mark()
        psi, rate = judged, moved
    if own:
        m.close()
    if own_pool:
        pool.close()
    if timed:
        torch.cuda.synchronize()
        t = [[ev[4 * j + k].elapsed_time(ev[4 * j + k + 1]) for k in range(3)] for j in range(jumps)]
        stats["member_fallbacks"] = members
        stats["fallback_members_per_interval"] = sizes
        stats["ms_network"] = sum(x[0] for x in t)
        stats["ms_judge"] = sum(x[1] for x in t)
        stats["ms_fallback_fd"] = sum(x[2] for x in t)
    return psi, fallbacks


def fd_run(psi0, steps, dt=0.01, m=None):
    b, n, _ = psi0.shape
    own = m is None
    if own:
        m = fd_model(n, b, dt)
    put_batch(m, psi0)
    m.step(dt, steps)
    out = get_batch(m, b, n)
    if own:
        m.close()
    return out


def rel_l2(a, b):
    return ((a - b).flatten(1).norm(dim=1) / b.flatten(1).norm(dim=1)).cpu().numpy()


def evaluate(net, batch=64, jumps=10, jump=100, judge_steps=4, dt=0.01, seed=777, warm=0,
             n=256, threshold=3.0):
    """Time to t_end (jumps x (jump + judge_steps) steps) of the judged
    surrogate and of plain FD on the same GPU, both on the same fresh
    seeded batch, with the relative L2 error of the surrogate at t_end."""
    m = fd_model(n, batch, dt)
    seed_fields(m, batch, seed)
    # plain FD on its fastest kernel shape for this batch (as the pool's)
    m.autotune(3)
    if warm:
        m.step(dt, warm)
    psi0 = get_batch(m, batch, n)
    steps = jumps * (jump + judge_steps)
    # warm both paths once (kernel selection, allocator, the fallback pool's
    # models and their graphs: set up once per run, not per interval)
    pool = FdPool(n, batch, dt)
    pool.warm(64)
    rollout(net, psi0, 1, jump, judge_steps, dt, threshold, m, pool)
    fd_run(psi0, jump, dt, m)
    stats = {}
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    ref = fd_run(psi0, steps, dt, m)
    ev[1].record()
    ev[2].record()
    sur, fb = rollout(net, psi0, jumps, jump, judge_steps, dt, threshold, m, pool, stats)
    ev[3].record()
    torch.cuda.synchronize()
    m.close()
    pool.close()
    t_fd, t_sur = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3])
    # the network alone: one jump of the batch, and its tensor-core throughput
    with torch.no_grad():
        net(psi0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            net(psi0)
        e1.record()
        torch.cuda.synchronize()
    t_net = e0.elapsed_time(e1) / 5
    flops = batch * net.flops(n)
    err = rel_l2(sur, ref)
    mass = float((sur.mean((1, 2)) - ref.mean((1, 2))).abs().max())
    return {"batch": batch, "t_end_steps": steps, "fd_ms": t_fd, "surrogate_ms": t_sur,
            "speedup": t_fd / t_sur, "rel_l2_mean": float(err.mean()),
            "rel_l2_max": float(err.max()), "fallback_intervals": fb, "intervals": jumps,
            "member_fallbacks": stats["member_fallbacks"],
            "fallback_members_per_interval": stats["fallback_members_per_interval"],
            "ms_network": stats["ms_network"], "ms_judge": stats["ms_judge"],
            "ms_fallback_fd": stats["ms_fallback_fd"],
            "max_mass_difference": mass, "net_ms_per_jump": t_net,
            "net_tflops": flops / (t_net * 1e-3) / 1e12,
            "fd_ms_per_jump": t_fd / jumps * jump / (jump + judge_steps)}


def time_conv(n, side, cin, cout, reps=5, inference=False):
    """Time one forward convolution layer of the network's kind (3x3
    circular, bias, GELU epilogue writing the pre-activation and the
    activation, or only the activation with `inference`) on random BF16 data:
    `reps` launches after two warm-up launches, CUDA events on the current
    stream."""
    g = torch.Generator().manual_seed(0)
    gd = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn(n, side, side, cin, device="cuda", generator=gd).to(torch.bfloat16)
    layer = ConvLayer(cin, cout, g)
    a = torch.empty(n, side, side, cout, device="cuda", dtype=torch.bfloat16)
    z = None if inference else torch.empty_like(a)
    scratch = layer.wt
    for _ in range(2):
        _fwd(x, layer.wb, layer.b, None, z, a, cin, cout, scratch)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        _fwd(x, layer.wb, layer.b, None, z, a, cin, cout, scratch)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    flops = 2.0 * n * side * side * cout * 9 * cin
    return {"kernel": KERNEL if _strip_ok(cin, cout, side) else "fallback", "n": n, "side": side,
            "cin": cin, "cout": cout, "ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}


@torch.no_grad()
def time_net(batch, n=256, channels=(32, 64, 128, 256), reps=5):
    """Time one forward pass (a jump) of the network on a batch of random
    fields: `reps` passes after two warm-up passes, CUDA events."""
    net = JumpNet(tuple(channels))
    g = torch.Generator(device="cuda").manual_seed(0)
    psi = 0.1 * torch.randn(batch, n, n, device="cuda", generator=g)
    for _ in range(2):
        net(psi)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net(psi)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    return {"batch": batch, "n": n, "ms": ms,
            "tflops": batch * net.flops(n) / (ms * 1e-3) / 1e12}


def main(argv=None):
    import argparse
    import json

    ap = argparse.ArgumentParser(description="train and evaluate the judged k-step jump")
    ap.add_argument("--time-conv", type=int, nargs=4, metavar=("N", "SIDE", "CIN", "COUT"),
                    help="only time one forward convolution layer of this shape and exit")
    ap.add_argument("--time-net", type=int, default=0, metavar="BATCH",
                    help="only time one forward pass of the network on this batch and exit")
    ap.add_argument("--inference", action="store_true",
                    help="--time-conv: write only the activation (the network's inference form)")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--ntraj", type=int, default=128, help="training trajectories")
    ap.add_argument("--nsnap", type=int, default=60, help="jumps per trajectory")
    ap.add_argument("--jump", type=int, default=100, help="FD steps per jump")
    ap.add_argument("--dt", type=float, default=0.01)
    ap.add_argument("--warm", type=int, default=0,
                    help="FD steps before the first snapshot (training and evaluation)")
    ap.add_argument("--steps", type=int, default=2000, help="optimiser steps")
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--channels", type=int, nargs="*", default=[32, 64, 128, 256])
    ap.add_argument("--eval-batch", type=int, default=64)
    ap.add_argument("--eval-jumps", type=int, default=20)
    ap.add_argument("--judge-steps", type=int, default=4)
    ap.add_argument("--threshold", type=float, default=3.0)
    ap.add_argument("--save", default="", help="write the trained weights here (torch.save)")
    ap.add_argument("--load", default="", help="skip training, load weights")
    ap.add_argument("--init", default="", help="train starting from these weights")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    if a.time_conv:
        print(json.dumps(time_conv(*a.time_conv, inference=a.inference)))
        return
    if a.time_net:
        print(json.dumps(time_net(a.time_net, a.n, tuple(a.channels))))
        return
    net = JumpNet(tuple(a.channels))
    report = {"params": net.nparams(), "channels": list(a.channels), "n": a.n, "jump": a.jump,
              "dt": a.dt, "warm": a.warm, "flops_per_sample": net.flops(a.n)}
    if a.load:
        net.load(torch.load(a.load))
    else:
        if a.init:
            net.load(torch.load(a.init))
        t0 = time.perf_counter()
        snaps = trajectories(a.ntraj, a.nsnap, a.jump, a.n, a.dt, seed=1, warm=a.warm)
        report["data_s"] = time.perf_counter() - t0
        report["pairs"] = a.ntraj * a.nsnap
        t0 = time.perf_counter()
        hist = train(net, snaps, a.steps, a.batch, a.lr)
        torch.cuda.synchronize()
        report["train_s"] = time.perf_counter() - t0
        report["loss"] = hist
        del snaps
        if a.save:
            torch.save(net.state(), a.save)
    report["eval"] = evaluate(net, a.eval_batch, a.eval_jumps, a.jump, a.judge_steps, a.dt,
                              warm=a.warm, n=a.n, threshold=a.threshold)
    print(json.dumps(report))


if __name__ == "__main__":
    main()
