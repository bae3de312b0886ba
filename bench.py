"""Throughput of the fused forward-Euler finite-difference step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload b3d|ensemble|c3d|regional]

Workloads (synthetic seeded fields; site-updates/s counts interior sites
advanced by one step, summed over instances):

  b3d       (default, the headline) Cahn-Hilliard (model B) on a 256^3
            periodic grid, dx 1, dt 0.005, Stencil3d2h<7,10,25>, FP32 fused
            step, psi_bar -0.2 +- 0.1.  A 256 MiB buffer is written before
            every timed step so the L2 (126 MB) holds none of the field; each
            step is timed with CUDA events on the solver's stream.
  ensemble  1024 independent 2D members, sides drawn from {64, 96, 128, 256,
            384, 512, 768, 1024}, first half model A (AMK: M, kappa), second
            half model B (BMK), M and kappa from U[0.5, 2], dt = 40% of each
            member's stability limit, +-0.1 noise, FP32 fused, periodic; one
            persistent launch per step, steps replayed from CUDA graphs.  The
            fields (~2.2 GB per buffer) exceed the L2, the K steps are timed
            as one region.
  c3d       model C (psi conserved, eta not, gamma 0.5), 8 instances of 256^3
            periodic, dx 1, dt 0.005, FP32 fused, psi_bar 0.1 +- 0.1 and eta
            +-0.1; one launch advances all 8 (2.1 GB per buffer, beyond L2).
  surrogate the metric's second half: time to t_end of the judged learned jump
            against plain FD on the same GPU.  2D model B 256^2 periodic, dx 1,
            dt 0.01, Stencil2d2h<5,6,13>, psi_bar U[-0.4,0.4] +- 0.1, 2000 FD
            steps of warm-up; a batch of 256 fields (the configuration's
            inference batch) advanced to t_end = 3 intervals of 2000 + 4 steps,
            by FP32 fused FD alone and by the network (jumps of 2000 steps,
            --surrogate-jump; tcgen05 convolutions; each member's jump judged
            by 4 FD steps, the members judged off the solution manifold
            redone by FD).  The network is trained first (256 FD
            trajectories, 10 snapshots each, Adam) unless --surrogate-load
            names saved weights.  value = effective
            site-updates/s of the surrogate path (t_end steps x sites / its
            time); the FD rate, the ratio and the relative L2 error at t_end
            are in the line.
  regional  model B 2D on a regional system (SymPhas's SolverSystemFDwSD):
            one droplet of radius 200 in a 4096^2 periodic domain, FP32 fused,
            dt 0.01; the window (about 1/15 of the domain) is re-centred every
            3.0 of time.  Rates count the window's interior sites; the L2 is
            flushed before every timed step; transfers of the end-to-end
            number are whole-domain fields.

With N > 1 (torchrun), every rank advances its own replica (the path runs on
one GPU; replicas only) and the job time is the maximum over ranks.  Prints
one JSON line (rank 0).

--impl reference times SymPhas's own CPU SolverFT (built from SymPhas's sources
into oracle/_ref/ by oracle/ref.mk; FP64, SymPhas's only scalar type) on the
same workload: one model per host thread, as SymPhas runs a model on one core
(b3d: the one 256^3 model; c3d: the 8 instances; ensemble: every 8th member
over all host threads).  SymPhas has no solver for the regional workload's
window search here, so --workload regional times the oracle's C restatement
(kind "port").  Without the built library every workload falls back to the
restatement.

--dtype f64 (b3d only) times the FP64 step in SymPhas's exact term order
(bit-identical to SymPhas's own solver), 16 algorithmic bytes per site.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "site-updates/s + %HBM roofline; time-to-t_end surrogate vs plain FD at ≤1% L2"
UNIT = "site-updates/s"
CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="b3d",
                    choices=["b3d", "ensemble", "c3d", "regional", "surrogate"])
    ap.add_argument("--surrogate-load", default="",
                    help="surrogate: weights of a trained jump network (else it is trained first)")
    ap.add_argument("--surrogate-train-steps", type=int, default=6000)
    ap.add_argument("--surrogate-save", default="",
                    help="surrogate: write the trained weights here (torch.save)")
    ap.add_argument("--surrogate-init", default="",
                    help="surrogate: start training from these weights")
    ap.add_argument("--surrogate-lr", type=float, default=1e-3)
    ap.add_argument("--surrogate-jump", type=int, default=2000,
                    help="surrogate: FD steps per learned jump (t_end stays about 6000 steps)")
    ap.add_argument("--surrogate-trajectories", type=int, default=256)
    ap.add_argument("--surrogate-snapshots", type=int, default=10,
                    help="surrogate: training snapshots per trajectory, one jump apart")
    ap.add_argument("--dtype", default="f32", choices=["f32", "f64"],
                    help="b3d only: FP32 fused step (default) or the FP64 exact step")
    ap.add_argument("--e2e-inner", type=int, default=100,
                    help="FD steps per end-to-end call (upload, steps, download)")
    return ap.parse_args()


class Clocks:
    """nvidia-smi samples of the GPU's clocks while the timed region runs."""

    def __init__(self, gpu):
        self.gpu = gpu
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--query-gpu=" + CLOCK_QUERY, "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.gpu)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # wait for the sampler's first line so even a short timed region is seen
        t0 = time.time()
        while time.time() - t0 < 5.0:
            try:
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.05)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        sm, mx, reasons, power = [], [], set(), []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for name, val in zip(names[1:], f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "power_w_max": max(power) if power else None, "reasons": sorted(reasons)}


def measured_peak():
    try:
        v = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        return float(v), "measured"
    except Exception:
        return 6650.0, "fallback"


def tune(model, reps):
    """The fastest tile shape (setup, not timed), unless SP_TILE names one: a
    profiler run of this script then gets the kernel a plain run chose."""
    if os.environ.get("SP_TILE"):
        return model.kernel_info()
    return model.autotune(reps)


def oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import spo

    return spo


def symphas():
    """SymPhas's own CPU solver (oracle/_ref), or None where it is not built."""
    oracle()
    import symref

    return symref if symref.loaded() is not None else None


class B3D:
    """Model B 3D 256^3 FP32 (the headline)."""

    name = "b3d"
    n = 256
    dt = 0.005
    dtype = "f32"
    form = "fused"
    bytes_per_site = 8  # one FP32 read and one FP32 write of the field per step
    flush_each_step = True
    kernel = "fused model B step (k_chrow / k_fd3d / k_ch3d, the autotuned tile variant)"
    traffic_file = os.path.join(ROOT, "profiles", "k_chrow_modelB_256cube_f32.json")
    workload = ("Cahn-Hilliard (model B) 3D 256^3 periodic, dx 1, dt 0.005, "
                "Stencil3d2h<7,10,25>, psi_bar -0.2 +- 0.1 seeded noise")

    def __init__(self, sp, rank, stream):
        n = self.n
        self.sites = float(n) ** 3
        self.model = sp.model_MB_t(3, sp.SolverFT(sp.Stencil3d2h(7, 10, 25), form=self.form),
                                   sp.ProblemParameters((n, n, n), h=1.0), dtype=self.dtype)
        self.model.set_stream(stream.cuda_stream)
        self.model.fill_uniform(0, 20261203 + rank, -0.3, -0.1)
        self.shape = tune(self.model, 20)
        self.fields = [(0, 0, int(self.sites))]  # (instance, field, sites)

    def step(self, k):
        self.model.step(self.dt, k)

    def config(self):
        return {"grid": [self.n] * 3, "form": self.form, "kernel_shape": self.shape}

    @classmethod
    def initial(cls):
        spo = oracle()
        n = cls.n
        return spo.seed_uniform(20261203, -0.3, -0.1, n ** 3).reshape(n, n, n)

    @classmethod
    def desc(cls):
        spo = oracle()
        n = cls.n
        return spo.make_desc(3, (n, n, n), spo.MODEL_B, 1.0, cls.dt)

    @classmethod
    def cpu_system(cls, threads):
        spo = oracle()
        sysm = spo.System(cls.desc(), cls.initial(), threads)
        return (lambda: sysm.step(1)), float(cls.n) ** 3, sysm.close, (
            "SolverFT steps of model B 256^3 FP64 (C restatement, %d threads)" % threads)

    @classmethod
    def ref_system(cls, ref, threads):
        """SymPhas's own solver on the same field: one model, one core."""
        sysm = ref.System(cls.desc(), cls.initial())
        return (lambda: sysm.step(1)), float(cls.n) ** 3, sysm.close, 1, (
            "SymPhas SolverFT steps of model B 256^3 FP64 (one model: SymPhas runs it on "
            "one core)")


class B3D64(B3D):
    """The same model B 256^3 step in FP64, SymPhas's exact term order."""

    dtype = "f64"
    form = "exact"
    bytes_per_site = 16  # one FP64 read and one FP64 write of the field per step
    kernel = "exact-form FP64 model B step (k_fd3d, the autotuned tile variant)"
    traffic_file = os.path.join(ROOT, "profiles", "k_fd3d_modelB_256cube_f64.json")


class C3D(B3D):
    """Model C, 8 instances of 256^3, FP32."""

    name = "c3d"
    batch = 8
    bytes_per_site = 16  # two fields, each read and written once per step
    flush_each_step = False
    kernel = "fused model C step (k_row / k_fd3d, two fields, the autotuned tile variant)"
    traffic_file = os.path.join(ROOT, "profiles", "k_row_modelC_8x256cube_f32.json")
    workload = ("model C (gamma 0.5) 3D, 8 instances of 256^3 periodic, dx 1, dt 0.005, "
                "Stencil3d2h<7,10,25>, psi 0.1 +- 0.1, eta +- 0.1 seeded noise")

    def __init__(self, sp, rank, stream):
        n = self.n
        self.sites = float(n) ** 3 * self.batch
        self.model = sp.model_MC_t(3, sp.SolverFT(sp.Stencil3d2h(7, 10, 25), form="fused"),
                                   sp.ProblemParameters((n, n, n), h=1.0), coeff=(0.5,),
                                   dtype="f32", batch=self.batch)
        self.model.set_stream(stream.cuda_stream)
        for i in range(self.batch):
            self.model.fill_uniform(0, 7000 + 64 * rank + 2 * i, 0.0, 0.2, inst=i)
            self.model.fill_uniform(1, 7001 + 64 * rank + 2 * i, -0.1, 0.1, inst=i)
        self.shape = tune(self.model, 5)
        self.fields = [(i, f, n ** 3) for i in range(self.batch) for f in range(2)]

    def config(self):
        return {"grid": [self.n] * 3, "instances": self.batch, "form": self.form,
                "kernel_shape": self.shape}

    @classmethod
    def instance(cls, i):
        spo = oracle()
        import numpy as np

        n = cls.n
        d = spo.make_desc(3, (n, n, n), spo.MODEL_C, 1.0, cls.dt, coeff=(0.5,))
        x = np.stack([spo.seed_uniform(7000 + 2 * i, 0.0, 0.2, n ** 3),
                      spo.seed_uniform(7001 + 2 * i, -0.1, 0.1, n ** 3)]).reshape(2, n, n, n)
        return d, x

    @classmethod
    def cpu_system(cls, threads):
        spo = oracle()
        d, x = cls.instance(0)
        sysm = spo.System(d, x, threads)
        return (lambda: sysm.step(1)), float(cls.n) ** 3, sysm.close, (
            "SolverFT steps of one model C 256^3 instance FP64 (C restatement, %d threads)"
            % threads)

    @classmethod
    def ref_system(cls, ref, threads):
        """SymPhas's own solver on the 8 instances, one model per core."""
        systems = [ref.System(*cls.instance(i)) for i in range(cls.batch)]
        used = min(threads, cls.batch)

        def close():
            for s in systems:
                s.close()

        return (lambda: ref.step_many(systems, 1, used)), float(cls.n) ** 3 * cls.batch, close, \
            used, ("SymPhas SolverFT steps of the 8 model C 256^3 instances FP64 (%d threads, "
                   "one model per thread)" % used)


class Ens:
    """1024 2D members of uneven sizes, models AMK / BMK, FP32."""

    name = "ensemble"
    count = 1024
    seed = 20261203
    dtype = "f32"
    bytes_per_site = 8
    flush_each_step = False
    kernel = "k_fd2d (persistent tile queue over every member, AMK and BMK right-hand sides)"
    traffic_file = os.path.join(ROOT, "profiles", "k_fd2d_ensemble1024_f32.json")
    workload = ("ensemble of 1024 2D periodic members, sides from {64,96,128,256,384,512,768,"
                "1024}, half model A (AMK) half model B (BMK), M and kappa U[0.5,2], dt 40% of "
                "each stability limit, Stencil2d2h<5,6,13>, +-0.1 seeded noise")

    def __init__(self, sp, rank, stream):
        self.members = sp.ensemble_members(self.count, seed=self.seed)
        self.model = sp.Ensemble(sp.SolverFT(sp.Stencil2d2h(5, 6, 13), form="fused"),
                                 self.members, dtype="f32")
        self.model.set_stream(stream.cuda_stream)
        for i in range(self.count):
            self.model.fill_uniform(0, self.seed + 4096 * rank + i, -0.1, 0.1, inst=i)
        self.sites = float(self.model.sites())
        self.shape = tune(self.model, 5)
        self.fields = [(i, 0, int(m["dims"][0] * m["dims"][1]))
                       for i, m in enumerate(self.members)]

    def step(self, k):
        self.model.step(k)

    def config(self):
        sides = sorted({m["dims"][0] for m in self.members})
        return {"members": self.count, "sides": sides, "sites": int(self.sites),
                "form": "fused", "kernel_shape": self.shape}

    @classmethod
    def sample(cls):
        """Every 8th member (128 of them, both models, all sizes)."""
        spo = oracle()

        import symphas_b200.model as spm  # the member generator only (host code)

        members = spm.ensemble_members(cls.count, seed=cls.seed)[::8]
        ids = {"AMK": spo.MODEL_AMK, "BMK": spo.MODEL_BMK}
        descs = [spo.make_desc(2, m["dims"], ids[m["model"]], 1.0, m["dt"], coeff=m["coeff"])
                 for m in members]
        fields = [spo.seed_uniform(cls.seed + 8 * i, -0.1, 0.1, m["dims"][0] * m["dims"][1])
                  .reshape(m["dims"][1], m["dims"][0]) for i, m in enumerate(members)]
        sites = float(sum(m["dims"][0] * m["dims"][1] for m in members))
        return descs, fields, sites

    @classmethod
    def ref_system(cls, ref, threads):
        """SymPhas's own solver on the sample, one model per thread."""
        descs, fields, sites = cls.sample()
        systems = [ref.System(d, f) for d, f in zip(descs, fields)]

        def close():
            for s in systems:
                s.close()

        return (lambda: ref.step_many(systems, 1, threads)), sites, close, threads, (
            "one SymPhas SolverFT step of 128 of the 1024 members (every 8th) FP64 "
            "(%d threads over members)" % threads)

    @classmethod
    def cpu_system(cls, threads):
        """The sample, all threads over members (one member per thread, as
        independent SymPhas models)."""
        spo = oracle()
        descs, fields, sites = cls.sample()
        fields = [f.reshape(-1).copy() for f in fields]

        def one():
            spo.run_batch(descs, fields, [1] * len(descs), threads)

        return one, sites, (lambda: None), (
            "one SolverFT step of 128 of the 1024 members (every 8th) FP64 "
            "(C restatement, %d threads over members)" % threads)


def droplet(n, radius, seed):
    """FP64 field of a 2D n x n periodic domain: +1 (+-1e-3 seeded noise) inside
    a disc of `radius` at the centre, -1 outside."""
    import numpy as np

    y, x = np.mgrid[0:n, 0:n]
    inside = (x - n // 2) ** 2 + (y - n // 2) ** 2 < radius * radius
    noise = np.random.default_rng(seed).uniform(-1e-3, 1e-3, (n, n))
    return np.where(inside, 1.0 + noise, -1.0)


class Reg2D:
    """Model B 2D on a regional system: one droplet in a 4096^2 domain, FP32."""

    name = "regional"
    n = 4096
    radius = 200
    dt = 0.01
    seed = 20261203
    dtype = "f32"
    bytes_per_site = 8
    flush_each_step = True
    kernel = "k_fd2d over the window's interior (the fused model B step of the window's handle)"
    traffic_file = os.path.join(ROOT, "profiles", "k_fd2d_regional_window_f32.json")
    workload = ("Cahn-Hilliard (model B) 2D regional system (SolverSystemFDwSD): one droplet of "
                "radius 200 (+1 in -1) in a 4096^2 periodic domain, dx 1, dt 0.01, "
                "Stencil2d2h<5,6,13>; window re-centred every 3.0 of time, padding "
                "factor 2, cutoff min + 1e-6; site-updates counted over the window's interior")

    def __init__(self, sp, rank, stream):
        n = self.n
        self.model = sp.RegionalModel(sp.model_MB_t, 2, sp.SolverFT(sp.Stencil2d2h(5, 6, 13),
                                                                     form="fused"),
                                      sp.ProblemParameters((n, n), h=1.0), dtype="f32",
                                      dt=self.dt, resize_delta=3.0, padding_factor=2.0,
                                      cutoff_eps=1e-6, fixed=True)
        self.model.set_stream(stream.cuda_stream)
        self.model.set_field(droplet(n, self.radius, self.seed + rank))
        self.model.step(1)  # the first window check shrinks the window
        self.shape = tune(self.model, 20)
        self.sites = float(self.model.interior_sites())
        # the window the timed steps run on (no re-centre falls due before 3.0 of time)
        self.window = self.model.window()
        self.fields = [(0, 0, n * n)]  # whole-domain transfers through the public API

    def step(self, k):
        self.model.step(k)

    def config(self):
        o, d = self.window
        return {"domain": [self.n] * 2, "window_origin": list(o), "window_dims": list(d),
                "window_interior_sites": int(self.sites),
                "domain_sites_per_window_site": self.n * self.n / self.sites,
                "kernel_shape": self.shape}

    @classmethod
    def cpu_system(cls, threads):
        spo = oracle()
        n = cls.n
        d = spo.make_desc(2, (n, n), spo.MODEL_B, 1.0, cls.dt)
        r = spo.Regional(d, droplet(n, cls.radius, cls.seed), resize_delta=3.0, factor=2.0,
                         eps=1e-6, fixed=True, threads=threads)
        r.step(1)
        o, dims = r.window()[:2]
        sites = float((dims[0] - 6) * (dims[1] - 6))
        return (lambda: r.step(1)), sites, r.close, (
            "SolverFT steps of the regional model B window (%d x %d interior) FP64 "
            "(C restatement, %d threads)" % (dims[0] - 6, dims[1] - 6, threads))


WORKLOADS = {"b3d": B3D, "c3d": C3D, "ensemble": Ens, "regional": Reg2D}


def workload(args):
    if args.dtype == "f64":
        if args.workload != "b3d":
            raise SystemExit("--dtype f64 is built for --workload b3d only")
        return B3D64
    return WORKLOADS[args.workload]


def max_over_ranks(ms, dist, device="cuda"):
    """The job's time: the slowest rank's (every rank gets it).  `dist` is
    torch.distributed when the job has more than one rank, else None."""
    if not dist:
        return float(ms)
    import torch

    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, steps, sites, ms):
    """Site-updates per second of the whole job: every rank advances its own
    replica of `sites` sites by `steps` steps in `ms` milliseconds."""
    return world * steps * sites / (ms * 1e-3)


def cpu_rate(W, seconds, threads):
    """Site-updates/s of the CPU restatement (oracle) on the workload, FP64."""
    step, sites, close, what = W.cpu_system(threads)
    step()  # warm-up
    steps, t0 = 0, time.perf_counter()
    while True:
        step()
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds and steps >= 2:
            break
    close()
    return steps * sites / el, "%d %s, %.1f s" % (steps, what, el)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    W = workload(args)
    threads = os.cpu_count() or 1
    ref = symphas() if hasattr(W, "ref_system") else None
    if ref is not None:
        step, sites, close, cores, what = W.ref_system(ref, threads)
        kind = "reference"
    else:
        step, sites, close, what = W.cpu_system(threads)
        cores, kind = threads, "port"
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t0
    close()
    value = args.steps * sites / el
    sample = "%d %s" % (args.steps, what)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": W.workload},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def run_surrogate(args):
    """The surrogate workload (see the module docstring): one JSON line."""
    import torch

    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    from symphas_b200 import surrogate as S

    n, warm, batch, judge = 256, 2000, 256, 4
    jump = args.surrogate_jump
    intervals = max(2, 6000 // jump)
    ntraj, nsnap = args.surrogate_trajectories, args.surrogate_snapshots
    net = S.JumpNet((32, 64, 128, 256))
    trained = {}
    if args.surrogate_load:
        net.load(torch.load(args.surrogate_load))
        trained = {"weights": os.path.basename(args.surrogate_load)}
    else:
        if args.surrogate_init:
            net.load(torch.load(args.surrogate_init))
        t0 = time.perf_counter()
        snaps = S.trajectories(ntraj, nsnap, jump, n, 0.01, seed=1, warm=warm)
        hist = S.train(net, snaps, args.surrogate_train_steps, 32, args.surrogate_lr,
                       log=lambda *_: None)
        torch.cuda.synchronize()
        trained = {"trajectories": ntraj, "pairs": ntraj * nsnap,
                   "adam_steps": args.surrogate_train_steps, "lr": args.surrogate_lr,
                   "init": os.path.basename(args.surrogate_init) or None,
                   "train_s": round(time.perf_counter() - t0, 1), "final_loss": hist[-1][1]}
        del snaps
        if args.surrogate_save:
            torch.save(net.state(), args.surrogate_save)
    ev = S.evaluate(net, batch=batch, jumps=intervals, jump=jump, judge_steps=judge, dt=0.01,
                    warm=warm, n=n, threshold=3.0)
    if rank != 0:
        return 0
    sites = float(batch * n * n * ev["t_end_steps"])
    value = sites / (ev["surrogate_ms"] * 1e-3)
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": intervals,
        "warmup": 1, "ms_per_step": ev["surrogate_ms"] / intervals, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16 network, f32 FD", "data": "synthetic",
        "config": {"workload": "learned jump (model B 2D 256^2, batch 256, jumps of %d steps "
                               "judged by 4 FD steps) to t_end = %d steps against plain FP32 "
                               "fused FD" % (jump, ev["t_end_steps"]),
                   "fd_site_updates_per_s": sites / (ev["fd_ms"] * 1e-3),
                   "speedup_vs_fd": ev["speedup"], "rel_l2_mean": ev["rel_l2_mean"],
                   "rel_l2_max": ev["rel_l2_max"], "fallback_intervals": ev["fallback_intervals"],
                   "member_fallbacks": ev["member_fallbacks"],
                   "fallback_members_per_interval": ev["fallback_members_per_interval"],
                   "ms_network": ev["ms_network"], "ms_judge": ev["ms_judge"],
                   "ms_fallback_fd": ev["ms_fallback_fd"],
                   "net_ms_per_jump": ev["net_ms_per_jump"], "net_tflops": ev["net_tflops"],
                   "training": trained},
        "roofline": {"bound": "tensor", "achieved": ev["net_tflops"],
                     "peak": measured_tensor_peak()[0], "unit": "TFLOP/s",
                     "frac": ev["net_tflops"] / measured_tensor_peak()[0],
                     "peak_kind": measured_tensor_peak()[1],
                     "kernel": "the jump network's convolutions (sp_conv3x3_fwd_strip)"},
    }))
    return 0


def measured_tensor_peak():
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"]), \
            "measured"
    except Exception:
        return 1590.0, "fallback"


def run_ours(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    import symphas_b200 as sp

    W = workload(args)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    w = W(sp, rank, stream)
    sites = w.sites
    warmup = max(args.warmup, 3)
    flush = None
    if W.flush_each_step:
        flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB
    for _ in range(warmup):
        if flush is not None:
            flush.zero_()
        w.step(1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    gpu_index = os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[local]
    clocks = Clocks(gpu_index)
    clocks.start()
    launches0 = w.model.launch_count()
    torch.cuda.synchronize()
    if flush is not None:
        # L2 flushed before every step; each step timed on the solver's stream
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        for e0, e1 in ev:
            flush.zero_()
            e0.record(stream)
            w.step(1)
            e1.record(stream)
        torch.cuda.synchronize()
        total_ms = sum(a.elapsed_time(b) for a, b in ev)
    else:
        # fields larger than the L2: the K steps (graph-replayed) as one region
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        w.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms = e0.elapsed_time(e1)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    launches = w.model.launch_count() - launches0
    job_ms = max_over_ranks(total_ms, dist)
    value = job_rate(world, args.steps, sites, job_ms)
    launch_ms = total_ms / args.steps

    # end to end through the public API: every field of the step's input from
    # pinned host memory, e2e_inner steps, every field back to pinned memory
    esz = 8 if W.dtype == "f64" else 4
    offs, total = [], 0
    for inst, f, cnt in w.fields:
        offs.append(total)
        total += cnt
    tdt = torch.float64 if W.dtype == "f64" else torch.float32
    host_in = torch.empty(total, dtype=tdt, pin_memory=True)
    host_out = torch.empty(total, dtype=tdt, pin_memory=True)
    nbytes = total * esz

    def download(buf):
        for (inst, f, cnt), o in zip(w.fields, offs):
            w.model.download_to(f, buf.data_ptr() + o * esz, cnt * esz, inst=inst)

    def upload(buf):
        for (inst, f, cnt), o in zip(w.fields, offs):
            w.model.upload_from(f, buf.data_ptr() + o * esz, cnt * esz, inst=inst)

    download(host_in)
    e2e_calls = 3
    for _ in range(2):
        upload(host_in)
        w.step(args.e2e_inner)
        download(host_out)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(e2e_calls):
        upload(host_in)
        w.step(args.e2e_inner)
        download(host_out)
    e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e_start.elapsed_time(e_end), dist) / e2e_calls
    e2e_value = job_rate(world, args.e2e_inner, sites, e2e_ms)
    w.model.close()

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    peak, peak_kind = measured_peak()
    alg_bytes = sites * W.bytes_per_site
    achieved = alg_bytes / (launch_ms * 1e-3) / 1e9
    traffic = None
    try:
        traffic = json.load(open(W.traffic_file))["dram_bytes_per_launch"]
    except Exception:
        pass
    cfg = {"workload": W.workload, "global_batch": world,
           "l2": ("256 MiB buffer written before every timed step (L2 flushed)"
                  if W.flush_each_step else
                  "fields larger than the 126 MB L2 (%.2f GB read per step)" % (alg_bytes / 2e9)),
           "parallelism": "replicas" if world > 1 else "single GPU"}
    cfg.update(w.config())
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": warmup, "ms_per_step": job_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": W.dtype,
        "data": "synthetic", "config": cfg,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind, "kernel": W.kernel,
                     "alg_bytes_per_launch": alg_bytes},
        # one call uploads every field, advances e2e_inner steps, downloads every
        # field: bytes per FD step are the call's bytes over its steps
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nbytes / args.e2e_inner,
                "d2h_bytes_per_step": nbytes / args.e2e_inner, "steps_per_call": args.e2e_inner,
                "h2d_bytes_per_call": nbytes, "d2h_bytes_per_call": nbytes,
                "call": "upload every field from pinned host, %d steps, download every field"
                        % args.e2e_inner},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if world == 1:
        threads = os.cpu_count() or 1
        rate, sample = cpu_rate(W, 10.0, threads)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": sample}
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0
def main():
    args = parse()
    if args.workload == "surrogate":
        if args.impl == "reference":
            if int(os.environ.get("RANK", "0")) == 0:
                print(json.dumps({"impl": "reference", "unavailable":
                                  "the learned jump has no counterpart in SymPhas"}))
            return 0
        return run_surrogate(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
