"""Headline benchmark: one fused forward-Euler step of Cahn-Hilliard (model B)
on a 256^3 periodic grid, dx = 1, dt = 0.005, Stencil3d2h<7,10,25>, FP32
(the bulk path), seeded uniform noise +-0.1 around psi_bar = -0.2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A timed step is one fused-step launch; a 256 MiB buffer is written before
every timed step so the L2 (126 MB) holds none of the field, and each step is
timed with CUDA events on the solver's stream.  With N > 1 (torchrun), every
rank advances its own replica (the path runs on one GPU; replicas only) and
the job time is the maximum over ranks.  Prints one JSON line (rank 0).

--impl reference times the CPU implementation of the same path (the C
restatement of SymPhas's SolverFT in oracle/, FP64 as SymPhas computes, all
host threads) on the same grid: one step per timed step.
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
N_GRID = 256
DT = 0.005
WORKLOAD = ("Cahn-Hilliard (model B) 3D 256^3 periodic, dx 1, dt 0.005, "
            "Stencil3d2h<7,10,25>, fused step, psi_bar -0.2 +- 0.1 seeded noise")
ALG_BYTES_PER_SITE = 8  # one FP32 read and one FP32 write of the field per step
CLOCK_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "k_fd3d_modelB_256cube_f32.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
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
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

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


def cpu_port_rate(seconds, threads):
    """Site-updates/s of the CPU restatement (oracle) on the same grid, FP64."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import spo

    n = N_GRID
    d = spo.make_desc(3, (n, n, n), spo.MODEL_B, 1.0, DT)
    x = spo.seed_uniform(20261203, -0.3, -0.1, n ** 3).reshape(n, n, n)
    sysm = spo.System(d, x, threads)
    sysm.step(1)  # warm-up
    steps, t0 = 0, time.perf_counter()
    while True:
        sysm.step(1)
        steps += 1
        el = time.perf_counter() - t0
        if el >= seconds and steps >= 2:
            break
    sysm.close()
    return steps * float(n ** 3) / el, steps, el, np


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import spo

    threads = os.cpu_count() or 1
    n = N_GRID
    d = spo.make_desc(3, (n, n, n), spo.MODEL_B, 1.0, DT)
    x = spo.seed_uniform(20261203, -0.3, -0.1, n ** 3).reshape(n, n, n)
    sysm = spo.System(d, x, threads)
    for _ in range(args.warmup):
        sysm.step(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sysm.step(1)
    el = time.perf_counter() - t0
    sysm.close()
    value = args.steps * float(n ** 3) / el
    sample = "%d SolverFT steps of model B 256^3 FP64 (C restatement, %d threads)" % (
        args.steps, threads)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD.replace("fused step", "SolverFT step"), "grid": n},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


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

    n = N_GRID
    sites = float(n) ** 3
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    model = sp.model_MB_t(3, sp.SolverFT(sp.Stencil3d2h(7, 10, 25), form="fused"),
                          sp.ProblemParameters((n, n, n), h=1.0), dtype="f32")
    model.set_stream(stream.cuda_stream)
    model.fill_uniform(0, 20261203 + rank, -0.3, -0.1)
    tile = model.autotune(20)  # pick the fastest tile shape (setup, not timed)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB

    for _ in range(max(args.warmup, 3)):
        flush.zero_()
        model.step(DT, 1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    gpu_index = os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[local]
    clocks = Clocks(gpu_index)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    launches0 = model.launch_count()
    torch.cuda.synchronize()
    for e0, e1 in ev:
        flush.zero_()
        e0.record(stream)
        model.step(DT, 1)
        e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    launches = model.launch_count() - launches0
    per = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(per)
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    job_ms = float(t.item())
    value = world * args.steps * sites / (job_ms * 1e-3)
    launch_ms = total_ms / args.steps

    # end to end: pinned host field -> upload -> e2e_inner steps -> download
    nbytes = int(sites) * 4
    host_in = torch.empty(int(sites), dtype=torch.float32, pin_memory=True)
    host_out = torch.empty(int(sites), dtype=torch.float32, pin_memory=True)
    model.download_to(0, host_in.data_ptr(), nbytes)
    e2e_calls = max(3, args.steps // 40)
    for _ in range(2):
        model.upload_from(0, host_in.data_ptr(), nbytes)
        model.step(DT, args.e2e_inner)
        model.download_to(0, host_out.data_ptr(), nbytes)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(e2e_calls):
        model.upload_from(0, host_in.data_ptr(), nbytes)
        model.step(DT, args.e2e_inner)
        model.download_to(0, host_out.data_ptr(), nbytes)
    e_end.record(stream)
    torch.cuda.synchronize()
    t = torch.tensor([e_start.elapsed_time(e_end)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t.item()) / e2e_calls
    e2e_value = world * args.e2e_inner * sites / (e2e_ms * 1e-3)
    model.close()

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    peak, peak_kind = measured_peak()
    achieved = sites * ALG_BYTES_PER_SITE / (launch_ms * 1e-3) / 1e9
    traffic = None
    try:
        traffic = json.load(open(PROFILE_TRAFFIC))["dram_bytes_per_launch"]
    except Exception:
        pass
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": job_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": [n, n, n], "global_batch": world,
                   "l2": "256 MiB buffer written before every timed step (L2 flushed)",
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "kernel_shape": tile},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind, "kernel": "k_fd3d (fused model B step)",
                     "alg_bytes_per_launch": sites * ALG_BYTES_PER_SITE},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes,
                "step": "upload field from pinned host, %d fused steps, download field" %
                        args.e2e_inner},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if world == 1:
        threads = os.cpu_count() or 1
        rate, steps, el, _ = cpu_port_rate(10.0, threads)
        line["cpu_baseline"] = {
            "value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "%d SolverFT steps of model B 256^3 FP64 (C restatement), %.1f s" % (
                steps, el)}
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
