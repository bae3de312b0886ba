"""Run a built-in model for a number of fused steps on seeded noise and print
the time per step.  Used for timing and for profiling single launches:

    python -m symphas_b200.run --model B --dim 3 --n 256 --dtype f32 --steps 8
    python -m symphas_b200.run --ensemble 128 --steps 8     (2D AMK/BMK members)
    python -m symphas_b200.run --regional 200 --n 4096 --steps 8
                        (model B 2D, one droplet of that radius, regional window)

Steps are launched one launch at a time (no CUDA graph), so a profiler sees
each fused-step launch separately: one step per launch, or k for a
temporally blocked kernel (the steps are rounded up to a multiple of k).

    python -m symphas_b200.run --model A --dim 2 --n 4096 --steps 256 --every-variant
                        (one line per tile shape and temporal-block depth)
"""
import os
import argparse
import json
import time

import symphas_b200 as sp

MODELS = {"A": sp.model_MA_t, "B": sp.model_MB_t, "C": sp.model_MC_t,
          "AMK": sp.model_MAMK_t, "BMK": sp.model_MBMK_t}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--model", default="B", choices=sorted(MODELS))
    ap.add_argument("--dim", type=int, default=3, choices=[2, 3])
    ap.add_argument("--n", type=int, default=256, help="interior points per axis")
    ap.add_argument("--dtype", default="f32", choices=["f32", "f64"])
    ap.add_argument("--form", default="fused", choices=["fused", "exact"])
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--dt", type=float, default=0.005)
    ap.add_argument("--h", type=float, default=1.0)
    ap.add_argument("--coeff", type=float, nargs="*", default=[])
    ap.add_argument("--ensemble", type=int, default=0,
                    help="run an ensemble of this many 2D members (sides 64..1024, models AMK "
                         "and BMK, FP32 fused) instead of one model")
    ap.add_argument("--regional", type=int, default=0,
                    help="run model B 2D on a regional system holding one droplet of this "
                         "radius (+1 in -1) at the centre of an n x n domain; the first step "
                         "shrinks the window, the steps after it are timed")
    ap.add_argument("--autotune", action="store_true",
                    help="pick the fastest tile shape first (its launches come before the steps)")
    ap.add_argument("--variant", type=int, default=-1,
                    help="run this tile variant (index into the kernel's shapes)")
    ap.add_argument("--every-variant", action="store_true",
                    help="time every tile variant of the kernel in turn, one line each")
    a = ap.parse_args(argv)
    if a.every_variant:
        nv = 1
        v = 0
        while v < nv:
            os.environ["SP_TILE"] = str(v)
            out = run_one(a, quiet=True)
            nv = out["kernel"]["variants"]
            if out["kernel"]["variant"] == v:
                print(json.dumps(out))
            v += 1
        del os.environ["SP_TILE"]
        return
    if a.variant >= 0:
        os.environ["SP_TILE"] = str(a.variant)
    if a.ensemble or a.regional:
        return run_ensemble(a) if a.ensemble else run_regional(a)
    print(json.dumps(run_one(a)))


def run_one(a, quiet=False):
    if a.ensemble:
        return run_ensemble(a, quiet)
    st = sp.Stencil2d2h(5, 6, 13) if a.dim == 2 else sp.Stencil3d2h(7, 10, 25)
    cls = MODELS[a.model]
    coeff = a.coeff or ([0.5] if a.model == "C" else [])
    m = cls(a.dim, sp.SolverFT(st, form=a.form), sp.ProblemParameters((a.n,) * a.dim, h=a.h),
            coeff=coeff, dtype=a.dtype)
    m.fill_uniform(0, 1, -0.3, -0.1)
    if cls.nfields > 1:
        m.fill_uniform(1, 2, -0.1, 0.1)
    info = m.autotune(5) if a.autotune else m.kernel_info()
    kt = info["steps_per_launch"]
    launches = -(-a.steps // kt)
    m.step(a.dt, kt)  # warm-up launch
    m.synchronize()
    l0 = m.launch_count()
    t0 = time.perf_counter()
    for _ in range(launches):
        m.step(a.dt, kt)
    m.synchronize()
    el = time.perf_counter() - t0
    out = {"model": a.model, "dim": a.dim, "n": a.n, "dtype": a.dtype, "form": a.form,
           "steps": launches * kt, "wall_ms_per_step": 1e3 * el / (launches * kt),
           "launches": m.launch_count() - l0, "kernel": info}
    m.close()
    return out


def run_ensemble(a, quiet=False):
    members = sp.ensemble_members(a.ensemble, seed=20261203)
    e = sp.Ensemble(sp.SolverFT(sp.Stencil2d2h(5, 6, 13), form=a.form), members, dtype=a.dtype)
    for i in range(len(members)):
        e.fill_uniform(0, 20261203 + i, -0.1, 0.1, inst=i)
    info = e.autotune(5) if a.autotune else e.kernel_info()
    kt = info["steps_per_launch"]
    launches = -(-a.steps // kt)
    e.step(kt)
    e.synchronize()
    l0 = e.launch_count()
    t0 = time.perf_counter()
    for _ in range(launches):
        e.step(kt)
    e.synchronize()
    el = time.perf_counter() - t0
    out = {"ensemble": len(members), "sites": e.sites(), "dtype": a.dtype, "form": a.form,
           "steps": launches * kt, "wall_ms_per_step": 1e3 * el / (launches * kt),
           "launches": e.launch_count() - l0, "kernel": info}
    e.close()
    if quiet:
        return out
    print(json.dumps(out))


def run_regional(a):
    import numpy as np

    n = a.n
    y, x = np.mgrid[0:n, 0:n]
    inside = (x - n // 2) ** 2 + (y - n // 2) ** 2 < a.regional ** 2
    field = np.where(inside, 1.0 + np.random.default_rng(1).uniform(-1e-3, 1e-3, (n, n)), -1.0)
    g = sp.RegionalModel(sp.model_MB_t, 2, sp.SolverFT(sp.Stencil2d2h(5, 6, 13), form=a.form),
                         sp.ProblemParameters((n, n), h=a.h), dtype=a.dtype, dt=a.dt)
    g.set_field(field)
    g.step(1)
    info = g.autotune(5) if a.autotune else g.kernel_info()
    t0 = time.perf_counter()
    g.step(a.steps)
    g.get_field()
    el = time.perf_counter() - t0
    o, d = g.window()
    print(json.dumps({"regional": a.regional, "n": n, "window_origin": o, "window_dims": d,
                      "dtype": a.dtype, "form": a.form, "steps": a.steps,
                      "wall_ms_per_step": 1e3 * el / a.steps, "launches": g.launch_count(),
                      "kernel": info}))
    g.close()


if __name__ == "__main__":
    main()
