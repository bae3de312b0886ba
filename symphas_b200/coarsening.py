"""Cahn-Hilliard (model B) coarsening on a periodic cube, run on the device in
FP64 (the exact form, bit-identical to the CPU solver step for step) and in
FP32 (the fused bulk path) from the same seeded field, reporting what the
model-B configuration asks for: the drift of the mass (reduced in FP64
inside the step kernel), the relative L-infinity distance of the FP32 field
from the FP64 one, and the peak of SymPhas's radially averaged structure
factor of both.  FP32 runs twice: as it rounds, and with its mass restored
every `conserve` steps (sp_conserve_mass).

    python -m symphas_b200.coarsening --n 256 --steps 20000 --mean 0 -0.2
"""
import argparse
import json
import time

import numpy as np

import symphas_b200 as sp


def run(n, steps, mean, dt=0.005, chunk=1000, seed=20261203, conserve=100):
    st = sp.Stencil3d2h(7, 10, 25)
    params = sp.ProblemParameters((n, n, n), h=1.0)
    out = {"n": n, "steps": steps, "dt": dt, "psi_bar": mean}
    fields, snaps = {}, {}
    checkpoints = [c for c in (1, 100, 1000) if c < steps]
    for key, dtype, form, every in (("f64", "f64", "exact", 0), ("f32", "f32", "fused", 0),
                                     ("f32_held", "f32", "fused", conserve)):
        if key == "f32_held" and not conserve:
            continue
        m = sp.model_MB_t(3, sp.SolverFT(st, form=form), params, dtype=dtype)
        m.fill_uniform(0, seed, mean - 0.1, mean + 0.1)
        m0, _ = m.reduce(0)
        if every:
            m.conserve_mass(every)
        masses = []
        snaps[key] = {}
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            # stop at the checkpoints to keep a copy of the field (not timed)
            nxt = min([c for c in checkpoints if c > done] + [done + chunk, steps])
            k = nxt - done
            masses.append(float(m.step_mass(dt, k)[0]))
            done += k
            if done in checkpoints:
                m.synchronize()
                t1 = time.perf_counter()
                snaps[key][done] = m.get_field(0).astype(np.float64)
                t0 += time.perf_counter() - t1
        m.synchronize()
        el = time.perf_counter() - t0
        mass, energy = m.reduce(0)
        k, s = m.structure_factor(threshold=True)
        b = int(np.argmax(s[1:])) + 1  # skip the k = 0 class
        out[key] = {"form": form, "conserve_every": every, "seconds": el, "site_updates_per_s": n ** 3 * steps / el,
                      "mass_initial": m0, "mass_final": mass,
                      "mass_drift_rel": abs(mass - m0) / max(abs(m0), 1e-300),
                      "mass_drift_rel_max": max(abs(x - m0) for x in masses) / max(abs(m0), 1e-300),
                      "energy_final": energy, "sf_peak_k": float(k[b]), "sf_peak": float(s[b])}
        fields[key] = m.get_field(0).astype(np.float64)
        m.close()
    def rel(a, b):
        return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))

    for key in fields:
        if key != "f64":
            out[key + "_vs_f64_rel_linf"] = rel(fields[key], fields["f64"])
            out[key + "_vs_f64_rel_linf_at"] = {str(c): rel(snaps[key][c], snaps["f64"][c])
                                                for c in checkpoints}
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--mean", type=float, nargs="*", default=[0.0, -0.2])
    ap.add_argument("--conserve", type=int, default=100,
                    help="also run FP32 with its mass restored every this many steps (0: no)")
    a = ap.parse_args(argv)
    for mean in a.mean:
        print(json.dumps(run(a.n, a.steps, mean, conserve=a.conserve)))


if __name__ == "__main__":
    main()
