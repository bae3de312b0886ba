"""Generates tests/golden/oracle_golden.npz: small seeded trajectories of the
CPU oracle (regression fixtures for the oracle and for the GPU path).

Run from the repository root after `make -C oracle`:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import spo  # noqa: E402

CASES = {
    # name: (dim, dims, model, h, dt, steps, coeff, [(seed, lo, hi) per field])
    "model_a_2d": (2, (16, 12), spo.MODEL_A, 0.5, 0.01, 100, (), [(3, -0.1, 0.1)]),
    "model_b_3d": (3, (8, 8, 6), spo.MODEL_B, 1.0, 0.005, 50, (), [(4, -0.3, -0.1)]),
    "model_c_3d": (3, (8, 6, 8), spo.MODEL_C, 1.0, 0.005, 30, (0.5,), [(5, 0.0, 0.2), (6, -0.1, 0.1)]),
    "model_bmk_2d": (2, (12, 16), spo.MODEL_BMK, 1.0, 0.004, 40, (1.5, 0.6), [(7, -0.1, 0.1)]),
}


def initial(dim, dims, fields):
    shape = tuple(reversed(dims))
    n = int(np.prod(dims))
    return np.stack([spo.seed_uniform(s, lo, hi, n).reshape(shape) for s, lo, hi in fields])


def main():
    out = {}
    for name, (dim, dims, model, h, dt, steps, coeff, fields) in CASES.items():
        x0 = initial(dim, dims, fields)
        x = x0[0] if len(fields) == 1 else x0
        d = spo.make_desc(dim, dims, model, h, dt, coeff=coeff)
        out[name + "_init"] = x
        out[name + "_final"] = spo.run(d, x, steps)
    out["splitmix_seed0_u01"] = spo.seed_uniform(0, 0.0, 1.0, 8)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, sorted(out))


if __name__ == "__main__":
    main()
