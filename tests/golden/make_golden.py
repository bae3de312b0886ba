"""Generates the golden fixtures: small seeded trajectories of
- the CPU oracle (tests/golden/oracle_golden.npz: regression fixtures for the
  oracle and for the GPU path), and
- SymPhas itself, its CPU SolverFT built by oracle/ref.mk
  (tests/golden/symphas_golden.npz: the oracle's pin, for machines that do not
  build SymPhas).

Run from the repository root after `make -C oracle` and
`make -C oracle -f ref.mk`:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import spo  # noqa: E402
import symref  # noqa: E402

CASES = {
    # name: (dim, dims, model, h, dt, steps, coeff, [(seed, lo, hi) per field])
    "model_a_2d": (2, (16, 12), spo.MODEL_A, 0.5, 0.01, 100, (), [(3, -0.1, 0.1)]),
    "model_b_3d": (3, (8, 8, 6), spo.MODEL_B, 1.0, 0.005, 50, (), [(4, -0.3, -0.1)]),
    "model_c_3d": (3, (8, 6, 8), spo.MODEL_C, 1.0, 0.005, 30, (0.5,), [(5, 0.0, 0.2), (6, -0.1, 0.1)]),
    "model_bmk_2d": (2, (12, 16), spo.MODEL_BMK, 1.0, 0.004, 40, (1.5, 0.6), [(7, -0.1, 0.1)]),
}


# SymPhas's own trajectories: the first configuration (model A 2D 64^2, dx 0.5,
# dt 0.01, 1000 steps), model B 3D around mean -0.2, and model B on SymPhas's
# default 3D stencil Stencil3d2h<> = <15,10,25>
REF_CASES = {
    "config_model_a_2d_64": (2, (64, 64), spo.MODEL_A, 0.5, 0.01, 1000, (), [(7, -0.1, 0.1)]),
    "model_b_3d_16": (3, (16, 16, 16), spo.MODEL_B, 1.0, 0.005, 100, (), [(11, -0.3, -0.1)]),
    "model_b_3d_default_stencil": (3, (12, 10, 8), spo.MODEL_B, 1.0, 0.002, 50, (),
                                   [(12, -0.1, 0.1)]),
}
REF_STENCIL = {"model_b_3d_default_stencil": (15, 10, 25)}


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
    here = os.path.dirname(os.path.abspath(__file__))
    path = os.path.join(here, "oracle_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, sorted(out))
    ref = {}
    for name, (dim, dims, model, h, dt, steps, coeff, fields) in REF_CASES.items():
        x0 = initial(dim, dims, fields)
        x = x0[0] if len(fields) == 1 else x0
        d = spo.make_desc(dim, dims, model, h, dt, coeff=coeff, stencil=REF_STENCIL.get(name))
        ref[name + "_init"] = x
        ref[name + "_final"] = symref.run(d, x, steps)
    path = os.path.join(here, "symphas_golden.npz")
    np.savez_compressed(path, **ref)
    print("wrote", path, sorted(ref))


if __name__ == "__main__":
    main()
