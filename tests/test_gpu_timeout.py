"""The bounded-wait failure path of the step kernels, on a GPU.

Every wait of a step kernel (an mbarrier for a TMA tile) is bounded: a CTA
that gives up sets the handle's device error flag, waits (bounded) for its
own copies in flight and returns; the host's next synchronising call returns
SP_ETIMEOUT, clears the flag and re-arms the 2D work queue, and the handle
stays usable.  sp_test_wait_timeout runs that path on its own: one warp waits
with a short limit on an mbarrier nothing completes (no copy in flight, so
nothing can land after it gives up) and, asked to, first takes an item from
the 2D work queue without re-arming it, as a CTA that gave up mid-step would.
"""
import ctypes
import time

import numpy as np
import pytest

import spo
import symphas_b200 as sp
from symphas_b200 import _capi as C

pytestmark = pytest.mark.gpu

S2 = sp.Stencil2d2h(5, 6, 13)
MEMBERS = [
    {"dims": (40, 24), "model": "BMK", "coeff": (0.7, 1.3), "dt": 0.002},
    {"dims": (130, 34), "model": "AMK", "coeff": (1.9, 0.6), "dt": 0.02},
    {"dims": (64, 64), "model": "BMK", "coeff": (0.5, 2.0), "dt": 0.002},
]
ORACLE_MODEL = {"AMK": spo.MODEL_AMK, "BMK": spo.MODEL_BMK}


@pytest.mark.parametrize("dirty_queue", [0, 1])
def test_a_wait_that_runs_out_is_reported_and_the_handle_recovers(dirty_queue):
    ens = sp.Ensemble(sp.SolverFT(S2, form="exact"), MEMBERS, dtype="f64")
    inits = []
    for i, m in enumerate(MEMBERS):
        ens.fill_uniform(0, 300 + i, -0.3, 0.3, inst=i)
        nx, ny = m["dims"]
        inits.append(spo.seed_uniform(300 + i, -0.3, 0.3, nx * ny).reshape(ny, nx))
    ens.step(10)
    lib = C.lib()
    t0 = time.perf_counter()
    assert lib.sp_test_wait_timeout(ens._h, 20000, dirty_queue) == C.SP_OK
    assert lib.sp_synchronize(ens._h) == C.SP_ETIMEOUT
    waited = time.perf_counter() - t0
    assert b"gave up" in lib.sp_last_error(ens._h)
    assert waited < 1.0, waited  # the wait is bounded: ~20000 cycles and one short sleep
    # the flag was cleared and the queue re-armed: the handle steps on as before
    assert lib.sp_synchronize(ens._h) == C.SP_OK
    ens.step(10)
    for i, m in enumerate(MEMBERS):
        d = spo.make_desc(2, m["dims"], ORACLE_MODEL[m["model"]], 1.0, m["dt"], coeff=m["coeff"])
        assert np.array_equal(ens.get_field(0, inst=i), spo.run(d, inits[i], 20)), i
    ens.close()


def test_the_hook_rejects_bad_arguments():
    ens = sp.Ensemble(sp.SolverFT(S2, form="exact"), MEMBERS, dtype="f64")
    assert C.lib().sp_test_wait_timeout(ens._h, -1, 0) == C.SP_EINVAL
    assert C.lib().sp_test_wait_timeout(ens._h, (1 << 31) + 1, 0) == C.SP_EINVAL
    ens.close()
