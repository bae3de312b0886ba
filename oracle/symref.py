"""ctypes wrapper of SymPhas's own CPU SolverFT (oracle/_ref/libsymphas_ref.so,
built by oracle/ref.mk from the SymPhas sources): the pin of the oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/ and by bench.py's reference arm.
The descriptor is the oracle's (spo.Desc), and the calls mirror spo.run /
spo.rhs, so a test hands both the same inputs.  Which combinations of model
and stencil the library holds is listed in oracle/ref_models_*.cpp and
oracle/ref_ops_*.cpp; `available(d)` answers for one descriptor.
"""
import ctypes
import os

import numpy as np

import spo

_HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(_HERE, "_ref", "libsymphas_ref.so")
MODEL_MBB = 5  # SymPhas's MBB (a provisional variable); not in the oracle

_lib = None


def loaded():
    """The library, or None when it was not built here."""
    global _lib
    if _lib is None and os.path.exists(PATH):
        lib = ctypes.CDLL(PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.symref_run.argtypes = [ctypes.POINTER(spo.Desc), dp, ctypes.c_int]
        lib.symref_rhs.argtypes = [ctypes.POINTER(spo.Desc), dp, dp]
        lib.symref_available.argtypes = [ctypes.POINTER(spo.Desc)]
        _lib = lib
    return _lib


def _need():
    lib = loaded()
    if lib is None:
        raise ImportError("%s is missing; build it with `make -C oracle -f ref.mk`" % PATH)
    return lib


def available(d):
    return bool(_need().symref_available(ctypes.byref(d)))


def _check(rc, what):
    if rc != 0:
        raise RuntimeError("%s: SymPhas driver status %d" % (what, rc))


def run(d, fields, steps):
    """`fields` ((nf, *shape) or (*shape), float64) after `steps` SolverFT
    iterations of SymPhas (update, equation, step per iteration)."""
    a = np.ascontiguousarray(fields, dtype=np.float64).copy()
    _check(_need().symref_run(ctypes.byref(d), spo._ptr(a), int(steps)), "symref_run")
    return a


def rhs(d, fields):
    """SymPhas's right-hand side (each system's dframe after update() and
    equation()), or one operator over the field."""
    a = np.ascontiguousarray(fields, dtype=np.float64)
    out = np.zeros_like(a)
    _check(_need().symref_rhs(ctypes.byref(d), spo._ptr(a), spo._ptr(out)), "symref_rhs")
    return out


class System:
    """A SymPhas model held between calls (the reference arm of bench.py times
    its steps): built from `fields`, stepped in place, read back."""

    def __init__(self, d, fields):
        lib = _need()
        lib.symref_create.argtypes = [ctypes.POINTER(spo.Desc), ctypes.POINTER(ctypes.c_double)]
        lib.symref_create.restype = ctypes.c_void_p
        lib.symref_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.symref_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        lib.symref_destroy.argtypes = [ctypes.c_void_p]
        self.d = d
        a = np.ascontiguousarray(fields, dtype=np.float64)
        self.shape = a.shape
        self.h = lib.symref_create(ctypes.byref(d), spo._ptr(a))
        if not self.h:
            raise RuntimeError("symref_create: combination not built or storage mismatch")

    def step(self, n=1):
        _need().symref_step(self.h, int(n))

    def get(self):
        out = np.empty(self.shape, dtype=np.float64)
        _need().symref_get(self.h, spo._ptr(out))
        return out

    def close(self):
        if self.h:
            _need().symref_destroy(self.h)
            self.h = None


def step_many(systems, nsteps, threads):
    """`nsteps` iterations of every system, spread over `threads` host threads
    (each model on one thread)."""
    lib = _need()
    lib.symref_step_many.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int]
    arr = (ctypes.c_void_p * len(systems))(*[s.h for s in systems])
    lib.symref_step_many(arr, len(systems), int(nsteps), int(threads))
