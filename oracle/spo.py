"""ctypes wrapper of the CPU oracle (oracle/spo.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, and only as the checker.  The product path never
imports this module.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

MODEL_A, MODEL_B, MODEL_C, MODEL_AMK, MODEL_BMK = 0, 1, 2, 3, 4
OP_LAP, OP_BILAP, OP_GRADLAP, OP_LAPCUBE = 10, 11, 12, 13
PERIODIC, DIRICHLET = 0, 1


class Desc(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("model", ctypes.c_int),
        ("lap_pts", ctypes.c_int),
        ("gradlap_pts", ctypes.c_int),
        ("bilap_pts", ctypes.c_int),
        ("h", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("c", ctypes.c_double * 8),
        ("bc", ctypes.c_int * 6),
        ("bcv", ctypes.c_double * 6),
        ("acc", ctypes.c_int),
    ]


def _load():
    path = os.path.join(_HERE, "libspo.so")
    if not os.path.exists(path):
        raise ImportError("oracle library %s is missing; run `make -C oracle`" % path)
    lib = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.spo_run.argtypes = [ctypes.POINTER(Desc), dp, ctypes.c_int, ctypes.c_int]
    lib.spo_rhs.argtypes = [ctypes.POINTER(Desc), dp, dp]
    lib.spo_seed_uniform.argtypes = [ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_longlong, ctypes.c_longlong, dp]
    lib.spo_fields.argtypes = [ctypes.c_int]
    lib.spo_mass.argtypes = [dp, ctypes.c_longlong]
    lib.spo_mass.restype = ctypes.c_double
    lib.spo_run_batch.argtypes = [ctypes.POINTER(Desc), ctypes.POINTER(dp), ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    lib.spo_omp_max_threads.restype = ctypes.c_int
    lib.spo_create.argtypes = [ctypes.POINTER(Desc), ctypes.c_int]
    lib.spo_create.restype = ctypes.c_void_p
    lib.spo_set.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
    lib.spo_get.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
    lib.spo_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.spo_destroy.argtypes = [ctypes.c_void_p]
    ip = ctypes.POINTER(ctypes.c_int)
    lib.spo_reg_create.argtypes = [ctypes.POINTER(Desc), ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int, ctypes.c_int]
    lib.spo_reg_create.restype = ctypes.c_void_p
    lib.spo_reg_set.argtypes = [ctypes.c_void_p, dp]
    lib.spo_reg_get.argtypes = [ctypes.c_void_p, dp]
    lib.spo_reg_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.spo_reg_adjust.argtypes = [ctypes.c_void_p, ip, ip]
    lib.spo_reg_window.argtypes = [ctypes.c_void_p, ip, ip, dp]
    lib.spo_reg_destroy.argtypes = [ctypes.c_void_p]
    lib.spo_reg_search.argtypes = [ctypes.c_int, ip, ip, ip, dp, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_double, ip, ip]
    return lib


_lib = _load()


def make_desc(dim, n, model, h, dt, coeff=(), stencil=None, bc=PERIODIC, bcv=0.0, acc=2):
    d = Desc()
    d.dim = dim
    nn = list(n) + [1] * (3 - len(n))
    for i in range(3):
        d.n[i] = nn[i]
    d.model = model
    if stencil is None:
        stencil = (5, 6, 13) if dim == 2 else (7, 10, 25)
    d.lap_pts, d.gradlap_pts, d.bilap_pts = stencil
    d.acc = acc
    d.h = h
    d.dt = dt
    cs = list(coeff) + [1.0] * (8 - len(coeff))
    for i in range(8):
        d.c[i] = cs[i]
    bcs = bc if isinstance(bc, (list, tuple)) else [bc] * 6
    vals = bcv if isinstance(bcv, (list, tuple)) else [bcv] * 6
    for i in range(6):
        d.bc[i] = bcs[i]
        d.bcv[i] = vals[i]
    return d


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def nfields(model):
    return _lib.spo_fields(model)


def shape_of(d):
    return (d.n[2], d.n[1], d.n[0]) if d.dim == 3 else (d.n[1], d.n[0])


def run(d, fields, steps, threads=1):
    """Advance `fields` (array (nf, *shape) or (*shape), float64) by `steps`."""
    a = np.ascontiguousarray(fields, dtype=np.float64).copy()
    _lib.spo_run(ctypes.byref(d), _ptr(a), int(steps), int(threads))
    return a


def rhs(d, fields):
    a = np.ascontiguousarray(fields, dtype=np.float64)
    out = np.empty_like(a)
    _lib.spo_rhs(ctypes.byref(d), _ptr(a), _ptr(out))
    return out


def seed_uniform(seed, lo, hi, count, first=0):
    out = np.empty(int(count), dtype=np.float64)
    _lib.spo_seed_uniform(ctypes.c_uint64(seed), lo, hi, int(count), int(first), _ptr(out))
    return out


def run_batch(descs, fields_list, steps_list, threads):
    """Run independent systems in parallel (one per thread).  Modifies arrays in place."""
    k = len(descs)
    arr = (Desc * k)(*descs)
    ptrs = (ctypes.POINTER(ctypes.c_double) * k)(*[_ptr(f) for f in fields_list])
    steps = (ctypes.c_int * k)(*[int(s) for s in steps_list])
    _lib.spo_run_batch(arr, ptrs, k, steps, int(threads))


def max_threads():
    return _lib.spo_omp_max_threads()


class System:
    """A persistent oracle system (no per-call allocation), for timing loops."""

    def __init__(self, d, fields, threads=1):
        self.d = d
        self.h = _lib.spo_create(ctypes.byref(d), int(threads))
        a = np.ascontiguousarray(fields, dtype=np.float64)
        nf = nfields(d.model)
        a = a.reshape((nf,) + shape_of(d))
        for f in range(nf):
            _lib.spo_set(self.h, f, _ptr(np.ascontiguousarray(a[f])))

    def step(self, n=1):
        _lib.spo_step(self.h, int(n))

    def get(self, f=0):
        out = np.empty(shape_of(self.d), dtype=np.float64)
        _lib.spo_get(self.h, f, _ptr(out))
        return out

    def close(self):
        if self.h:
            _lib.spo_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def _i3(v):
    a = (ctypes.c_int * 3)(0, 0, 0)
    for i, x in enumerate(v):
        a[i] = int(x)
    return a


class Regional:
    """The oracle's regional system (the moving window of SolverSystemFDwSD):
    whole-domain fields in and out, `empty` outside the window's interior."""

    def __init__(self, d, field, resize_delta=3.0, factor=2.0, eps=1e-6, fixed=True, threads=1):
        self.d = d
        self.h = _lib.spo_reg_create(ctypes.byref(d), float(resize_delta), float(factor),
                                     float(eps), int(bool(fixed)), int(threads))
        self.set(field)

    def set(self, field):
        a = np.ascontiguousarray(field, dtype=np.float64).reshape(shape_of(self.d))
        _lib.spo_reg_set(self.h, _ptr(a))

    def get(self):
        out = np.empty(shape_of(self.d), dtype=np.float64)
        _lib.spo_reg_get(self.h, _ptr(out))
        return out

    def step(self, n=1):
        _lib.spo_reg_step(self.h, int(n))

    def adjust(self, origin, dims):
        _lib.spo_reg_adjust(self.h, _i3(origin), _i3(dims))

    def window(self):
        """(origin, dims, empty, cutoff, time, next_resize) of the window."""
        o, dd = _i3(()), _i3(())
        st = (ctypes.c_double * 4)()
        _lib.spo_reg_window(self.h, o, dd, st)
        D = self.d.dim
        return (tuple(o[:D]), tuple(dd[:D]), st[0], st[1], st[2], int(st[3]))

    def close(self):
        if self.h:
            _lib.spo_reg_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def reg_search(dim, G, o, d, buf, cutoff, mode, factor=2.0, rel_eps=0.0):
    """Target window (origin, dims) of the oracle's search on a window buffer
    of values (rim included, x-fastest): mode 0 re-centres, mode 1 resizes."""
    b = np.ascontiguousarray(buf, dtype=np.float64).ravel()
    no, nd = _i3(()), _i3(())
    _lib.spo_reg_search(int(dim), _i3(G), _i3(o), _i3(d), _ptr(b), float(cutoff), int(mode),
                        float(factor), float(rel_eps), no, nd)
    return tuple(no[:dim]), tuple(nd[:dim])
