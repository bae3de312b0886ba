"""Regional systems: a model whose system keeps only a moving window of the
domain (SymPhas's SolverSystemFDwSD, sol/inc/solversystem.h:62-77, over a
RegionalGrid, datatypes/inc/grid.h:2038-2158).

The window (origin and dims in storage coordinates, each with a 3-deep rim)
is evolved by the fused kernels; everything outside its interior reads
`empty`.  At the first step the cutoff becomes min + eps and `empty` the
minimum, and the window shrinks to the values >= cutoff times the padding
factor; afterwards, every `resize_delta` of time, it is re-centred (fixed
size) or resized again (sol/inc/boundarysystem.h:438-471, with SymPhas's
defaults from sol/src/boundarysystem.cpp:24-27).
"""
import ctypes

import numpy as np

from . import _capi as C
from .model import _DTYPES


def _i3(v=()):
    a = (ctypes.c_int * 3)(0, 0, 0)
    for i, x in enumerate(v):
        a[i] = int(x)
    return a


class RegionalModel:
    """A single-field model on a regional system.  `model` is a model class
    (model_MA_t, model_MB_t, ...) or an SP_MODEL_* id; the domain must be
    periodic on every side."""

    def __init__(self, model, dim, solver, params, coeff=(), dtype="f64", dt=0.0,
                 resize_delta=3.0, padding_factor=2.0, cutoff_eps=1e-6, fixed=True):
        model_id = getattr(model, "model_id", model)
        if model_id is None:
            raise TypeError("model must be a model class or an SP_MODEL_* id")
        if solver.stencil.dim != dim or len(params.dims) != dim:
            raise ValueError("dimension of the model, stencil and problem parameters differ")
        if dtype not in _DTYPES:
            raise ValueError("dtype must be 'f32' or 'f64'")
        self.dim = dim
        self.dims = tuple(params.dims)
        self.dtype_code, self.np_dtype = _DTYPES[dtype]
        d = C.SpDesc()
        d.dim = dim
        for i, v in enumerate(list(params.dims) + [1] * (3 - dim)):
            d.n[i] = v
        d.dtype = self.dtype_code
        d.model = int(model_id)
        d.form = C.SP_FORM_EXACT if solver.form == "exact" else C.SP_FORM_FUSED
        d.lap_pts, d.gradlap_pts, d.bilap_pts = solver.stencil.points
        d.accuracy = solver.stencil.accuracy
        for i in range(6):
            d.boundary[i] = params.boundary[i]
            d.boundary_value[i] = params.boundary_value[i]
        d.h = params.h
        d.dt = float(dt)
        cs = list(coeff) + [1.0] * (8 - len(coeff))
        for i in range(8):
            d.coeff[i] = float(cs[i])
        d.ncoeff = len(coeff)
        d.batch = 1
        p = C.SpRegionalParams()
        p.resize_delta = float(resize_delta)
        p.padding_factor = float(padding_factor)
        p.cutoff_eps = float(cutoff_eps)
        p.fixed = int(bool(fixed))
        self.desc = d
        self.dt = float(dt)
        self._r = ctypes.c_void_p()
        rc = C.lib().sp_regional_create(ctypes.byref(d), ctypes.byref(p), ctypes.byref(self._r))
        if rc != C.SP_OK:
            raise C.SymPhasError(rc, (C.lib().sp_regional_error(None) or b"").decode())

    def _check(self, rc):
        if rc != C.SP_OK:
            raise C.SymPhasError(rc, (C.lib().sp_regional_error(self._r) or b"").decode())

    # --- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_r", None):
            C.lib().sp_regional_destroy(self._r)
            self._r = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- fields (whole domain) -------------------------------------------------
    @property
    def shape(self):
        return tuple(reversed(self.dims))

    def set_field(self, values):
        a = np.ascontiguousarray(values, dtype=self.np_dtype).reshape(self.shape)
        self._check(C.lib().sp_regional_upload(self._r, a.ctypes.data, a.nbytes))

    def get_field(self):
        out = np.empty(self.shape, dtype=self.np_dtype)
        self._check(C.lib().sp_regional_download(self._r, out.ctypes.data, out.nbytes))
        return out

    def upload_from(self, field, host_ptr, nbytes, inst=0):
        """Whole-domain values from host memory at `host_ptr` (the Model
        signature; field and inst must be 0)."""
        if field != 0 or inst != 0:
            raise ValueError("a regional system holds one field of one instance")
        self._check(C.lib().sp_regional_upload(self._r, ctypes.c_void_p(host_ptr), int(nbytes)))

    def download_to(self, field, host_ptr, nbytes, inst=0):
        if field != 0 or inst != 0:
            raise ValueError("a regional system holds one field of one instance")
        self._check(C.lib().sp_regional_download(self._r, ctypes.c_void_p(host_ptr), int(nbytes)))

    def set_stream(self, stream_ptr):
        """Run all further work on the CUDA stream `stream_ptr`."""
        self._check(C.lib().sp_regional_set_stream(self._r, ctypes.c_void_p(stream_ptr)))

    # --- stepping and the window ---------------------------------------------
    def step(self, n=1):
        self._check(C.lib().sp_regional_step(self._r, int(n)))

    def set_dt(self, dt):
        """Time step of further steps."""
        self._check(C.lib().sp_regional_set_dt(self._r, float(dt)))
        self.dt = float(dt)

    def adjust(self, origin, dims):
        self._check(C.lib().sp_regional_adjust(self._r, _i3(origin), _i3(dims)))

    def window(self):
        """(origin, dims) of the window, storage coordinates, rim included."""
        o, d = _i3(), _i3()
        st = (ctypes.c_double * 4)()
        self._check(C.lib().sp_regional_window(self._r, o, d, st))
        return tuple(o[:self.dim]), tuple(d[:self.dim])

    def state(self):
        """(empty, cutoff, time, next window-update index)."""
        st = (ctypes.c_double * 4)()
        self._check(C.lib().sp_regional_window(self._r, None, None, st))
        return st[0], st[1], st[2], int(st[3])

    @property
    def time(self):
        return self.state()[2]

    def handle(self):
        """The window's sp_handle (None while the window has no interior)."""
        h = C.lib().sp_regional_handle(self._r)
        return h or None

    def kernel_info(self):
        h = self.handle()
        if h is None:
            return None
        info = (ctypes.c_int * 8)()
        C.check(C.lib().sp_kernel_info(h, info), h)
        return list(info)

    def autotune(self, reps=20):
        """Time the tile shapes on the present window's handle, keep the fastest."""
        h = self.handle()
        if h is None:
            return None
        C.check(C.lib().sp_autotune(h, int(reps)), h)
        return self.kernel_info()

    def interior_sites(self):
        """Sites of the window's interior (the sites a step advances)."""
        o, d = self.window()
        s = 1
        for x in d:
            s *= max(0, x - 6)
        return s

    def launch_count(self):
        h = self.handle()
        return 0 if h is None else C.lib().sp_launch_count(h)


def region_search(dim, G, origin, dims, mask, mode, factor=2.0, rel_eps=0.0):
    """The library's window search alone, on the host: the target (origin,
    dims) after a re-centre (mode 0) or a resize (mode 1) of window
    (origin, dims) in a domain of storage extents G, given the byte mask of
    the window's buffer (rim included, x-fastest)."""
    m = np.ascontiguousarray(mask, dtype=np.uint8).ravel()
    no, nd = _i3(), _i3()
    rc = C.lib().sp_region_search(int(dim), _i3(G), _i3(origin), _i3(dims), m.ctypes.data,
                                  int(mode), float(factor), float(rel_eps), no, nd)
    if rc != C.SP_OK:
        raise C.SymPhasError(rc, "region search")
    return tuple(no[:dim]), tuple(nd[:dim])
