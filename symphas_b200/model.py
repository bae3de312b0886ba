"""Python mirror of SymPhas's model / solver / find_solution surface for the
explicit finite-difference path, running on the B200 library.

    SymPhas (C++)                                         here
    ---------------------------------------------------   ---------------------------------
    SolverFT<Stencil2d2h<5,6,13>>                         SolverFT(Stencil2d2h(5, 6, 13))
    BoundaryType::PERIODIC || 64_h / 0.5_dh (x, y)        ProblemParameters((64, 64), h=0.5)
    model_MA_t<2, SolverFT<...>> m{coeff, n, params}      model_MA_t(2, solver, params, coeff)
    symphas::find_solution(m, dt, steps)                  find_solution(m, dt, steps)
    m.update(t); m.equation(); m.step(dt)                 same names (equation/update fold
                                                          into the fused step kernel)
    m.system<0>().values / get_field<0>()                 m.get_field(0)

References (paths inside the SymPhas tree): MODEL macros
sol/inc/modelmacros.h:597-626; Model constructors sol/inc/model.h:100-128;
find_solution modules-io.h:747-753 and modules-none.h:42-54; model_iteration
modules-models.h:435-467; Stencil2d2h/Stencil3d2h sol/inc/stencilincludes.h:315-409
(defaults <9,6,13> and <15,10,25>, :758-792 and :884-921).
"""
import ctypes

import numpy as np

from . import _capi as C


class Stencil2d2h:
    """Stencil2d2h<L, G, B>: laplacian, gradlaplacian and bilaplacian point counts."""

    dim = 2
    accuracy = 2

    def __init__(self, L=9, G=6, B=13):
        self.points = (int(L), int(G), int(B))


class Stencil3d2h:
    """Stencil3d2h<L, G, B>."""

    dim = 3
    accuracy = 2

    def __init__(self, L=15, G=10, B=25):
        self.points = (int(L), int(G), int(B))


class Stencil2d4h:
    """Stencil2d4h<L, G, B>: the 2D stencils of 4th order of accuracy
    (sol/inc/stencilh4.h; defaults Stencil2d4h<> = <9, 14, 21>).  As in the
    reference, every operator is scaled by 1/h^3 (stencilincludes.h:446-460),
    which is exact for the Laplacian and bilaplacian only at h = 1."""

    dim = 2
    accuracy = 4

    def __init__(self, L=9, G=14, B=21):
        self.points = (int(L), int(G), int(B))


class SolverFT:
    """Forward-Euler finite-difference solver (examples/solvers/solverft.h).

    form="exact" evaluates the printed scheme term by term without FMA, which
    is bit-identical to the CPU solver in FP64; form="fused" uses the
    algebraically equal fused form (fewer operations, rounding differs)."""

    def __init__(self, stencil, form="fused"):
        if form not in ("exact", "fused"):
            raise ValueError("form must be 'exact' or 'fused'")
        self.stencil = stencil
        self.form = form


class BoundaryType:
    PERIODIC = C.SP_PERIODIC
    DEFAULT = C.SP_DIRICHLET  # with BoundaryTag::CONSTANT


class ProblemParameters:
    """Grid extents (interior points per axis, x first), uniform spacing h and
    one boundary per side (LEFT RIGHT TOP BOTTOM FRONT BACK).  A single
    boundary value applies to every side."""

    def __init__(self, dims, h=1.0, boundary=BoundaryType.PERIODIC, boundary_value=0.0):
        self.dims = tuple(int(x) for x in dims)
        self.h = float(h)
        self.boundary = list(boundary) if isinstance(boundary, (list, tuple)) else [boundary] * 6
        bv = boundary_value
        self.boundary_value = list(bv) if isinstance(bv, (list, tuple)) else [float(bv)] * 6


_DTYPES = {"f32": (C.SP_F32, np.float32), "f64": (C.SP_F64, np.float64)}


class Model:
    """A device-resident model: fields live in HBM between steps and are read
    back only by get_field / reduce."""

    model_id = None
    nfields = 1

    def __init__(self, dim, solver, params, coeff=(), dtype="f64", batch=1, dt=0.0):
        if self.model_id is None:
            raise TypeError("use one of the model_*_t classes")
        if solver.stencil.dim != dim or len(params.dims) != dim:
            raise ValueError("dimension of the model, stencil and problem parameters differ")
        if dtype not in _DTYPES:
            raise ValueError("dtype must be 'f32' or 'f64'")
        self.dim = dim
        self.dims = params.dims
        self.dtype_code, self.np_dtype = _DTYPES[dtype]
        d = C.SpDesc()
        d.dim = dim
        for i, v in enumerate(list(params.dims) + [1] * (3 - dim)):
            d.n[i] = v
        d.dtype = self.dtype_code
        d.model = self.model_id
        d.form = C.SP_FORM_EXACT if solver.form == "exact" else C.SP_FORM_FUSED
        d.lap_pts, d.gradlap_pts, d.bilap_pts = solver.stencil.points
        d.accuracy = solver.stencil.accuracy
        for i in range(6):
            d.boundary[i] = params.boundary[i]
            d.boundary_value[i] = params.boundary_value[i]
        d.h = params.h
        d.dt = float(dt)
        cs = list(coeff) + [1.0] * (8 - len(coeff))  # c(i) defaults to 1
        for i in range(8):
            d.coeff[i] = float(cs[i])
        d.ncoeff = len(coeff)
        d.batch = int(batch)
        self.desc = d
        self.batch = int(batch)
        self._h = C._H()
        C.check(C.lib().sp_create(ctypes.byref(d), ctypes.byref(self._h)))
        self.index = 0
        self.time = 0.0
        self.dt = float(dt)

    # --- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            C.lib().sp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- fields -------------------------------------------------------------
    @property
    def shape(self):
        return tuple(reversed(self.dims))

    def _nbytes(self):
        return int(np.prod(self.dims)) * np.dtype(self.np_dtype).itemsize

    def _inst_sites(self, inst):
        return int(np.prod(self.dims))

    def set_field(self, field, values, inst=0):
        a = np.ascontiguousarray(values, dtype=self.np_dtype)
        if a.shape != self.shape:
            raise ValueError("field shape %s != %s" % (a.shape, self.shape))
        C.check(C.lib().sp_upload(self._h, inst, field, a.ctypes.data, a.nbytes), self._h)

    def upload_from(self, field, host_ptr, nbytes, inst=0):
        """Upload interior values from a raw host pointer (e.g. pinned memory)."""
        C.check(C.lib().sp_upload(self._h, inst, field, ctypes.c_void_p(host_ptr), nbytes),
                self._h)

    def download_to(self, field, host_ptr, nbytes, inst=0):
        """Download interior values to a raw host pointer and wait for them."""
        C.check(C.lib().sp_download(self._h, inst, field, ctypes.c_void_p(host_ptr), nbytes),
                self._h)

    def field_to_device(self, field, dev_ptr, nbytes, inst=0):
        """Copy the interior to device memory (compact, x fastest), in the
        order of the handle's stream (no host wait)."""
        C.check(C.lib().sp_download_device(self._h, inst, field, ctypes.c_void_p(dev_ptr),
                                           nbytes), self._h)

    def field_from_device(self, field, dev_ptr, nbytes, inst=0):
        """Set the interior from device memory (compact, x fastest) and refresh
        the halo, in the order of the handle's stream."""
        C.check(C.lib().sp_upload_device(self._h, inst, field, ctypes.c_void_p(dev_ptr),
                                         nbytes), self._h)

    def batch_to_device(self, field, dev_ptr, nbytes):
        """Copy the interiors of every instance to device memory as one dense
        array [instance][interior, x fastest], one kernel, in the order of the
        handle's stream (instances of equal extents)."""
        C.check(C.lib().sp_download_batch_device(self._h, field, ctypes.c_void_p(dev_ptr),
                                                 nbytes), self._h)

    def batch_from_device(self, field, dev_ptr, nbytes):
        """Set every instance's interior from one dense device array and
        refresh all halos, two launches in the order of the handle's stream."""
        C.check(C.lib().sp_upload_batch_device(self._h, field, ctypes.c_void_p(dev_ptr),
                                               nbytes), self._h)

    def fill_uniform(self, field, seed, lo, hi, inst=0):
        """Seeded SplitMix64 initial values, bit-identical to the oracle."""
        C.check(C.lib().sp_fill_uniform(self._h, inst, field, seed, lo, hi), self._h)

    def get_field(self, field=0, inst=0):
        out = np.empty(self.shape, dtype=self.np_dtype)
        C.check(C.lib().sp_download(self._h, inst, field, out.ctypes.data, out.nbytes), self._h)
        return out

    def eval_rhs(self, field=0, inst=0):
        """dframe of the current state (one evaluation of the equations)."""
        out = np.empty(self.shape, dtype=self.np_dtype)
        C.check(C.lib().sp_eval_rhs(self._h, inst, field, out.ctypes.data, out.nbytes), self._h)
        return out

    # --- time stepping (SolverFT) -----------------------------------------------
    def update(self, t=None):
        """Halo refresh: done inside every fused step, nothing to do here."""

    def equation(self):
        """Evaluation of dframe: fused into step()."""

    def step(self, dt, n=1):
        if dt != self.dt:
            C.check(C.lib().sp_set_dt(self._h, float(dt)), self._h)
            self.dt = float(dt)
        C.check(C.lib().sp_step(self._h, int(n)), self._h)
        self.index += n
        self.time += n * dt

    def step_mass(self, dt, n):
        """n steps; the last one also returns the FP64 mass of field 0 of every
        instance, reduced inside the step kernel."""
        if dt != self.dt:
            C.check(C.lib().sp_set_dt(self._h, float(dt)), self._h)
            self.dt = float(dt)
        out = (ctypes.c_double * self.batch)()
        C.check(C.lib().sp_step_mass(self._h, int(n), out), self._h)
        self.index += n
        self.time += n * dt
        return np.array(out[:])

    def conserve_mass(self, every=100):
        """From now on restore the FP64 mass of field 0 every `every` steps
        (uniform shift; 0 turns it off)."""
        C.check(C.lib().sp_conserve_mass(self._h, int(every)), self._h)

    def reduce(self, field=0, inst=0):
        """(mass, free energy) in FP64: the sum of the field's values and h^D
        times the sum of a Landau free-energy density (no SymPhas
        counterpart; sp_reduce in include/symphas_b200.h gives the formula)."""
        m = ctypes.c_double()
        e = ctypes.c_double()
        C.check(C.lib().sp_reduce(self._h, inst, field, ctypes.byref(m), ctypes.byref(e)),
                self._h)
        return m.value, e.value

    def density(self, field=0, inst=0):
        """SymPhas's Density collector (dataprocesses/datadensity.h:11-19): the
        sum of the field's values, in FP64."""
        return self.reduce(field, inst)[0]

    def energy(self, field=0, inst=0):
        """SymPhas's Energy collector (dataprocesses/dataenergy.h:11-19): the
        sum of the field's values over the number of sites, in FP64."""
        return self.reduce(field, inst)[0] * (1.0 / self._inst_sites(inst))

    def structure_factor(self, field=0, inst=0, threshold=True):
        """(k, S): SymPhas's radially averaged structure factor of the field
        (thresholded at 0 when `threshold`), computed on the device.  k is in
        units of the wave-number step 2 pi / (n h)."""
        nb = ctypes.c_int(0)
        C.check(C.lib().sp_structure_factor(self._h, inst, field, int(bool(threshold)), None,
                                            None, ctypes.byref(nb)), self._h)
        k = (ctypes.c_double * nb.value)()
        sf = (ctypes.c_double * nb.value)()
        C.check(C.lib().sp_structure_factor(self._h, inst, field, int(bool(threshold)), k, sf,
                                            ctypes.byref(nb)), self._h)
        return np.array(k[:nb.value]), np.array(sf[:nb.value])

    def autotune(self, reps=20):
        """Pick the fastest tile shape for this kernel and size on this GPU."""
        C.check(C.lib().sp_autotune(self._h, int(reps)), self._h)
        return self.kernel_info()

    def kernel_info(self):
        v = (ctypes.c_int * 8)()
        C.check(C.lib().sp_kernel_info(self._h, v), self._h)
        keys = ("tile_x", "tile_y", "rows_per_thread", "stages_in_flight", "variant",
                "variants", "threads", "z_per_cta_or_ctas")
        info = dict(zip(keys, v[:]))
        kt = ctypes.c_int(0)
        C.check(C.lib().sp_steps_per_launch(self._h, ctypes.byref(kt)), self._h)
        info["steps_per_launch"] = kt.value
        return info

    def synchronize(self):
        C.check(C.lib().sp_synchronize(self._h), self._h)

    def set_stream(self, stream_ptr):
        C.check(C.lib().sp_set_stream(self._h, ctypes.c_void_p(stream_ptr)), self._h)

    def launch_count(self):
        return C.lib().sp_launch_count(self._h)

    def get_index(self):
        return self.index

    def get_time(self):
        return self.time


class model_MA_t(Model):
    """MODEL(MA, (SCALAR), EVOLUTION(dpsi = lap(psi) + (c(1) - c(2) psi^2) psi))."""

    model_id = C.SP_MODEL_A


class model_MB_t(Model):
    """MODEL(MB, (SCALAR), EVOLUTION(dpsi = -bilap(psi) - lap((c(1) - c(2) psi^2) psi)))."""

    model_id = C.SP_MODEL_B


class model_MC_t(Model):
    """Model C with coupling gamma = c(1): conserved psi, non-conserved eta."""

    model_id = C.SP_MODEL_C
    nfields = 2


class model_MAMK_t(Model):
    """dpsi = M (kappa lap(psi) - psi^3 + psi), M = c(1), kappa = c(2)."""

    model_id = C.SP_MODEL_AMK


class model_MBMK_t(Model):
    """dpsi = M lap(psi^3 - psi - kappa lap(psi)), M = c(1), kappa = c(2)."""

    model_id = C.SP_MODEL_BMK


class model_OP_t(Model):
    """Single-operator model dframe = op(psi), to check a stencil point set."""

    def __init__(self, op, dim, solver, params, dtype="f64"):
        self.model_id = {"lap": C.SP_OP_LAP, "bilap": C.SP_OP_BILAP,
                         "gradlap": C.SP_OP_GRADLAP, "lapcube": C.SP_OP_LAPCUBE}[op]
        super().__init__(dim, solver, params, dtype=dtype)


class Ensemble(Model):
    """Independent 2D systems of differing size, model (model_MAMK_t or
    model_MBMK_t, or all of one model), coefficients and time step, advanced
    together: every step is one persistent kernel launch over the tiles of
    all members.  `members` is a list of dicts with keys dims (x, y),
    model ("AMK", "BMK", or another model class's name), dt and coeff.
    Instance i is member i in every per-instance call."""

    _IDS = {"A": C.SP_MODEL_A, "B": C.SP_MODEL_B, "AMK": C.SP_MODEL_AMK,
            "BMK": C.SP_MODEL_BMK}

    def __init__(self, solver, members, h=1.0, boundary=BoundaryType.PERIODIC,
                 dtype="f32"):
        if solver.stencil.dim != 2:
            raise ValueError("ensembles are two-dimensional")
        if dtype not in _DTYPES:
            raise ValueError("dtype must be 'f32' or 'f64'")
        self.dim = 2
        self.dtype_code, self.np_dtype = _DTYPES[dtype]
        params = ProblemParameters(members[0]["dims"], h=h, boundary=boundary)
        d = C.SpDesc()
        d.dim = 2
        d.dtype = self.dtype_code
        d.form = C.SP_FORM_EXACT if solver.form == "exact" else C.SP_FORM_FUSED
        d.lap_pts, d.gradlap_pts, d.bilap_pts = solver.stencil.points
        d.accuracy = solver.stencil.accuracy
        for i in range(6):
            d.boundary[i] = params.boundary[i]
            d.boundary_value[i] = params.boundary_value[i]
        d.h = float(h)
        arr = (C.SpMember * len(members))()
        for i, m in enumerate(members):
            dims = tuple(int(x) for x in m["dims"])
            if len(dims) != 2:
                raise ValueError("member %d: two extents (x, y) expected" % i)
            arr[i].n[0], arr[i].n[1], arr[i].n[2] = dims[0], dims[1], 1
            arr[i].model = self._IDS[m["model"]]
            arr[i].dt = float(m["dt"])
            cs = list(m.get("coeff", ())) + [1.0] * (8 - len(m.get("coeff", ())))
            for c in range(8):
                arr[i].coeff[c] = float(cs[c])
        self.desc = d
        self.members = [dict(m) for m in members]
        self.member_dims = [tuple(int(x) for x in m["dims"]) for m in members]
        self.batch = len(members)
        self._h = C._H()
        C.check(C.lib().sp_create_ensemble(ctypes.byref(d), arr, len(members),
                                           ctypes.byref(self._h)))
        self.index = 0
        self.time = None  # members advance by their own dt
        self.dt = None

    def _shape(self, inst):
        return tuple(reversed(self.member_dims[inst]))

    def _inst_sites(self, inst):
        return int(np.prod(self.member_dims[inst]))

    def sites(self):
        return sum(int(np.prod(x)) for x in self.member_dims)

    def set_field(self, field, values, inst=0):
        a = np.ascontiguousarray(values, dtype=self.np_dtype)
        if a.shape != self._shape(inst):
            raise ValueError("field shape %s != %s" % (a.shape, self._shape(inst)))
        C.check(C.lib().sp_upload(self._h, inst, field, a.ctypes.data, a.nbytes), self._h)

    def get_field(self, field=0, inst=0):
        out = np.empty(self._shape(inst), dtype=self.np_dtype)
        C.check(C.lib().sp_download(self._h, inst, field, out.ctypes.data, out.nbytes), self._h)
        return out

    def eval_rhs(self, field=0, inst=0):
        out = np.empty(self._shape(inst), dtype=self.np_dtype)
        C.check(C.lib().sp_eval_rhs(self._h, inst, field, out.ctypes.data, out.nbytes), self._h)
        return out

    def step(self, n=1):
        """Advance every member by n steps of its own dt."""
        C.check(C.lib().sp_step(self._h, int(n)), self._h)
        self.index += n

    def step_mass(self, *a, **k):
        raise NotImplementedError("use reduce(inst=i) on ensembles")


def ensemble_members(count, seed=0, sides=(64, 96, 128, 256, 384, 512, 768, 1024), h=1.0,
                     safety=0.4):
    """A sweep of `count` 2D members: square sides drawn from `sides`, the first
    half model_MAMK_t and the second half model_MBMK_t, M and kappa drawn from
    U[0.5, 2], and dt = safety x the forward-Euler stability limit of each
    member with the 5-point Laplacian (largest eigenvalue 8 / h^2):
    AMK  2 / (M (8 kappa / h^2 + 2)),  BMK  2 / (M (64 kappa / h^4 + 16 / h^2))."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.choice(sides))
        M, kappa = (float(v) for v in rng.uniform(0.5, 2.0, 2))
        if i < count // 2:
            model, lim = "AMK", 2.0 / (M * (8.0 * kappa / h ** 2 + 2.0))
        else:
            model, lim = "BMK", 2.0 / (M * (64.0 * kappa / h ** 4 + 16.0 / h ** 2))
        out.append({"dims": (n, n), "model": model, "dt": safety * lim, "coeff": (M, kappa)})
    return out


def find_solution(model, dt, steps):
    """symphas::find_solution(model, dt, steps): advance `steps` iterations."""
    model.update(model.time)
    model.step(dt, steps)
    return model
