"""ctypes binding of the C ABI in include/symphas_b200.h.

The shared library lib/libsymphas_b200.so is loaded from inside the package
directory.  There is no fallback: if the library is missing or a call fails,
an exception says so.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libsymphas_b200.so")

# status codes
SP_OK, SP_EINVAL, SP_ECUDA, SP_ENOMEM, SP_ETIMEOUT, SP_ENONFINITE = range(6)
SP_F32, SP_F64 = 0, 1
SP_PERIODIC, SP_DIRICHLET = 0, 1
SP_MODEL_A, SP_MODEL_B, SP_MODEL_C, SP_MODEL_AMK, SP_MODEL_BMK = 0, 1, 2, 3, 4
SP_OP_LAP, SP_OP_BILAP, SP_OP_GRADLAP, SP_OP_LAPCUBE = 10, 11, 12, 13
SP_FORM_EXACT, SP_FORM_FUSED = 1, 0
SP_ENSEMBLE_AMK_BMK = 5
SP_NOALLOC_MAX_INSTANCES = 64

_STATUS = {
    SP_EINVAL: "invalid argument",
    SP_ECUDA: "CUDA error",
    SP_ENOMEM: "out of device memory",
    SP_ETIMEOUT: "device wait timed out",
    SP_ENONFINITE: "non-finite values",
}


class SymPhasError(RuntimeError):
    """A call into the B200 library failed."""

    def __init__(self, code, message):
        super().__init__("%s (status %d): %s" % (_STATUS.get(code, "error"), code, message))
        self.code = code


class SpDesc(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("dtype", ctypes.c_int),
        ("model", ctypes.c_int),
        ("form", ctypes.c_int),
        ("lap_pts", ctypes.c_int),
        ("gradlap_pts", ctypes.c_int),
        ("bilap_pts", ctypes.c_int),
        ("boundary", ctypes.c_int * 6),
        ("boundary_value", ctypes.c_double * 6),
        ("h", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("coeff", ctypes.c_double * 8),
        ("ncoeff", ctypes.c_int),
        ("batch", ctypes.c_int),
        ("accuracy", ctypes.c_int),
    ]


class SpMember(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int * 3),
        ("model", ctypes.c_int),
        ("dt", ctypes.c_double),
        ("coeff", ctypes.c_double * 8),
    ]


class SpRegionalParams(ctypes.Structure):
    _fields_ = [
        ("resize_delta", ctypes.c_double),
        ("padding_factor", ctypes.c_double),
        ("cutoff_eps", ctypes.c_double),
        ("fixed", ctypes.c_int),
    ]


_H = ctypes.c_void_p
_P = ctypes.c_void_p
_SZ = ctypes.c_size_t

# name -> (restype, argtypes); every function declared in include/symphas_b200.h
SIGNATURES = {
    "sp_create": (ctypes.c_int, [ctypes.POINTER(SpDesc), ctypes.POINTER(_H)]),
    "sp_create_ensemble": (ctypes.c_int, [ctypes.POINTER(SpDesc), ctypes.POINTER(SpMember),
                                          ctypes.c_int, ctypes.POINTER(_H)]),
    "sp_upload": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, _P, _SZ]),
    "sp_upload_device": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, _P, _SZ]),
    "sp_fill_uniform": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                       ctypes.c_double, ctypes.c_double]),
    "sp_step": (ctypes.c_int, [_H, ctypes.c_int]),
    "sp_step_mass": (ctypes.c_int, [_H, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "sp_eval_rhs": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, _P, _SZ]),
    "sp_download": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, _P, _SZ]),
    "sp_download_device": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, _P, _SZ]),
    "sp_upload_batch_device": (ctypes.c_int, [_H, ctypes.c_int, _P, _SZ]),
    "sp_download_batch_device": (ctypes.c_int, [_H, ctypes.c_int, _P, _SZ]),
    "sp_reduce": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_double)]),
    "sp_autotune": (ctypes.c_int, [_H, ctypes.c_int]),
    "sp_kernel_info": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int)]),
    "sp_steps_per_launch": (ctypes.c_int, [_H, ctypes.POINTER(ctypes.c_int)]),
    "sp_test_wait_timeout": (ctypes.c_int, [_H, ctypes.c_longlong, ctypes.c_int]),
    "sp_set_stream": (ctypes.c_int, [_H, _P]),
    "sp_set_dt": (ctypes.c_int, [_H, ctypes.c_double]),
    "sp_synchronize": (ctypes.c_int, [_H]),
    "sp_launch_count": (ctypes.c_longlong, [_H]),
    "sp_field_geometry": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_P),
                                         ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_int)]),
    "sp_reduce_fields_noalloc": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int,
                                                 ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                                 ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                                 ctypes.c_int, _P, _P]),
    "sp_structure_factor": (ctypes.c_int, [_H, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_int)]),
    "sp_conv3x3_fwd": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, _P]),
    "sp_conv3x3_fwd_tc": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, _P]),
    "sp_conv3x3_fwd_strip": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, _P]),
    "sp_conv3x3_fwd_strip_up2": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, _P]),
    "sp_conv_tc_status": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    "sp_avgpool2_bf16": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, _P]),
    "sp_embed_channel0_bf16": (ctypes.c_int, [_P, _P, ctypes.c_longlong, ctypes.c_int, _P]),
    "sp_conv3x3_wgrad": (ctypes.c_int, [_P, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, _P]),
    "sp_conv3x3_flip": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_int, _P]),
    "sp_adam_step": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_longlong, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                    ctypes.c_float, _P]),
    "sp_conserve_mass": (ctypes.c_int, [_H, ctypes.c_int]),
    "sp_regional_create": (ctypes.c_int, [ctypes.POINTER(SpDesc), ctypes.POINTER(SpRegionalParams),
                                          ctypes.POINTER(_P)]),
    "sp_regional_upload": (ctypes.c_int, [_P, _P, _SZ]),
    "sp_regional_download": (ctypes.c_int, [_P, _P, _SZ]),
    "sp_regional_step": (ctypes.c_int, [_P, ctypes.c_int]),
    "sp_regional_adjust": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int)]),
    "sp_regional_window": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_double)]),
    "sp_regional_set_dt": (ctypes.c_int, [_P, ctypes.c_double]),
    "sp_regional_set_stream": (ctypes.c_int, [_P, _P]),
    "sp_regional_handle": (_H, [_P]),
    "sp_regional_error": (ctypes.c_char_p, [_P]),
    "sp_regional_destroy": (None, [_P]),
    "sp_region_search": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                        _P, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                        ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]),
    "sp_noalloc_error": (ctypes.c_char_p, []),
    "sp_last_error": (ctypes.c_char_p, [_H]),
    "sp_create_error": (ctypes.c_char_p, []),
    "sp_destroy": (None, [_H]),
}

_lib = None


def lib():
    """The loaded library (loaded on first use; raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                "symphas_b200: %s is missing; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'` or "
                "`make -C symphas_b200/csrc`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc, handle=None):
    if rc != SP_OK:
        L = lib()
        msg = L.sp_last_error(handle) if handle else L.sp_create_error()
        raise SymPhasError(rc, (msg or b"").decode())
