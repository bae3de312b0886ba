"""The C-ABI library loads on a machine without a GPU and exports every
function declared in include/symphas_b200.h."""
import ctypes
import os
import re

import symphas_b200 as sp
from symphas_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "symphas_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_ ]+\**\s*\**(sp_[a-z_0-9]+)\s*\(", text, re.M)
    return sorted(set(names))


def test_header_declares_the_abi():
    names = declared_functions()
    for n in ("sp_create", "sp_upload", "sp_step", "sp_download", "sp_reduce", "sp_last_error",
              "sp_destroy"):
        assert n in names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_capi.LIB_PATH)
    for name in declared_functions():
        assert hasattr(L, name), name
    assert set(declared_functions()) == set(_capi.SIGNATURES)


def test_binding_loads():
    assert sp.lib() is not None


def test_create_rejects_bad_description_without_gpu_work():
    d = _capi.SpDesc()
    d.dim = 4  # invalid: checked before any device call
    h = _capi._H()
    rc = sp.lib().sp_create(ctypes.byref(d), ctypes.byref(h))
    assert rc == _capi.SP_EINVAL
    assert b"dim" in sp.lib().sp_create_error()
