"""The C-ABI library loads on a machine without a GPU and exports every
function declared in include/symphas_b200.h."""
import ctypes
import os
import re

import pytest

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


def _valid_desc(dim):
    d = _capi.SpDesc()
    d.dim = dim
    for a in range(3):
        d.n[a] = 16
    d.dtype, d.model, d.form = _capi.SP_F64, 0, 1
    d.h, d.batch = 1.0, 1
    return d


@pytest.mark.parametrize("dim,acc,word", [(2, 3, b"accuracy"), (3, 4, b"two-dimensional")])
def test_create_rejects_bad_stencil_accuracy_without_gpu_work(dim, acc, word):
    d = _valid_desc(dim)
    d.accuracy = acc  # checked before any device call
    h = _capi._H()
    assert sp.lib().sp_create(ctypes.byref(d), ctypes.byref(h)) == _capi.SP_EINVAL
    assert word in sp.lib().sp_create_error()


def test_struct_layouts_match_the_header(tmp_path):
    """sizeof and field offsets of sp_desc and sp_member as a C compiler lays
    them out from the header, against the ctypes mirrors."""
    import subprocess
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "symphas_b200.h"\n'
        "int main(void) {\n"
        '  printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(sp_desc), offsetof(sp_desc, h),\n'
        "         offsetof(sp_desc, batch), sizeof(sp_member), offsetof(sp_member, dt),\n"
        "         offsetof(sp_member, coeff));\n"
        "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    D, M = _capi.SpDesc, _capi.SpMember
    assert got == [ctypes.sizeof(D), D.h.offset, D.batch.offset, ctypes.sizeof(M), M.dt.offset,
                   M.coeff.offset]


def test_ensemble_rejects_bad_members_without_gpu_work():
    d = _capi.SpDesc()
    d.dim = 2
    mem = (_capi.SpMember * 2)()
    for i, model in enumerate((_capi.SP_MODEL_A, _capi.SP_MODEL_B)):
        mem[i].n[0] = mem[i].n[1] = 32
        mem[i].model = model
    h = _capi._H()
    assert sp.lib().sp_create_ensemble(ctypes.byref(d), mem, 2, ctypes.byref(h)) == _capi.SP_EINVAL
    assert b"AMK" in sp.lib().sp_create_error()
    d.dim = 3
    assert sp.lib().sp_create_ensemble(ctypes.byref(d), mem, 2, ctypes.byref(h)) == _capi.SP_EINVAL
    assert b"two-dimensional" in sp.lib().sp_create_error()
    d.dim = 2
    mem[1].n[0] = 2
    assert sp.lib().sp_create_ensemble(ctypes.byref(d), mem, 2, ctypes.byref(h)) == _capi.SP_EINVAL
