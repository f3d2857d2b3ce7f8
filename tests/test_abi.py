"""The C-ABI library loads without a GPU and exports every symbol that
include/tmsolve.h declares; the Python mirror binds all of them."""
import ctypes
import os
import re

from conftest import ROOT
from nissa_b200 import _lib


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "tmsolve.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tms_[A-Za-z0-9_]+)\s*\(", text)))


def test_library_exports_declared_symbols():
    lib = ctypes.CDLL(_lib.load().__dict__["_name"])
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_python_mirror_binds_every_symbol():
    assert set(declared_symbols()) == set(_lib.SIGNATURES)


def test_library_is_built_for_sm100a():
    from nissa_b200 import build
    assert "arch=compute_100a,code=sm_100a" in build.NVCC_FLAGS


def test_bad_arguments_rejected_without_gpu():
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.tms_create(ctypes.byref(h), 5, 4, -1.0, 0) == 3  # odd extent -> BAD_ARG
    assert lib.tms_create(None, 4, 4, -1.0, 0) == 3
