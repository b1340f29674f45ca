"""The C-ABI library on the CPU: it loads, exports every entry point declared
in include/gpv.h, keeps the documented record layouts, and fails cleanly
(error code + message, no abort) when no GPU is present.  No compute call is
made here."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

from conftest import HAS_GPU, ROOT

HEADER = os.path.join(ROOT, "include", "gpv.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gpv_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("gpv_image_create", "gpv_image_destroy", "gpv_solve_batch", "gpv_solve_batch_device",
                 "gpv_last_error", "gpv_version", "gpv_context_create"):
        assert must in names


def test_library_exports_every_declared_symbol(gpv_mod):
    from gpv import _lib
    L = ct.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding gives every declared function a signature
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_record_layouts(gpv_mod, oracle):
    from gpv import _lib
    assert _lib.DESC_DTYPE.itemsize == 120
    assert _lib.RESULT_DTYPE.itemsize == 200
    assert ct.sizeof(_lib.SolveParams) == 48
    assert _lib.SolveParams.mask.offset == 32 and _lib.SolveParams.history.offset == 40
    # the oracle reads the same records
    assert oracle.DESC_DTYPE == _lib.DESC_DTYPE
    assert oracle.RESULT_DTYPE == _lib.RESULT_DTYPE


def test_version_and_abi(gpv_mod):
    from gpv import _lib
    assert _lib.lib().gpv_abi_version() == 1
    assert b"sm_100a" in _lib.lib().gpv_version()


@pytest.mark.skipif(HAS_GPU, reason="checks the no-GPU failure path")
def test_context_create_fails_cleanly_without_gpu(gpv_mod):
    from gpv import _lib
    h = ct.c_void_p()
    rc = _lib.lib().gpv_context_create(0, ct.byref(h))
    assert rc != 0 and not h.value
    assert len(_lib.last_error()) > 0


def test_null_arguments_are_rejected(gpv_mod):
    from gpv import _lib
    L = _lib.lib()
    assert L.gpv_image_destroy(None) == 0          # NULL handle: no-op
    assert L.gpv_context_destroy(None) == 0
    assert L.gpv_image_shape(None, None, None, None) == _lib_err(-1)
    assert "NULL" in _lib.last_error() or "img" in _lib.last_error()
    assert L.gpv_solve_batch(None, None, None, None, 0, None, None) == -1
    assert L.gpv_image_create(None, None, 1, 4, 4, 20, 0, None) == -1


def _lib_err(v):
    return v


def test_python_api_validation(gpv_mod):
    with pytest.raises(ValueError):
        gpv_mod.Mask("local")                           # shape required
    with pytest.raises(RuntimeError):
        gpv_mod.Mask("local", shape="circle", size=0)   # LocalMask::circle(0) -> Err
    with pytest.raises(ValueError):
        gpv_mod.Mask("bogus")
    with pytest.raises(NotImplementedError):
        gpv_mod.Mask("local", shape="square", size=5)
    with pytest.raises(ValueError):
        gpv_mod.Image(filepath="a.png", image_gs=np.zeros((4, 4)))
    assert gpv_mod.Mask("local", shape="circle", size=25).n_px == 1961
    d = gpv_mod.make_desc([[1.0, 2.0], [3.0, 4.0]], [5, 6], 2, [[0.1, 0.2]])
    assert list(d["radius"]) == [5, 6] and list(d["order"]) == [2, 2]
    assert d["p0"][1, 0] == 0.1 and d["p0"][0, 2] == 0.0
