"""The C-ABI library builds, loads and exports every symbol ippi_lbm.h
declares; without a GPU every entry point fails cleanly (no compute calls)."""
import ctypes as C
import os
import re

import pytest

from conftest import REPO

ip = pytest.importorskip("ippi_lbm")
from ippi_lbm import _lib  # noqa: E402


def header_symbols():
    src = open(os.path.join(REPO, "include", "ippi_lbm.h")).read()
    return sorted(set(re.findall(r"^\w[\w\s\*]*?\b(ippi_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = ip.lib()
    syms = header_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(L, s), s
    assert set(_lib.EXPORTS) <= set(syms)
    assert L.ippi_abi_version() == 3


def test_params_default_is_reference_main():
    p = _lib.Params()
    ip.lib().ippi_params_default(C.byref(p), 2401, 501)
    assert (p.nx, p.ny, p.collision, p.storage, p.les_model) == (2401, 501, 0, 0, 1)
    assert abs(p.tau0 - (0.5 + 6.0 * 501 * 0.1 / 5e5)) < 1e-15
    assert abs(p.cs - 0.173) < 1e-15 and p.plate_x0 == 400 and p.avg_start == 30000


def test_bad_parameters_rejected_before_device_use():
    p = _lib.Params()
    ip.lib().ippi_params_default(C.byref(p), 2, 2)
    h = C.c_void_p()
    assert ip.lib().ippi_create(C.byref(p), C.byref(h)) == _lib.IPPI_ERR_ARG
    ip.lib().ippi_params_default(C.byref(p), 64, 64)
    p.tau0 = 0.5
    assert ip.lib().ippi_create(C.byref(p), C.byref(h)) == _lib.IPPI_ERR_ARG
    assert "tau0" in _lib.last_error()


def test_null_handle_calls_fail_cleanly():
    L = ip.lib()
    assert L.ippi_step(None, 1, 1) == _lib.IPPI_ERR_ARG
    assert L.ippi_download(None, 0, None, 0) == _lib.IPPI_ERR_ARG
    assert L.ippi_destroy(None) == 0
