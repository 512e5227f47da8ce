"""The C-ABI library loads and exports every symbol include/*.h declares.

Runs without a GPU: only dlopen/dlsym, no compute call.
"""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT

LIB = os.path.join(ROOT, "krigekit_b200", "libkrigecuda.so")


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(?:int|void|char)\s*\**\s*(krige_\w+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_reference_entry_points():
    names = _declared()
    for ref in ("krige_create", "krige_initialize", "krige_set_obs", "krige_set_vgm", "krige_set_grid",
                "krige_set_search", "krige_solve", "krige_get_estimate_all", "krige_get_variance_all",
                "krige_get_last_error", "krige_solver_stats"):
        assert ref in names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.fail("libkrigecuda.so is not built (run python -m krigekit_b200.build)")
    lib = ctypes.CDLL(LIB)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"


def test_error_slot_without_device():
    lib = ctypes.CDLL(LIB)
    lib.krige_solve.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int]
    lib.krige_solve.restype = ctypes.c_int
    assert lib.krige_solve(ctypes.c_int64(999999), 0, -1) == 1
    buf = ctypes.create_string_buffer(256)
    lib.krige_get_last_error(buf, 256)
    assert b"invalid kriging handle" in buf.value
