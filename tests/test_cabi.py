"""The C ABI library: loads, exports what include/qesb.h declares, and
reports errors as status codes (no GPU compute here)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import qesb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if hdr.endswith(".h"):
            text = open(os.path.join(ROOT, "include", hdr)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"\b(qesb_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(qesb.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in qesb.lib().qesb_version()


def test_create_rejects_bad_grid():
    g = qesb.Grid(2, 5, 5, 1.0, 1.0, None)
    h = C.c_void_p()
    st = qesb.lib().qesb_create(C.byref(g), 1e-9, 0, C.byref(h))
    assert st == 1 and not h
    assert b"grid" in qesb.lib().qesb_last_error()


def test_create_without_gpu_is_an_error_not_a_crash():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    d = qesb.Domain(8, 8, 6, 1.0, 1.0, 1.0)
    with pytest.raises(qesb.QesbError) as ei:
        qesb.Solver_B200(d, 1e-9)
    assert ei.value.status == 6


def test_null_handle_calls_fail_cleanly():
    L = qesb.lib()
    assert L.qesb_reset_lambda(None) == 1
    assert L.qesb_solve(None, 10, None, None, None, None) == 1
    assert L.qesb_set_option(None, b"path", 1) == 1
    assert L.qesb_destroy(None) == 0


def test_factory_rejects_other_types():
    d = qesb.Domain(8, 8, 6, 1.0, 1.0, 1.0)
    with pytest.raises(qesb.QesbError, match="Invalid solver type"):
        qesb.SolverFactory.create(qesb.CPU_Type, d, 1e-9)


def test_domain_index_math_matches_reference_formulas():
    d = qesb.Domain(10, 7, 5, 2.0, 3.0, 1.0)
    assert (d.nx(), d.ny(), d.nz()) == (11, 8, 7)
    assert d.numCellCentered() == 10 * 7 * 6
    assert d.numFaceCentered() == 11 * 8 * 7
    assert d.cell(3, 4, 5) == 3 + 4 * 10 + 5 * 70
    assert d.face(3, 4, 5) == 3 + 4 * 11 + 5 * 88
    assert d.z_face[1] == 0 and d.z[1] == 0.5 and d.z_face[0] == -1


def test_every_called_entry_point_has_a_ctypes_signature():
    """Floats and 64-bit sizes only cross ctypes correctly with declared
    argtypes: every qesb_* the Python package calls must be in the table."""
    pkg = os.path.join(ROOT, "qes-public_b200", "qesb")
    called = set()
    for fn in os.listdir(pkg):
        if fn.endswith(".py"):
            called |= set(re.findall(r"lib\(\)\.(qesb_[a-z0-9_]+)", open(os.path.join(pkg, fn)).read()))
    L = qesb.lib()
    for name in sorted(called):
        assert getattr(L, name).argtypes is not None, name
    assert len(called) >= 20


def test_noalloc_rejects_rows_beyond_the_launch_limit():
    """A long thin grid under the cell cap still needs Ny + 1 <= 65535 rows
    in a launch's y dimension: refused as an argument error before any
    device work (so this runs without a GPU)."""
    d = qesb.Domain(3, 65535, 2, 2.0, 2.0, 1.0)
    with pytest.raises(qesb.QesbError) as ei:
        qesb.solve_noalloc(d, 1e-3, 10, *([16] * 14))
    assert ei.value.status == 1
    assert "65534 rows" in str(ei.value)
