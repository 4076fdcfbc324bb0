"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and its host-side table builders are bit-exact with the
reference's lattice.py:86-120 / boundary_conditions.py:10-20 (golden tables)."""
import ctypes
import os
import re

import numpy as np

from tests.conftest import ROOT, load_golden
from tfleonardym_b200 import _lib

HEADER = os.path.join(ROOT, "include", "lym.h")


def header_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lym_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(lib, s), s
    # and the ctypes signature table covers exactly the header
    assert set(syms) == set(_lib.SIGNATURES)


def test_version_and_status_strings():
    lib = _lib.lib()
    assert lib.lym_version() >= 10000
    assert lib.lym_status_string(_lib.LYM_ERR_NOT_CONVERGED) == b"not converged"


def test_host_tables_bit_exact():
    z = load_golden("tables")
    for key in sorted({k.split("/")[0] for k in z}):
        geom = tuple(int(g) for g in key.split("x"))
        sup, sdn, coords = _lib.host_lookup_tables(geom)
        np.testing.assert_array_equal(sup, z[f"{key}/sup"])
        np.testing.assert_array_equal(sdn, z[f"{key}/sdn"])
        np.testing.assert_array_equal(coords, z[f"{key}/coords"])
        np.testing.assert_array_equal(_lib.host_antiperiodic_field(geom), z[f"{key}/bc"])


def test_bad_arguments_are_rejected():
    lib = _lib.lib()
    dims = _lib.dims_array((4, 4))
    assert lib.lym_lookup_tables(0, dims, None, None, None) == _lib.LYM_ERR_BAD_ARG
    assert lib.lym_lookup_tables(2, dims, None, None, None) == _lib.LYM_ERR_BAD_ARG
    bad = _lib.dims_array((4, 0))
    out = np.empty((2, 16), np.int64)
    assert lib.lym_lookup_tables(2, bad, out.ctypes.data, None, None) == _lib.LYM_ERR_BAD_ARG
    assert b"extent" in lib.lym_last_error()


def test_solver_entry_points_validate_before_any_device_work():
    """The multi-lattice and even-odd multishift entry points reject bad arguments
    (null pointers, counts out of range) before touching a device."""
    import ctypes
    lib = _lib.lib()
    prm = _lib.SolverParams(1e-10, 100, 1, 0.1, 0, 8, 0, 0, 0, 0.0)
    reps = (_lib.SolverReport * 4)()
    one = (ctypes.c_void_p * 1)(None)
    k = (ctypes.c_double * 1)(0.1)
    n = (ctypes.c_int * 1)(1)
    assert lib.lym_wilson_solve_multi(0, one, k, None, n, one, one, ctypes.byref(prm), reps, None) == \
        _lib.LYM_ERR_BAD_ARG
    assert lib.lym_wilson_solve_multi(1, None, k, None, n, one, one, ctypes.byref(prm), reps, None) == \
        _lib.LYM_ERR_BAD_ARG
    assert lib.lym_wilson_solve_multi(1, one, k, None, n, one, one, None, reps, None) == _lib.LYM_ERR_BAD_ARG
    # a null first gauge object is refused before its fields are read
    assert lib.lym_wilson_solve_multi(1, one, k, None, n, one, one, ctypes.byref(prm), reps, None) == \
        _lib.LYM_ERR_BAD_ARG
    assert b"lattice 0" in lib.lym_last_error()
    sh =(ctypes.c_double * 1)(0.1)
    assert lib.lym_multishift_solve_eo(None, 0.1, 1, 1, sh, None, None, ctypes.byref(prm), reps, None) == \
        _lib.LYM_ERR_BAD_ARG
    zero = _lib.SolverParams(0.0, 100, 1, 0.1, 0, 8, 0, 0, 0, 0.0)
    assert lib.lym_wilson_solve_multi(1, one, k, None, n, one, one, ctypes.byref(zero), reps, None) == \
        _lib.LYM_ERR_BAD_ARG
    assert b"tol" in lib.lym_last_error()


def test_multi_lattice_hmc_step_validates_before_any_device_work():
    """lym_gauge_hmc_step_multi refuses an empty or oversized lattice list and null
    arrays or entries before reading a lattice or launching anything."""
    import ctypes
    lib = _lib.lib()
    one = (ctypes.c_void_p * 1)(None)
    nc = (ctypes.c_int * 1)(3)
    beta = (ctypes.c_double * 1)(5.6)
    f = lib.lym_gauge_hmc_step_multi
    assert f(0, one, nc, beta, one, one, 0.1, 0.1, None) == _lib.LYM_ERR_BAD_ARG
    assert f(257, one, nc, beta, one, one, 0.1, 0.1, None) == _lib.LYM_ERR_BAD_ARG
    assert f(1, None, nc, beta, one, one, 0.1, 0.1, None) == _lib.LYM_ERR_BAD_ARG
    assert f(1, one, nc, beta, one, one, 0.1, 0.1, None) == _lib.LYM_ERR_BAD_ARG
    assert b"lattice 0" in lib.lym_last_error()
