"""ctypes binding of liblym.so (the C ABI declared in include/lym.h).

There is no CPU fallback: every device entry point raises if the library or a
CUDA device is missing.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblym.so")

LYM_OK = 0
LYM_ERR_BAD_ARG = 1
LYM_ERR_BAD_SHAPE = 2
LYM_ERR_UNSUPPORTED = 3
LYM_ERR_NOT_CONVERGED = 4
LYM_ERR_CUDA = 5
LYM_ERR_OOM = 6
LYM_ERR_REJECTED = 7
LYM_ERR_TIMEOUT = 8

PREC = {"f64": 0, "f32": 1, "f16": 2, "bf16": 3}

c_void_p = ctypes.c_void_p
c_int = ctypes.c_int
c_double = ctypes.c_double
c_int64 = ctypes.c_int64
c_uint = ctypes.c_uint
P = ctypes.POINTER


class SolverParams(ctypes.Structure):
    _fields_ = [("tol", c_double), ("max_iter", c_int), ("precision", c_int),
                ("delta", c_double), ("hermitian", c_int), ("chunk", c_int), ("rhs_per_thread", c_int),
                ("compressed_links", c_int), ("mixed_fma", c_int), ("switch_residual", c_double)]


class SolverReport(ctypes.Structure):
    _fields_ = [("status", c_int), ("iterations", c_int), ("reliable_updates", c_int),
                ("true_residual", c_double), ("kernel_launches", c_int64), ("rhs_per_thread", c_int),
                ("compressed_links", c_int), ("mixed_fma", c_int)]


# name -> (restype, argtypes); every symbol include/lym.h declares
SIGNATURES = {
    "lym_version": (c_int, []),
    "lym_last_error": (ctypes.c_char_p, []),
    "lym_status_string": (ctypes.c_char_p, [c_int]),
    "lym_lookup_tables": (c_int, [c_int, P(c_int64), c_void_p, c_void_p, c_void_p]),
    "lym_antiperiodic_field": (c_int, [c_int, P(c_int64), c_double, c_double, c_void_p]),
    "lym_lattice_create": (c_int, [c_int, P(c_int64), P(c_void_p)]),
    "lym_lattice_destroy": (c_int, [c_void_p]),
    "lym_lattice_tables_device": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "lym_wilson_apply": (c_int, [c_void_p, c_int, c_double, c_int, c_double, c_double,
                                 c_void_p, c_void_p, c_void_p, c_void_p]),
    "lym_wilson_apply_batch": (c_int, [c_void_p, c_int, c_double, c_int, c_double, c_double,
                                       c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "lym_cdot": (c_int, [c_int64, c_void_p, c_void_p, P(c_double), c_void_p]),
    "lym_caxpby": (c_int, [c_int64, P(c_double), c_void_p, P(c_double), c_void_p, c_void_p]),
    "lym_cdot_batch_noalloc": (c_int, [c_int, c_int64, c_void_p, c_void_p, P(c_double), c_void_p]),
    "lym_gauge_create": (c_int, [c_void_p, c_int, c_void_p, c_double, c_double, c_uint, c_void_p,
                                 P(c_void_p)]),
    "lym_gauge_update": (c_int, [c_void_p, c_void_p, c_void_p]),
    "lym_gauge_destroy": (c_int, [c_void_p]),
    "lym_wilson_solve": (c_int, [c_void_p, c_double, c_int, c_void_p, c_void_p, P(SolverParams),
                                 P(SolverReport), c_void_p]),
    "lym_dslash_eo": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p]),
    "lym_wilson_solve_multi": (c_int, [c_int, P(c_void_p), P(c_double), P(c_double), P(c_int), P(c_void_p),
                                       P(c_void_p), P(SolverParams), P(SolverReport), c_void_p]),
    "lym_multishift_solve": (c_int, [c_void_p, c_double, c_int, P(c_double), c_void_p, c_void_p,
                                     c_double, c_int, P(c_int), c_void_p]),
    "lym_multishift_solve_eo": (c_int, [c_void_p, c_double, c_int, c_int, P(c_double), c_void_p, c_void_p,
                                        P(SolverParams), P(SolverReport), c_void_p]),
    "lym_mmmr_solve": (c_int, [c_void_p, c_double, c_int, P(c_double), c_void_p, c_void_p, c_int,
                               c_double, c_double, P(c_int), c_void_p]),
    "lym_gauge_force": (c_int, [c_void_p, c_int, c_double, c_void_p, c_void_p, c_void_p, c_double,
                                c_void_p]),
    "lym_staples": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p]),
    "lym_staple_terms": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p]),
    "lym_momenta_from_normals": (c_int, [c_int, c_int, c_int64, c_void_p, c_void_p, c_void_p]),
    "lym_gauge_hmc_step_multi": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_double,
                                         c_double, c_void_p]),
    "lym_plaquette_sum": (c_int, [c_void_p, c_int, c_void_p, P(c_double), c_void_p]),
    "lym_momenta_energy": (c_int, [c_int, c_int, c_int64, c_void_p, P(c_double), c_void_p]),
    "lym_update_momenta": (c_int, [c_int64, c_void_p, c_void_p, c_double, c_void_p]),
    "lym_update_links": (c_int, [c_int, c_int, c_int64, c_void_p, c_void_p, c_double, c_int, c_void_p]),
    "lym_unitary_projection": (c_int, [c_int, c_int, c_int64, c_void_p, c_void_p, c_void_p]),
    "lym_fermion_force": (c_int, [c_void_p, c_int, c_double, c_int, c_double, c_double, c_void_p, c_int,
                                  P(c_double), c_void_p, c_void_p, c_int, c_double, c_void_p, c_void_p]),
    "lym_wilson_apply_adjoint": (c_int, [c_void_p, c_int, c_double, c_int, c_double, c_double, c_void_p,
                                         c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "lym_adjoint_links": (c_int, [c_void_p, c_int, c_double, c_double, c_void_p, c_void_p, c_void_p]),
    "lym_decode_xdr_gauge": (c_int, [c_int, c_int, c_int64, c_void_p, c_void_p, c_void_p]),
    "lym_path_product": (c_int, [c_void_p, c_int, c_void_p, c_int, P(c_int), c_int, c_void_p, c_void_p]),
    "lym_slice_sums": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "lym_timeslice_sums": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "lym_fermion_force_adjoint": (c_int, [c_void_p, c_int, c_double, c_int, c_double, c_double, c_void_p, c_int,
                                          P(c_double), c_void_p, c_void_p, c_int, c_double, c_void_p,
                                          c_void_p]),
}

_lib = None


class LymError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(msg)
        self.status = status


class NotConverged(LymError):
    pass


def lib():
    """Load liblym.so once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m tfleonardym_b200.build` "
                              "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status, what=""):
    if status == LYM_OK:
        return
    L = lib()
    msg = f"{what}: {L.lym_status_string(status).decode()}: {L.lym_last_error().decode()}"
    if status == LYM_ERR_NOT_CONVERGED:
        raise NotConverged(status, msg)
    if status in (LYM_ERR_BAD_SHAPE, LYM_ERR_UNSUPPORTED):
        # the reference raises RuntimeError for both (algebra_utils.py:6-7, dirac.py:299-300)
        raise RuntimeError(msg)
    raise LymError(status, msg)


def dims_array(geometry):
    arr = (c_int64 * len(geometry))(*[int(g) for g in geometry])
    return arr


def host_lookup_tables(geometry):
    """sup, sdn, coords as int64 (nd, V) numpy arrays (lattice.py:86-120)."""
    nd = len(geometry)
    vol = int(np.prod(geometry))
    sup = np.empty((nd, vol), dtype=np.int64)
    sdn = np.empty((nd, vol), dtype=np.int64)
    coords = np.empty((nd, vol), dtype=np.int64)
    check(lib().lym_lookup_tables(nd, dims_array(geometry), sup.ctypes.data, sdn.ctypes.data,
                                  coords.ctypes.data), "lym_lookup_tables")
    return sup, sdn, coords


def host_antiperiodic_field(geometry, factor=-1):
    vol = int(np.prod(geometry))
    out = np.empty(vol, dtype=np.complex128)
    f = complex(factor)
    check(lib().lym_antiperiodic_field(len(geometry), dims_array(geometry), f.real, f.imag,
                                       out.ctypes.data), "lym_antiperiodic_field")
    return out
