"""B200 (sm_100a) implementation of the TfLeonardYM Wilson-fermion / SU(N)
gauge hot path, behind mirrors of the reference's own Python modules:

    lattice, translate, boundary_conditions, algebra_utils, dirac,
    dirac_solver, gauge_action, staples, measurements, smearing, hmc,
    fermion_action, approximations

All arithmetic runs in liblym.so (hand-written CUDA, include/lym.h) through
ctypes; tensors are complex128 CUDA tensors in the reference's layouts.
"""
from . import _lib  # noqa: F401

__all__ = ["lattice", "translate", "boundary_conditions", "algebra_utils", "dirac", "dirac_solver",
           "gauge_action", "staples", "measurements", "smearing", "hmc", "fermion_action", "approximations"]
