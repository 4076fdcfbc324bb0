"""Fermion measurements (mirror of the reference's fermion_measurements.py on the GPU).

``pion_correlator`` and ``chiral_condensate`` keep the reference's signatures
and results (fermion_measurements.py:41-115).  Their propagators go through
``dirac.Propagator``; by default, for a fundamental-representation Wilson
operator, every source is solved in one batched even-odd CG call
(lym_wilson_solve, FP64 reliable updates, true relative residual 1e-12) instead
of one BiCGStab run per source, and the per-slice sums of the correlator run in
lym_timeslice_sums.  ``inverter=`` takes any solver with the reference's
``solve(operator, source)`` (for instance ``dirac_solver.biconjugate_gradient``,
the reference's own choice, which the adjoint representation uses).
"""
import numpy as np
import torch

from . import _dev, _lib, dirac, dirac_solver, lie_generators
from .measurements import Measurement


def generate_random_z2_noise(volume, nc=3, spinor_dimension=4, representation="fundamental", generator=None):
    """+-1 noise (fermion_measurements.py:11-24); adjoint: sum_a n_a T^a."""
    dev = torch.device("cuda")
    if representation == "fundamental":
        bits = torch.randint(0, 2, (spinor_dimension, nc, volume), device=dev, generator=generator)
        return ((bits.to(torch.float64) - 0.5) * 2).to(torch.complex128)
    if representation == "adjoint":
        bits = torch.randint(0, 2, (spinor_dimension, nc * nc - 1, volume), device=dev, generator=generator)
        v = ((bits.to(torch.float64) - 0.5) * 2).to(torch.complex128)
        gens = torch.from_numpy(lie_generators.generators(nc, "fundamental")).to(dev)
        return torch.einsum("mic,ijk->mjkc", v, gens)
    raise RuntimeError(f"Unknown representation {representation}")


def generate_point_source(site, color, spin, volume, nc=3, spinor_dimension=4, representation="fundamental"):
    """Unit source at (spin, colour, site) (fermion_measurements.py:27-38); adjoint: T^color."""
    if representation == "fundamental":
        v = torch.zeros((spinor_dimension, nc, volume), dtype=torch.complex128, device="cuda")
        v[spin, color, site] = 1
        return v
    if representation == "adjoint":
        v = torch.zeros((spinor_dimension, nc, nc, volume), dtype=torch.complex128, device="cuda")
        v[spin, :, :, site] = torch.from_numpy(lie_generators.generators(nc, "fundamental")[color]).to(v.device)
        return v
    raise RuntimeError(f"Unknown representation {representation}")


def _default_inverter(dirac_operator, tol):
    if getattr(dirac_operator, "representation", "fundamental") == "fundamental":
        return dirac_solver.conjugate_gradient(max_steps=20000, tol=1e-12)
    return dirac_solver.biconjugate_gradient(5000, tol)


def slice_sums(solutions, dirac_operator, direction):
    """sum over the solutions of the per-site colour-spin products, summed per slice
    of `direction` (fermion_measurements.py:76-90), as a complex numpy array."""
    s = _dev.as_c128(solutions)
    adjoint = dirac_operator.representation == "adjoint"
    per = 5 if adjoint else 4
    if s.dim() == per - 1:
        s = s[None]
    length = dirac_operator.cfg.geometry[direction]
    out = torch.empty(2 * length, dtype=torch.float64, device=s.device)
    _lib.check(_lib.lib().lym_timeslice_sums(dirac_operator.lattice.handle, int(direction), s.shape[0], s.shape[1],
                                             dirac_operator.number_of_colors, int(adjoint), _dev.ptr(s),
                                             _dev.ptr(out), _dev.stream()), "lym_timeslice_sums")
    o = out.cpu().numpy()
    return o[0::2] + 1j * o[1::2]


def pion_correlator(dirac_operator, correlator_direction, lookup_tables=None, global_summator=None, inverter=None):
    """Pion correlator from the ns x colour point sources at site 0 (fermion_measurements.py:41-96)."""
    inverter = inverter or _default_inverter(dirac_operator, 1e-13)
    propagator = dirac.Propagator(dirac_operator, inverter)
    nc = dirac_operator.number_of_colors
    ncol = nc * nc - 1 if dirac_operator.representation == "adjoint" else nc
    sources = torch.stack([generate_point_source(0, c, spin, dirac_operator.volume, nc, dirac_operator.spinor_dimension,
                                                 dirac_operator.representation)
                           for spin in range(dirac_operator.spinor_dimension) for c in range(ncol)])
    solutions = propagator.apply(sources)
    correlator = slice_sums(solutions, dirac_operator, correlator_direction)
    if global_summator is not None:
        correlator = np.array([global_summator(c) for c in correlator])
    return Measurement(name="pion_operator", value=np.array(correlator), geometry=dirac_operator.cfg.geometry,
                       colors=dirac_operator.cfg.colors)


def chiral_condensate(dirac_operator, num_estimators=20, inverter=None, sources=None, generator=None):
    """Mean over Z2-noise estimators of <source, propagator(source)> / V
    (fermion_measurements.py:99-115).  ``sources`` (num_estimators stacked) replaces
    the random noise when given."""
    inverter = inverter or _default_inverter(dirac_operator, 1e-10)
    propagator = dirac.Propagator(dirac_operator, inverter)
    if sources is None:
        sources = torch.stack([generate_random_z2_noise(dirac_operator.volume, dirac_operator.number_of_colors,
                                                        dirac_operator.spinor_dimension, dirac_operator.representation,
                                                        generator) for _ in range(num_estimators)])
    sources = _dev.as_c128(sources)
    solutions = propagator.apply(sources)
    values = [_dev.cdot(sources[i], solutions[i]) / dirac_operator.volume for i in range(sources.shape[0])]
    return Measurement(name="chiral_condensate", value=np.mean(values), geometry=dirac_operator.cfg.geometry,
                       colors=dirac_operator.cfg.colors)
