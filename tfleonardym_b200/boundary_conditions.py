"""Fermion boundary conditions (mirror of boundary_conditions.py:10-46).

The reference multiplies the last direction's links on the last time slice
by ``factor``.  The device kernels take that factor as a scalar, so the
providers below carry it in ``lym_time_factor``; any other provider callable
is applied to the gauge tensor itself and the kernels then see periodic links.
"""
import numpy as np
import torch

from . import _lib
from . import lattice as lt

antiperiodic_field_in_t_direction = None
_factor = -1.0
_geometry = None


def set_antiperiodic_field_in_t_direction(lattice_geometry: tuple, factor=-1):
    global antiperiodic_field_in_t_direction, _factor, _geometry
    _geometry = tuple(lattice_geometry)
    _factor = complex(factor)
    antiperiodic_field_in_t_direction = torch.from_numpy(
        _lib.host_antiperiodic_field(_geometry, factor)).to("cuda")


def apply_antiboundary_conditions_in_t_direction(cfg):
    """Return the configuration (or bare (nd,N,N,V) tensor) with the time links twisted."""
    field = antiperiodic_field_in_t_direction
    if isinstance(cfg, lt.Configuration):
        g = cfg.gauge_field.clone()
        g[-1] = g[-1] * field
        return lt.Configuration(gauge_field=g, geometry=cfg.geometry, colors=cfg.colors,
                                number_of_dimensions=cfg.number_of_dimensions)
    g = cfg.clone()
    g[-1] = g[-1] * field
    return g


def _tag(f, factor):
    f.lym_time_factor = complex(factor)
    return f


def time_antiperiodic_provider(factor=None):
    """Provider equivalent to ``lambda x: apply_antiboundary_conditions_in_t_direction(x)``
    that the kernels recognise and apply in registers."""
    fac = _factor if factor is None else complex(factor)
    return _tag(lambda x: apply_antiboundary_conditions_in_t_direction(x), fac)


def periodic_provider():
    return _tag(lambda x: x, 1.0)


def factor_provider(factor):
    """Provider for an arbitrary time-boundary factor (1 periodic, -1 antiperiodic),
    applied by the kernels in registers."""
    f = complex(factor)

    def apply(x):
        g = x.clone()
        geom_last = _geometry[-1] if _geometry else None
        if geom_last is None:
            raise RuntimeError("set_antiperiodic_field_in_t_direction was not called")
        g[-1][..., geom_last - 1::geom_last] *= f
        return g
    return _tag(apply, f)


def provider_factor(provider):
    """(factor, needs_tensor_application) for a boundary_condition_provider."""
    if provider is None:
        return 1.0 + 0j, False
    fac = getattr(provider, "lym_time_factor", None)
    if fac is not None:
        return complex(fac), False
    if provider is apply_antiboundary_conditions_in_t_direction:
        return _factor, False
    return 1.0 + 0j, True
