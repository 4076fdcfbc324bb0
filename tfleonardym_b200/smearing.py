"""Reunitarisation and APE smearing (mirror of the reference's smearing.py on the GPU).

``unitary_sqrt_projection`` (smearing.py:17-31): X (X^dag X)^{-1/2} / det^{1/N}
(lym_unitary_projection).  ``ape_smearing`` (smearing.py:34-51): summed staples
(staples.get_staple_sums, lym_staples), the fat-link combination (lym_caxpby) and
the projection.
``multi_smearing_operators`` (smearing.py:54-86) keeps the reference's loop.
"""
import torch

from . import _dev, _lib
from . import lattice as lt
from .measurements import Measurement


def unitary_sqrt_projection(link_config):
    x = _dev.as_c128(link_config)
    out = torch.empty_like(x)
    _lib.check(_lib.lib().lym_unitary_projection(x.shape[0], x.shape[1], x.shape[-1], _dev.ptr(x), _dev.ptr(out),
                                                 _dev.stream()), "lym_unitary_projection")
    return out


def ape_smearing(cfg, rho, no_smear_direction=3):
    """P_SU(N)[(rho/6) S_mu + (1 - rho) U_mu]; a direction without staples (the
    no-smear one) gets rho U_mu + (1 - rho) U_mu, as in the reference."""
    from .staples import get_staple_sums
    u = _dev.as_c128(cfg.gauge_field)
    nd = u.shape[0]
    nodir = no_smear_direction if 0 <= no_smear_direction < nd else -1
    st = get_staple_sums(cfg, nodir)
    fat = torch.empty_like(u)
    for mu in range(nd):
        if mu == nodir:
            fat[mu] = _dev.axpby(rho, u[mu], 1 - rho, u[mu])
        else:
            fat[mu] = _dev.axpby(rho / 6, st[mu], 1 - rho, u[mu])
    return lt.Configuration(gauge_field=unitary_sqrt_projection(fat), geometry=cfg.geometry, colors=cfg.colors,
                            number_of_dimensions=nd)


def multi_smearing_operators(cfg, operators_to_measure, smearing_levels=10, rho=0.3, no_smear_direction=3, skip=1):
    """Measure, smear `skip` times, measure again, for smearing_levels // skip levels
    (smearing.py:54-86)."""
    result = []
    next_cfg = cfg
    for operator in operators_to_measure:
        result.extend(operator(next_cfg))
    for level in range(smearing_levels // skip):
        for _ in range(skip):
            next_cfg = ape_smearing(next_cfg, rho, no_smear_direction=no_smear_direction)
        for operator in operators_to_measure:
            for meas in operator(next_cfg):
                result.append(Measurement(name=meas.name, value=meas.value, geometry=meas.geometry,
                                          colors=meas.colors, smearing_levels=level))
    return result
