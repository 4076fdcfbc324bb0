"""Wilson gauge action (mirror of gauge_action.py:5-113) on the GPU.

``force`` is one fused kernel per link (staples + traceless anti-Hermitian
projection, lym_gauge_force); ``force_into_momenta`` fuses the momentum update
of hmc.py:59-61 as well, so the force is never materialised.
"""
import ctypes

import torch

from . import _dev, _lib
from . import lattice as lt


def _lat(cfg):
    return lt.get_lattice(tuple(cfg.geometry))


class yang_mills:  # noqa: N801 - reference name
    def __init__(self, cfg: lt.Configuration, beta):
        self.beta = beta
        self.cfg = cfg

    def set_gauge_configuration(self, cfg):
        self.cfg = cfg

    def force(self):
        u = _dev.as_c128(self.cfg.gauge_field)
        f = torch.empty_like(u)
        _lib.check(_lib.lib().lym_gauge_force(_lat(self.cfg).handle, u.shape[1], float(self.beta), _dev.ptr(u),
                                              _dev.ptr(f), None, 0.0, _dev.stream()), "lym_gauge_force")
        return f

    def force_into_momenta(self, momenta, eps):
        """momenta += eps * force() in one kernel (in place)."""
        u = _dev.as_c128(self.cfg.gauge_field)
        _lib.check(_lib.lib().lym_gauge_force(_lat(self.cfg).handle, u.shape[1], float(self.beta), _dev.ptr(u),
                                              None, _dev.ptr(momenta), float(eps), _dev.stream()), "lym_gauge_force")
        return momenta

    def energy(self):
        re, _ = plaquette_trace_sum(self.cfg)
        return -self.beta * re / self.cfg.gauge_field.shape[1]


def plaquette_trace_sum(cfg):
    """(Re, Im) of sum_{x, mu<nu} Tr P_mu nu(x) (gauge_action.py:110-113 summed over planes)."""
    u = _dev.as_c128(cfg.gauge_field)
    out = (ctypes.c_double * 2)()
    _lib.check(_lib.lib().lym_plaquette_sum(_lat(cfg).handle, u.shape[1], _dev.ptr(u), out, _dev.stream()),
               "lym_plaquette_sum")
    return out[0], out[1]
