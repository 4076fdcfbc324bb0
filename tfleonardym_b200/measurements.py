"""Gauge measurements (mirror of the reference's measurements.py on the GPU).

Every observable is a trace of a link product along a closed path: the products
run in lym_path_product (one thread per starting site), the sums over slices in
lym_slice_sums and the totals in lym_cdot / lym_plaquette_sum.  Signatures,
orders and normalisations are the reference's (measurements.py:22-290).
"""
import ctypes
from collections import namedtuple

import numpy as np
import torch

from . import _dev, _lib
from . import lattice as lt
from .gauge_action import plaquette_trace_sum

Measurement = namedtuple("Measurement", ["geometry", "colors", "value", "name", "smearing_levels"])
Measurement.__new__.__defaults__ = (None, None, None, None, 0)


def plaquette(cfg) -> Measurement:
    nd, nc = cfg.gauge_field.shape[0], cfg.gauge_field.shape[1]
    vol = cfg.gauge_field.shape[-1]
    re, _ = plaquette_trace_sum(cfg)
    return Measurement(name="plaquette", value=re / (nd * (nd - 1) // 2 * nc * vol), geometry=cfg.geometry,
                       colors=nc)


def _lattice(cfg):
    return lt.get_lattice(tuple(cfg.geometry))


def path_field(cfg, steps, trace=True):
    """Per site, Tr (or the matrix) of the link product along `steps`
    (+(mu+1) forward, -(mu+1) backward)."""
    u = _dev.as_c128(cfg.gauge_field)
    nc, vol = u.shape[1], u.shape[-1]
    out = torch.empty((vol,) if trace else (nc, nc, vol), dtype=torch.complex128, device=u.device)
    arr = (ctypes.c_int * len(steps))(*[int(s) for s in steps])
    _lib.check(_lib.lib().lym_path_product(_lattice(cfg).handle, nc, _dev.ptr(u), len(steps), arr, int(trace),
                                           _dev.ptr(out), _dev.stream()), "lym_path_product")
    return out


def _total(field):
    ones = torch.ones_like(field)
    return _dev.cdot(ones, field)  # sum of the field (conj(1) = 1)


def _slice_sums(cfg, field, direction, mask_direction=-1):
    length = cfg.geometry[direction]
    out = torch.empty(2 * length, dtype=torch.float64, device=field.device)
    _lib.check(_lib.lib().lym_slice_sums(_lattice(cfg).handle, int(direction), int(mask_direction),
                                         _dev.ptr(_dev.as_c128(field)), _dev.ptr(out), _dev.stream()),
               "lym_slice_sums")
    o = out.cpu().numpy()
    return o[0::2] + 1j * o[1::2]


def temporal_plaquette(cfg) -> Measurement:
    """measurements.py:46-66."""
    nd, nc, vol = cfg.gauge_field.shape[0], cfg.gauge_field.shape[1], cfg.gauge_field.shape[-1]
    t = nd - 1
    tot = sum(_total(path_field(cfg, [mu + 1, t + 1, -(mu + 1), -(t + 1)])) for mu in range(nd - 1))
    return Measurement(name="temporal_plaquette", value=np.real(tot) / ((nd - 1) * nc * vol), geometry=cfg.geometry,
                       colors=cfg.colors)


def polyakov_loop_field(cfg, direction):
    """Trace of the links around the compact `direction` at every site (measurements.py:74-84)."""
    return path_field(cfg, [direction + 1] * cfg.geometry[direction])


def wilson_lines_field(cfg, direction, maxT):  # noqa: N803 - reference argument name
    """[U(x), U(x)U(x+d), ...] up to maxT + 1 links, each (N, N, V) (measurements.py:87-96)."""
    return [path_field(cfg, [direction + 1] * (k + 1), trace=False) for k in range(maxT + 1)]


def wilson_loops(cfg, direction_R, direction_T, max_R, max_T):  # noqa: N803 - reference argument names
    """Rectangular r x t Wilson loops, r = 1..max_R, t = 1..max_T (measurements.py:99-140)."""
    nc, vol = cfg.gauge_field.shape[1], cfg.gauge_field.shape[-1]
    a, b = direction_R + 1, direction_T + 1
    loops = []
    for r in range(1, max_R + 1):
        for t in range(1, max_T + 1):
            field = path_field(cfg, [a] * r + [b] * t + [-a] * r + [-b] * t)
            loops.append(Measurement(name=f"wilson_loop_{r}_{t}", value=_total(field) / (nc * vol),
                                     geometry=cfg.geometry, colors=cfg.colors))
    return loops


def polyakov_operators(cfg, correlator_direction=2, polyakov_direction=3):
    """Meson operator, Polyakov-loop correlator and Polyakov loop (measurements.py:143-194;
    the meson pairs P(x) with P(x + e_1), as the reference does)."""
    vol = cfg.gauge_field.shape[-1]
    lat = _lattice(cfg)
    p = polyakov_loop_field(cfg, polyakov_direction)
    meson = p * torch.conj(lt.mth_translate(p, 1, +1, lat))
    count = vol // (cfg.geometry[correlator_direction] * cfg.geometry[polyakov_direction])
    mz = _slice_sums(cfg, meson, correlator_direction, polyakov_direction) / count
    corr = []
    pdt = p
    for _ in range(cfg.geometry[correlator_direction]):
        corr.append(_dev.cdot(pdt, p) / vol)  # mean of p * conj(p_dt)
        pdt = lt.mth_translate(pdt, correlator_direction, +1, lat)
    return [Measurement(name="meson_operator", value=np.array(mz), geometry=cfg.geometry, colors=cfg.colors),
            Measurement(name="polyakov_correlator", value=np.array(corr), geometry=cfg.geometry, colors=cfg.colors),
            Measurement(name="polyakov_loop", value=_total(p) / vol, geometry=cfg.geometry, colors=cfg.colors)]


def glueball_operators(cfg, correlator_direction=2):
    """Per-slice means of the summed 1x1 plaquette and 2x2 square traces over the planes
    without `correlator_direction` (measurements.py:197-290)."""
    nd, vol = cfg.gauge_field.shape[0], cfg.gauge_field.shape[-1]
    plaq = None
    square = None
    for mu in range(nd):
        for nu in range(mu + 1, nd):
            if correlator_direction in (mu, nu):
                continue
            a, b = mu + 1, nu + 1
            p1 = path_field(cfg, [a, b, -a, -b])
            s1 = path_field(cfg, [a, a, b, b, -a, -a, -b, -b])
            plaq = p1 if plaq is None else plaq + p1
            square = s1 if square is None else square + s1
    count = vol // cfg.geometry[correlator_direction]
    pz = _slice_sums(cfg, plaq, correlator_direction) / count
    sz = _slice_sums(cfg, square, correlator_direction) / count
    return [Measurement(name="zpp_operator", value=np.array(pz), geometry=cfg.geometry, colors=cfg.colors),
            Measurement(name="square_operator", value=np.array(sz), geometry=cfg.geometry, colors=cfg.colors)]
