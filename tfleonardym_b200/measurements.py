"""Plaquette measurement (mirror of measurements.py:7-43)."""
from collections import namedtuple

from .gauge_action import plaquette_trace_sum

Measurement = namedtuple("Measurement", ["geometry", "colors", "value", "name", "smearing_levels"])
Measurement.__new__.__defaults__ = (None, None, None, None, 0)


def plaquette(cfg) -> Measurement:
    nd, nc = cfg.gauge_field.shape[0], cfg.gauge_field.shape[1]
    vol = cfg.gauge_field.shape[-1]
    re, _ = plaquette_trace_sum(cfg)
    return Measurement(name="plaquette", value=re / (nd * (nd - 1) // 2 * nc * vol), geometry=cfg.geometry,
                       colors=nc)
