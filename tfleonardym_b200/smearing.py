"""Reunitarisation (mirror of smearing.py:17-31): X (X^dag X)^{-1/2} / det^{1/N}."""
import torch

from . import _dev, _lib


def unitary_sqrt_projection(link_config):
    x = _dev.as_c128(link_config)
    out = torch.empty_like(x)
    _lib.check(_lib.lib().lym_unitary_projection(x.shape[0], x.shape[1], x.shape[-1], _dev.ptr(x), _dev.ptr(out),
                                                 _dev.stream()), "lym_unitary_projection")
    return out
