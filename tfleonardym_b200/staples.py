"""Staple fields (mirror of staples.py:23-58 on the GPU).

``get_staple_fields`` keeps the reference's return value: a list with one entry
per direction, each the list of per-plane (N, N, V) terms in the reference's
order (for every plane (mu, nu) the "up" then the "down" term), an empty list
for the excluded direction.  One kernel launch (lym_staple_terms) writes all the
terms into one (nd, 2(nd-1), N, N, V) tensor; the lists hold views of it.
``get_staple_sums`` is the fused form every caller of the reference ends up
with (the sum of each direction's list, gauge_action.py:130-132,
smearing.py:39-41): one (nd, N, N, V) tensor from lym_staples.
"""
import torch

from . import _dev, _lib
from . import lattice as lt


def _no_dir(no_direction, nd):
    return no_direction if 0 <= no_direction < nd else -1


def get_staple_fields(cfg: lt.Configuration, no_direction: int = 3):
    u = _dev.as_c128(cfg.gauge_field)
    nd, nc = u.shape[0], u.shape[1]
    nodir = _no_dir(no_direction, nd)
    terms = torch.empty((nd, 2 * (nd - 1)) + tuple(u.shape[1:]), dtype=u.dtype, device=u.device)
    _lib.check(_lib.lib().lym_staple_terms(lt.get_lattice(tuple(cfg.geometry)).handle, nc, _dev.ptr(u), nodir,
                                           _dev.ptr(terms), _dev.stream()), "lym_staple_terms")
    nplanes = nd - 1 - (1 if nodir >= 0 else 0)
    return [[] if mu == nodir else [terms[mu, k] for k in range(2 * nplanes)] for mu in range(nd)]


def get_staple_sums(cfg: lt.Configuration, no_direction: int = 3):
    """(nd, N, N, V): the sum of each direction's staple terms (zero for the excluded one)."""
    u = _dev.as_c128(cfg.gauge_field)
    out = torch.empty_like(u)
    nd = u.shape[0]
    _lib.check(_lib.lib().lym_staples(lt.get_lattice(tuple(cfg.geometry)).handle, u.shape[1], _dev.ptr(u),
                                      _no_dir(no_direction, nd), _dev.ptr(out), _dev.stream()), "lym_staples")
    return out
