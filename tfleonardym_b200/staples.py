"""Staple fields (mirror of staples.py:23-58): summed per direction on the GPU."""
import torch

from . import _dev, _lib
from . import lattice as lt


def get_staple_fields(cfg: lt.Configuration, no_direction: int = 3):
    """(nd, N, N, V) staple sums; direction ``no_direction`` is excluded (zero staple).
    The reference returns, per direction, the list of per-plane terms; their sum
    is what every caller uses (gauge_action.py:130-132, smearing.py:39-41)."""
    u = _dev.as_c128(cfg.gauge_field)
    out = torch.empty_like(u)
    nd = u.shape[0]
    nodir = no_direction if 0 <= no_direction < nd else -1
    _lib.check(_lib.lib().lym_staples(lt.get_lattice(tuple(cfg.geometry)).handle, u.shape[1], _dev.ptr(u), nodir,
                                      _dev.ptr(out), _dev.stream()), "lym_staples")
    return out
