"""Lattice runtime (mirror of the reference's lattice.py for one GPU).

``Configuration`` keeps the reference's fields (lattice.py:7); ``gauge_field``
is a complex128 CUDA tensor of shape (nd, N, N, V).  Neighbour tables are
built by the C ABI (lym_lookup_tables) bit-exactly as lattice.py:86-120 does,
and live on the device inside a ``Lattice`` handle shared by every operator of
that geometry.
"""
import ctypes
import functools
from collections import namedtuple

import numpy as np
import torch

from . import _dev, _lib

Configuration = namedtuple("Configuration", ["gauge_field", "geometry", "colors", "number_of_dimensions"])
Configuration.__new__.__defaults__ = (None,)

def read_config(cfg_name, lattice_size, Nc=3):  # noqa: N803 - reference argument name
    """Read the reference's XDR configuration file (lattice.py:10-70).

    The link section (V x nd x 3 x 2 x 2 big-endian float32: the first two columns
    of conj(U)) is copied to the device as bytes and decoded there by
    lym_decode_xdr_gauge (Gram-Schmidt of the two columns, third column =
    conj(col0 x col1)); the trailing extents and three parameters are printed as
    the reference prints them.  The Configuration carries number_of_dimensions,
    which the reference's omits (it raises there)."""
    nd = len(lattice_size)
    vol = int(np.prod(lattice_size))
    if Nc != 3:
        raise RuntimeError("the XDR configuration format holds SU(3) links")
    raw = np.fromfile(cfg_name, dtype=np.uint8)
    nbytes = vol * nd * Nc * (Nc - 1) * 2 * 4
    trailer = 4 * nd + 8 * 3
    if raw.size < nbytes + trailer:
        raise RuntimeError(f"{cfg_name}: {raw.size} bytes, expected {nbytes + trailer} for {tuple(lattice_size)}")
    words = torch.from_numpy(raw[:nbytes].copy()).to("cuda")
    gauge = torch.empty((nd, Nc, Nc, vol), dtype=torch.complex128, device="cuda")
    _lib.check(_lib.lib().lym_decode_xdr_gauge(nd, Nc, vol, _dev.ptr(words), _dev.ptr(gauge), _dev.stream()),
               "lym_decode_xdr_gauge")
    dims = [int(d) for d in np.frombuffer(raw.tobytes(), dtype=">i4", count=nd, offset=nbytes)]
    params = [float(p) for p in np.frombuffer(raw.tobytes(), dtype=">f8", count=3, offset=nbytes + 4 * nd)]
    print(cfg_name, dims, ", params", params)
    return Configuration(gauge_field=gauge, geometry=tuple(lattice_size), colors=Nc, number_of_dimensions=nd)


MthLookupTables = namedtuple("MthLookupTables", ["sup", "sdn", "global_coordinates", "global_volume",
                                                 "local_volume"])


@functools.lru_cache(maxsize=100)
def mth_lookup_tables(lattice_geometry: tuple):
    """Same tables as lattice.py:86-120 (int64 numpy arrays (nd, V))."""
    sup, sdn, coords = _lib.host_lookup_tables(tuple(lattice_geometry))
    vol = int(np.prod(lattice_geometry))
    return MthLookupTables(sup, sdn, coords, vol, vol)


class Lattice:
    """Device-resident tables for one geometry on the current CUDA device."""

    def __init__(self, geometry):
        _dev.require_cuda()
        self.geometry = tuple(int(g) for g in geometry)
        self.nd = len(self.geometry)
        self.volume = int(np.prod(self.geometry))
        self.device = torch.cuda.current_device()
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().lym_lattice_create(self.nd, _lib.dims_array(self.geometry), ctypes.byref(h)),
                   "lym_lattice_create")
        self.handle = h
        self._tables = None

    @property
    def even(self):
        return all(g % 2 == 0 for g in self.geometry)

    def device_tables(self):
        """(sup, sdn) int64 CUDA tensors (nd, V), widened from the device copies."""
        if self._tables is None:
            sup = torch.empty((self.nd, self.volume), dtype=torch.int64, device="cuda")
            sdn = torch.empty_like(sup)
            _lib.check(_lib.lib().lym_lattice_tables_device(self.handle, _dev.ptr(sup), _dev.ptr(sdn),
                                                             _dev.stream()), "lym_lattice_tables_device")
            self._tables = (sup, sdn)
        return self._tables

    def __del__(self):
        h = getattr(self, "handle", None)
        # at interpreter exit the module globals may already be gone
        if h is not None and _lib is not None and getattr(_lib, "_lib", None) is not None:
            try:
                torch.cuda.synchronize()
            except Exception:
                pass
            _lib.lib().lym_lattice_destroy(h)
            self.handle = None


_lattices = {}


def get_lattice(geometry) -> Lattice:
    key = (tuple(int(g) for g in geometry), torch.cuda.current_device())
    lat = _lattices.get(key)
    if lat is None:
        lat = Lattice(key[0])
        _lattices[key] = lat
    return lat


def mth_translate(tensor, direction, sign, lattice: Lattice):
    """Shift along the site axis (lattice.py:124-128) on the device."""
    sup, sdn = lattice.device_tables()
    idx = sup[direction] if sign > 0 else sdn[direction]
    return torch.index_select(tensor, tensor.dim() - 1, idx)


def mth_global_sum(to_sum):
    """Single GPU: identity (lattice.py:375-376)."""
    return to_sum


translate = None
global_sum = mth_global_sum
