"""Backend switch (mirror of translate.py:9-36): binds translate / lookup_tables /
global_sum for one geometry.  Only the single-process path exists on the GPU."""
import functools

from . import lattice as lt

translate = None
lookup_tables = None
global_sum = None
geometry = None


def set_translate(use_mpi, geometry_, mpi_grid=None):
    global translate, lookup_tables, global_sum, geometry
    if use_mpi:
        raise NotImplementedError("MPI domain decomposition is not part of the single-GPU path")
    geometry = tuple(int(g) for g in geometry_)
    lt.global_sum = lt.mth_global_sum
    global_sum = lt.mth_global_sum
    lookup_tables = lt.mth_lookup_tables(geometry)
    lat = lt.get_lattice(geometry)
    lt.translate = functools.partial(lt.mth_translate, lattice=lat)
    translate = lt.translate
