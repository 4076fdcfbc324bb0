"""Index arithmetic of the even-odd hop forms, checked on the CPU against the
oracle's neighbour tables (lattice.py:86-120 restated): the checkerboard ordering
(checkerboard index = lexicographic index / 2 within a parity) and the t-shuffle
form's choice between the own-index load and the neighbouring lane of the t row
(csrc/lym_eo.cuh, hop_tile_mx with TSH).  The GPU tests check the kernels'
results; this pins the formulas they implement."""
import numpy as np
import pytest

from oracle import lym_oracle as O


def _eo_sites(geometry, par):
    """lexicographic sites of parity par in checkerboard order, and their coordinates"""
    _, _, coords = O.lookup_tables(geometry)
    parity = coords.sum(axis=0) % 2
    lex = np.nonzero(parity == par)[0]
    return lex, coords[:, lex]


@pytest.mark.parametrize("geometry", [(4, 4, 4, 8), (4, 4, 2, 16), (2, 4, 4, 4), (8, 64), (4, 2, 2, 32)])
def test_t_shuffle_sources_are_the_t_neighbours(geometry):
    sup, sdn, _ = O.lookup_tables(geometry)
    nd = len(geometry)
    lh = geometry[-1] // 2
    vh = int(np.prod(geometry)) // 2
    assert lh <= 32 and lh & (lh - 1) == 0 and vh % 32 == 0
    lhm = lh - 1
    for par in (0, 1):
        lex, x = _eo_sites(geometry, par)
        cb = np.arange(vh)
        assert np.array_equal(lex // 2, cb)  # checkerboard index = lex / 2
        lane = cb & 31
        seg = lane & ~lhm
        srcf = seg | ((lane + 1) & lhm)
        srcb = seg | ((lane - 1) & lhm)
        odd = (x[nd - 1] & 1) == 1
        # +t: own index when the site's t is even, else the next lane of the row
        fwd = np.where(~odd, cb, cb - lane + srcf)
        bwd = np.where(odd, cb, cb - lane + srcb)
        assert np.array_equal(fwd, sup[nd - 1][lex] // 2), (geometry, par)
        assert np.array_equal(bwd, sdn[nd - 1][lex] // 2), (geometry, par)
        # the -t neighbour's index the kernel computes for the backward link
        ncb_b = (cb & ~lhm) | ((cb - np.where(odd, 0, 1)) & lhm)
        assert np.array_equal(ncb_b, sdn[nd - 1][lex] // 2), (geometry, par)
        # every source lane lies in the same warp and the same t row
        assert np.all((cb - lane + srcf) // 32 == cb // 32)
        assert np.all((cb - lane + srcb) // lh == cb // lh)


@pytest.mark.parametrize("geometry", [(4, 4, 4, 8), (2, 4, 4, 6), (6, 10), (4, 6, 4)])
def test_arithmetic_neighbours_match_the_tables(geometry):
    """nb_fwd / nb_bwd on the coordinates (last coordinate fastest, periodic) give the
    tables' neighbours in every direction; the neighbour's checkerboard index is its
    lexicographic index / 2."""
    sup, sdn, coords = O.lookup_tables(geometry)
    nd = len(geometry)
    stride = [int(np.prod(geometry[m + 1:])) for m in range(nd)]
    lex = np.arange(int(np.prod(geometry)))
    for mu in range(nd):
        xm = coords[mu]
        fwd = np.where(xm == geometry[mu] - 1, lex - (geometry[mu] - 1) * stride[mu], lex + stride[mu])
        bwd = np.where(xm == 0, lex + (geometry[mu] - 1) * stride[mu], lex - stride[mu])
        assert np.array_equal(fwd, sup[mu]) and np.array_equal(bwd, sdn[mu]), (geometry, mu)
