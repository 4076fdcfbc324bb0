"""SU(N) generators (mirror of the reference's lie_generators.py).

``generators(nc, "fundamental")``: T^a = lambda^a / 2 (Pauli for N = 2,
Gell-Mann for N = 3) in the reference's order, Tr T^a T^b = delta^ab / 2 --
the basis in which the adjoint-representation spinors and links are
expressed, so it must be the reference's.  ``generators(nc, "adjoint")``:
(T_adj^i)_{jk} = -2 Tr([T_i, T_j] T_k) (lie_generators.py:22-36).  Host-side
constants; the device kernels build their own copies.
"""
import numpy as np

_cache = {}


def _fundamental(nc):
    if nc == 2:
        g = np.zeros((3, 2, 2), dtype=np.complex128)
        g[0, 0, 1] = g[0, 1, 0] = 1
        g[1, 0, 1], g[1, 1, 0] = -1j, 1j
        g[2, 0, 0], g[2, 1, 1] = 1, -1
        return g / 2
    if nc == 3:
        g = np.zeros((8, 3, 3), dtype=np.complex128)
        # symmetric off-diagonal pairs (0,1), (0,2), (1,2); then antisymmetric ones; then the diagonal two
        for a, (i, j) in enumerate(((0, 1), (0, 2), (1, 2))):
            g[a, i, j] = g[a, j, i] = 1
            g[a + 3, i, j], g[a + 3, j, i] = -1j, 1j
        g[6, 0, 0], g[6, 1, 1] = 1, -1
        g[7] = np.diag([1, 1, -2]) / np.sqrt(3.0)
        return g / 2
    raise ValueError(f"N={nc} has no generator table")


def generators(nc, representation="fundamental"):
    key = (nc, representation)
    if key not in _cache:
        t = _fundamental(nc)
        if representation == "fundamental":
            _cache[key] = t
        elif representation == "adjoint":
            comm = np.einsum("iab,jbc->ijac", t, t) - np.einsum("jab,ibc->ijac", t, t)
            _cache[key] = -2 * np.einsum("ijab,kba->ijk", comm, t)
        else:
            raise RuntimeError(f"Unknown representation {representation}")
    return _cache[key]
