"""Three-dimensional Wilson fermions (builder-defined: the reference has fermions in
D = 2 and 4 only, dirac.py:283-300): two-component spinors, gamma_mu = sigma_{mu+1}.
No reference parity exists, so the CUDA path is checked against
  * the oracle's restatement of the operator with the Pauli gammas (1e-13),
  * the free-field known answer: with unit links a plane wave psi(x) = e^{ip.x} chi
    (antiperiodic in time) is an eigenvector, D psi = [1 + 2 kappa sum cos p_mu
    - 2 i kappa sum sigma_mu sin p_mu] psi,
  * the oracle's true residual |b - D x| / |b| of the even-odd CG solutions (its
    M^dag is the adjoint hop, gamma -> -gamma, checked against <phi, D psi> =
    <D^dag phi, psi> on the CPU in tests/test_oracle_golden.py),
and the solves of several 3D lattices in the same launches against single solves.
"""
import numpy as np
import pytest
import torch

from oracle import lym_oracle as O
from tests.conftest import relerr

pytestmark = pytest.mark.gpu


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def np_(t):
    return t.detach().cpu().numpy()


def links(geometry, nc, seed, spread=None):
    rng = np.random.default_rng(seed)
    vol = int(np.prod(geometry))
    a = rng.normal(size=(3, nc, nc, vol)) + 1j * rng.normal(size=(3, nc, nc, vol))
    if spread is not None:  # near unity, for solves at a moderate condition number
        a = np.eye(nc)[None, :, :, None] + spread * a
    return O.unitary_sqrt_projection(a)


def operator(u, geometry, kappa):
    from tfleonardym_b200 import boundary_conditions as bcs
    from tfleonardym_b200 import dirac
    from tfleonardym_b200 import lattice as lt
    cfg = lt.Configuration(cu(u), tuple(geometry), u.shape[1], 3)
    return dirac.DiracWilsonOperator(cfg, kappa, False, representation="fundamental",
                                     boundary_condition_provider=bcs.time_antiperiodic_provider(-1))


@pytest.mark.parametrize("geometry,nc", [((4, 6, 8), 2), ((6, 4, 4), 3), ((5, 3, 4), 2)])
def test_apply_vs_oracle(cuda_device, geometry, nc):
    u = links(geometry, nc, 31 + nc)
    op = operator(u, geometry, 0.13)
    rng = np.random.default_rng(3)
    vol = int(np.prod(geometry))
    psi = rng.normal(size=(3, 2, nc, vol)) + 1j * rng.normal(size=(3, 2, nc, vol))
    out = np_(op.apply(cu(psi)))
    tables = O.lookup_tables(geometry)
    ub = O.apply_time_bc(u, O.antiperiodic_field(geometry))
    for i in range(3):
        assert relerr(out[i], O.wilson_apply(ub, psi[i], 0.13, False, tables)) < 1e-13


def test_free_field_plane_wave(cuda_device):
    geometry, nc, kappa = (6, 4, 8), 2, 0.11
    vol = int(np.prod(geometry))
    u = np.zeros((3, nc, nc, vol), complex)
    for i in range(nc):
        u[:, i, i] = 1.0
    op = operator(u, geometry, kappa)
    sig = np.array([[[0, 1], [1, 0]], [[0, -1j], [1j, 0]], [[1, 0], [0, -1]]])
    coords = np.indices(geometry).reshape(3, -1)
    rng = np.random.default_rng(1)
    for n in [(1, 0, 0), (0, 3, 1), (2, 1, 3), (5, 2, 7)]:
        # momenta allowed by periodic space and antiperiodic time
        p = np.array([2 * np.pi * n[0] / geometry[0], 2 * np.pi * n[1] / geometry[1],
                      (2 * n[2] + 1) * np.pi / geometry[2]])
        chi = rng.normal(size=(2, nc)) + 1j * rng.normal(size=(2, nc))
        phase = np.exp(1j * (p[:, None] * coords).sum(0))
        psi = chi[:, :, None] * phase[None, None, :]
        dp = (1 + 2 * kappa * np.cos(p).sum()) * np.eye(2) - 2j * kappa * np.einsum("m,mab->ab", np.sin(p), sig)
        want = np.einsum("ab,bcv->acv", dp, psi)
        assert relerr(np_(op.apply(cu(psi))), want) < 1e-13, n


@pytest.mark.parametrize("precision", ["f64", "f32", "f16", "bf16"])
@pytest.mark.parametrize("geometry,nc", [((8, 6, 8), 2), ((4, 6, 6), 3)])
def test_eo_cg_true_residual(cuda_device, geometry, nc, precision):
    from tfleonardym_b200 import dirac_solver
    u = links(geometry, nc, 7, spread=0.4)
    kappa = 0.14
    op = operator(u, geometry, kappa)
    vol = int(np.prod(geometry))
    rng = np.random.default_rng(11)
    b = rng.normal(size=(4, 2, nc, vol)) + 1j * rng.normal(size=(4, 2, nc, vol))
    solver = dirac_solver.conjugate_gradient(tol=1e-10, precision=precision, delta=0.01)
    x = np_(solver.solve(op, cu(b)))
    tables = O.lookup_tables(geometry)
    ub = O.apply_time_bc(u, O.antiperiodic_field(geometry))
    for i in range(4):
        res = np.linalg.norm(b[i] - O.wilson_apply(ub, x[i], kappa, False, tables)) / np.linalg.norm(b[i])
        assert res < 1e-10, (precision, i, res, solver.reports[i])


def test_lattices_solved_together(cuda_device):
    """3D SU(2) lattices of different extents and kappa in the same launches give the
    answers of single solves."""
    from tfleonardym_b200 import dirac_solver
    geoms = [(8, 8, 8), (6, 4, 10), (12, 12, 12), (4, 4, 4)]
    ops, bs = [], []
    for k, g in enumerate(geoms):
        u = links(g, 2, 50 + k, spread=0.3)
        ops.append(operator(u, g, 0.10 + 0.01 * k))
        rng = np.random.default_rng(k)
        vol = int(np.prod(g))
        bs.append(cu(rng.normal(size=(3, 2, 2, vol)) + 1j * rng.normal(size=(3, 2, 2, vol))))
    for precision in ("f32", "f16"):
        xs, reps = dirac_solver.solve_lattices(ops, bs, tol=1e-10, precision=precision, delta=0.01)
        for k in range(len(geoms)):
            alone = dirac_solver.conjugate_gradient(tol=1e-10, precision="f64").solve(ops[k], bs[k])
            assert relerr(np_(xs[k]), np_(alone)) < 1e-8, (precision, k)
            assert all(r["true_residual"] < 1e-10 for r in reps[k])


def test_hermitian_and_square_operator_solvers_refuse_three_dimensions(cuda_device):
    """Q = gamma_d D (and so Q^2 + sigma) does not exist in three dimensions: the
    C ABI refuses hermitian solves and the Q^2 solvers with LYM_ERR_UNSUPPORTED."""
    import ctypes

    from tfleonardym_b200 import _dev, _lib
    u = links((4, 4, 4), 2, 1)
    op = operator(u, (4, 4, 4), 0.1)
    b = cu(np.ones((1, 2, 2, 64), complex))
    x = torch.empty_like(b)
    g = op.solver_gauge(())
    reps = (_lib.SolverReport * 4)()
    herm = _lib.SolverParams(1e-10, 100, 0, 0.1, 1, 8, 0, 0, 0, 0.0)
    rc = _lib.lib().lym_wilson_solve(g, 0.1, 1, _dev.ptr(b), _dev.ptr(x), ctypes.byref(herm), reps, _dev.stream())
    assert rc == _lib.LYM_ERR_UNSUPPORTED and b"hermitian" in _lib.lib().lym_last_error()
    plain = _lib.SolverParams(1e-10, 100, 0, 0.1, 0, 8, 0, 0, 0, 0.0)
    sh = (ctypes.c_double * 1)(0.1)
    xs = torch.empty((1, 1, 2, 2, 64), dtype=torch.complex128, device="cuda")
    rc = _lib.lib().lym_multishift_solve_eo(g, 0.1, 1, 1, sh, _dev.ptr(b), _dev.ptr(xs), ctypes.byref(plain), reps,
                                            _dev.stream())
    assert rc == _lib.LYM_ERR_UNSUPPORTED and b"hermitian" in _lib.lib().lym_last_error()
