"""GPU parity at the workload sizes: the CUDA path (through the C ABI) against the
pinned CPU oracle on the lattices the throughput figures are quoted on.

* 16^4 SU(3), kappa = 0.13, links exp(i 0.25 H): the full-lattice FP64 Wilson
  operator against oracle.wilson_apply (1e-13 relative); the even-odd CG with FP64
  and with FP16 inner iterations, each solution's true residual |b - D x| / |b|
  recomputed by the oracle (1e-10), and the FP16-inner solution's relative
  difference to the FP64 one (bounded by cond(D) x 2e-10, asserted below 1e-8).
* 32^4 SU(3): the full-lattice operator at a sample of sites (every site of the
  four time-boundary and corner classes plus random ones) against the oracle's
  site-restricted apply; the FP16-inner CG's residual through that same apply.
* 24^3 x 48 SU(3), kappa = 0.13, links exp(i 0.3 H): even-odd multishift CG, one
  source and 3 shifts, FP32 inner iterations; every shift's oracle residual
  |(Q^2 + sigma) x - b| / |b| <= 1e-10.
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


def exp_links(geometry, nc, eps, seed):
    """U = exp(i eps H) per link, H traceless Hermitian with unit-variance complex
    entries, by eigendecomposition (exactly unitary with det 1 up to rounding);
    (nd, N, N, V) complex128."""
    rng = np.random.default_rng(seed)
    nd, vol = len(geometry), int(np.prod(geometry))
    a = (rng.normal(size=(nd, vol, nc, nc)) + 1j * rng.normal(size=(nd, vol, nc, nc))) / np.sqrt(2)
    h = (a + np.conj(np.swapaxes(a, -1, -2))) / 2
    h = h - (np.trace(h, axis1=-2, axis2=-1) / nc)[..., None, None] * np.eye(nc)
    w, v = np.linalg.eigh(h)
    u = np.einsum("...ik,...k,...jk->...ij", v, np.exp(1j * eps * w), np.conj(v))
    return np.ascontiguousarray(np.transpose(u, (0, 2, 3, 1)))


def sources(geometry, nc, n, seed):
    rng = np.random.default_rng(seed)
    vol = int(np.prod(geometry))
    ns = 2 if len(geometry) == 2 else 4
    return (rng.normal(size=(n, ns, nc, vol)) + 1j * rng.normal(size=(n, ns, nc, vol))) / np.sqrt(2)


def operator(gauge, geometry, kappa, hermitian):
    from tfleonardym_b200 import boundary_conditions as bc
    from tfleonardym_b200 import dirac
    from tfleonardym_b200 import lattice as lt
    nd, nc = gauge.shape[0], gauge.shape[1]
    cfg = lt.Configuration(gauge if torch.is_tensor(gauge) else cu(gauge), tuple(geometry), nc, nd)
    return dirac.DiracWilsonOperator(cfg, kappa, hermitian, representation="fundamental",
                                     boundary_condition_provider=bc.time_antiperiodic_provider(-1))


GEOM16 = (16, 16, 16, 16)


@pytest.fixture(scope="module")
def lattice16():
    u = exp_links(GEOM16, 3, 0.25, 2026)
    tables = O.lookup_tables(GEOM16)
    ub = O.apply_time_bc(u, O.antiperiodic_field(GEOM16))
    return u, ub, tables


@pytest.mark.parametrize("hermitian", [False, True])
def test_wilson_apply_16x16x16x16_vs_oracle(cuda_device, lattice16, hermitian):
    u, ub, tables = lattice16
    b = sources(GEOM16, 3, 2, 7)
    op = operator(u, GEOM16, 0.13, hermitian)
    out = np_(op.apply(cu(b)))
    for i in range(2):
        err = relerr(out[i], O.wilson_apply(ub, b[i], 0.13, hermitian, tables))
        assert err < 1e-13, (hermitian, i, err)


def test_eo_cg_16x16x16x16_fp64_and_fp16_vs_oracle(cuda_device, lattice16):
    """The headline solve (D x = b at kappa = 0.13, tol 1e-10) in FP64 and with FP16
    inner iterations; the residuals are the oracle's, not the solver's report."""
    from tfleonardym_b200 import dirac_solver
    u, ub, tables = lattice16
    b = sources(GEOM16, 3, 4, 99)
    op = operator(u, GEOM16, 0.13, False)
    sols = {}
    for prec in ("f64", "f16"):
        solver = dirac_solver.conjugate_gradient(max_steps=2000, tol=1e-10, precision=prec, delta=0.01)
        x = np_(solver.solve(op, cu(b)))
        sols[prec] = x
        for i in range(len(b)):
            res = np.linalg.norm(b[i] - O.wilson_apply(ub, x[i], 0.13, False, tables)) / np.linalg.norm(b[i])
            assert res < 1e-10, (prec, i, res, solver.reports[i])
            assert solver.reports[i]["status"] == 0
    for i in range(len(b)):
        diff = relerr(sols["f16"][i], sols["f64"][i])
        print(f"16^4 rhs {i}: |x_f16 - x_f64| / |x_f64| = {diff:.3e}")
        assert diff < 1e-8, (i, diff)


def _sample_sites(geometry, n, seed):
    """Random sites plus every site on the first and last time slices of one
    spatial row and the lattice's corner sites (the boundary-crossing hops)."""
    rng = np.random.default_rng(seed)
    vol = int(np.prod(geometry))
    picked = set(rng.choice(vol, n, replace=False).tolist())
    lt = geometry[-1]
    for x0 in (0, geometry[0] - 1):
        for x1 in (0, geometry[1] - 1):
            for x2 in (0, geometry[2] - 1):
                for t in (0, 1, lt - 2, lt - 1):
                    picked.add(int(np.ravel_multi_index((x0, x1, x2, t), geometry)))
    return np.array(sorted(picked), dtype=np.int64)


def test_wilson_apply_and_fp16_cg_32x32x32x32_sampled(cuda_device):
    from tfleonardym_b200 import dirac_solver, hmc
    geom = (32, 32, 32, 32)
    nd, nc, vol = 4, 3, 32 ** 4
    dev = torch.device("cuda")
    g = torch.Generator(device=dev)
    g.manual_seed(32)
    a = torch.complex(torch.randn((nd, nc, nc, vol), generator=g, device=dev, dtype=torch.float64),
                      torch.randn((nd, nc, nc, vol), generator=g, device=dev, dtype=torch.float64)) / np.sqrt(2)
    h = (a + torch.conj(a.transpose(1, 2))) / 2
    tr = torch.diagonal(h, dim1=1, dim2=2).sum(-1) / nc
    for i in range(nc):
        h[:, i, i] -= tr
    del a
    ident = torch.zeros_like(h)
    for i in range(nc):
        ident[:, i, i] = 1
    links = hmc.update_link_field(ident, 1j * h, 0.25, reunitarize=True)
    del h, ident
    op = operator(links, geom, 0.13, False)
    b = cu(sources(geom, nc, 1, 5)[0])
    out = np_(op.apply(b))
    u_host = np_(links)
    tables = O.lookup_tables(geom)
    ub = O.apply_time_bc(u_host, O.antiperiodic_field(geom))
    sites = _sample_sites(geom, 512, 11)
    b_host = np_(b)
    ref = O.wilson_apply_sites(ub, b_host, 0.13, False, tables, sites)
    assert relerr(out[:, :, sites], ref) < 1e-13
    # FP16-inner CG: the residual through the apply checked above
    solver = dirac_solver.conjugate_gradient(max_steps=3000, tol=1e-10, precision="f16", delta=0.01)
    x = solver.solve(op, b)
    res = float(torch.linalg.vector_norm(b - op.apply(x)) / torch.linalg.vector_norm(b))
    assert res < 1e-10, (res, solver.reports)
    # and the solution itself at the sampled sites: D x reproduces b there
    dx = O.wilson_apply_sites(ub, np_(x), 0.13, False, tables, sites)
    assert relerr(dx, b_host[:, :, sites]) < 1e-9


@pytest.mark.parametrize("precision", ["f32", "f16"])
def test_multishift_eo_24x24x24x48_vs_oracle(cuda_device, precision):
    """Every shift's oracle Q^2 residual <= 1e-10 (FP16: the mixed-precision hop with
    arithmetic neighbours, which the multishift takes at this size)."""
    from tfleonardym_b200 import dirac, dirac_solver
    geom = (24, 24, 24, 48)
    u = exp_links(geom, 3, 0.3, 48)
    tables = O.lookup_tables(geom)
    ub = O.apply_time_bc(u, O.antiperiodic_field(geom))
    b = sources(geom, 3, 1, 3)[0]
    op = operator(u, geom, 0.13, True)
    shifts = [0.0001, 0.01, 0.5]
    ms = dirac_solver.multishift_cg(8000, 1e-10, precision=precision, delta=0.01)
    xs = ms.solve(dirac.SquareOperator(op), cu(b), shifts)
    nb = np.linalg.norm(b)
    for s, xk in zip(shifts, xs):
        xk = np_(xk)
        q2x = O.wilson_apply(ub, O.wilson_apply(ub, xk, 0.13, True, tables), 0.13, True, tables)
        res = np.linalg.norm(q2x + s * xk - b) / nb
        assert res < 1e-10, (s, res)
