"""GPU parity: the CUDA path (through the C ABI) against the reference's golden
vectors and the pinned CPU oracle, on identical inputs.

Tolerances: integer tables bit-exact; FP64 straight-line kernels 1e-13
relative (summation order only); solver outputs against the tolerance they
were solved to.
"""
import numpy as np
import pytest
import torch

from oracle import lym_oracle as O
from tests.conftest import ADJOINT_CASES, GOLDEN_CASES, MEASUREMENT_CASES, OBSERVABLE_CASES, load_golden, relerr

pytestmark = pytest.mark.gpu

TOL = 1e-13


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def np_(t):
    return t.detach().cpu().numpy()


def make_cfg(gauge, geometry):
    from tfleonardym_b200 import lattice as lt
    nd, nc = gauge.shape[0], gauge.shape[1]
    return lt.Configuration(cu(gauge), tuple(geometry), nc, nd)


def make_op(g, spec, hermitian=True, anti=True):
    from tfleonardym_b200 import boundary_conditions as bc
    from tfleonardym_b200 import dirac
    prov = bc.time_antiperiodic_provider(-1) if anti else bc.periodic_provider()
    return dirac.DiracWilsonOperator(make_cfg(g["gauge"], spec["geometry"]), spec["kappa"], hermitian,
                                     representation="fundamental", boundary_condition_provider=prov)


def test_device_tables_bit_exact(cuda_device):
    from tfleonardym_b200 import lattice as lt
    z = load_golden("tables")
    for key in sorted({k.split("/")[0] for k in z}):
        geom = tuple(int(g) for g in key.split("x"))
        sup, sdn = lt.get_lattice(geom).device_tables()
        np.testing.assert_array_equal(np_(sup), z[f"{key}/sup"])
        np.testing.assert_array_equal(np_(sdn), z[f"{key}/sdn"])


@pytest.mark.parametrize("case", list(GOLDEN_CASES))
def test_wilson_apply_vs_reference(cuda_device, case):
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    for herm in (0, 1):
        for bcname in ("periodic", "anti"):
            op = make_op(g, spec, bool(herm), bcname == "anti")
            out = np_(op.apply(cu(g["eta"])))
            assert relerr(out, g[f"apply/h{herm}/{bcname}/projected"]) < TOL, (herm, bcname)


def test_wilson_apply_generic_provider(cuda_device):
    """An arbitrary provider callable is applied to the tensor (dirac.py:368-370)."""
    from tfleonardym_b200 import boundary_conditions as bc
    from tfleonardym_b200 import dirac
    g = load_golden("d2")
    spec = GOLDEN_CASES["d2"]
    bc.set_antiperiodic_field_in_t_direction(spec["geometry"])
    op = dirac.DiracWilsonOperator(make_cfg(g["gauge"], spec["geometry"]), spec["kappa"], True,
                                   representation="fundamental",
                                   boundary_condition_provider=lambda x: bc.apply_antiboundary_conditions_in_t_direction(x))
    assert relerr(np_(op.apply(cu(g["eta"]))), g["apply/h1/anti/projected"]) < TOL


@pytest.mark.parametrize("geom,nc", [((4, 6, 4, 8), 3), ((8, 6), 2), ((6, 4, 2, 4), 2), ((10, 6), 3)])
def test_wilson_apply_vs_oracle_random(cuda_device, geom, nc):
    rng = np.random.default_rng(sum(geom) + nc)
    nd = len(geom)
    vol = int(np.prod(geom))
    ns = 2 if nd == 2 else 4
    u = O.unitary_sqrt_projection(rng.normal(size=(nd, nc, nc, vol)) + 1j * rng.normal(size=(nd, nc, nc, vol)))
    psi = rng.normal(size=(3, ns, nc, vol)) + 1j * rng.normal(size=(3, ns, nc, vol))
    spec = dict(geometry=geom, kappa=0.137)
    op = make_op(dict(gauge=u), spec, True, True)
    out = np_(op.apply(cu(psi)))  # batched over 3 vectors
    tables = O.lookup_tables(geom)
    ub = O.apply_time_bc(u, O.antiperiodic_field(geom))
    for i in range(3):
        assert relerr(out[i], O.wilson_apply(ub, psi[i], 0.137, True, tables)) < TOL


def test_unsupported_dimension_raises(cuda_device):
    """The reference's message for dimensions without fermions (dirac.py:299-300); the
    three-dimensional extension has no hermitian form and no adjoint representation."""
    from tfleonardym_b200 import dirac
    g1 = np.zeros((1, 2, 2, 64), complex)
    with pytest.raises(RuntimeError, match="not supported for fermions"):
        dirac.DiracWilsonOperator(make_cfg(g1, (64,)), 0.1, False, representation="fundamental")
    g3 = np.zeros((3, 2, 2, 64), complex)
    with pytest.raises(RuntimeError, match="no hermitian form"):
        dirac.DiracWilsonOperator(make_cfg(g3, (4, 4, 4)), 0.1, True, representation="fundamental")
    with pytest.raises(RuntimeError, match="not supported for fermions"):
        dirac.DiracWilsonOperator(make_cfg(g3, (4, 4, 4)), 0.1, False, representation="adjoint")


def test_dot_and_shape_error(cuda_device):
    from tfleonardym_b200 import algebra_utils
    g = load_golden("d4")
    d = algebra_utils.dot(cu(g["eta"]), cu(g["eta2"]))
    assert abs(d - complex(g["dot/eta_eta2"])) < 1e-12 * abs(d)
    with pytest.raises(RuntimeError, match="Incompatible"):
        algebra_utils.dot(cu(g["eta"]), cu(g["eta"][:, :, :-1]))


@pytest.mark.parametrize("case", list(GOLDEN_CASES))
def test_gauge_side_vs_reference(cuda_device, case):
    from tfleonardym_b200 import gauge_action, hmc, measurements, smearing, staples
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    cfg = make_cfg(g["gauge"], spec["geometry"])
    nd = g["gauge"].shape[0]
    ym = gauge_action.yang_mills(cfg, spec["beta"])
    assert relerr(np_(ym.force()), g["gauge_force"]) < TOL
    assert abs(ym.energy() - g["gauge_energy"]) < 1e-12 * abs(g["gauge_energy"])
    assert abs(measurements.plaquette(cfg).value - g["plaquette"]) < 1e-14
    assert relerr(np_(staples.get_staple_sums(cfg, no_direction=nd)), g["staples_all"]) < TOL
    if "staples_no3" in g:
        assert relerr(np_(staples.get_staple_sums(cfg)), g["staples_no3"]) < TOL
    # the reference's return value: per direction, the list of per-plane terms (staples.py:49-58)
    for key, nodir in (("staple_terms_all", nd), ("staple_terms_no3", 3)):
        if f"{key}/0" not in g:
            continue
        lists = staples.get_staple_fields(cfg, no_direction=nodir)
        assert len(lists) == nd
        for mu in range(nd):
            want = g[f"{key}/{mu}"]
            assert len(lists[mu]) == want.shape[0], (key, mu)
            for k, term in enumerate(lists[mu]):
                assert relerr(np_(term), want[k]) < TOL, (key, mu, k)
    assert abs(hmc.momenta_energy(cu(g["momenta"])) - g["momenta_energy"]) < 1e-12 * abs(g["momenta_energy"])
    assert relerr(np_(hmc.update_momenta(cu(g["momenta"]), cu(g["gauge_force"]), -0.05)), g["update_momenta"]) < TOL
    assert relerr(np_(hmc.update_link_field(cu(g["gauge"]), cu(g["momenta"]), 0.1)), g["update_link_field"]) < 1e-13
    assert relerr(np_(smearing.unitary_sqrt_projection(cu(g["unitary_in"]))), g["unitary_out"]) < 1e-12
    # fused force + momentum update
    p = cu(g["momenta"]).clone()
    ym.force_into_momenta(p, -0.05)
    assert relerr(np_(p), g["update_momenta"]) < TOL


@pytest.mark.parametrize("case", list(GOLDEN_CASES))
def test_lie_derivative_vs_reference(cuda_device, case):
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    op = make_op(g, spec)
    assert relerr(np_(op.lie_derivative(cu(g["eta"]), cu(g["eta2"]))), g["lie_derivative"]) < TOL


def test_link_update_large_and_small_steps(cuda_device):
    """exp(eps P) U for eps from 1e-7 to 2 against scipy expm (the oracle)."""
    from tfleonardym_b200 import hmc
    g = load_golden("d4")
    for eps in (1e-7, 1e-3, 0.3, 2.0):
        out = np_(hmc.update_link_field(cu(g["gauge"]), cu(g["momenta"]), eps))
        ref = O.update_link_field(g["gauge"], g["momenta"], eps)
        assert relerr(out, ref) < 1e-13, eps


@pytest.mark.parametrize("case", ["d2", "d4"])
def test_mmmr_vs_reference(cuda_device, case):
    from tfleonardym_b200 import dirac, dirac_solver
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    op = make_op(g, spec)
    solver = dirac_solver.multishift_solver(2000, float(g["mmmr/precision"]))
    sols = solver.solve(dirac.SquareOperator(op), cu(g["eta"]), list(g["mmmr/shifts"]))
    # same arithmetic as the reference: the printed step agrees (reduction order may move it by one)
    assert abs(solver.last_steps - int(g["mmmr/iterations"][0])) <= 1
    for s, ref in zip(sols, g["mmmr/solutions"]):
        assert relerr(np_(s), ref) < 1e-9


@pytest.mark.parametrize("case", ["d2", "d4"])
def test_bicgstab_vs_reference(cuda_device, case):
    from tfleonardym_b200 import dirac, dirac_solver
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    op = dirac.ShiftedOperator(dirac.SquareOperator(make_op(g, spec)), float(g["mmmr/shifts"][-1]))
    solver = dirac_solver.biconjugate_gradient(2000, 1e-11)
    x = solver.solve(op, cu(g["eta"]))
    assert abs(solver.last_steps - int(g["bicgstab/iterations"][0])) <= 1
    assert relerr(np_(x), g["bicgstab/solution"]) < 1e-8


@pytest.mark.parametrize("case", ["d2", "d4"])
def test_multishift_cg(cuda_device, case):
    from tfleonardym_b200 import dirac, dirac_solver
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    op = make_op(g, spec)
    shifts = list(g["mmmr/shifts"])
    xs = dirac_solver.multishift_cg(5000, 1e-12).solve(dirac.SquareOperator(op), cu(g["eta"]), shifts)
    setup = O.WilsonSetup(g["gauge"], spec["kappa"], spec["geometry"])
    for x, s, ref in zip(xs, shifts, g["mmmr/solutions"]):
        xn = np_(x)
        res = np.linalg.norm(setup.Q2(xn) + s * xn - g["eta"]) / np.linalg.norm(g["eta"])
        assert res < 1e-11, (s, res)
        # the golden MMMR solution stopped at |r|^2 < 1e-11 (absolute), so it is
        # itself only accurate to ~1e-7; the residual above is the real check
        assert relerr(xn, ref) < 1e-6


@pytest.mark.parametrize("precision", ["f64", "f32", "f16", "bf16"])
@pytest.mark.parametrize("case", ["d2", "d4", "d4su2", "d2su3"])
def test_multishift_eo(cuda_device, case, precision):
    """Even-odd multishift CG, two sources, shifts out of order (0 included):
    every (source, shift) meets 1e-10 by the oracle's Q^2 and agrees with the
    full-lattice FP64 multishift CG."""
    from tfleonardym_b200 import dirac, dirac_solver
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    op = make_op(g, spec)
    setup = O.WilsonSetup(g["gauge"], spec["kappa"], spec["geometry"])
    shifts = [0.5, 0.0, 2.0, 0.01]
    b = np.stack([g["eta"], g["eta2"]])
    ms = dirac_solver.multishift_cg(5000, 1e-10, precision=precision, delta=0.01)
    xs = ms.solve(dirac.SquareOperator(op), cu(b), shifts)
    full = [dirac_solver.multishift_cg(5000, 1e-12).solve(dirac.SquareOperator(op), cu(b[i]), shifts)
            for i in range(2)]
    for k, s in enumerate(shifts):
        x = np_(xs[k])
        assert x.shape == b.shape
        for i in range(2):
            rep = ms.reports[i * len(shifts) + k]
            res = np.linalg.norm(setup.Q2(x[i]) + s * x[i] - b[i]) / np.linalg.norm(b[i])
            assert res < 1e-10, (precision, i, s, res, rep)
            assert rep["status"] == 0 and rep["true_residual"] < 1e-10, rep
            assert relerr(x[i], np_(full[i][k])) < 1e-7, (i, s)


@pytest.mark.parametrize("precision", ["f32", "f16"])
@pytest.mark.parametrize("tile", [0, 1])
def test_multishift_eo_padded_groups(cuda_device, precision, tile):
    """Five sources (FP32: four per hop thread and three padding groups, or
    one per thread; FP16: one per thread, mixed-precision hop), 17 shifts from
    1e-4 to 300 (a rational approximation's spread): true residual 1e-10 each."""
    from tfleonardym_b200 import dirac, dirac_solver
    g = load_golden("d4")
    spec = GOLDEN_CASES["d4"]
    op = make_op(g, spec)
    setup = O.WilsonSetup(g["gauge"], spec["kappa"], spec["geometry"])
    shifts = list(np.geomspace(1e-4, 300.0, 17))
    rng = np.random.default_rng(11)
    b = (rng.normal(size=(5,) + g["eta"].shape) + 1j * rng.normal(size=(5,) + g["eta"].shape)) / np.sqrt(2)
    ms = dirac_solver.multishift_cg(5000, 1e-10, precision=precision, delta=0.01, rhs_per_thread=tile)
    xs = ms.solve(dirac.SquareOperator(op), cu(b), shifts)
    # four groups per thread in FP32 unless forced to one; FP16 always one (mixed-precision hop)
    assert ms.reports[0]["rhs_per_thread"] == (4 if precision == "f32" and tile == 0 else 1)
    for k, s in enumerate(shifts):
        x = np_(xs[k])
        for i in range(5):
            res = np.linalg.norm(setup.Q2(x[i]) + s * x[i] - b[i]) / np.linalg.norm(b[i])
            assert res < 1e-10, (i, s, res, ms.reports[i * len(shifts) + k])


def test_multishift_eo_edge_cases(cuda_device):
    """A zero source gives zero solutions; one shift; a repeated shift gives the
    same solution twice; too few iterations report NOT_CONVERGED per pair and
    return the last iterate (as the reference's solvers do)."""
    from tfleonardym_b200 import _lib, dirac, dirac_solver
    dirac_solver.VERBOSE = False
    g = load_golden("d4")
    spec = GOLDEN_CASES["d4"]
    sq = dirac.SquareOperator(make_op(g, spec))
    setup = O.WilsonSetup(g["gauge"], spec["kappa"], spec["geometry"])
    b = np.stack([np.zeros_like(g["eta"]), g["eta"]])
    ms = dirac_solver.multishift_cg(5000, 1e-10, precision="f32")
    xs = ms.solve(sq, cu(b), [0.1])
    x = np_(xs[0])
    assert np.all(x[0] == 0) and ms.reports[0]["status"] == 0
    res = np.linalg.norm(setup.Q2(x[1]) + 0.1 * x[1] - b[1]) / np.linalg.norm(b[1])
    assert res < 1e-10
    xs = ms.solve(sq, cu(g["eta"]), [0.2, 0.05, 0.2])
    assert relerr(np_(xs[0]), np_(xs[2])) < 1e-12
    short = dirac_solver.multishift_cg(3, 1e-10, precision="f64")
    xs = short.solve(sq, cu(g["eta"]), [0.05, 0.5])
    assert all(r["status"] == _lib.LYM_ERR_NOT_CONVERGED for r in short.reports)
    assert all(np.isfinite(np_(x)).all() and np.linalg.norm(np_(x)) > 0 for x in xs)


@pytest.mark.parametrize("switch", [-1.0, 1e-3, 1e-12])
def test_multishift_eo_switch_points(cuda_device, switch):
    """Inner precision from the start (-1), after an FP64 head to 1e-3, and an
    FP64 head past tol (the whole solve in FP64): 1e-10 for every shift."""
    from tfleonardym_b200 import dirac, dirac_solver
    g = load_golden("d4")
    spec = GOLDEN_CASES["d4"]
    op = make_op(g, spec)
    setup = O.WilsonSetup(g["gauge"], spec["kappa"], spec["geometry"])
    shifts = [0.02, 0.001, 0.3]
    b = np.stack([g["eta"], g["eta2"], g["eta"] - g["eta2"]])
    ms = dirac_solver.multishift_cg(5000, 1e-10, precision="f16", delta=0.01, switch_residual=switch)
    xs = ms.solve(dirac.SquareOperator(op), cu(b), shifts)
    for k, s in enumerate(shifts):
        x = np_(xs[k])
        for i in range(3):
            res = np.linalg.norm(setup.Q2(x[i]) + s * x[i] - b[i]) / np.linalg.norm(b[i])
            assert res < 1e-10, (switch, i, s, res, ms.reports[i * len(shifts) + k])


@pytest.mark.parametrize("precision", ["f64", "f32", "f16", "bf16"])
@pytest.mark.parametrize("case", ["d2", "d4", "d4su2", "d2su3"])
def test_eo_cg_true_residual(cuda_device, case, precision):
    """D x = b (and Q x = b) by even-odd CG: true residual recomputed by the oracle."""
    from tfleonardym_b200 import dirac_solver
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    tables = O.lookup_tables(spec["geometry"])
    ub = O.apply_time_bc(g["gauge"], O.antiperiodic_field(spec["geometry"]))
    b = np.stack([g["eta"], g["eta2"]])
    for herm in (False, True):
        op = make_op(g, spec, herm, True)
        solver = dirac_solver.conjugate_gradient(tol=1e-10, precision=precision)
        x = np_(solver.solve(op, cu(b)))
        for i in range(2):
            res = np.linalg.norm(b[i] - O.wilson_apply(ub, x[i], spec["kappa"], herm, tables)) / np.linalg.norm(b[i])
            assert res < 1e-10, (herm, i, res, solver.reports)
            assert solver.reports[i]["true_residual"] < 1e-10


@pytest.mark.parametrize("precision", ["f32", "f16"])
def test_eo_cg_every_hop_tile(cuda_device, precision):
    """Every hop-kernel variant (1, 2, 4 rhs per thread with full links, and the
    autotuned pick, which may use compressed links) meets the true residual."""
    from tfleonardym_b200 import dirac_solver
    g = load_golden("d4")
    spec = GOLDEN_CASES["d4"]
    tables = O.lookup_tables(spec["geometry"])
    ub = O.apply_time_bc(g["gauge"], O.antiperiodic_field(spec["geometry"]))
    rng = np.random.default_rng(3)
    b = rng.normal(size=(8,) + g["eta"].shape) + 1j * rng.normal(size=(8,) + g["eta"].shape)
    op = make_op(g, spec, False, True)
    for tile in (1, 2, 4, 0):
        solver = dirac_solver.conjugate_gradient(tol=1e-10, precision=precision, rhs_per_thread=tile)
        x = np_(solver.solve(op, cu(b)))
        if tile:
            assert solver.reports[0]["rhs_per_thread"] == tile and solver.reports[0]["compressed_links"] == 0
        for i in range(8):
            res = np.linalg.norm(b[i] - O.wilson_apply(ub, x[i], spec["kappa"], False, tables)) / np.linalg.norm(b[i])
            assert res < 1e-10, (tile, i, res)


def _smooth_links(geometry, nc, seed, spread=0.3):
    """SU(N) links near unity: the polar projection of 1 + spread * Gaussian."""
    rng = np.random.default_rng(seed)
    nd, vol = len(geometry), int(np.prod(geometry))
    a = rng.normal(size=(nd, vol, nc, nc)) + 1j * rng.normal(size=(nd, vol, nc, nc))
    x = np.eye(nc) + spread * a
    u = O.unitary_sqrt_projection(np.ascontiguousarray(np.transpose(x, (0, 2, 3, 1))))
    return u


@pytest.mark.parametrize("precision", ["f64", "f32", "f16"])
@pytest.mark.parametrize("nd_nc", [(4, 3), (2, 2)])
def test_solve_lattices_together(cuda_device, precision, nd_nc):
    """Independent lattices of different geometry, kappa and rhs count in the same
    launches (lym_wilson_solve_multi): every solution meets 1e-10 by the oracle's
    operator and matches the lattice solved alone."""
    from tfleonardym_b200 import boundary_conditions as bc
    from tfleonardym_b200 import dirac, dirac_solver
    from tfleonardym_b200 import lattice as lt
    nd, nc = nd_nc
    geoms = [(4, 4, 4, 8), (6, 4, 2, 4), (4, 2, 4, 4)] if nd == 4 else [(8, 6), (16, 12), (6, 4)]
    kappas, counts = [0.11, 0.13, 0.12], [2, 1, 3]
    rng = np.random.default_rng(5)
    ops, srcs, links = [], [], []
    for k, geom in enumerate(geoms):
        u = _smooth_links(geom, nc, seed=31 + k)
        links.append(u)
        cfg = lt.Configuration(cu(u), geom, nc, nd)
        ops.append(dirac.DiracWilsonOperator(cfg, kappas[k], False, representation="fundamental",
                                             boundary_condition_provider=bc.time_antiperiodic_provider(-1)))
        ns = 2 if nd == 2 else 4
        shape = (counts[k], ns, nc, int(np.prod(geom)))
        b = (rng.normal(size=shape) + 1j * rng.normal(size=shape)) / np.sqrt(2)
        srcs.append(b if counts[k] > 1 else b[0])
    xs, reps = dirac_solver.solve_lattices(ops, [cu(b) for b in srcs], tol=1e-10, precision=precision, delta=0.01)
    for k, geom in enumerate(geoms):
        tables = O.lookup_tables(geom)
        ub = O.apply_time_bc(links[k], O.antiperiodic_field(geom))
        x, b = np_(xs[k]), srcs[k]
        assert x.shape == b.shape
        xb, bb = (x, b) if counts[k] > 1 else (x[None], b[None])
        alone = np_(dirac_solver.conjugate_gradient(tol=1e-10, precision="f64").solve(ops[k], cu(b)))
        alone = alone if counts[k] > 1 else alone[None]
        for i in range(counts[k]):
            res = np.linalg.norm(bb[i] - O.wilson_apply(ub, xb[i], kappas[k], False, tables)) / np.linalg.norm(bb[i])
            assert res < 1e-10, (k, i, res, reps[k][i])
            assert reps[k][i]["status"] == 0 and reps[k][i]["true_residual"] < 1e-10
            assert relerr(xb[i], alone[i]) < 1e-8


@pytest.mark.parametrize("geometry,nc", [((4, 4, 4, 8), 3), ((2, 4, 4, 6), 3), ((4, 4, 4, 4), 2),
                                         ((8, 6), 2), ((12, 4), 3), ((4, 4, 2, 16), 3), ((8, 64), 2)])
def test_eo_cg_mixed_fma_hop(cuda_device, geometry, nc):
    """The mixed-precision FP16 hop (half spinor in FP16, U h through
    f16 x f16 + f32 FMAs) at 1, 2 and 4 rhs per thread, with neighbour indices from
    the table (mixed_fma 1), from coordinate arithmetic (4) or with the t neighbours
    by warp shuffle (5, where the t rows fill whole warps), meets the true residual
    in about the iterations of the FP32-arithmetic FP16 hop; both neighbour forms give
    the same solutions to the tolerance's scale (the same arithmetic on the same
    neighbours; the compiler may fuse a multiply-add differently in the two kernels)."""
    from tfleonardym_b200 import boundary_conditions as bcs
    from tfleonardym_b200 import dirac, dirac_solver
    from tfleonardym_b200 import lattice as lt
    u = _smooth_links(geometry, nc, seed=sum(geometry) + nc)
    kappa = 0.12
    tables = O.lookup_tables(geometry)
    ub = O.apply_time_bc(u, O.antiperiodic_field(geometry))
    cfg = lt.Configuration(cu(u), tuple(geometry), nc, len(geometry))
    op = dirac.DiracWilsonOperator(cfg, kappa, False, representation="fundamental",
                                   boundary_condition_provider=bcs.time_antiperiodic_provider(-1))
    rng = np.random.default_rng(5)
    ns = 4 if len(geometry) == 4 else 2
    b = rng.normal(size=(4, ns, nc, u.shape[-1])) + 1j * rng.normal(size=(4, ns, nc, u.shape[-1]))
    ref = dirac_solver.conjugate_gradient(tol=1e-10, precision="f16", rhs_per_thread=1)
    ref.solve(op, cu(b))
    assert ref.reports[0]["mixed_fma"] == 0
    base = max(r["iterations"] for r in ref.reports)
    xs = {}
    forms = [(1, 1), (1, 2), (1, 4), (4, 1), (4, 2), (4, 4)]
    lh, vh = geometry[-1] // 2, int(np.prod(geometry)) // 2
    if lh <= 32 and lh & (lh - 1) == 0 and vh % 32 == 0:
        forms += [(5, 1), (5, 2)]  # t neighbours by warp shuffle: full warps, t rows aligned to them
    for arith, tile in forms:
        mx = dirac_solver.conjugate_gradient(tol=1e-10, precision="f16", rhs_per_thread=tile, mixed_fma=arith)
        x = np_(mx.solve(op, cu(b)))
        xs[(arith, tile)] = x
        rep = mx.reports[0]
        assert rep["mixed_fma"] == arith and rep["rhs_per_thread"] == tile and rep["compressed_links"] == 0, rep
        for i in range(4):
            res = np.linalg.norm(b[i] - O.wilson_apply(ub, x[i], kappa, False, tables)) / np.linalg.norm(b[i])
            assert res < 1e-10, (tile, i, res)
        its = max(r["iterations"] for r in mx.reports)
        assert abs(its - base) <= max(3, base // 10), (arith, tile, its, base)
    for tile in (1, 2, 4):
        assert relerr(xs[(4, tile)], xs[(1, tile)]) < 1e-8, tile
        if (5, tile) in xs:
            assert relerr(xs[(5, tile)], xs[(1, tile)]) < 1e-8, tile


@pytest.mark.parametrize("geometry,nrhs", [((4, 4, 4, 8), 16), ((2, 4, 4, 6), 16), ((6, 4, 2, 4), 32)])
def test_eo_cg_tensor_core_hop(cuda_device, geometry, nrhs):
    """The tensor-core FP16 hop (4D SU(3); projected FP16 spinors x FP16 links on
    mma.sync, FP32 accumulation; 16 rhs per CTA, so 32 rhs run as two groups)
    meets the oracle's true residual for every rhs in about the iterations of the
    FP32-arithmetic FP16 hop."""
    from tfleonardym_b200 import boundary_conditions as bcs
    from tfleonardym_b200 import dirac, dirac_solver
    from tfleonardym_b200 import lattice as lt
    nc = 3
    u = _smooth_links(geometry, nc, seed=sum(geometry) + nrhs)
    kappa = 0.12
    tables = O.lookup_tables(geometry)
    ub = O.apply_time_bc(u, O.antiperiodic_field(geometry))
    cfg = lt.Configuration(cu(u), tuple(geometry), nc, len(geometry))
    rng = np.random.default_rng(nrhs)
    b = rng.normal(size=(nrhs, 4, nc, u.shape[-1])) + 1j * rng.normal(size=(nrhs, 4, nc, u.shape[-1]))
    for herm in (False, True):
        op = dirac.DiracWilsonOperator(cfg, kappa, herm, representation="fundamental",
                                       boundary_condition_provider=bcs.time_antiperiodic_provider(-1))
        ref = dirac_solver.conjugate_gradient(tol=1e-10, precision="f16", rhs_per_thread=1)
        ref.solve(op, cu(b))
        base = max(r["iterations"] for r in ref.reports)
        tcg = dirac_solver.conjugate_gradient(tol=1e-10, precision="f16", rhs_per_thread=16, mixed_fma=2)
        x = np_(tcg.solve(op, cu(b)))
        rep = tcg.reports[0]
        assert rep["mixed_fma"] == 2 and rep["compressed_links"] == 0, rep
        assert rep["rhs_per_thread"] == 16, rep
        for i in range(nrhs):
            res = np.linalg.norm(b[i] - O.wilson_apply(ub, x[i], kappa, herm, tables)) / np.linalg.norm(b[i])
            assert res < 1e-10, (herm, i, res, tcg.reports[i])
        its = max(r["iterations"] for r in tcg.reports)
        assert abs(its - base) <= max(3, base // 10), (herm, its, base)


@pytest.mark.parametrize("geometry,nc", [((8, 8, 8, 16), 3), ((4, 6, 4, 8), 2), ((16, 12), 3)])
def test_eo_cg_packed_half_hop(cuda_device, geometry, nc):
    """The packed-half FP16 hop (colour contraction of each direction in half2 FMAs,
    FP32 over the directions; mixed_fma = 3) meets the oracle's true residual for every
    rhs, with the iteration count of the mixed-precision hop within 10 %."""
    from tfleonardym_b200 import boundary_conditions as bcs
    from tfleonardym_b200 import dirac, dirac_solver
    from tfleonardym_b200 import lattice as lt
    u = _smooth_links(geometry, nc, seed=sum(geometry) + nc)
    kappa = 0.12
    tables = O.lookup_tables(geometry)
    ub = O.apply_time_bc(u, O.antiperiodic_field(geometry))
    cfg = lt.Configuration(cu(u), tuple(geometry), nc, len(geometry))
    ns = 4 if len(geometry) == 4 else 2
    nrhs = 8
    rng = np.random.default_rng(nc)
    b = rng.normal(size=(nrhs, ns, nc, u.shape[-1])) + 1j * rng.normal(size=(nrhs, ns, nc, u.shape[-1]))
    for herm in (False, True):
        op = dirac.DiracWilsonOperator(cfg, kappa, herm, representation="fundamental",
                                       boundary_condition_provider=bcs.time_antiperiodic_provider(-1))
        ref = dirac_solver.conjugate_gradient(tol=1e-10, precision="f16", rhs_per_thread=1, mixed_fma=1)
        ref.solve(op, cu(b))
        assert ref.reports[0]["mixed_fma"] == 1
        base = max(r["iterations"] for r in ref.reports)
        h2 = dirac_solver.conjugate_gradient(tol=1e-10, precision="f16", rhs_per_thread=1, mixed_fma=3)
        x = np_(h2.solve(op, cu(b)))
        rep = h2.reports[0]
        assert rep["mixed_fma"] == 3 and rep["rhs_per_thread"] == 1 and rep["compressed_links"] == 0, rep
        for i in range(nrhs):
            res = np.linalg.norm(b[i] - O.wilson_apply(ub, x[i], kappa, herm, tables)) / np.linalg.norm(b[i])
            assert res < 1e-10, (herm, i, res, h2.reports[i])
        its = max(r["iterations"] for r in h2.reports)
        assert abs(its - base) <= max(3, base // 10), (herm, its, base)


def test_eo_cg_workspace_reused_across_batch_sizes(cuda_device):
    """Batches of 8, 5, 4, 3 and 1 right-hand sides share workspaces by capacity (8, 8,
    4, 4, 1 in the sloppy precisions): every answer meets the oracle's true residual and
    equals the answer of a solve of that right-hand side alone (a smaller batch clears
    the slots a larger one left behind, so nothing of the earlier sources leaks in)."""
    from tfleonardym_b200 import boundary_conditions as bcs
    from tfleonardym_b200 import dirac, dirac_solver
    from tfleonardym_b200 import lattice as lt
    geometry, nc, kappa = (4, 4, 4, 8), 3, 0.12
    u = _smooth_links(geometry, nc, seed=77)
    tables = O.lookup_tables(geometry)
    ub = O.apply_time_bc(u, O.antiperiodic_field(geometry))
    cfg = lt.Configuration(cu(u), tuple(geometry), nc, len(geometry))
    op = dirac.DiracWilsonOperator(cfg, kappa, False, representation="fundamental",
                                   boundary_condition_provider=bcs.time_antiperiodic_provider(-1))
    rng = np.random.default_rng(5)
    b = rng.normal(size=(21, 4, nc, u.shape[-1])) + 1j * rng.normal(size=(21, 4, nc, u.shape[-1]))
    for precision in ("f64", "f16"):
        solver = dirac_solver.conjugate_gradient(tol=1e-10, precision=precision, delta=0.01)
        alone = dirac_solver.conjugate_gradient(tol=1e-10, precision=precision, delta=0.01)
        start = 0
        for n in (8, 5, 4, 3, 1):
            x = np_(solver.solve(op, cu(b[start:start + n])))
            if x.ndim == 3:
                x = x[None]
            assert len(solver.reports) == n
            for i in range(n):
                bi = b[start + i]
                res = np.linalg.norm(bi - O.wilson_apply(ub, x[i], kappa, False, tables)) / np.linalg.norm(bi)
                assert res < 1e-10, (precision, n, i, res)
                xa = np_(alone.solve(op, cu(bi)))
                assert np.linalg.norm(x[i] - xa) / np.linalg.norm(xa) < 1e-9, (precision, n, i)
            start += n


def test_eo_cg_batch_equals_single(cuda_device):
    """A right-hand side gives the same answer alone and inside a batch."""
    from tfleonardym_b200 import dirac_solver
    g = load_golden("d4")
    spec = GOLDEN_CASES["d4"]
    op = make_op(g, spec, True, True)
    b = np.stack([g["eta"], g["eta2"], g["eta"] * 0.5 + 1j * g["eta2"]])
    for precision in ("f64", "f16"):
        solver = dirac_solver.conjugate_gradient(tol=1e-10, precision=precision)
        xb = np_(solver.solve(op, cu(b)))
        x1 = np_(solver.solve(op, cu(b[1])))
        assert relerr(xb[1], x1) < 1e-9


@pytest.mark.parametrize("case", ["d2", "d4"])
def test_nf2_force_and_energy_vs_reference(cuda_device, case):
    from tfleonardym_b200 import dirac, dirac_solver, fermion_action
    dirac_solver.VERBOSE = False
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    q = make_op(g, spec)
    solver = dirac_solver.multishift_solver(5000, 1e-22)
    ra = dirac.RationalApproximation(dirac.SquareOperator(q), [1.0], [0.0], 0, solver)
    nf = fermion_action.n_flavor([ra], [ra], [q], solver, q)
    nf.initialize_pseudofermions([cu(g["eta"])])
    assert relerr(np_(nf.pseudofermions[0]), g["nf2/phi"]) < TOL
    assert abs(nf.energy() - g["nf2/energy"]) < 1e-9 * abs(g["nf2/energy"])
    assert relerr(np_(nf.force()), g["nf2/force"]) < 1e-9


@pytest.mark.parametrize("case,precision", [("d2", "f64"), ("d4", "f64"), ("d4", "f16")])
def test_nf2_force_with_eo_square_solver(cuda_device, case, precision):
    """The even-odd square solver (two CG solves of Q for the zero shift) in
    place of the reference's MMMR gives the reference's Nf=2 energy and force to
    the accuracy of the solves."""
    from tfleonardym_b200 import dirac, dirac_solver, fermion_action
    dirac_solver.VERBOSE = False
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    q = make_op(g, spec)
    solver = dirac_solver.eo_square_solver(tol=1e-12, precision=precision)
    ra = dirac.RationalApproximation(dirac.SquareOperator(q), [1.0], [0.0], 0, solver)
    nf = fermion_action.n_flavor([ra], [ra], [q], solver, q)
    nf.initialize_pseudofermions([cu(g["eta"])])
    assert abs(nf.energy() - g["nf2/energy"]) < 1e-9 * abs(g["nf2/energy"])
    assert relerr(np_(nf.force()), g["nf2/force"]) < 1e-8
    assert solver.total_iterations > 0


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_rational_approximation_with_eo_square_solver(cuda_device, precision):
    """RationalApproximation.apply (dirac.py:52-59) with positive poles: the even-odd
    square solver (even-odd multishift) against the reference's MMMR."""
    from tfleonardym_b200 import dirac, dirac_solver
    dirac_solver.VERBOSE = False
    g = load_golden("d4")
    spec = GOLDEN_CASES["d4"]
    q = make_op(g, spec)
    # descending poles: the reference's MMMR iterates on the last (smallest) one
    alphas, betas = [0.1, 0.25, 0.4], [1.5, 0.05, 0.002]
    ra_ref = dirac.RationalApproximation(dirac.SquareOperator(q), alphas, betas, 0.3,
                                         dirac_solver.multishift_solver(5000, 1e-24))
    solver = dirac_solver.eo_square_solver(tol=1e-12, precision=precision)
    ra = dirac.RationalApproximation(dirac.SquareOperator(q), alphas, betas, 0.3, solver)
    v = cu(g["eta"])
    assert relerr(np_(ra.apply(v)), np_(ra_ref.apply(v))) < 1e-9
    assert solver.total_iterations > 0


@pytest.mark.parametrize("case", ["d2", "d4"])
def test_md_trajectory_vs_reference(cuda_device, case):
    """integrate_om (hmc.py:133-162) with the Nf=2 and gauge actions from the golden inputs."""
    from tfleonardym_b200 import dirac, dirac_solver, fermion_action, gauge_action, hmc
    dirac_solver.VERBOSE = False
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    q = make_op(g, spec)
    solver = dirac_solver.multishift_solver(5000, 1e-22)
    ra = dirac.RationalApproximation(dirac.SquareOperator(q), [1.0], [0.0], 0, solver)
    nf = fermion_action.n_flavor([ra], [ra], [q], solver, q)
    cfg = make_cfg(g["gauge"], spec["geometry"])
    nf.set_gauge_configuration(cfg)
    nf.initialize_pseudofermions([cu(g["eta"])])
    ym = gauge_action.yang_mills(cfg, spec["beta"])
    new_cfg, p = hmc.integrate_om(cfg, cu(g["md/momenta_in"]), [nf, ym], list(g["hmc/steps"]), 1.0)
    assert relerr(np_(new_cfg.gauge_field), g["md/cfg_out"]) < 1e-9
    assert relerr(np_(p), g["md/momenta_out"]) < 1e-9


def test_hmc_chain_config1(cuda_device):
    """The CPU-runnable HMC case (D=2 24x16 SU(2), beta=3, kappa=-0.15, antiperiodic time,
    Omelyan [4,3], t=1): 10 trajectories fed the reference's momenta, eta and
    uniforms; dH, acceptance and plaquette per trajectory against the reference."""
    from tfleonardym_b200 import dirac, dirac_solver, fermion_action, gauge_action, hmc, measurements
    dirac_solver.VERBOSE = False
    g = load_golden("d2")
    spec = GOLDEN_CASES["d2"]
    q = make_op(g, spec)
    solver = dirac_solver.multishift_solver(5000, 1e-22)
    ra = dirac.RationalApproximation(dirac.SquareOperator(q), [1.0], [0.0], 0, solver)
    nf = fermion_action.n_flavor([ra], [ra], [q], solver, q)
    cfg = make_cfg(g["gauge"], spec["geometry"])
    ym = gauge_action.yang_mills(cfg, spec["beta"])
    steps = list(g["hmc/steps"])
    for k in range(len(g["hmc/dH"])):
        nf.set_gauge_configuration(cfg)
        nf.initialize_pseudofermions([cu(g["hmc/eta"][k])])
        cfg, minus_dh, acc = hmc.hybrid_mc(cfg, [nf, ym], steps, 1.0, momenta=cu(g["hmc/momenta"][k]),
                                           uniform=float(g["hmc/uniform"][k]))
        assert abs(-minus_dh - g["hmc/dH"][k]) < 1e-7, k
        assert acc == bool(g["hmc/accepted"][k])
        assert abs(measurements.plaquette(cfg).value - g["hmc/plaquette"][k]) < 1e-10
    assert relerr(np_(cfg.gauge_field), g["hmc/cfg_out"]) < 1e-8


def test_reversibility(cuda_device):
    from tfleonardym_b200 import dirac, dirac_solver, fermion_action, gauge_action, hmc
    dirac_solver.VERBOSE = False
    g = load_golden("d2")
    spec = GOLDEN_CASES["d2"]
    q = make_op(g, spec)
    solver = dirac_solver.multishift_solver(5000, 1e-24)
    ra = dirac.RationalApproximation(dirac.SquareOperator(q), [1.0], [0.0], 0, solver)
    nf = fermion_action.n_flavor([ra], [ra], [q], solver, q)
    cfg = make_cfg(g["hmc/cfg_out"], spec["geometry"])
    nf.set_gauge_configuration(cfg)
    nf.initialize_pseudofermions([cu(g["hmc/eta"][0])])
    ym = gauge_action.yang_mills(cfg, spec["beta"])
    dh = hmc.reversibility_check(cfg, [nf, ym], list(g["hmc/steps"]), 1.0,
                                 momenta=cu(g["hmc/reversibility_momenta"]))
    assert abs(dh) < 1e-9
    assert abs(dh - g["hmc/reversibility_dH"]) < 1e-9


# ---------------------------------------------------------------------------
# adjoint representation (dirac.py:358-370, 380-456, 525-565)
# ---------------------------------------------------------------------------
def make_adj_op(g, spec, hermitian, anti=True, provider=None):
    from tfleonardym_b200 import boundary_conditions as bc
    from tfleonardym_b200 import dirac
    prov = provider or (bc.time_antiperiodic_provider(-1) if anti else bc.periodic_provider())
    return dirac.DiracWilsonOperator(make_cfg(g["gauge"], spec["geometry"]), spec["kappa"], hermitian,
                                     representation="adjoint", boundary_condition_provider=prov)


@pytest.mark.parametrize("case", list(ADJOINT_CASES))
def test_adjoint_apply_links_force_vs_reference(cuda_device, case):
    """Adjoint operator (both reference modes, all hermiticity / BC pairs, batched),
    adjoint links and Lie derivative against the reference's outputs."""
    g = load_golden(case)
    spec = ADJOINT_CASES[case]
    for herm in (0, 1):
        for bcname in ("periodic", "anti"):
            op = make_adj_op(g, spec, bool(herm), bcname == "anti")
            ref = g[f"apply/h{herm}/{bcname}/projected"]
            assert relerr(np_(op.multiply_in_adjoint_representation(cu(g["eta"]))), ref) < TOL, (herm, bcname)
            assert relerr(np_(op.simple_multiply_in_adjoint_representation(cu(g["eta"]))),
                          g[f"apply/h{herm}/{bcname}/simple"]) < TOL
            both = np_(op.apply(cu(np.stack([g["eta"], g["eta2"]]))))
            assert relerr(both[0], ref) < TOL
            if bcname == "anti":
                d = np_(op.lie_derivative(cu(g["eta"]), cu(g["eta2"])))
                assert relerr(d, g[f"lie_derivative/h{herm}"]) < 1e-12, herm
    q = make_adj_op(g, spec, True)
    assert relerr(np_(q.fermion_gauge_field), g["fermion_gauge_field"]) < TOL


def test_adjoint_generic_provider(cuda_device):
    """An arbitrary provider callable multiplies the left links and the adjoint links."""
    from tfleonardym_b200 import boundary_conditions as bc
    g = load_golden("adj_d2su2")
    spec = ADJOINT_CASES["adj_d2su2"]
    bc.set_antiperiodic_field_in_t_direction(spec["geometry"])
    op = make_adj_op(g, spec, True, provider=lambda x: bc.apply_antiboundary_conditions_in_t_direction(x))
    assert relerr(np_(op.apply(cu(g["eta"]))), g["apply/h1/anti/projected"]) < TOL
    assert relerr(np_(op.fermion_gauge_field), g["fermion_gauge_field"]) < TOL


@pytest.mark.parametrize("case", list(ADJOINT_CASES))
def test_adjoint_nf2_vs_reference(cuda_device, case):
    """Nf=2 adjoint fermions through the reference's MMMR (generic operator path):
    pseudofermion, energy and force against the reference's."""
    from tfleonardym_b200 import dirac, dirac_solver, fermion_action
    dirac_solver.VERBOSE = False
    g = load_golden(case)
    spec = ADJOINT_CASES[case]
    q = make_adj_op(g, spec, True)
    solver = dirac_solver.multishift_solver(5000, 1e-22)
    ra = dirac.RationalApproximation(dirac.SquareOperator(q), [1.0], [0.0], 0, solver)
    nf = fermion_action.n_flavor([ra], [ra], [q], solver, q)
    nf.initialize_pseudofermions([cu(g["eta"])])
    assert relerr(np_(nf.pseudofermions[0]), g["nf2/phi"]) < TOL
    assert abs(nf.energy() - g["nf2/energy"]) < 1e-9 * abs(g["nf2/energy"])
    assert relerr(np_(nf.force()), g["nf2/force"]) < 1e-8


def test_adjoint_rejected_by_even_odd_solvers(cuda_device):
    from tfleonardym_b200 import dirac_solver
    g = load_golden("adj_d2su2")
    q = make_adj_op(g, ADJOINT_CASES["adj_d2su2"], True)
    with pytest.raises(TypeError):
        dirac_solver.conjugate_gradient().solve(q, cu(g["eta"]))


# ---------------------------------------------------------------------------
# fermion measurements (fermion_measurements.py:41-115, dirac.py:665-696)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("case", list(MEASUREMENT_CASES))
def test_measurements_vs_reference(cuda_device, case):
    """Propagator, pion correlator and chiral condensate (recorded Z2 sources)
    against the reference: fundamental through the batched even-odd CG (default
    inverter), adjoint through the reference's BiCGStab; the reference's own
    BiCGStab tolerances bound the agreement."""
    from tfleonardym_b200 import dirac, dirac_solver, fermion_measurements
    dirac_solver.VERBOSE = False
    g = load_golden(case)
    spec = MEASUREMENT_CASES[case]
    from tfleonardym_b200 import boundary_conditions as bc
    q = dirac.DiracWilsonOperator(make_cfg(g["gauge"], spec["geometry"]), spec["kappa"], True,
                                  representation=spec["representation"],
                                  boundary_condition_provider=bc.time_antiperiodic_provider(-1))
    inv = dirac_solver.conjugate_gradient(tol=1e-12) if spec["representation"] == "fundamental" else \
        dirac_solver.biconjugate_gradient(5000, 1e-24)
    prop = dirac.Propagator(q, inv)
    assert relerr(np_(prop.apply(cu(g["propagator/source"]))), g["propagator/out"]) < 1e-8
    nd = len(spec["geometry"])
    corr = fermion_measurements.pion_correlator(q, nd - 1, None, lambda x: x)
    assert relerr(corr.value, g["pion_correlator"]) < 1e-5
    cc = fermion_measurements.chiral_condensate(q, sources=cu(g["chiral_condensate/sources"]))
    assert abs(cc.value - g["chiral_condensate"]) < 1e-4 * abs(g["chiral_condensate"])


def test_pion_correlator_vs_oracle_exact(cuda_device):
    """The batched-CG pion correlator against the oracle's exact-solve one (1e-9)."""
    from tfleonardym_b200 import boundary_conditions as bc
    from tfleonardym_b200 import dirac, fermion_measurements
    g = load_golden("meas_d4")
    spec = MEASUREMENT_CASES["meas_d4"]
    geometry, kappa = spec["geometry"], spec["kappa"]
    q = dirac.DiracWilsonOperator(make_cfg(g["gauge"], geometry), kappa, True, representation="fundamental",
                                  boundary_condition_provider=bc.time_antiperiodic_provider(-1))
    corr = fermion_measurements.pion_correlator(q, 1, None, None).value  # along x1 this time
    tables = O.lookup_tables(geometry)
    ub = O.apply_time_bc(g["gauge"], O.antiperiodic_field(geometry))
    vol = int(np.prod(geometry))
    sols = [O.propagator(lambda v: O.wilson_apply(ub, v, kappa, True, tables), O.point_source(0, c, s, vol, 3, 4))
            for s in range(4) for c in range(3)]
    assert relerr(corr, O.pion_correlator(sols, tables[2], 1, geometry[1])) < 1e-9


# ---------------------------------------------------------------------------
# on-disk gauge format (lattice.py:10-70)
# ---------------------------------------------------------------------------
def test_read_config_vs_reference(cuda_device, tmp_path):
    """read_config decodes the XDR file on the device to the reference's links."""
    from tfleonardym_b200 import lattice as lt
    g = load_golden("xdr_su3")
    path = tmp_path / "cfg.xdr"
    g["raw"].tofile(path)
    geometry = tuple(int(d) for d in g["geometry"])
    cfg = lt.read_config(str(path), geometry)
    assert cfg.number_of_dimensions == len(geometry) and cfg.colors == 3
    assert relerr(np_(cfg.gauge_field), g["gauge"]) < 1e-15


def test_xdr_decode_round_trip_large(cuda_device):
    """Size-independent property at 16^4: SU(3) links written in the XDR convention
    (float32 conj columns) decode to SU(3) matrices within float32 of the originals,
    and the oracle decodes the same bytes to the same links."""
    from tfleonardym_b200 import _dev, _lib
    geometry = (16, 16, 16, 16)
    nd, vol = 4, 16 ** 4
    rng = np.random.default_rng(9)
    a = rng.normal(size=(vol, nd, 3, 3)) + 1j * rng.normal(size=(vol, nd, 3, 3))
    q, _ = np.linalg.qr(a)
    q = q / np.linalg.det(q)[..., None, None] ** (1 / 3)
    cols = np.conj(q[..., :2])
    raw = np.stack([cols.real, cols.imag], axis=-1).astype(">f4").tobytes()
    words = torch.from_numpy(np.frombuffer(raw, dtype=np.uint8).copy()).cuda()
    out = torch.empty((nd, 3, 3, vol), dtype=torch.complex128, device="cuda")
    _lib.check(_lib.lib().lym_decode_xdr_gauge(nd, 3, vol, _dev.ptr(words), _dev.ptr(out), _dev.stream()))
    u = np_(out)
    ref = np.transpose(q, (1, 2, 3, 0))
    assert np.abs(u - ref).max() < 1e-6
    sample = u[:, :, :, :4096]
    uu = np.einsum("mijc,mkjc->mikc", sample, np.conj(sample))
    assert np.abs(uu - np.eye(3)[None, :, :, None]).max() < 1e-13
    head = nd * 3 * 2 * 2 * 4 * 4096  # the first 4096 sites (site index slowest in the file)
    o, _, _ = O.read_config_xdr(np.frombuffer(raw[:head] + bytes(4 * nd + 24), dtype=np.uint8), (8, 8, 8, 8))
    assert relerr(sample, o) < 1e-15


# ---------------------------------------------------------------------------
# gauge observables and smearing (measurements.py:46-290, smearing.py:34-86)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("case", list(OBSERVABLE_CASES))
def test_gauge_observables_vs_reference(cuda_device, case):
    from tfleonardym_b200 import measurements as M
    from tfleonardym_b200 import smearing
    g = load_golden(case)
    geometry = OBSERVABLE_CASES[case]["geometry"]
    cfg = make_cfg(g["gauge"], geometry)
    assert abs(M.temporal_plaquette(cfg).value - g["temporal_plaquette"]) < 1e-13
    mz, corr, ploop = M.polyakov_operators(cfg, 2, 3)
    assert relerr(mz.value, g["polyakov/meson_operator"]) < 1e-12
    assert relerr(corr.value, g["polyakov/polyakov_correlator"]) < 1e-12
    assert abs(ploop.value - g["polyakov/polyakov_loop"]) < 1e-13
    assert relerr(np_(M.polyakov_loop_field(cfg, 1)), g["polyakov_loop_field/1"]) < 1e-13
    pz, sz = M.glueball_operators(cfg, 2)
    assert relerr(pz.value, g["glueball/zpp_operator"]) < 1e-12
    assert relerr(sz.value, g["glueball/square_operator"]) < 1e-12
    loops = M.wilson_loops(cfg, 0, 3, 2, 3)
    assert [m.name for m in loops] == [f"wilson_loop_{r}_{t}" for r in (1, 2) for t in (1, 2, 3)]
    for m in loops:
        assert abs(m.value - g[f"wilson/{m.name}"]) < 1e-13, m.name
    tables = O.lookup_tables(geometry)
    lines = M.wilson_lines_field(cfg, 2, 2)
    for k, line in enumerate(lines):
        assert relerr(np_(line), O.path_product(g["gauge"], tables, [3] * (k + 1))) < 1e-14
    sm = smearing.ape_smearing(cfg, 0.3, no_smear_direction=3)
    assert relerr(np_(sm.gauge_field), g["ape/gauge"]) < 1e-13
    # a caller that consumes get_staple_fields the way smearing.py:38-44 does (len of
    # each direction's list, their sum) gets the reference's APE links too
    from tfleonardym_b200 import staples
    rho = 0.3
    fat = []
    for mu, elem in enumerate(staples.get_staple_fields(cfg, 3)):
        if len(elem) != 0:
            fat.append((rho / 6) * torch.stack(elem).sum(0))
        else:
            fat.append(rho * cfg.gauge_field[mu])
    unitary = smearing.unitary_sqrt_projection(torch.stack(fat) + (1 - rho) * cfg.gauge_field)
    assert relerr(np_(unitary), g["ape/gauge"]) < 1e-13
    res = smearing.multi_smearing_operators(cfg, [lambda c: M.glueball_operators(c, 2)], smearing_levels=2, rho=0.3,
                                            no_smear_direction=3, skip=1)
    assert relerr(np.stack([m.value for m in res]), g["multi/values"]) < 1e-12
    assert [m.smearing_levels for m in res] == list(g["multi/levels"])


@pytest.mark.parametrize("nc", [2, 3])
def test_random_momenta_kernel(cuda_device, nc):
    """Momenta from normals on the device (one kernel) equal the oracle's
    restatement of random_momenta (hmc.py:69-96) for the same draws; a large draw
    is anti-Hermitian and traceless to rounding, with zero mean and unit variance
    per generator (omega_a = -2i Tr(P T^a), T^a = lambda^a / 2)."""
    from tfleonardym_b200 import hmc, lie_generators
    nd, vol = 4, 6 * 4 * 4 * 8
    g = torch.Generator(device="cuda")
    g.manual_seed(5 + nc)
    normals = torch.randn((nd, nc * nc - 1, vol), dtype=torch.float64, device="cuda", generator=g)
    p = np_(hmc.momenta_from_normals(normals, nc))
    assert relerr(p, O.random_momenta_from_normals(np_(normals), nc)) < 1e-15
    big = hmc.random_momenta(nc, 2, 200000, generator=g)
    pb = np_(big)
    herm = pb + np.conj(np.swapaxes(pb, 1, 2))
    assert np.abs(herm).max() < 1e-15
    assert np.abs(np.trace(pb, axis1=1, axis2=2)).max() < 1e-15
    gens = lie_generators.generators(nc, "fundamental")  # (N^2-1, N, N)
    omega = -2j * np.einsum("mijv,aji->mav", pb, gens)
    assert np.abs(omega.imag).max() < 1e-13
    w = omega.real
    n = w.shape[-1]
    assert np.abs(w.mean(-1)).max() < 5 / np.sqrt(n)
    assert np.abs(w.var(-1) - 1.0).max() < 6 * np.sqrt(2.0 / n)


def test_gauge_hmc_step_on_many_lattices_in_two_launches(cuda_device):
    """lym_gauge_hmc_step_multi over a mix of 2D SU(2), 3D SU(2), 4D SU(2) and 4D SU(3)
    lattices equals, lattice by lattice, the fused force-into-momenta kernel followed
    by the link update (1e-13)."""
    from tfleonardym_b200 import gauge_action, hmc
    from tfleonardym_b200 import lattice as lt
    specs = [((8, 6), 2, 2.3), ((4, 6, 4), 2, 2.0), ((4, 4, 2, 6), 2, 2.3), ((2, 4, 4, 6), 3, 5.6),
             ((10, 12), 2, 3.0), ((4, 4, 4, 4), 3, 5.8)]
    rng = np.random.default_rng(9)
    cfgs, moms, ref_u, ref_p = [], [], [], []
    for geom, nc, beta in specs:
        nd, vol = len(geom), int(np.prod(geom))
        u = O.unitary_sqrt_projection(rng.normal(size=(nd, nc, nc, vol)) + 1j * rng.normal(size=(nd, nc, nc, vol)))
        p = np_(hmc.random_momenta(nc, nd, vol))
        cfg = lt.Configuration(cu(u), geom, nc, nd)
        pr = cu(p)
        gauge_action.yang_mills(cfg, beta).force_into_momenta(pr, -0.07)
        ref_p.append(np_(pr))
        ref_u.append(np_(hmc.update_link_field(cu(u), pr, 0.05)))
        cfgs.append(lt.Configuration(cu(u), geom, nc, nd))
        moms.append(cu(p))
    hmc.gauge_step_lattices(cfgs, moms, [b for _, _, b in specs], -0.07, 0.05)
    for k in range(len(specs)):
        assert relerr(np_(moms[k]), ref_p[k]) < 1e-13, k
        assert relerr(np_(cfgs[k].gauge_field), ref_u[k]) < 1e-13, k
    # two lattices on one momenta buffer would race in the same launch: refused
    with pytest.raises(RuntimeError, match="share a buffer"):
        hmc.gauge_step_lattices(cfgs[:2], [moms[0], moms[0]], [2.3, 2.3], -0.07, 0.05)


def test_md_energy_violation_is_second_order(cuda_device):
    """Nf = 2 Wilson + Wilson gauge action on 2x4x4x6 SU(3), Omelyan [n, 1], t = 1, the same
    momenta and pseudofermions for every n: the energy violation of the second-order
    integrator (hmc.py:104-162) falls by four when the step halves -- the molecular
    dynamics integrates the Hamiltonian whose energy the Metropolis step measures."""
    from tfleonardym_b200 import dirac, dirac_solver, fermion_action, gauge_action, hmc
    dirac_solver.VERBOSE = False
    g = load_golden("d4")
    spec = GOLDEN_CASES["d4"]
    q = make_op(g, spec)
    solver = dirac_solver.multishift_solver(5000, 1e-24)
    ra = dirac.RationalApproximation(dirac.SquareOperator(q), [1.0], [0.0], 0, solver)
    nf = fermion_action.n_flavor([ra], [ra], [q], solver, q)
    dhs = []
    for n in (4, 8, 16):
        cfg = make_cfg(g["gauge"], spec["geometry"])
        nf.set_gauge_configuration(cfg)
        nf.initialize_pseudofermions([cu(g["eta"])])
        ym = gauge_action.yang_mills(cfg, spec["beta"])
        _, minus_dh, _ = hmc.hybrid_mc(cfg, [nf, ym], [n, 1], 1.0, momenta=cu(g["momenta"]), uniform=1.0)
        dhs.append(abs(minus_dh))
    assert dhs[0] > dhs[1] > dhs[2] > 0, dhs
    for a, b in zip(dhs, dhs[1:]):
        assert 3.0 < a / b < 5.5, dhs
