"""Pin the CPU oracle to golden vectors produced by the unmodified reference.

Every reference-restating function of ``oracle/lym_oracle.py`` is compared to
the reference's own outputs on identical inputs (``tests/golden/*.npz``).
Tolerances: 1e-13 relative for straight-line arithmetic (differences are
summation order only); bit-exact for the integer tables.
"""
import numpy as np
import pytest

from oracle import lym_oracle as O
from tests.conftest import ADJOINT_CASES, GOLDEN_CASES, MEASUREMENT_CASES, OBSERVABLE_CASES, load_golden, relerr

TOL = 1e-13


def test_lookup_tables_bit_exact():
    z = load_golden("tables")
    geoms = sorted({k.split("/")[0] for k in z})
    assert len(geoms) >= 5
    for key in geoms:
        geom = tuple(int(g) for g in key.split("x"))
        sup, sdn, coords = O.lookup_tables(geom)
        assert sup.dtype == np.int64
        np.testing.assert_array_equal(sup, z[f"{key}/sup"])
        np.testing.assert_array_equal(sdn, z[f"{key}/sdn"])
        np.testing.assert_array_equal(coords, z[f"{key}/coords"])
        np.testing.assert_array_equal(O.antiperiodic_field(geom), z[f"{key}/bc"])


@pytest.mark.parametrize("case", list(GOLDEN_CASES))
def test_wilson_apply(case):
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    tables = O.lookup_tables(spec["geometry"])
    bcf = O.antiperiodic_field(spec["geometry"])
    for herm in (0, 1):
        for bcname in ("periodic", "anti"):
            gauge = O.apply_time_bc(g["gauge"], bcf) if bcname == "anti" else g["gauge"]
            out = O.wilson_apply(gauge, g["eta"], spec["kappa"], bool(herm), tables)
            assert relerr(out, g[f"apply/h{herm}/{bcname}/projected"]) < TOL
    # projected == simple in the reference itself (tests.py:51-59)
    assert relerr(g["apply/h1/anti/simple"], g["apply/h1/anti/projected"]) < TOL


@pytest.mark.parametrize("case", list(GOLDEN_CASES))
def test_gauge_side(case):
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    geom = spec["geometry"]
    tables = O.lookup_tables(geom)
    u = g["gauge"]
    assert relerr(O.dot(g["eta"], g["eta2"]), g["dot/eta_eta2"]) < TOL
    assert abs(O.plaquette(u, tables) - g["plaquette"]) < 1e-14
    assert relerr(O.staples(u, tables), g["staples_all"]) < TOL
    if "staples_no3" in g:
        assert relerr(O.staples(u, tables, no_direction=3), g["staples_no3"]) < TOL
    for key, nodir in (("staple_terms_all", len(geom)), ("staple_terms_no3", 3)):
        if f"{key}/0" not in g:
            continue
        lists = O.staple_terms(u, tables, no_direction=nodir)
        for mu, elem in enumerate(lists):
            want = g[f"{key}/{mu}"]
            assert len(elem) == want.shape[0], (key, mu)
            for k, term in enumerate(elem):
                assert relerr(term, want[k]) < TOL, (key, mu, k)
    assert relerr(O.gauge_force(u, spec["beta"], tables), g["gauge_force"]) < TOL
    assert abs(O.gauge_energy(u, spec["beta"], tables) - g["gauge_energy"]) < 1e-12 * abs(g["gauge_energy"])
    assert abs(O.momenta_energy(g["momenta"]) - g["momenta_energy"]) < 1e-12 * abs(g["momenta_energy"])
    assert relerr(O.update_link_field(u, g["momenta"], 0.1), g["update_link_field"]) < 1e-13
    assert relerr(O.update_momenta(g["momenta"], g["gauge_force"], -0.05), g["update_momenta"]) < TOL
    assert relerr(O.unitary_sqrt_projection(g["unitary_in"]), g["unitary_out"]) < 1e-12
    bcf = O.antiperiodic_field(geom)
    ld = O.lie_derivative(O.apply_time_bc(u, bcf), g["eta"], g["eta2"], spec["kappa"], True, tables)
    assert relerr(ld, g["lie_derivative"]) < TOL


def test_momenta_structure():
    """random_momenta output (hmc.py:69-96) is anti-Hermitian and traceless."""
    g = load_golden("d4")
    p = g["momenta"]
    assert np.abs(p + np.conj(np.transpose(p, (0, 2, 1, 3)))).max() < 1e-15
    assert np.abs(np.einsum("miic->mc", p)).max() < 1e-15


@pytest.mark.parametrize("case", ["d2", "d4"])
def test_mmmr_and_bicgstab(case):
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    setup = O.WilsonSetup(g["gauge"], spec["kappa"], spec["geometry"])
    shifts = list(g["mmmr/shifts"])
    sols, step, ok = O.mmmr_multishift(setup.Q2, g["eta"], shifts, 2000, float(g["mmmr/precision"]))
    assert ok
    # the reference prints `step`; identical arithmetic gives the identical count
    assert step == int(g["mmmr/iterations"][0])
    for s, ref in zip(sols, g["mmmr/solutions"]):
        assert relerr(s, ref) < 1e-10
    x, step_b, ok_b = O.bicgstab(lambda v: setup.Q2(v) + shifts[-1] * v, g["eta"], 2000, 1e-11)
    assert ok_b and abs(step_b - int(g["bicgstab/iterations"][0])) <= 1
    assert relerr(x, g["bicgstab/solution"]) < 1e-8


@pytest.mark.parametrize("case", ["d2", "d4"])
def test_nf2_energy_force(case):
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    setup = O.WilsonSetup(g["gauge"], spec["kappa"], spec["geometry"])
    phi = setup.Q(g["eta"])
    assert relerr(phi, g["nf2/phi"]) < TOL

    def solve(a, b, shifts):
        return O.mmmr_multishift(a, b, shifts, 5000, 1e-22)[0]

    e = O.fermion_energy(setup, phi, [1.0], [0.0], solve)
    assert abs(e - g["nf2/energy"]) < 1e-9 * abs(g["nf2/energy"])
    f = O.fermion_force(setup, phi, [1.0], [0.0], solve)
    assert relerr(f, g["nf2/force"]) < 1e-9


@pytest.mark.parametrize("case", ["d2", "d4"])
def test_md_trajectory(case):
    """integrate_om (hmc.py:133-162) with the Nf=2 and gauge forces."""
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    setup = O.WilsonSetup(g["gauge"], spec["kappa"], spec["geometry"])
    tables = setup.tables
    phi = setup.Q(g["eta"])

    def solve(a, b, shifts):
        return O.mmmr_multishift(a, b, shifts, 5000, 1e-22)[0]

    def f_ferm(u):
        setup.set_gauge(u)
        return O.fermion_force(setup, phi, [1.0], [0.0], solve)

    def f_gauge(u):
        return O.gauge_force(u, spec["beta"], tables)

    u, p = O.integrate_om(g["gauge"], g["md/momenta_in"], [f_ferm, f_gauge], list(g["hmc/steps"]), 1.0)
    assert relerr(u, g["md/cfg_out"]) < 1e-10
    assert relerr(p, g["md/momenta_out"]) < 1e-10


# ---------------------------------------------------------------------------
# adjoint representation
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("case", list(ADJOINT_CASES))
def test_adjoint_apply_links_and_lie_derivative(case):
    """Adjoint Wilson operator (projected and simple forms, all hermiticity / BC
    pairs), adjoint links and Lie derivative against the reference's outputs."""
    g = load_golden(case)
    spec = ADJOINT_CASES[case]
    tables = O.lookup_tables(spec["geometry"])
    bcf = O.antiperiodic_field(spec["geometry"])
    u = g["gauge"]
    for herm in (0, 1):
        for bcname in ("periodic", "anti"):
            ub = O.apply_time_bc(u, bcf) if bcname == "anti" else u
            out = O.wilson_apply_adjoint(ub, u, g["eta"], spec["kappa"], bool(herm), tables)
            assert relerr(out, g[f"apply/h{herm}/{bcname}/projected"]) < TOL, (herm, bcname)
            assert relerr(out, g[f"apply/h{herm}/{bcname}/simple"]) < TOL, (herm, bcname)
    v = O.adjoint_links(u, bcf)
    assert relerr(v, g["fermion_gauge_field"]) < TOL
    for herm in (0, 1):
        d = O.lie_derivative_adjoint(v, g["eta"], g["eta2"], spec["kappa"], bool(herm), tables)
        assert relerr(d, g[f"lie_derivative/h{herm}"]) < 1e-12, herm


@pytest.mark.parametrize("case", list(ADJOINT_CASES))
def test_adjoint_nf2_energy_force(case):
    """Nf=2 in the adjoint: phi = Q eta, S = <phi, (Q^2)^-1 phi>, force from the
    Lie derivatives of x = (Q^2)^-1 phi and Q x (fermion_action.py:64-93)."""
    g = load_golden(case)
    spec = ADJOINT_CASES[case]
    geometry, kappa = spec["geometry"], spec["kappa"]
    tables = O.lookup_tables(geometry)
    bcf = O.antiperiodic_field(geometry)
    u = g["gauge"]
    ub = O.apply_time_bc(u, bcf)

    def q(v):
        return O.wilson_apply_adjoint(ub, u, v, kappa, True, tables)

    phi = q(g["eta"])
    assert relerr(phi, g["nf2/phi"]) < TOL
    # (Q^2)^-1 phi by CG to full precision
    x = np.zeros_like(phi)
    r = phi.copy()
    p = r.copy()
    rr = np.vdot(r, r).real
    for _ in range(2000):
        ap = q(q(p))
        a = rr / np.vdot(p, ap).real
        x += a * p
        r -= a * ap
        rn = np.vdot(r, r).real
        if rn < 1e-28 * np.vdot(phi, phi).real:
            break
        p = r + (rn / rr) * p
        rr = rn
    assert abs(np.vdot(phi, x).real - g["nf2/energy"]) < 1e-9 * abs(g["nf2/energy"])
    v = O.adjoint_links(u, bcf)
    y = q(x)
    force = O.lie_derivative_adjoint(v, x, y, kappa, True, tables) + \
        O.lie_derivative_adjoint(v, y, x, kappa, True, tables)
    assert relerr(force, g["nf2/force"]) < 1e-8


# ---------------------------------------------------------------------------
# fermion measurements
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("case", list(MEASUREMENT_CASES))
def test_measurements(case):
    """Propagator, pion correlator (all ns x colour point sources at site 0) and the
    chiral condensate on the recorded Z2 noise, against the reference (whose
    BiCGStab stops at |r|^2 < 1e-13 for the correlator and 1e-10 for the condensate,
    so those two agree to the solves' accuracy only)."""
    g = load_golden(case)
    spec = MEASUREMENT_CASES[case]
    geometry, kappa = spec["geometry"], spec["kappa"]
    adjoint = spec["representation"] == "adjoint"
    tables = O.lookup_tables(geometry)
    u = g["gauge"]
    ub = O.apply_time_bc(u, O.antiperiodic_field(geometry))
    nd, nc, vol = len(geometry), u.shape[1], u.shape[-1]
    ns = 2 if nd == 2 else 4

    def q(v):
        if adjoint:
            return O.wilson_apply_adjoint(ub, u, v, kappa, True, tables)
        return O.wilson_apply(ub, v, kappa, True, tables)

    assert relerr(O.propagator(q, g["propagator/source"]), g["propagator/out"]) < 1e-8
    ncol = nc * nc - 1 if adjoint else nc
    sols = [O.propagator(q, O.point_source(0, c, s, vol, nc, ns, adjoint)) for s in range(ns) for c in range(ncol)]
    corr = O.pion_correlator(sols, tables[2], nd - 1, geometry[-1], adjoint)
    assert relerr(corr, g["pion_correlator"]) < 1e-5
    cc = np.mean([O.dot(src, O.propagator(q, src)) / vol for src in g["chiral_condensate/sources"]])
    assert abs(cc - g["chiral_condensate"]) < 1e-4 * abs(g["chiral_condensate"])


def test_read_config_xdr():
    """The XDR configuration reader (lattice.py:10-70) against the reference's output."""
    g = load_golden("xdr_su3")
    geometry = tuple(int(d) for d in g["geometry"])
    gauge, dims, params = O.read_config_xdr(g["raw"], geometry)
    assert relerr(gauge, g["gauge"]) < 1e-15
    assert dims == list(geometry) and params == [5.6, 0.13, 1.0]


# ---------------------------------------------------------------------------
# gauge observables and smearing
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("case", list(OBSERVABLE_CASES))
def test_gauge_observables_and_smearing(case):
    g = load_golden(case)
    geometry = OBSERVABLE_CASES[case]["geometry"]
    tables = O.lookup_tables(geometry)
    u = g["gauge"]
    assert abs(O.temporal_plaquette(u, tables) - g["temporal_plaquette"]) < 1e-13
    mz, corr, ploop = O.polyakov_operators(u, tables, geometry, 2, 3)
    assert relerr(mz, g["polyakov/meson_operator"]) < 1e-12
    assert relerr(corr, g["polyakov/polyakov_correlator"]) < 1e-12
    assert abs(ploop - g["polyakov/polyakov_loop"]) < 1e-13
    assert relerr(O.polyakov_loop_field(u, tables, geometry, 1), g["polyakov_loop_field/1"]) < 1e-13
    pz, sz = O.glueball_operators(u, tables, geometry, 2)
    assert relerr(pz, g["glueball/zpp_operator"]) < 1e-12
    assert relerr(sz, g["glueball/square_operator"]) < 1e-12
    loops = O.wilson_loops(u, tables, 0, 3, 2, 3)
    ref = [g[f"wilson/wilson_loop_{r}_{t}"] for r in range(1, 3) for t in range(1, 4)]
    assert relerr(np.array(loops), np.array(ref)) < 1e-12
    assert relerr(O.ape_smearing(u, tables, 0.3, 3), g["ape/gauge"]) < 1e-13
    # multi_smearing_operators: unsmeared glueball operators, then after each smearing step
    vals, v = [], u
    vals.extend(O.glueball_operators(v, tables, geometry, 2))
    for _ in range(2):
        v = O.ape_smearing(v, tables, 0.3, 3)
        vals.extend(O.glueball_operators(v, tables, geometry, 2))
    assert relerr(np.stack(vals), g["multi/values"]) < 1e-12
    assert list(g["multi/levels"]) == [0, 0, 0, 0, 1, 1]


@pytest.mark.parametrize("case", list(GOLDEN_CASES))
def test_wilson_apply_sites_matches_golden(case):
    """The site-restricted oracle apply (used at lattice sizes too large for a
    whole-field numpy apply) reproduces the reference's apply at every site."""
    g = load_golden(case)
    spec = GOLDEN_CASES[case]
    geom = spec["geometry"]
    tables = O.lookup_tables(geom)
    ub = O.apply_time_bc(g["gauge"], O.antiperiodic_field(geom))
    sites = np.arange(int(np.prod(geom)))[::3]
    for herm in (0, 1):
        out = O.wilson_apply_sites(ub, g["eta"], spec["kappa"], bool(herm), tables, sites)
        assert relerr(out, g[f"apply/h{herm}/anti/projected"][:, :, sites]) < TOL


def test_three_dimensional_adjoint_hop():
    """The oracle's D^dag (gamma -> -gamma, builder-defined for D = 3) is the adjoint of
    its D: <phi, D psi> = <D^dag phi, psi>; in 4D it equals gamma_d D gamma_d."""
    rng = np.random.default_rng(0)
    geom = (4, 4, 6)
    vol = int(np.prod(geom))
    u = O.unitary_sqrt_projection(rng.normal(size=(3, 3, 3, vol)) + 1j * rng.normal(size=(3, 3, 3, vol)))
    t = O.lookup_tables(geom)
    ub = O.apply_time_bc(u, O.antiperiodic_field(geom))
    phi = rng.normal(size=(2, 3, vol)) + 1j * rng.normal(size=(2, 3, vol))
    psi = rng.normal(size=(2, 3, vol)) + 1j * rng.normal(size=(2, 3, vol))
    a = np.vdot(phi, O.wilson_apply(ub, psi, 0.13, False, t))
    b = np.vdot(O.wilson_apply(ub, phi, 0.13, False, t, dagger=True), psi)
    assert abs(a - b) < 1e-13 * abs(a)
    with pytest.raises(RuntimeError, match="hermitian"):
        O.wilson_apply(ub, psi, 0.13, True, t)
    g = load_golden("d4")
    geom4 = GOLDEN_CASES["d4"]["geometry"]
    t4 = O.lookup_tables(geom4)
    u4 = O.apply_time_bc(g["gauge"], O.antiperiodic_field(geom4))
    d4 = O.wilson_apply(u4, g["eta"], 0.13, False, t4, dagger=True)
    assert np.abs(d4 - O.gamma_d(O.wilson_apply(u4, O.gamma_d(g["eta"]), 0.13, False, t4))).max() < 1e-14
