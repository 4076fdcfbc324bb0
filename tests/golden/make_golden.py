"""Generate golden vectors by running the unmodified reference on CPU.

Test infrastructure only.  Run where a checkout of the reference tree is
available, naming it with --reference (or the LYM_REFERENCE_DIR environment
variable):

    python tests/golden/make_golden.py --reference <reference tree>            # all cases
    python tests/golden/make_golden.py --reference <reference tree> --case d2  # one case

Each case runs in its own subprocess because the reference binds its
lookup tables at import time (``from translate import lookup_tables`` in
boundary_conditions.py:3, hmc.py:2, staples.py:2, measurements.py:4), so one
process can hold one geometry only.  The reference runs on the numpy-backed
``tensorflow`` stand-in in ``tfshim/``; all randomness comes from that
stand-in's seeded generator and is saved next to the outputs, so the oracle
and the GPU path can be fed the identical inputs.

Harness-side deviations from the shipped reference scripts (the reference
files themselves are never modified):
  * the boundary-condition provider takes one argument, as
    dirac.py:369 calls it (tests.py:17-25 passes two and crashes);
  * ``hmc.metropolis`` is replaced by the same rule (metropolis.py:11-18)
    with a uniform drawn from a seeded generator on every call and saved;
  * ``dirac_solver.print`` is captured to record solver iteration counts
    (dirac_solver.py:49,102);
  * ``lattice.Configuration`` fills in ``number_of_dimensions`` from the gauge
    field when a caller leaves it out: ``read_config`` (lattice.py:69-70) and
    ``ape_smearing`` (smearing.py:49-51) build it with three fields and raise.
"""
import argparse
import os
import re
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("LYM_REFERENCE_DIR", "")

CASES = {
    # the CPU-runnable HMC case: D=2 24x16 SU(2), kappa=-0.15, beta=3.0
    "d2": dict(geometry=(24, 16), nc=2, kappa=-0.15, beta=3.0, seed=11,
               hmc_steps=[4, 3], n_traj=10, shifts=[0.5, 0.1, 0.01]),
    # 4D SU(3) on an asymmetric small lattice, kappa=0.13, beta=5.6
    "d4": dict(geometry=(2, 4, 4, 6), nc=3, kappa=0.13, beta=5.6, seed=12,
               hmc_steps=[2, 2], n_traj=1, shifts=[0.5, 0.1, 0.01]),
    # extra (D, N) combinations: operator application only
    "d4su2": dict(geometry=(4, 4, 2, 4), nc=2, kappa=0.12, beta=2.3, seed=13,
                  apply_only=True),
    "d2su3": dict(geometry=(6, 8), nc=3, kappa=0.11, beta=5.0, seed=14,
                  apply_only=True),
}

# adjoint representation (dirac.py:380-456, 358-364, 525-565): operator, adjoint
# links, lie derivative, and the Nf=2 energy/force through the reference's MMMR
ADJOINT_CASES = {
    "adj_d2su2": dict(geometry=(8, 6), nc=2, kappa=0.17, seed=21),
    "adj_d4su3": dict(geometry=(2, 4, 2, 4), nc=3, kappa=0.12, seed=22),
    "adj_d4su2": dict(geometry=(4, 2, 2, 4), nc=2, kappa=0.13, seed=23),
}

# fermion measurements (fermion_measurements.py:41-115, dirac.py:665-696): pion
# correlator from point sources, chiral condensate from recorded Z2 noise,
# one propagator application
MEASUREMENT_CASES = {
    "meas_d2": dict(geometry=(8, 6), nc=2, kappa=0.12, seed=31, representation="fundamental"),
    "meas_d4": dict(geometry=(2, 4, 2, 6), nc=3, kappa=0.11, seed=32, representation="fundamental"),
    "meas_adj": dict(geometry=(4, 6), nc=2, kappa=0.1, seed=33, representation="adjoint"),
}

# on-disk gauge format (lattice.py:10-70): an XDR file of two-column SU(3) links
# (U* stored, float32) written here, read by the reference's read_config
XDR_CASES = {
    "xdr_su3": dict(geometry=(4, 2, 4, 6), seed=41),
}

# gauge observables and smearing (measurements.py:46-330, smearing.py:34-86)
OBSERVABLE_CASES = {
    "obs_su3": dict(geometry=(4, 4, 4, 6), nc=3, seed=51),
    "obs_su2": dict(geometry=(4, 6, 4, 4), nc=2, seed=52),
}

TABLE_GEOMETRIES = [(2, 4, 6, 8), (3, 5, 2, 4), (4, 6, 8), (5, 7), (8, 8), (1, 4, 2, 2)]


def _complete_configuration():
    """lattice.Configuration with number_of_dimensions filled in from the gauge field
    when a caller leaves it out (read_config, lattice.py:69-70; ape_smearing,
    smearing.py:49-51 build it with three fields and raise)."""
    import lattice
    orig = lattice.Configuration

    def configuration(gauge_field, geometry, colors, number_of_dimensions=None):
        if number_of_dimensions is None:
            number_of_dimensions = int(np.asarray(gauge_field).shape[0])
        return orig(gauge_field, geometry, colors, number_of_dimensions)

    lattice.Configuration = configuration


def _setup_reference(geometry):
    sys.path.insert(0, REFERENCE)
    sys.path.insert(0, os.path.join(HERE, "tfshim"))
    import metropolis
    metropolis.set_metropolis(False)
    import translate
    translate.set_translate(False, list(geometry), [1] * len(geometry))
    import boundary_conditions
    boundary_conditions.set_antiperiodic_field_in_t_direction(tuple(geometry))


class _IterLog:
    """Collects the iteration counts the reference solvers print."""

    def __init__(self):
        self.records = []

    def __call__(self, *args, **_kw):
        msg = " ".join(str(a) for a in args)
        m = re.search(r"(MMMRMultishiftsolver|BiconjugateGradient): (convergence|failed to find convergence) after (\d+) steps", msg)
        if m:
            self.records.append((m.group(1), m.group(2) == "convergence", int(m.group(3))))

    def take(self):
        out, self.records = self.records, []
        return out


def run_tables():
    out = {}
    for geom in TABLE_GEOMETRIES:
        code = (
            "import sys, numpy as np\n"
            f"sys.path.insert(0, {REFERENCE!r}); sys.path.insert(0, {os.path.join(HERE, 'tfshim')!r})\n"
            "import lattice as lt\n"
            f"t = lt.mth_lookup_tables({tuple(geom)!r})\n"
            "import translate\n"
            f"translate.set_translate(False, {list(geom)!r}, {[1] * len(geom)!r})\n"
            "import boundary_conditions as bc\n"
            f"bc.set_antiperiodic_field_in_t_direction({tuple(geom)!r})\n"
            "np.savez(sys.argv[1], sup=np.asarray(t.sup), sdn=np.asarray(t.sdn),"
            " coords=np.asarray(t.global_coordinates), bc=np.asarray(bc.antiperiodic_field_in_t_direction))\n"
        )
        tmp = os.path.join(HERE, "_tmp_tables.npz")
        subprocess.run([sys.executable, "-c", code, tmp], check=True)
        with np.load(tmp) as z:
            key = "x".join(str(g) for g in geom)
            for k in z.files:
                out[f"{key}/{k}"] = z[k]
        os.remove(tmp)
    np.savez_compressed(os.path.join(HERE, "tables.npz"), **out)
    print("wrote tables.npz", len(out), "arrays")


# nested integrators whose call sequence is recorded (the reference's hmc.py run
# with recording stand-ins for update_momenta / update_configuration and the actions)
SCHEDULE_CASES = [("integrate_om", [4, 3], 1.0), ("integrate_om", [2, 2], 1.0), ("integrate_om", [10, 2], 1.0),
                  ("integrate_om", [3, 2, 2], 0.5), ("integrate_om", [4, 3], -1.0), ("integrate_om", [1], 1.0),
                  ("integrate_lp", [4, 3], 1.0), ("integrate_lp", [2, 3, 2], 1.0)]


def run_schedules():
    """The sequence of momentum kicks (level, weight) and link drifts (weight) the
    reference's integrate_om / integrate_lp (hmc.py:104-162) perform, with two
    kicks in a row that reuse one force (the closing kick) summed into one."""
    _setup_reference((4, 4))
    import hmc

    class Force:
        def __init__(self, level, ident):
            self.level, self.ident = level, ident

    class Action:
        def __init__(self, level, counter):
            self.level, self.counter = level, counter

        def set_gauge_configuration(self, cfg):
            pass

        def force(self):
            self.counter[0] += 1
            return Force(self.level, self.counter[0])

    out = {}
    for fn, steps, dt in SCHEDULE_CASES:
        seq = []

        def update_momenta(m, f, eps, seq=seq):
            if seq and seq[-1][0] == "kick" and seq[-1][3] == f.ident:
                seq[-1] = ("kick", f.level, seq[-1][2] + eps, f.ident)
            else:
                seq.append(("kick", f.level, eps, f.ident))
            return m

        def update_configuration(cfg, m, eps, seq=seq):
            seq.append(("drift", len(steps) - 1, eps, None))
            return cfg

        hmc.update_momenta = update_momenta
        hmc.update_configuration = update_configuration
        counter = [0]
        actions = [Action(level, counter) for level in range(len(steps))]
        getattr(hmc, fn)(None, None, actions, steps, dt)
        key = f"{fn}/{'_'.join(str(k) for k in steps)}/{dt}"
        out[key] = [[kind, level, weight] for kind, level, weight, _ in seq]
    import json
    with open(os.path.join(HERE, "md_schedules.json"), "w") as f:
        f.write("{\n" + ",\n".join(f"{json.dumps(k)}: {json.dumps(v)}" for k, v in out.items()) + "\n}\n")
    print("wrote md_schedules.json", len(out), "schedules")


def run_case(name):
    spec = CASES[name]
    geometry = spec["geometry"]
    nd, nc = len(geometry), spec["nc"]
    _setup_reference(geometry)
    import tensorflow as tf
    tf.set_seed(spec["seed"])
    np.random.seed(spec["seed"])

    import boundary_conditions
    import dirac
    import dirac_solver
    import hmc
    import gauge_action
    import staples
    import measurements
    import fermion_action
    import smearing
    import algebra_utils

    log = _IterLog()
    dirac_solver.print = log

    def bc_anti(x):
        return boundary_conditions.apply_antiboundary_conditions_in_t_direction(x)

    def bc_periodic(x):
        return x

    out = {}
    kappa, beta = spec["kappa"], spec["beta"]
    cfg = hmc.hotstart(list(geometry), nc, nd)
    out["gauge"] = np.asarray(cfg.gauge_field)
    ns = 2 if nd == 2 else 4
    eta = hmc.generate_random_vector(nc, ns)
    eta2 = hmc.generate_random_vector(nc, ns)
    out["eta"], out["eta2"] = np.asarray(eta), np.asarray(eta2)

    # dirac.py:458-523,649-662 -- all (hermitian, bc, mode) combinations
    for herm in (False, True):
        for bcname, prov in (("periodic", bc_periodic), ("anti", bc_anti)):
            op = dirac.DiracWilsonOperator(cfg, kappa, herm, representation="fundamental",
                                           boundary_condition_provider=prov)
            out[f"apply/h{int(herm)}/{bcname}/projected"] = np.asarray(op.multiply_in_fundamental_representation(eta))
            if herm and bcname == "anti":
                out[f"apply/h{int(herm)}/{bcname}/simple"] = np.asarray(
                    op.simple_multiply_in_fundamental_representation(eta))
    out["dot/eta_eta2"] = np.asarray(algebra_utils.dot(eta, eta2))
    out["plaquette"] = np.asarray(measurements.plaquette(cfg).value)

    ym = gauge_action.yang_mills(cfg, beta)
    out["gauge_force"] = np.asarray(ym.force())
    out["gauge_energy"] = np.asarray(ym.energy())
    st = gauge_action._get_staple_fields(cfg, no_direction=nd)
    out["staples_all"] = np.asarray([np.sum([np.asarray(s) for s in elem], axis=0) for elem in st])
    if nd > 3:
        st3 = staples.get_staple_fields(cfg)  # default no_direction=3 (staples.py:23)
        out["staples_no3"] = np.asarray([np.sum([np.asarray(s) for s in elem], axis=0) if elem else
                                         np.zeros((nc, nc, cfg.gauge_field.shape[-1]), complex) for elem in st3])
        # the per-plane terms themselves, in the reference's list order (staples.py:49-58)
        for mu, elem in enumerate(st3):
            out[f"staple_terms_no3/{mu}"] = (np.stack([np.asarray(s) for s in elem]) if elem else
                                             np.zeros((0, nc, nc, cfg.gauge_field.shape[-1]), complex))
    st_all = staples.get_staple_fields(cfg, no_direction=nd)
    for mu, elem in enumerate(st_all):
        out[f"staple_terms_all/{mu}"] = np.stack([np.asarray(s) for s in elem])

    mom = hmc.random_momenta(nc, nd)
    out["momenta"] = np.asarray(mom)
    out["momenta_energy"] = np.asarray(hmc.momenta_energy(mom))
    out["update_link_field/eps"] = np.asarray(0.1)
    out["update_link_field"] = np.asarray(hmc.update_link_field(cfg.gauge_field, mom, 0.1))
    out["update_momenta"] = np.asarray(hmc.update_momenta(mom, out["gauge_force"], -0.05))
    gauss = tf.complex(tf.random.normal(shape=(nd, nc, nc, cfg.gauge_field.shape[-1]), dtype=tf.float64),
                       tf.random.normal(shape=(nd, nc, nc, cfg.gauge_field.shape[-1]), dtype=tf.float64))
    out["unitary_in"] = np.asarray(gauss)
    out["unitary_out"] = np.asarray(smearing.unitary_sqrt_projection(gauss))

    Q = dirac.DiracWilsonOperator(cfg, kappa, True, representation="fundamental", boundary_condition_provider=bc_anti)
    out["lie_derivative"] = np.asarray(Q.lie_derivative(eta, eta2))

    if spec.get("apply_only"):
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print("wrote", name)
        return

    # dirac_solver.py:19-53 multishift MMMR on Q^2 (absolute |r|^2 stop), tests.py:96-106
    Q2 = dirac.SquareOperator(Q)
    shifts = spec["shifts"]
    sols = dirac_solver.multishift_solver(2000, 1e-11).solve(Q2, eta, shifts)
    out["mmmr/shifts"] = np.asarray(shifts)
    out["mmmr/precision"] = np.asarray(1e-11)
    out["mmmr/solutions"] = np.asarray([np.asarray(s) for s in sols])
    rec = log.take()
    out["mmmr/iterations"] = np.asarray([r[2] for r in rec])
    # dirac_solver.py:61-110 BiCGStab on Q^2 + 0.01, tests.py:108-113
    bic = dirac_solver.biconjugate_gradient(2000, 1e-11).solve(dirac.ShiftedOperator(Q2, shifts[-1]), eta)
    out["bicgstab/solution"] = np.asarray(bic)
    out["bicgstab/iterations"] = np.asarray([r[2] for r in log.take()])

    # Nf=2 fundamental: fermion_action.py with R(Q^2) = (Q^2)^-1 and heatbath = Q
    solver = dirac_solver.multishift_solver(5000, 1e-22)
    ra = dirac.RationalApproximation(dirac.SquareOperator(Q), [1.0], [0.0], 0, solver)
    nf = fermion_action.n_flavor([ra], [ra], [Q], solver, Q)
    nf.set_gauge_configuration(cfg)
    nf.initialize_pseudofermions([eta])
    out["nf2/phi"] = np.asarray(nf.pseudofermions[0])
    out["nf2/energy"] = np.asarray(nf.energy())
    out["nf2/force"] = np.asarray(nf.force())
    log.take()

    # hmc.py:218-278 -- trajectories with harness-supplied momenta / eta / uniform
    rng = np.random.default_rng(spec["seed"] + 1000)
    state = {}

    orig_random_momenta = hmc.random_momenta

    def recording_momenta(ncol, ndim):
        m = orig_random_momenta(ncol, ndim)
        state.setdefault("momenta", []).append(np.asarray(m))
        return m

    def recording_metropolis(new_energy, old_energy):
        u = rng.uniform()
        state.setdefault("uniform", []).append(u)
        if new_energy < old_energy:
            return True
        return bool(u < np.exp(-(new_energy - old_energy)))

    hmc.random_momenta = recording_momenta
    hmc.metropolis = recording_metropolis
    actions = [nf, ym]

    # one molecular-dynamics trajectory, hmc.py:133-162, outputs kept
    md_mom = orig_random_momenta(nc, nd)
    nf.set_gauge_configuration(cfg)
    nf.initialize_pseudofermions([eta])
    md_cfg, md_p = hmc.integrate_om(cfg, md_mom, actions, spec["hmc_steps"], 1.0)
    out["md/momenta_in"] = np.asarray(md_mom)
    out["md/cfg_out"] = np.asarray(md_cfg.gauge_field)
    out["md/momenta_out"] = np.asarray(md_p)
    out["md/iterations"] = np.asarray(sum(r[2] for r in log.take()))

    traj = {"dH": [], "accepted": [], "plaquette": [], "iterations": [], "eta": []}
    out["hmc/steps"] = np.asarray(spec["hmc_steps"])
    cur = cfg
    for _ in range(spec["n_traj"]):
        e = hmc.generate_random_vector(nc, ns)
        traj["eta"].append(np.asarray(e))
        nf.set_gauge_configuration(cur)
        nf.initialize_pseudofermions([e])
        cur, minus_dh, acc = hmc.hybrid_mc(cur, actions, spec["hmc_steps"], 1.0)
        traj["dH"].append(-float(np.real(minus_dh)))
        traj["accepted"].append(bool(acc))
        traj["plaquette"].append(float(measurements.plaquette(cur).value))
        traj["iterations"].append(sum(r[2] for r in log.take()))
    for k, v in traj.items():
        out[f"hmc/{k}"] = np.asarray(v)
    out["hmc/momenta"] = np.asarray(state["momenta"])
    out["hmc/uniform"] = np.asarray(state["uniform"])
    out["hmc/cfg_out"] = np.asarray(cur.gauge_field)

    # hmc.py:249-278 reversibility on the final configuration
    hmc.random_momenta = recording_momenta
    nf.set_gauge_configuration(cur)
    nf.initialize_pseudofermions([traj["eta"][0]])
    state["momenta"] = []
    out["hmc/reversibility_dH"] = np.asarray(hmc.reversibility_check(cur, actions, spec["hmc_steps"], 1.0))
    out["hmc/reversibility_momenta"] = np.asarray(state["momenta"][0])
    log.take()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print("wrote", name)


def run_adjoint_case(name):
    spec = ADJOINT_CASES[name]
    geometry = spec["geometry"]
    nd, nc = len(geometry), spec["nc"]
    _setup_reference(geometry)
    import tensorflow as tf
    tf.set_seed(spec["seed"])
    np.random.seed(spec["seed"])

    import boundary_conditions
    import dirac
    import dirac_solver
    import fermion_action
    import hmc

    log = _IterLog()
    dirac_solver.print = log

    def bc_anti(x):
        return boundary_conditions.apply_antiboundary_conditions_in_t_direction(x)

    def bc_periodic(x):
        return x

    out = {}
    kappa = spec["kappa"]
    cfg = hmc.hotstart(list(geometry), nc, nd)
    out["gauge"] = np.asarray(cfg.gauge_field)
    ns = 2 if nd == 2 else 4
    eta = hmc.generate_random_vector(nc, ns, "adjoint")
    eta2 = hmc.generate_random_vector(nc, ns, "adjoint")
    out["eta"], out["eta2"] = np.asarray(eta), np.asarray(eta2)
    for herm in (False, True):
        for bcname, prov in (("periodic", bc_periodic), ("anti", bc_anti)):
            op = dirac.DiracWilsonOperator(cfg, kappa, herm, representation="adjoint",
                                           boundary_condition_provider=prov)
            out[f"apply/h{int(herm)}/{bcname}/projected"] = np.asarray(op.multiply_in_adjoint_representation(eta))
            out[f"apply/h{int(herm)}/{bcname}/simple"] = np.asarray(op.simple_multiply_in_adjoint_representation(eta))
            if bcname == "anti":
                out[f"lie_derivative/h{int(herm)}"] = np.asarray(op.lie_derivative(eta, eta2))
    Q = dirac.DiracWilsonOperator(cfg, kappa, True, representation="adjoint", boundary_condition_provider=bc_anti)
    out["fermion_gauge_field"] = np.asarray(Q.fermion_gauge_field)
    # Nf=2 in the adjoint: phi = Q eta, S = <phi, (Q^2)^-1 phi>, F = the lie derivatives of the solution
    solver = dirac_solver.multishift_solver(5000, 1e-22)
    ra = dirac.RationalApproximation(dirac.SquareOperator(Q), [1.0], [0.0], 0, solver)
    nf = fermion_action.n_flavor([ra], [ra], [Q], solver, Q)
    nf.set_gauge_configuration(cfg)
    nf.initialize_pseudofermions([eta])
    out["nf2/phi"] = np.asarray(nf.pseudofermions[0])
    out["nf2/energy"] = np.asarray(nf.energy())
    out["nf2/force"] = np.asarray(nf.force())
    log.take()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print("wrote", name)


def run_measurement_case(name):
    spec = MEASUREMENT_CASES[name]
    geometry = spec["geometry"]
    nd, nc, rep = len(geometry), spec["nc"], spec["representation"]
    _setup_reference(geometry)
    import tensorflow as tf
    tf.set_seed(spec["seed"])
    np.random.seed(spec["seed"])

    import boundary_conditions
    import dirac
    import dirac_solver
    import fermion_measurements
    import hmc
    import translate

    log = _IterLog()
    dirac_solver.print = log

    def bc_anti(x):
        return boundary_conditions.apply_antiboundary_conditions_in_t_direction(x)

    out = {}
    cfg = hmc.hotstart(list(geometry), nc, nd)
    out["gauge"] = np.asarray(cfg.gauge_field)
    Q = dirac.DiracWilsonOperator(cfg, spec["kappa"], True, representation=rep, boundary_condition_provider=bc_anti)
    corr = fermion_measurements.pion_correlator(Q, nd - 1, translate.lookup_tables, lambda x: x)
    out["pion_correlator"] = np.asarray(corr.value)
    recorded = []
    noise = fermion_measurements.generate_random_z2_noise

    def recording_noise(*a, **k):
        v = noise(*a, **k)
        recorded.append(np.asarray(v))
        return v

    fermion_measurements.generate_random_z2_noise = recording_noise
    cc = fermion_measurements.chiral_condensate(Q, num_estimators=3)
    out["chiral_condensate"] = np.asarray(cc.value)
    out["chiral_condensate/sources"] = np.stack(recorded)
    prop = dirac.Propagator(Q, dirac_solver.biconjugate_gradient(5000, 1e-20))
    src = fermion_measurements.generate_point_source(1, 0, 1, Q.volume, nc, Q.spinor_dimension, rep)
    out["propagator/source"] = np.asarray(src)
    out["propagator/out"] = np.asarray(prop.apply(src))
    log.take()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print("wrote", name)


def run_xdr_case(name):
    import xdrlib  # Python <= 3.12 (the reference's own reader uses it)
    spec = XDR_CASES[name]
    geometry = spec["geometry"]
    nd, nc, vol = len(geometry), 3, int(np.prod(geometry))
    rng = np.random.default_rng(spec["seed"])
    # near-SU(3) links; the file holds conj(U)'s first two columns in float32
    a = rng.normal(size=(vol, nd, nc, nc)) + 1j * rng.normal(size=(vol, nd, nc, nc))
    q, _ = np.linalg.qr(a)
    cols = np.conj(q[..., :2])  # (V, nd, row, col<2)
    words = np.stack([cols.real, cols.imag], axis=-1).astype(np.float32).ravel()
    pk = xdrlib.Packer()
    pk.pack_farray(words.size, [float(w) for w in words], pk.pack_float)
    for d in geometry:
        pk.pack_int(int(d))
    for prm in (5.6, 0.13, 1.0):
        pk.pack_double(prm)
    raw = pk.get_buffer()
    path = os.path.join(HERE, f"_tmp_{name}.xdr")
    with open(path, "wb") as f:
        f.write(raw)
    _setup_reference(geometry)
    import lattice
    _complete_configuration()
    cfg = lattice.read_config(path, list(geometry), 3)
    os.remove(path)
    out = {"raw": np.frombuffer(raw, dtype=np.uint8), "gauge": np.asarray(cfg.gauge_field),
           "geometry": np.asarray(geometry)}
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print("wrote", name)


def run_observable_case(name):
    spec = OBSERVABLE_CASES[name]
    geometry = spec["geometry"]
    nd, nc = len(geometry), spec["nc"]
    _setup_reference(geometry)
    import tensorflow as tf
    tf.set_seed(spec["seed"])
    np.random.seed(spec["seed"])
    import hmc
    import measurements
    import smearing
    _complete_configuration()

    out = {}
    cfg = hmc.hotstart(list(geometry), nc, nd)
    # smooth the hot start a little so that loops are not pure noise
    cfg = smearing.ape_smearing(cfg, 0.5, no_smear_direction=-1)
    cfg = cfg._replace(geometry=list(geometry))
    out["gauge"] = np.asarray(cfg.gauge_field)
    out["temporal_plaquette"] = np.asarray(measurements.temporal_plaquette(cfg).value)
    for m in measurements.polyakov_operators(cfg, 2, 3):
        out[f"polyakov/{m.name}"] = np.asarray(m.value)
    for m in measurements.glueball_operators(cfg, 2):
        out[f"glueball/{m.name}"] = np.asarray(m.value)
    for m in measurements.wilson_loops(cfg, 0, 3, 2, 3):
        out[f"wilson/{m.name}"] = np.asarray(m.value)
    out["polyakov_loop_field/1"] = np.asarray(measurements.polyakov_loop_field(cfg, 1))
    sm = smearing.ape_smearing(cfg, 0.3, no_smear_direction=3)
    out["ape/gauge"] = np.asarray(sm.gauge_field)
    res = smearing.multi_smearing_operators(cfg, [lambda c: measurements.glueball_operators(c, 2)], smearing_levels=2,
                                            rho=0.3, no_smear_direction=3, skip=1)
    out["multi/values"] = np.stack([np.asarray(m.value) for m in res])
    out["multi/levels"] = np.asarray([m.smearing_levels for m in res])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print("wrote", name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default=None)
    ap.add_argument("--inproc", action="store_true")
    ap.add_argument("--reference", default=os.environ.get("LYM_REFERENCE_DIR"),
                    help="the reference source tree (default: $LYM_REFERENCE_DIR)")
    args = ap.parse_args()
    global REFERENCE
    if not args.reference or not os.path.isdir(args.reference):
        ap.error("give the reference tree with --reference or LYM_REFERENCE_DIR")
    REFERENCE = os.path.abspath(args.reference)
    if args.case and args.inproc:
        if args.case == "tables":
            run_tables()
        elif args.case == "md_schedules":
            run_schedules()
        elif args.case in ADJOINT_CASES:
            run_adjoint_case(args.case)
        elif args.case in MEASUREMENT_CASES:
            run_measurement_case(args.case)
        elif args.case in XDR_CASES:
            run_xdr_case(args.case)
        elif args.case in OBSERVABLE_CASES:
            run_observable_case(args.case)
        else:
            run_case(args.case)
        return
    names = [args.case] if args.case else (["tables", "md_schedules"] + list(CASES) + list(ADJOINT_CASES) + list(MEASUREMENT_CASES)
                                           + list(XDR_CASES) + list(OBSERVABLE_CASES))
    for n in names:
        subprocess.run([sys.executable, os.path.abspath(__file__), "--case", n, "--inproc", "--reference", REFERENCE],
                       check=True)


if __name__ == "__main__":
    main()
