"""Hybrid Monte Carlo (mirror of the reference's hmc.py on the GPU).

The per-link kernels replace the reference's TF ops: ``update_link_field``
(hmc.py:40-43, tf.linalg.expm) runs lym_update_links (SU(2) closed form,
SU(3) Cayley-Hamilton), ``update_momenta`` (hmc.py:59-61) runs
lym_update_momenta, ``momenta_energy`` (hmc.py:170-176) lym_momenta_energy.
The integrators are compiled into flat schedules of drifts and kicks (below)
and run over these device tensors; ``integrate_om`` / ``integrate_lp`` /
``hybrid_mc`` / ``reversibility_check`` keep the reference's signatures and
results (hmc.py:104-278).
"""
import copy
import ctypes

import numpy as np
import torch

from . import _dev, _lib, lie_generators
from . import lattice as lt
from . import smearing

OMELYAN_LAMBDA = 0.19318332275037863


def update_link_field(link_field, momenta, epsilon, reunitarize=False):
    """expm(eps P) U per link, as a new tensor (hmc.py:40-43)."""
    u = _dev.as_c128(link_field).clone()
    p = _dev.as_c128(momenta)
    _lib.check(_lib.lib().lym_update_links(u.shape[0], u.shape[1], u.shape[-1], _dev.ptr(u), _dev.ptr(p),
                                           float(epsilon), int(bool(reunitarize)), _dev.stream()),
               "lym_update_links")
    return u


def update_configuration(config: lt.Configuration, momenta, epsilon):
    return lt.Configuration(gauge_field=update_link_field(config.gauge_field, momenta, epsilon),
                            geometry=config.geometry, colors=config.colors,
                            number_of_dimensions=config.number_of_dimensions)


def update_momenta(momenta, gauge_force, epsilon):
    """P + eps F as a new tensor (hmc.py:59-61)."""
    p = _dev.as_c128(momenta).clone()
    f = _dev.as_c128(gauge_force)
    _lib.check(_lib.lib().lym_update_momenta(p.numel(), _dev.ptr(p), _dev.ptr(f), float(epsilon), _dev.stream()),
               "lym_update_momenta")
    return p


def momenta_from_normals(normals, nc):
    """Anti-Hermitian traceless momenta from unit normals (nd, N*N-1, V) on the
    device, built as random_momenta builds them from its draws (hmc.py:69-96)
    in one kernel (lym_momenta_from_normals)."""
    nrm = normals.to(torch.float64).contiguous()
    nd, ng, vol = nrm.shape
    if ng != nc * nc - 1:
        raise ValueError(f"normals need N*N-1 = {nc * nc - 1} rows per direction, got {ng}")
    p = torch.empty((nd, nc, nc, vol), dtype=torch.complex128, device=nrm.device)
    _lib.check(_lib.lib().lym_momenta_from_normals(nd, nc, vol, nrm.data_ptr(), _dev.ptr(p), _dev.stream()),
               "lym_momenta_from_normals")
    return p


def random_momenta(nc=3, nd=4, volume=None, generator=None):
    """Gaussian su(N) momenta, unit variance per generator (hmc.py:69-96)."""
    if volume is None:
        from . import translate
        volume = translate.lookup_tables.local_volume
    normals = torch.randn((nd, nc * nc - 1, volume), dtype=torch.float64, device="cuda", generator=generator)
    return momenta_from_normals(normals, nc)


def trace_momenta(momenta):
    p = _dev.as_c128(momenta)
    out = ctypes.c_double()
    _lib.check(_lib.lib().lym_momenta_energy(p.shape[0], p.shape[1], p.shape[-1], _dev.ptr(p), ctypes.byref(out),
                                             _dev.stream()), "lym_momenta_energy")
    return out.value


def momenta_energy(momenta):
    return lt.global_sum(trace_momenta(momenta))


def random_gauge_field(nc=3, nd=4, volume=None, generator=None):
    """Hot start: complex Gaussian links projected to SU(N) (hmc.py:16-24)."""
    if volume is None:
        from . import translate
        volume = translate.lookup_tables.local_volume
    re = torch.randn((nd, nc, nc, volume), dtype=torch.float64, device="cuda", generator=generator)
    im = torch.randn((nd, nc, nc, volume), dtype=torch.float64, device="cuda", generator=generator)
    return smearing.unitary_sqrt_projection(torch.complex(re, im))


def hotstart(geometry, nc=3, nd=4, generator=None):
    return lt.Configuration(gauge_field=random_gauge_field(nc, nd, int(np.prod(geometry)), generator),
                            geometry=tuple(geometry), colors=nc, number_of_dimensions=nd)


def generate_random_vector(nc=3, spinor_dimension=4, representation="fundamental", stddev=1, volume=None,
                           generator=None):
    """Complex Gaussian spinor (hmc.py:196-210): (ns, N, V) fundamental, or the
    matrix-valued adjoint one sum_a v_a T^a, (ns, N, N, V)."""
    if representation not in ("fundamental", "adjoint"):
        raise RuntimeError(f"Unknown representation {representation}")
    if volume is None:
        from . import translate
        volume = translate.lookup_tables.local_volume
    if representation == "adjoint":
        ncomp = nc * nc - 1
        shape = (spinor_dimension, ncomp, volume)
        re = torch.randn(shape, dtype=torch.float64, device="cuda", generator=generator) * stddev
        im = torch.randn(shape, dtype=torch.float64, device="cuda", generator=generator) * stddev
        gens = torch.from_numpy(lie_generators.generators(nc, "fundamental")).to(re.device)
        return torch.einsum("mic,ijk->mjkc", torch.complex(re, im), gens)
    shape = (spinor_dimension, nc, volume)
    re = torch.randn(shape, dtype=torch.float64, device="cuda", generator=generator) * stddev
    im = torch.randn(shape, dtype=torch.float64, device="cuda", generator=generator) * stddev
    return torch.complex(re, im)


def gauge_step_lattices(configs, momenta, betas, eps_p, eps_u):
    """The gauge part of one HMC step on many independent lattices at once (any mix of
    dimension, N and size; builder-defined: the reference runs one lattice per process):
    momenta[l] += eps_p * F_gauge(configs[l]) for every lattice, then every link
    U <- exp(eps_u P) U, in two launches (lym_gauge_hmc_step_multi).  Updates the
    momenta tensors and the configurations' gauge fields in place."""
    n = len(configs)
    if n != len(momenta) or n != len(betas):
        raise ValueError("one momenta tensor and one beta per configuration")
    us = [_dev.as_c128(c.gauge_field, "gauge_field") for c in configs]
    ps = [_dev.as_c128(p, "momenta") for p in momenta]
    lats = (ctypes.c_void_p * n)(*[lt.get_lattice(tuple(c.geometry)).handle.value for c in configs])
    ncs = (ctypes.c_int * n)(*[int(u.shape[1]) for u in us])
    bs = (ctypes.c_double * n)(*[float(b) for b in betas])
    up = (ctypes.c_void_p * n)(*[u.data_ptr() for u in us])
    pp = (ctypes.c_void_p * n)(*[p.data_ptr() for p in ps])
    _lib.check(_lib.lib().lym_gauge_hmc_step_multi(n, lats, ncs, bs, up, pp, float(eps_p), float(eps_u),
                                                   _dev.stream()), "lym_gauge_hmc_step_multi")


# ---------------------------------------------------------------------------
# Molecular dynamics as a flat schedule
#
# The reference integrates recursively, calling update_momenta and
# update_configuration as it goes (hmc.py:104-162).  Here an integrator is first
# compiled into a flat list of operations -- a drift U <- exp(w P) U, or a kick
# P <- P + w F_level(U) -- and then run.  Compilation writes each step as the
# symmetric product of the scheme and fuses neighbouring kicks of one level that
# no drift separates into one kick with the summed weight: the reference's closing
# kick reuses the force of the kick just before it (hmc.py:122, 160), so the fused
# list asks for exactly the force evaluations the reference makes.  The runner
# sets an action's gauge configuration only when the links changed since it last
# saw them, and applies each kick through the action's fused force-into-momenta
# kernel where it has one.
# ---------------------------------------------------------------------------
DRIFT, KICK = 0, 1


class Op:
    __slots__ = ("kind", "level", "weight")

    def __init__(self, kind, level, weight):
        self.kind, self.level, self.weight = kind, level, weight

    def __repr__(self):
        return f"{'drift' if self.kind == DRIFT else 'kick'}({self.level}, {self.weight!r})"


def _fuse(ops):
    out = []
    for op in ops:
        if out and op.kind == KICK and out[-1].kind == KICK and out[-1].level == op.level:
            out[-1] = Op(KICK, op.level, out[-1].weight + op.weight)
        else:
            out.append(op)
    return out


def _compile(scheme, steps, delta_t, level=0):
    """The flat schedule of `scheme` ("omelyan" or "leapfrog") on nested levels:
    level l takes steps[l] steps of delta_t / steps[l] (times the scheme's inner
    fractions for the levels below); the last level's inner move is the drift."""
    n = steps[level]
    eps = delta_t / n
    last = level == len(steps) - 1

    def inner(dt):
        return [Op(DRIFT, level, dt)] if last else _compile(scheme, steps, dt, level + 1)

    one = []
    if scheme == "omelyan":
        lam = OMELYAN_LAMBDA
        # K(lam e) I(e/2) K((1 - 2 lam) e) I(e/2) K(lam e); kick weights carry the
        # force's sign convention of hmc.py (P + w F with w = -c e)
        one = [Op(KICK, level, -lam * eps)] + inner(eps / 2) + [Op(KICK, level, -(1 - 2 * lam) * eps)] + \
            inner(eps / 2) + [Op(KICK, level, -lam * eps)]
    elif scheme == "leapfrog":
        one = [Op(KICK, level, -eps / 2)] + inner(eps) + [Op(KICK, level, -eps / 2)]
    else:
        raise ValueError(f"unknown integrator {scheme!r}")
    return _fuse(one * n)


def schedule(scheme, steps, delta_t):
    """Compiled molecular-dynamics schedule (a list of Op) for `steps` per level."""
    if not steps or any(int(k) < 1 for k in steps):
        raise ValueError("every level needs at least one step")
    return _compile(scheme, [int(k) for k in steps], float(delta_t))


def force_evaluations(ops):
    """Forces a schedule evaluates, per level."""
    counts = {}
    for op in ops:
        if op.kind == KICK:
            counts[op.level] = counts.get(op.level, 0) + 1
    return counts


def _kick(action, momenta, w):
    fused = getattr(action, "force_into_momenta", None)
    if fused is not None:
        return fused(momenta.clone(), w)
    return update_momenta(momenta, action.force(), w)


def run_schedule(config, momenta, actions, ops, level_offset=0):
    """Run a compiled schedule; kick level l uses actions[level_offset + l]."""
    version, seen = 0, {}
    for op in ops:
        if op.kind == DRIFT:
            config = update_configuration(config, momenta, op.weight)
            version += 1
            continue
        a = level_offset + op.level
        if seen.get(a) != version:
            actions[a].set_gauge_configuration(config)
            seen[a] = version
        momenta = _kick(actions[a], momenta, op.weight)
    return config, momenta


def integrate_om(config, momenta, actions, steps, delta_t, action_index=0):
    """Nested Omelyan integrator with the reference's interface (hmc.py:133-162)."""
    return run_schedule(config, momenta, actions, schedule("omelyan", steps[action_index:len(actions)], delta_t),
                        action_index)


def integrate_lp(config, momenta, actions, steps, delta_t, action_index=0):
    """Nested leap-frog integrator with the reference's interface (hmc.py:104-124)."""
    return run_schedule(config, momenta, actions, schedule("leapfrog", steps[action_index:len(actions)], delta_t),
                        action_index)


def gauge_energy(cfg, beta):
    from .measurements import plaquette
    nd = cfg.gauge_field.shape[0]
    return -beta * (nd - 1) * nd / 2 * cfg.gauge_field.shape[-1] * plaquette(cfg).value


def hamiltonian(config, momenta, actions):
    """Kinetic energy of the momenta plus every action's energy on `config`."""
    h = momenta_energy(momenta)
    for a in actions:
        a.set_gauge_configuration(config)
        h += a.energy()
    return h


def accept(delta_h, uniform=None):
    """Metropolis test on delta_h = H_new - H_old (metropolis.py:11-18); the caller
    may supply the uniform deviate."""
    if delta_h < 0:
        return True
    u = np.random.uniform(0, 1) if uniform is None else uniform
    return bool(u < np.exp(-delta_h))


def _fresh_momenta(config):
    return random_momenta(config.colors, config.number_of_dimensions, config.gauge_field.shape[-1])


def hybrid_mc(config, actions, steps, delta_t, momenta=None, uniform=None):
    """One HMC trajectory with the reference's interface and result (hmc.py:218-246):
    returns (configuration, -dH, accepted)."""
    p0 = _fresh_momenta(config) if momenta is None else momenta
    h0 = hamiltonian(config, p0, actions)
    ops = schedule("omelyan", steps[:len(actions)], delta_t)
    cfg1, p1 = run_schedule(config, p0, actions, ops)
    dh = hamiltonian(cfg1, p1, actions) - h0
    if accept(dh, uniform):
        return cfg1, -dh, True
    return copy.copy(config), -dh, False


def reversibility_check(config, actions, steps, delta_t, momenta=None):
    """H after integrating forward by delta_t and back by -delta_t, minus H before
    (hmc.py:249-278)."""
    p0 = _fresh_momenta(config) if momenta is None else momenta
    h0 = hamiltonian(config, p0, actions)
    lv = steps[:len(actions)]
    cfg1, p1 = run_schedule(config, p0, actions, schedule("omelyan", lv, delta_t))
    cfg2, p2 = run_schedule(cfg1, p1, actions, schedule("omelyan", lv, -delta_t))
    return hamiltonian(cfg2, p2, actions) - h0
