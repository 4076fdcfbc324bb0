"""Hybrid Monte Carlo (mirror of the reference's hmc.py on the GPU).

The per-link kernels replace the reference's TF ops: ``update_link_field``
(hmc.py:40-43, tf.linalg.expm) runs lym_update_links (SU(2) closed form,
SU(3) Cayley-Hamilton), ``update_momenta`` (hmc.py:59-61) runs
lym_update_momenta, ``momenta_energy`` (hmc.py:170-176) lym_momenta_energy.
The integrators and ``hybrid_mc`` / ``reversibility_check`` keep the
reference's control flow (hmc.py:104-278) over these device tensors.
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
    """Anti-Hermitian traceless momenta from unit normals (nd, N*N-1, V), built
    exactly as random_momenta does from its draws (hmc.py:69-96)."""
    nd, _, vol = normals.shape
    p = torch.zeros((nd, nc, nc, vol), dtype=torch.complex128, device=normals.device)
    for mu in range(nd):
        k = 0
        for i in range(nc):
            for j in range(i + 1, nc):
                re, im = normals[mu, k] / 2, normals[mu, k + 1] / 2
                k += 2
                p[mu, i, j] = torch.complex(re, im)
                p[mu, j, i] = torch.complex(-re, im)
        diag = torch.zeros((nc, vol), dtype=torch.float64, device=normals.device)
        for i in range(1, nc):
            r = normals[mu, k] / 2
            k += 1
            for j in range(i):
                diag[j] += r / np.sqrt(i * (i + 1) / 2.0)
            diag[i] += -r * (i * np.sqrt(2.0 / (i * (i + 1))))
        for i in range(nc):
            p[mu, i, i] = torch.complex(torch.zeros_like(diag[i]), diag[i])
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


def _apply_force(action, momenta, eps):
    """momenta + eps * action.force(), fusing the update when the action allows it."""
    fused = getattr(action, "force_into_momenta", None)
    if fused is not None:
        out = momenta.clone()
        return fused(out, eps)
    return update_momenta(momenta, action.force(), eps)


def integrate_lp(config, momenta, actions, steps, delta_t, action_index=0):
    """Leap-frog (hmc.py:104-124)."""
    epsilon = delta_t / steps[action_index]
    actions[action_index].set_gauge_configuration(config)
    momenta = _apply_force(actions[action_index], momenta, -(epsilon / 2))
    for k in range(steps[action_index]):
        if action_index == len(actions) - 1:
            config = update_configuration(config, momenta, epsilon)
        else:
            config, momenta = integrate_lp(config, momenta, actions, steps, epsilon, action_index + 1)
        actions[action_index].set_gauge_configuration(config)
        # -eps inside the loop; after the last step also the closing +eps/2 with the same force
        w = -epsilon if k < steps[action_index] - 1 else -epsilon / 2
        momenta = _apply_force(actions[action_index], momenta, w)
    return config, momenta


def integrate_om(config, momenta, actions, steps, delta_t, action_index=0):
    """Nested Omelyan integrator (hmc.py:133-162).

    The reference evaluates the last force of the loop twice in a row with the
    same links (once inside the loop, once for the closing +lambda*eps kick);
    here the closing kick reuses that force through eps-weight merging, which
    is the same arithmetic on the momenta."""
    ll = OMELYAN_LAMBDA
    epsilon = delta_t / steps[action_index]
    last = action_index == len(actions) - 1
    actions[action_index].set_gauge_configuration(config)
    momenta = _apply_force(actions[action_index], momenta, -ll * epsilon)
    for k in range(steps[action_index]):
        if last:
            config = update_configuration(config, momenta, epsilon / 2)
        else:
            config, momenta = integrate_om(config, momenta, actions, steps, epsilon / 2, action_index + 1)
        actions[action_index].set_gauge_configuration(config)
        momenta = _apply_force(actions[action_index], momenta, -(1 - 2 * ll) * epsilon)
        if last:
            config = update_configuration(config, momenta, epsilon / 2)
        else:
            config, momenta = integrate_om(config, momenta, actions, steps, epsilon / 2, action_index + 1)
        actions[action_index].set_gauge_configuration(config)
        # -2 ll eps inside the loop and, after the last step, +ll eps with the same force
        w = -2 * ll * epsilon if k < steps[action_index] - 1 else -ll * epsilon
        momenta = _apply_force(actions[action_index], momenta, w)
    return config, momenta


def gauge_energy(cfg, beta):
    from .measurements import plaquette
    nd = cfg.gauge_field.shape[0]
    return -beta * (nd - 1) * nd / 2 * cfg.gauge_field.shape[-1] * plaquette(cfg).value


def _metropolis(new_energy, old_energy, uniform=None):
    """metropolis.py:11-18; ``uniform`` may be supplied by the caller."""
    if new_energy < old_energy:
        return True
    u = np.random.uniform(0, 1) if uniform is None else uniform
    return bool(u < np.exp(-(new_energy - old_energy)))


def hybrid_mc(config, actions, steps, delta_t, momenta=None, uniform=None):
    """One HMC trajectory (hmc.py:218-246).  Returns (cfg, -dH, accepted)."""
    if momenta is None:
        momenta = random_momenta(config.colors, config.number_of_dimensions, config.gauge_field.shape[-1])
    old_energy = momenta_energy(momenta)
    for action in actions:
        action.set_gauge_configuration(config)
        old_energy += action.energy()
    new_config, new_momenta = integrate_om(config, momenta, actions, steps, delta_t)
    new_energy = momenta_energy(new_momenta)
    for action in actions:
        action.set_gauge_configuration(new_config)
        new_energy += action.energy()
    if _metropolis(new_energy, old_energy, uniform):
        return new_config, -(new_energy - old_energy), True
    return copy.copy(config), -(new_energy - old_energy), False


def reversibility_check(config, actions, steps, delta_t, momenta=None):
    """Forward then backward trajectory; returns H_end - H_start (hmc.py:249-278)."""
    if momenta is None:
        momenta = random_momenta(config.colors, config.number_of_dimensions, config.gauge_field.shape[-1])
    old_energy = momenta_energy(momenta)
    for action in actions:
        action.set_gauge_configuration(config)
        old_energy += action.energy()
    new_config, new_momenta = integrate_om(config, momenta, actions, steps, delta_t)
    new_config, new_momenta = integrate_om(new_config, new_momenta, actions, steps, -delta_t)
    new_energy = momenta_energy(new_momenta)
    for action in actions:
        action.set_gauge_configuration(new_config)
        new_energy += action.energy()
    return new_energy - old_energy
