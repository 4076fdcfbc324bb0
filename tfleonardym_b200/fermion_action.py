"""Pseudofermion action (mirror of fermion_action.py:7-93) on the GPU.

``force`` solves all poles of each force approximation with the configured
solver, applies the Dirac operator to the whole stack of solutions in one
batched launch, and accumulates sum_i alpha_i [L(X_i, Y_i) + L(Y_i, X_i)] in
one fused per-link kernel (lym_fermion_force) instead of the reference's
2 x n_poles x nd separate einsums.
"""
import numpy as np
import torch

from . import _dev
from . import dirac


def _operator_chain(op):
    """Every operator object reachable from `op` through the wrappers' fields."""
    seen = []
    stack = [op]
    while stack:
        o = stack.pop()
        if o is None or any(o is s for s in seen):
            continue
        seen.append(o)
        for attr in ("operator", "operator_to_square", "operator_to_shift"):
            stack.append(getattr(o, attr, None))
    return seen


def _rational_apply_many(approximation, vectors):
    """shift v + sum_i alpha_i (A + beta_i)^-1 v for every v in `vectors` (dirac.py:52-59):
    one batched multishift solve when the solver takes several sources at once."""
    batched = getattr(approximation.solver, "precision", None) is not None and len(vectors) > 1 and \
        hasattr(approximation.solver, "_solve_eo")
    if not batched:
        return [approximation.apply(v) for v in vectors]
    stack = torch.stack([_dev.as_c128(v) for v in vectors])
    sols = approximation.solver.solve(approximation.operator, stack, approximation.betas)  # per shift (n, ...)
    out = stack * approximation.shift
    for sol, alpha in zip(sols, approximation.alphas):
        out = out + alpha * sol
    return list(out)


class n_flavor:  # noqa: N801 - reference name
    """Rational pseudofermion action sum_k Re <phi_k, M_k phi_k> with the reference's
    constructor, attributes and methods (fermion_action.py:7-93).  Device-side
    differences: a new gauge configuration reaches each distinct operator object once
    (the approximations usually wrap one Dirac operator); pseudofermions whose
    approximations share operator, poles and a batching solver are solved together;
    the force is one fused kernel over all poles (below)."""

    def __init__(self, force_operators, metropolis_operators, heatbath_operators, solver, dirac_operator):
        self.force_operators = force_operators
        self.metropolis_operators = metropolis_operators
        self.heatbath_operators = heatbath_operators
        self.solver = solver
        self.dirac_operator = dirac_operator
        self.square_dirac_operator = dirac.SquareOperator(dirac_operator)
        self.pseudofermions = None

    def set_gauge_configuration(self, cfg):
        done = []
        for root in [self.dirac_operator, *self.force_operators, *self.metropolis_operators,
                     *self.heatbath_operators]:
            for op in _operator_chain(root):
                if hasattr(op, "number_of_dimensions") and not any(op is d for d in done):
                    op.set_gauge_configuration(cfg)  # the Dirac operators themselves
                    done.append(op)
        self.square_dirac_operator = dirac.SquareOperator(self.dirac_operator)

    def _apply_each(self, approximations, vectors):
        """approximations[k] applied to vectors[k], batching runs of equal rational
        approximations; any other operator (e.g. the Dirac operator as heatbath) is
        applied on its own."""
        out = [None] * len(vectors)
        groups = {}
        for k, a in enumerate(approximations):
            if not all(hasattr(a, f) for f in ("operator", "solver", "alphas", "betas", "shift")):
                out[k] = a.apply(vectors[k])
                continue
            key = (id(a.operator), id(a.solver), tuple(np.asarray(a.betas).tolist()),
                   tuple(np.asarray(a.alphas).tolist()), float(a.shift))
            groups.setdefault(key, []).append(k)
        for ks in groups.values():
            res = _rational_apply_many(approximations[ks[0]], [vectors[k] for k in ks])
            for k, r in zip(ks, res):
                out[k] = r
        return out

    def initialize_pseudofermions(self, random_vectors):
        n = min(len(random_vectors), len(self.heatbath_operators))
        self.pseudofermions = self._apply_each(self.heatbath_operators[:n], list(random_vectors)[:n])

    def energy(self):
        n = min(len(self.pseudofermions), len(self.metropolis_operators))
        applied = self._apply_each(self.metropolis_operators[:n], self.pseudofermions[:n])
        return float(sum(np.real(_dev.cdot(phi, m)) for phi, m in zip(self.pseudofermions, applied)))

    def number_of_flavors(self):
        """2 log2 of the product of the Metropolis approximations at x = 1/2."""
        return 2.0 * float(np.log2(np.prod([a.evaluate(0.5) for a in self.metropolis_operators])))

    def check_rational_approximations(self, vector):
        """sum over pseudofermion slots of |H M H v - v|^2 (H heatbath, M Metropolis)."""
        total = 0.0
        for m, h in zip(self.metropolis_operators, self.heatbath_operators):
            d = _dev.axpby(1.0, h.apply(m.apply(h.apply(vector))), -1.0, vector)
            total += _dev.cdot(d, d)
        return total

    def force(self):
        d = self.dirac_operator
        f = torch.zeros((d.number_of_dimensions, d.number_of_colors, d.number_of_colors, d.volume),
                        dtype=torch.complex128, device="cuda")
        for approximation, phi in zip(self.force_operators, self.pseudofermions):
            xs = self.solver.solve(approximation.operator, phi, approximation.betas)
            X = torch.stack([_dev.as_c128(x) for x in xs])
            Y = d.apply(X)  # one batched launch over all poles
            d.accumulate_force(f, approximation.alphas, X, Y, symmetric=True)
        return f

    def force_into_momenta(self, momenta, eps):
        """momenta += eps * force(): the force kernel accumulates straight into the momenta."""
        d = self.dirac_operator
        for approximation, phi in zip(self.force_operators, self.pseudofermions):
            xs = self.solver.solve(approximation.operator, phi, approximation.betas)
            X = torch.stack([_dev.as_c128(x) for x in xs])
            Y = d.apply(X)
            d.accumulate_force(momenta, approximation.alphas, X, Y, symmetric=True, scale=eps)
        return momenta
