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


class n_flavor:  # noqa: N801 - reference name
    def __init__(self, force_operators, metropolis_operators, heatbath_operators, solver, dirac_operator):
        self.force_operators = force_operators
        self.metropolis_operators = metropolis_operators
        self.heatbath_operators = heatbath_operators
        self.solver = solver
        self.dirac_operator = dirac_operator
        self.square_dirac_operator = dirac.SquareOperator(dirac_operator)
        self.pseudofermions = None

    def initialize_pseudofermions(self, random_vectors):
        self.pseudofermions = [op.apply(v) for v, op in zip(random_vectors, self.heatbath_operators)]

    def set_gauge_configuration(self, cfg):
        self.dirac_operator.set_gauge_configuration(cfg)
        self.square_dirac_operator = dirac.SquareOperator(self.dirac_operator)
        for approximation in self.force_operators:
            approximation.set_gauge_configuration(cfg)
        for approximation in self.metropolis_operators:
            approximation.set_gauge_configuration(cfg)
        for approximation in self.heatbath_operators:
            approximation.set_gauge_configuration(cfg)

    def energy(self):
        energy = 0
        for vector, operator in zip(self.pseudofermions, self.metropolis_operators):
            energy += _dev.cdot(vector, operator.apply(vector))
        return float(np.real(energy))

    def number_of_flavors(self):
        result = 1
        for approximation in self.metropolis_operators:
            result *= approximation.evaluate(0.5)
        return 2 * np.log(result) / np.log(2.0)

    def check_rational_approximations(self, vector):
        result = 0.0
        for metropolis, heatbath in zip(self.metropolis_operators, self.heatbath_operators):
            third = heatbath.apply(metropolis.apply(heatbath.apply(vector)))
            d = _dev.axpby(1.0, third, -1.0, vector)
            result += _dev.cdot(d, d)
        return result

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
