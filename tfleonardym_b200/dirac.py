"""Dirac operators (mirror of the reference's dirac.py on the GPU).

``DiracWilsonOperator`` keeps the reference constructor and attributes
(dirac.py:253-378).  ``apply`` runs the fused FP64 Wilson kernel
(lym_wilson_apply, replacing dirac.py:458-523 + 649-662); ``lie_derivative``
runs the fused per-link force kernel (lym_fermion_force, dirac.py:525-565).
The adjoint representation (matrix-valued spinors (ns, N, N, V), dirac.py:358-370,
380-456) runs lym_wilson_apply_adjoint and lym_fermion_force_adjoint; its
``fermion_gauge_field`` (the adjoint links) is built on demand by lym_adjoint_links.
The even-odd solvers take the fundamental representation only.
"""
import ctypes

import numpy as np
import torch

from . import _dev, _lib
from . import boundary_conditions as bcs
from . import lattice as lt


class Operator:
    def __init__(self, hermitian=False):
        self.hermitian = hermitian


class ShiftedOperator(Operator):
    """(A + shift) (dirac.py:15-25)."""

    def __init__(self, operator_to_shift: Operator, shift: float):
        super().__init__(operator_to_shift.hermitian)
        self.operator_to_shift = operator_to_shift
        self.shift = shift

    def set_gauge_configuration(self, cfg):
        self.operator_to_shift.set_gauge_configuration(cfg)

    def apply(self, vector):
        return _dev.axpby(1.0, self.operator_to_shift.apply(vector), self.shift, vector)


class SquareOperator(Operator):
    """A A (dirac.py:28-37)."""

    def __init__(self, operator_to_square: Operator):
        super().__init__(operator_to_square.hermitian)
        self.operator_to_square = operator_to_square

    def set_gauge_configuration(self, cfg):
        self.operator_to_square.set_gauge_configuration(cfg)

    def apply(self, vector):
        return self.operator_to_square.apply(self.operator_to_square.apply(vector))


class RationalApproximation(Operator):
    """shift + sum_i alpha_i (A + beta_i)^-1 (dirac.py:40-73)."""

    def __init__(self, operator, alphas, betas, shift, solver):
        super().__init__(operator.hermitian)
        self.operator = operator
        self.alphas = alphas
        self.betas = betas
        self.shift = shift
        self.solver = solver

    def set_gauge_configuration(self, cfg):
        self.operator.set_gauge_configuration(cfg)

    def apply(self, vector):
        solutions = self.solver.solve(self.operator, vector, self.betas)
        result = _dev.axpby(0.0, vector, self.shift, vector)
        for solution, alpha in zip(solutions, self.alphas):
            _dev.axpby_(alpha, solution, 1.0, result)
        return result

    def evaluate(self, x: float):
        result = self.shift
        for alpha, beta in zip(self.alphas, self.betas):
            result += alpha / (x + beta)
        return result

    def test_inverter(self, vector):
        """Residual |A x - v|^2 per pole (the reference prints them, dirac.py:69-73)."""
        out = []
        for solution, beta in zip(self.solver.solve(self.operator, vector, self.betas), self.betas):
            v = _dev.axpby(1.0, self.operator.apply(solution), beta, solution)
            d = _dev.axpby(1.0, v, -1.0, vector)
            out.append(_dev.cdot(d, d))
        return out


class DiracWilsonOperator(Operator):
    """Wilson operator D = 1 + kappa sum_mu [U(1-g_mu)T_+mu + U^dag(1+g_mu)T_-mu],
    Q = gamma_d D when hermitian (dirac.py:253-662)."""

    def __init__(self, cfg: lt.Configuration, kappa, hermitian=False, mode="projected",
                 representation="adjoint", boundary_condition_provider=None):
        super().__init__(hermitian)
        self.kappa = kappa
        self.mode = mode
        self.representation = representation
        if mode not in ("projected", "simple"):
            raise RuntimeError(f"Unknown dirac multiplication mode {mode}")
        if representation not in ("fundamental", "adjoint"):
            raise RuntimeError(f"Unknown representation {representation}")
        self.boundary_condition_provider = boundary_condition_provider
        self._solver_gauge = None
        self._solver_gauge_key = None
        self.set_gauge_configuration(cfg)
        self.set_gamma_matrices()

    # dirac.py:283-300: only D = 2 and 4 carry fermions
    def set_gamma_matrices(self):
        if self.number_of_dimensions == 2:
            self.spinor_dimension = 2
        elif self.number_of_dimensions == 4:
            self.spinor_dimension = 4
        elif self.number_of_dimensions == 3 and self.representation == "fundamental":
            # builder-defined extension (the reference stops here): two-component
            # spinors with gamma_mu = sigma_{mu+1}; odd dimensions have no gamma_5,
            # so only D itself (hermitian=False) exists
            if self.hermitian:
                raise RuntimeError("Number of dimensions 3 has no hermitian form gamma_d D (two-component spinors)")
            self.spinor_dimension = 2
        else:
            raise RuntimeError(f"Number of dimensions {self.number_of_dimensions} not supported for fermions!")

    def set_gauge_configuration(self, cfg):
        gauge = _dev.as_c128(cfg.gauge_field, "gauge_field")
        self.number_of_dimensions = gauge.shape[0]
        self.number_of_colors = gauge.shape[1]
        self.volume = gauge.shape[-1]
        self.cfg = cfg
        self.original_cfg = cfg
        factor, apply_tensor = bcs.provider_factor(self.boundary_condition_provider)
        self._generic_bc = apply_tensor
        self._gauge_orig = gauge
        if apply_tensor:
            gauge = _dev.as_c128(self.boundary_condition_provider(gauge))
        self.bc = factor
        self._gauge_left = gauge  # links with the boundary condition (the reference's cfg)
        self._adjoint_links = None
        if self.representation == "fundamental":
            self.fermion_gauge_field = gauge
        geometry = tuple(cfg.geometry) if cfg.geometry is not None else None
        if geometry is None or int(np.prod(geometry)) != self.volume:
            raise RuntimeError("Configuration.geometry does not match the gauge field volume")
        self.geometry = geometry
        self.lattice = lt.get_lattice(geometry)
        self._gauge_version = getattr(self, "_gauge_version", 0) + 1

    @property
    def fermion_gauge_field(self):
        """Fundamental: the links with the boundary condition.  Adjoint: the adjoint links
        V^{ab} = 2 Tr(T_a U T_b U^dag) with the boundary condition (dirac.py:358-370)."""
        if self.representation == "fundamental":
            return self._fermion_gauge_field
        if self._adjoint_links is None:
            nc, nd = self.number_of_colors, self.number_of_dimensions
            a = nc * nc - 1
            v = torch.empty((nd, a, a, self.volume), dtype=torch.complex128, device=self._gauge_orig.device)
            bc = 1.0 + 0j if self._generic_bc else self.bc
            _lib.check(_lib.lib().lym_adjoint_links(self.lattice.handle, nc, bc.real, bc.imag,
                                                    _dev.ptr(self._gauge_orig), _dev.ptr(v), _dev.stream()),
                       "lym_adjoint_links")
            if self._generic_bc:
                v = _dev.as_c128(self.boundary_condition_provider(v))
            self._adjoint_links = v
        return self._adjoint_links

    @fermion_gauge_field.setter
    def fermion_gauge_field(self, value):
        self._fermion_gauge_field = value

    # -- operator application ------------------------------------------------
    def apply(self, input_vector):
        if self.representation == "adjoint":
            return self._apply_adjoint(input_vector)
        v = _dev.as_c128(input_vector, "input_vector")
        out = torch.empty_like(v)
        nvec = 1
        if v.dim() == 4:  # a batch (nvec, ns, N, V)
            nvec = v.shape[0]
        elif v.dim() != 3:
            raise RuntimeError("spinor must be (ns, N, V) or (nvec, ns, N, V)")
        _lib.check(_lib.lib().lym_wilson_apply_batch(
            self.lattice.handle, self.number_of_colors, float(self.kappa), int(bool(self.hermitian)),
            self.bc.real, self.bc.imag, _dev.ptr(self.fermion_gauge_field), nvec, _dev.ptr(v), _dev.ptr(out),
            _dev.stream()), "lym_wilson_apply")
        return out

    multiply_in_fundamental_representation = apply
    simple_multiply_in_fundamental_representation = apply
    multiply_in_adjoint_representation = apply
    simple_multiply_in_adjoint_representation = apply

    def _apply_adjoint(self, input_vector):
        v = _dev.as_c128(input_vector, "input_vector")
        out = torch.empty_like(v)
        nvec = 1
        if v.dim() == 5:  # a batch (nvec, ns, N, N, V)
            nvec = v.shape[0]
        elif v.dim() != 4:
            raise RuntimeError("adjoint spinor must be (ns, N, N, V) or (nvec, ns, N, N, V)")
        bc = 1.0 + 0j if self._generic_bc else self.bc
        _lib.check(_lib.lib().lym_wilson_apply_adjoint(
            self.lattice.handle, self.number_of_colors, float(self.kappa), int(bool(self.hermitian)),
            bc.real, bc.imag, _dev.ptr(self._gauge_left), _dev.ptr(self._gauge_orig), nvec, _dev.ptr(v),
            _dev.ptr(out), _dev.stream()), "lym_wilson_apply_adjoint")
        return out

    def apply_hermiticity(self, input_vector):
        if not self.hermitian:
            return input_vector.clone()
        out = input_vector.clone()
        out[input_vector.shape[0] // 2:] *= -1
        return out

    def lie_derivative(self, X, Y):
        """kappa-weighted Lie derivative (nd, N, N, V) of dirac.py:525-565 (either representation)."""
        force = torch.zeros((self.number_of_dimensions, self.number_of_colors, self.number_of_colors,
                             self.volume), dtype=torch.complex128, device="cuda")
        self.accumulate_force(force, [1.0], _dev.as_c128(X)[None], _dev.as_c128(Y)[None], symmetric=False)
        return force

    def accumulate_force(self, force, alphas, X, Y, symmetric=True, scale=1.0):
        """force += scale * sum_i alpha_i [L(X_i, Y_i) (+ L(Y_i, X_i) if symmetric)];
        X, Y stacked (nterms, ns, N, V).  Fused n_flavor.force (fermion_action.py:87-91)."""
        X = _dev.as_c128(X)
        Y = _dev.as_c128(Y)
        n = X.shape[0]
        al = (ctypes.c_double * n)(*[float(np.real(a)) for a in alphas])
        if self.representation == "adjoint":
            if self._generic_bc:
                raise NotImplementedError("the adjoint force takes a tagged boundary_condition_provider "
                                          "(boundary_conditions.*_provider)")
            _lib.check(_lib.lib().lym_fermion_force_adjoint(
                self.lattice.handle, self.number_of_colors, float(self.kappa), int(bool(self.hermitian)),
                self.bc.real, self.bc.imag, _dev.ptr(self._gauge_orig), n, al, _dev.ptr(X), _dev.ptr(Y),
                int(bool(symmetric)), float(scale), _dev.ptr(force), _dev.stream()), "lym_fermion_force_adjoint")
            return force
        _lib.check(_lib.lib().lym_fermion_force(
            self.lattice.handle, self.number_of_colors, float(self.kappa), int(bool(self.hermitian)),
            self.bc.real, self.bc.imag, _dev.ptr(self.fermion_gauge_field), n, al, _dev.ptr(X), _dev.ptr(Y),
            int(bool(symmetric)), float(scale), _dev.ptr(force), _dev.stream()), "lym_fermion_force")
        return force

    # -- device gauge for the solvers -----------------------------------------
    def solver_gauge(self, precisions=("f32", "f16", "bf16")):
        """lym_gauge handle (even-odd links) for the current configuration."""
        if self.representation != "fundamental":
            raise TypeError("the even-odd solvers take the fundamental representation")
        mask = 0
        for p in precisions:
            mask |= 1 << _lib.PREC[p]
        if self._solver_gauge is not None:
            held = self._solver_gauge_key[1]
            if mask & ~held:
                mask |= held  # widen: keep every precision asked for so far
            else:
                mask = held
        key = (self._gauge_version, mask)
        if self._solver_gauge is not None and self._solver_gauge_key == key:
            return self._solver_gauge
        if self._solver_gauge is not None and self._solver_gauge_key[1] == mask:
            _lib.check(_lib.lib().lym_gauge_update(self._solver_gauge, _dev.ptr(self.fermion_gauge_field),
                                                   _dev.stream()), "lym_gauge_update")
        else:
            self._free_solver_gauge()
            h = ctypes.c_void_p()
            _lib.check(_lib.lib().lym_gauge_create(self.lattice.handle, self.number_of_colors,
                                                   _dev.ptr(self.fermion_gauge_field), self.bc.real, self.bc.imag,
                                                   mask, _dev.stream(), ctypes.byref(h)), "lym_gauge_create")
            self._solver_gauge = h
        self._solver_gauge_key = key
        self._gauge_ref = self.fermion_gauge_field  # keep the source alive while the handle is used
        return self._solver_gauge

    def _free_solver_gauge(self):
        if self._solver_gauge is not None and _lib._lib is not None:
            torch.cuda.synchronize()
            _lib.lib().lym_gauge_destroy(self._solver_gauge)
        self._solver_gauge = None

    def release(self):
        """Frees the solver's device objects (lym_gauge, workspaces, graphs) now, on the
        calling thread; the next solve builds them again."""
        self._free_solver_gauge()
        self._solver_gauge_key = None

    def __del__(self):
        try:
            self._free_solver_gauge()
        except Exception:
            pass


class Propagator:
    """gamma_d op^-1 source (dirac.py:665-696 for a Wilson operator: the reference
    computes op (op^2)^-1 source with its inverter, then applies gamma_d).

    With ``dirac_solver.conjugate_gradient`` as the inverter and a fundamental
    DiracWilsonOperator, op x = source is solved directly by the even-odd CG, all
    stacked sources (nsrc, ns, N, V) in one batched call; any other inverter
    follows the reference's steps (inverter.solve(SquareOperator(op), source), then
    op.apply) one source at a time."""

    def __init__(self, operator, inverter):
        self.operator = operator
        self.inverter = inverter

    def apply(self, source):
        from . import dirac_solver
        src = _dev.as_c128(source)
        op = self.operator
        fundamental = isinstance(op, DiracWilsonOperator) and op.representation == "fundamental"
        if isinstance(self.inverter, dirac_solver.conjugate_gradient) and fundamental:
            return self.apply_gammad(self.inverter.solve(op, src))
        per = 4 if (isinstance(op, DiracWilsonOperator) and op.representation == "adjoint") else 3
        if src.dim() == per + 1:  # a stack of sources, one reference-style solve each
            return torch.stack([self.apply(src[i]) for i in range(src.shape[0])])
        square_solution = self.inverter.solve(SquareOperator(op), src)
        return self.apply_gammad(op.apply(square_solution))

    def apply_gammad(self, input_vector):
        """Negate the lower half of the spin components (dirac.py:684-696), of one vector
        or of each vector of a stack."""
        adjoint = isinstance(self.operator, DiracWilsonOperator) and self.operator.representation == "adjoint"
        spin_axis = input_vector.dim() - (4 if adjoint else 3)
        out = input_vector.clone()
        ns = out.shape[spin_axis]
        index = [slice(None)] * out.dim()
        index[spin_axis] = slice(ns // 2, ns)
        out[tuple(index)] *= -1
        return out
