"""Krylov solvers (mirror of the reference's dirac_solver.py on the GPU).

* ``multishift_solver`` -- the reference's multishift MMMR (dirac_solver.py:13-53):
  same constructor, same ``solve(operator, source, shifts)`` returning a list,
  absolute stop |<r,r>| < precision, negative leading shifts handed to
  BiCGStab, "failed to converge" printed and the last iterate returned.  On a
  ``SquareOperator(DiracWilsonOperator)`` the whole solve runs in lym_mmmr_solve;
  on any other operator the loop calls ``operator.apply`` with lym vector kernels.
* ``biconjugate_gradient`` -- BiCGStab of dirac_solver.py:56-110.
* ``multishift_cg`` -- builder-defined drop-in for ``multishift_solver`` on
  Q^2 + sigma (lym_multishift_solve, FP64; or with ``precision`` the even-odd
  lym_multishift_solve_eo with FP64 / FP32 / FP16 / BF16 inner iterations and
  batched sources); tolerance is relative, tol * |b|.
* ``conjugate_gradient`` -- builder-defined even-odd CG for D x = b (or Q x = b)
  with FP64 reliable updates and FP64 / FP32 / FP16 / BF16 inner iterations
  (lym_wilson_solve).
* ``solve_lattices`` -- builder-defined: independent lattices (their own geometry,
  kappa, links and sources) solved together, the CG iterations of all of them in
  the same launches (lym_wilson_solve_multi).
* ``eo_square_solver`` -- builder-defined drop-in for ``multishift_solver`` on
  SquareOperator(Q): shift 0 by two even-odd CG solves of Q, positive shifts by
  ``multishift_cg``.
"""
import ctypes

import numpy as np
import torch

from . import _dev, _lib
from .dirac import DiracWilsonOperator, ShiftedOperator, SquareOperator

VERBOSE = True


def _print(*args):
    if VERBOSE:
        print(*args)


def _wilson_square(operator):
    """The DiracWilsonOperator behind SquareOperator(Q) with hermitian Q, else None."""
    if isinstance(operator, SquareOperator) and isinstance(operator.operator_to_square, DiracWilsonOperator):
        q = operator.operator_to_square
        if q.hermitian and q.representation == "fundamental":
            return q
    return None


class multishift_solver:  # noqa: N801 - reference name
    def __init__(self, max_steps, precision, omega=0.95):
        self.max_steps = max_steps
        self.precision = precision
        self.omega = omega
        self.last_steps = None

    def solve(self, operator, source, shifts: list):
        source = _dev.as_c128(source, "source")
        shifts = list(shifts)
        solutions = [torch.zeros_like(source) for _ in shifts]
        first = 0
        while first < len(shifts) and shifts[first] < 0:  # dirac_solver.py:26-30
            solver = biconjugate_gradient(self.max_steps, self.precision)
            solutions[first] = solver.solve(ShiftedOperator(operator, shifts[first]), source)
            first += 1
        rest = shifts[first:]
        if not rest:
            return solutions
        q = _wilson_square(operator)
        if q is not None:
            xs = torch.empty((len(rest),) + tuple(source.shape), dtype=torch.complex128, device=source.device)
            steps = ctypes.c_int()
            sh = (ctypes.c_double * len(rest))(*[float(s) for s in rest])
            rc = _lib.lib().lym_mmmr_solve(q.solver_gauge(()), float(q.kappa), len(rest), sh, _dev.ptr(source),
                                           _dev.ptr(xs), int(self.max_steps), float(self.precision),
                                           float(self.omega), ctypes.byref(steps), _dev.stream())
            self.last_steps = steps.value
            if rc == _lib.LYM_ERR_NOT_CONVERGED:
                _print(f"MMMRMultishiftsolver: failed to find convergence after {steps.value} steps")
            else:
                _lib.check(rc, "lym_mmmr_solve")
                _print(f"MMMRMultishiftsolver: convergence after {steps.value} steps")
            for i in range(len(rest)):
                solutions[first + i] = xs[i]
            return solutions
        return self._generic(operator, source, rest, solutions, first)

    def _generic(self, operator, source, shifts, solutions, first):
        f = [1.0 for _ in shifts]
        r = source.clone()
        xs = [torch.zeros_like(source) for _ in shifts]
        step = 0
        for step in range(self.max_steps):
            p = _dev.axpby(1.0, operator.apply(r), shifts[-1], r)
            alpha = self.omega * _dev.cdot(p, r) / _dev.cdot(p, p)
            _dev.axpby_(alpha, r, 1.0, xs[-1])
            for i, s in enumerate(shifts[:-1]):
                f[i] = f[i] / (1 + (s - shifts[-1]) * alpha)
                _dev.axpby_(alpha * f[i], r, 1.0, xs[i])
            _dev.axpby_(-alpha, p, 1.0, r)
            if abs(_dev.cdot(r, r)) < self.precision:
                self.last_steps = step
                _print(f"MMMRMultishiftsolver: convergence after {step} steps")
                break
        else:
            self.last_steps = step
            _print(f"MMMRMultishiftsolver: failed to find convergence after {step} steps")
        for i, x in enumerate(xs):
            solutions[first + i] = x
        return solutions


class biconjugate_gradient:  # noqa: N801 - reference name
    """BiCGStab of dirac_solver.py:61-110 (x0 = source or guess, r0 = x0 - A x0,
    r_hat = x0 + A x0, absolute stop), with lym vector kernels."""

    def __init__(self, max_steps, precision):
        self.max_steps = max_steps
        self.precision = precision
        self.last_steps = None

    def solve(self, operator, source, initial_guess=None):
        source = _dev.as_c128(source)
        x = (source if initial_guess is None else _dev.as_c128(initial_guess)).clone()
        init = operator.apply(x)
        r = _dev.axpby(1.0, x, -1.0, init)
        rhat = _dev.axpby(1.0, x, 1.0, init)
        alpha = omega = rho = 1.0
        p = torch.zeros_like(source)
        nu = torch.zeros_like(source)
        step = 0
        for step in range(self.max_steps):
            rho_next = _dev.cdot(rhat, r)
            beta = (rho_next / rho) * (alpha / omega)
            p = _dev.axpby(1.0, r, beta, _dev.axpby(1.0, p, -omega, nu))
            nu = operator.apply(p)
            alpha = rho_next / _dev.cdot(rhat, nu)
            s = _dev.axpby(1.0, r, -alpha, nu)
            t = operator.apply(s)
            omega = _dev.cdot(t, s) / _dev.cdot(t, t)
            _dev.axpby_(alpha, p, 1.0, x)
            _dev.axpby_(omega, s, 1.0, x)
            r = _dev.axpby(1.0, s, -omega, t)
            if abs(_dev.cdot(r, r)) < self.precision:
                self.last_steps = step
                _print(f"BiconjugateGradient: convergence after {step} steps")
                return x
            rho = rho_next
        self.last_steps = step
        _print(f"BiconjugateGradient: failed to find convergence after {step} steps")
        return x


class multishift_cg:  # noqa: N801 - named like the reference solvers
    """Multishift CG on (Q^2 + sigma_k): same interface as multishift_solver;
    stops when every shift's residual is below tol * |source|.

    ``precision=None``: the full-lattice FP64 multishift (lym_multishift_solve),
    one source.  ``precision`` in {"f64", "f32", "f16", "bf16"}: the even-odd
    multishift (lym_multishift_solve_eo) with inner iterations in that precision,
    FP64 reliable updates and every shift's FP64 true residual verified (and
    refined where needed); ``source`` may then be a batch (nrhs, ns, N, V), each
    returned solution then has the batch shape.  ``switch_residual``: FP64
    iterations until the smallest shift's true relative residual is below it,
    then the inner precision (0: the library's default per precision, < 0: the
    inner precision from the start).  ``reports`` holds one dict per (rhs,
    shift) after an even-odd solve."""

    def __init__(self, max_steps, tol, precision=None, delta=0.1, chunk=8, rhs_per_thread=0, switch_residual=0.0):
        self.max_steps = max_steps
        self.tol = tol
        self.precision = precision
        self.delta = delta
        self.chunk = chunk
        self.rhs_per_thread = rhs_per_thread
        self.switch_residual = switch_residual
        self.last_steps = None
        self.reports = None

    def solve(self, operator, source, shifts):
        q = _wilson_square(operator)
        if q is None:
            raise TypeError("multishift_cg needs SquareOperator(DiracWilsonOperator(hermitian=True))")
        source = _dev.as_c128(source)
        if self.precision is not None:
            return self._solve_eo(q, source, shifts)
        xs = torch.empty((len(shifts),) + tuple(source.shape), dtype=torch.complex128, device=source.device)
        it = ctypes.c_int()
        sh = (ctypes.c_double * len(shifts))(*[float(s) for s in shifts])
        rc = _lib.lib().lym_multishift_solve(q.solver_gauge(()), float(q.kappa), len(shifts), sh, _dev.ptr(source),
                                             _dev.ptr(xs), float(self.tol), int(self.max_steps), ctypes.byref(it),
                                             _dev.stream())
        self.last_steps = it.value
        if rc == _lib.LYM_ERR_NOT_CONVERGED:
            _print(f"multishift CG: failed to find convergence after {it.value} steps")
        else:
            _lib.check(rc, "lym_multishift_solve")
        return [xs[i] for i in range(len(shifts))]

    def _solve_eo(self, q, source, shifts):
        batched = source.dim() == 4
        bb = source if batched else source[None]
        n, ns = bb.shape[0], len(shifts)
        xs = torch.empty((n, ns) + tuple(bb.shape[1:]), dtype=torch.complex128, device=bb.device)
        sh = (ctypes.c_double * ns)(*[float(s) for s in shifts])
        prm = _lib.SolverParams(float(self.tol), int(self.max_steps), _lib.PREC[self.precision], float(self.delta),
                                1, int(self.chunk), int(self.rhs_per_thread), 0, 0, float(self.switch_residual))
        reps = (_lib.SolverReport * (n * ns))()
        precs = () if self.precision == "f64" else (self.precision,)
        rc = _lib.lib().lym_multishift_solve_eo(q.solver_gauge(precs), float(q.kappa), n, ns, sh, _dev.ptr(bb),
                                                _dev.ptr(xs), ctypes.byref(prm), reps, _dev.stream())
        self.reports = [dict(status=r.status, iterations=r.iterations, reliable_updates=r.reliable_updates,
                             true_residual=r.true_residual, kernel_launches=r.kernel_launches,
                             rhs_per_thread=r.rhs_per_thread, compressed_links=r.compressed_links) for r in reps]
        self.last_steps = max(r.iterations for r in reps)
        if rc == _lib.LYM_ERR_NOT_CONVERGED:
            _print(f"multishift CG: failed to find convergence ({self.reports})")
        else:
            _lib.check(rc, "lym_multishift_solve_eo")
        if batched:
            return [xs[:, k] for k in range(ns)]
        return [xs[0, k] for k in range(ns)]


class conjugate_gradient:  # noqa: N801 - named like the reference solvers
    """Even-odd CG for D x = b (Q x = b when the operator is hermitian) with FP64
    reliable updates.  ``precision`` in {"f64", "f32", "f16", "bf16"} is the inner
    precision; ``tol`` the target true relative residual |b - D x| / |b|."""

    def __init__(self, max_steps=20000, tol=1e-10, precision="f64", delta=0.1, chunk=8, rhs_per_thread=0,
                 compressed_links=0, mixed_fma=0):
        self.max_steps = max_steps
        self.tol = tol
        self.precision = precision
        self.delta = delta
        self.chunk = chunk
        self.rhs_per_thread = rhs_per_thread  # 0: the library's autotuner picks the hop tile
        self.compressed_links = compressed_links  # with a forced tile: 1 = N-1-row links
        self.mixed_fma = mixed_fma  # with a forced tile and FP16: 1 = the mixed-precision hop
        self.reports = None

    def solve(self, operator, source):
        if not isinstance(operator, DiracWilsonOperator) or operator.representation != "fundamental":
            raise TypeError("conjugate_gradient solves with a fundamental-representation DiracWilsonOperator")
        b = _dev.as_c128(source)
        batched = b.dim() == 4
        bb = b if batched else b[None]
        x = torch.empty_like(bb)
        n = bb.shape[0]
        prm = _lib.SolverParams(float(self.tol), int(self.max_steps), _lib.PREC[self.precision], float(self.delta),
                                int(bool(operator.hermitian)), int(self.chunk), int(self.rhs_per_thread),
                                int(self.compressed_links), int(self.mixed_fma))
        reps = (_lib.SolverReport * n)()
        precs = () if self.precision == "f64" else (self.precision,)
        rc = _lib.lib().lym_wilson_solve(operator.solver_gauge(precs), float(operator.kappa), n, _dev.ptr(bb),
                                         _dev.ptr(x), ctypes.byref(prm), reps, _dev.stream())
        self.reports = [dict(status=r.status, iterations=r.iterations, reliable_updates=r.reliable_updates,
                             true_residual=r.true_residual, kernel_launches=r.kernel_launches,
                             rhs_per_thread=r.rhs_per_thread, compressed_links=r.compressed_links,
                             mixed_fma=r.mixed_fma) for r in reps]
        if rc == _lib.LYM_ERR_NOT_CONVERGED:
            _print(f"conjugate_gradient: failed to find convergence ({self.reports})")
        else:
            _lib.check(rc, "lym_wilson_solve")
        return x if batched else x[0]


def solve_lattices(operators, sources, tol=1e-10, precision="f32", max_steps=20000, delta=0.1, chunk=8, tols=None):
    """Independent lattices solved together (lym_wilson_solve_multi): D x = b (Q x = b
    when the operators are hermitian) for every fundamental DiracWilsonOperator in
    ``operators`` (distinct objects, same dimension and N, each with its own geometry,
    kappa and links) and its ``sources[l]`` ((ns, N, V) or a batch (nrhs, ns, N, V)).
    The sloppy CG iterations of all lattices run in the same launches.  Returns the
    solutions (shaped like the sources) and one list of report dicts per lattice.
    ``tols``: one target true relative residual per lattice (default ``tol`` for all).
    Builder-defined (the reference solves one lattice per process)."""
    n = len(operators)
    if n == 0 or len(sources) != n:
        raise ValueError("one source (batch) per operator")
    herm = bool(operators[0].hermitian)
    for op in operators:
        if not isinstance(op, DiracWilsonOperator) or op.representation != "fundamental":
            raise TypeError("solve_lattices takes fundamental-representation DiracWilsonOperators")
        if bool(op.hermitian) != herm:
            raise ValueError("every operator needs the same hermitian flag")
    bs = [_dev.as_c128(b) for b in sources]
    batched = [b.dim() == 4 for b in bs]
    bb = [b if bt else b[None] for b, bt in zip(bs, batched)]
    xs = [torch.empty_like(b) for b in bb]
    precs = () if precision == "f64" else (precision,)
    handles = [op.solver_gauge(precs) for op in operators]
    gauges = (ctypes.c_void_p * n)(*[h.value for h in handles])
    kappas = (ctypes.c_double * n)(*[float(op.kappa) for op in operators])
    nrhs = (ctypes.c_int * n)(*[int(b.shape[0]) for b in bb])
    bptr = (ctypes.c_void_p * n)(*[b.data_ptr() for b in bb])
    xptr = (ctypes.c_void_p * n)(*[x.data_ptr() for x in xs])
    prm = _lib.SolverParams(float(tol), int(max_steps), _lib.PREC[precision], float(delta), int(herm), int(chunk),
                            0, 0, 0, 0.0)
    total = sum(int(b.shape[0]) for b in bb)
    reps = (_lib.SolverReport * total)()
    tol_arr = None if tols is None else (ctypes.c_double * n)(*[float(t) for t in tols])
    rc = _lib.lib().lym_wilson_solve_multi(n, gauges, kappas, tol_arr, nrhs, bptr, xptr, ctypes.byref(prm), reps,
                                           _dev.stream())
    flat = [dict(status=r.status, iterations=r.iterations, reliable_updates=r.reliable_updates,
                 true_residual=r.true_residual, kernel_launches=r.kernel_launches) for r in reps]
    if rc == _lib.LYM_ERR_NOT_CONVERGED:
        _print("solve_lattices: failed to find convergence for some right-hand sides")
    else:
        _lib.check(rc, "lym_wilson_solve_multi")
    out, reports, k = [], [], 0
    for x, bt in zip(xs, batched):
        out.append(x if bt else x[0])
        reports.append(flat[k:k + x.shape[0]])
        k += x.shape[0]
    return out, reports


class eo_square_solver:  # noqa: N801 - named like the reference solvers
    """(Q^2 + sigma_k) x_k = b for SquareOperator(DiracWilsonOperator(hermitian=True)),
    with the interface of multishift_solver (dirac_solver.py:19), so that it plugs
    into RationalApproximation and fermion_action.n_flavor.  sigma = 0: two
    even-odd CG solves Q y = b, Q x = y (conjugate_gradient, relative true residual
    ``tol`` each, inner ``precision``); sigma > 0: the even-odd multishift_cg in the
    same inner precision (relative tolerance ``tol`` per shift).  ``last_iterations`` holds the CG iterations of the last call."""

    def __init__(self, tol=1e-10, precision="f64", max_steps=20000, **cg_options):
        self.tol = tol
        self.precision = precision
        self.max_steps = max_steps
        self.cg_options = cg_options
        self.last_iterations = 0
        self.total_iterations = 0

    def solve(self, operator, source, shifts):
        q = _wilson_square(operator)
        if q is None:
            raise TypeError("eo_square_solver needs SquareOperator(DiracWilsonOperator(hermitian=True))")
        shifts = [float(s) for s in shifts]
        out = [None] * len(shifts)
        self.last_iterations = 0
        zero = [i for i, s in enumerate(shifts) if s == 0.0]
        rest = [i for i, s in enumerate(shifts) if s != 0.0]
        if zero:
            cg = conjugate_gradient(max_steps=self.max_steps, tol=self.tol, precision=self.precision,
                                    **self.cg_options)
            y = cg.solve(q, source)
            self.last_iterations += max(r["iterations"] for r in cg.reports)
            x = cg.solve(q, y)
            self.last_iterations += max(r["iterations"] for r in cg.reports)
            for i in zero:
                out[i] = x
        if rest:
            if any(shifts[i] < 0 for i in rest):
                raise ValueError("eo_square_solver takes shifts >= 0")
            ms = multishift_cg(self.max_steps, self.tol, precision=self.precision,
                               delta=self.cg_options.get("delta", 0.1), chunk=self.cg_options.get("chunk", 8))
            xs = ms.solve(operator, source, [shifts[i] for i in rest])
            self.last_iterations += ms.last_steps
            for k, i in enumerate(rest):
                out[i] = xs[k]
        self.total_iterations += self.last_iterations
        return out
