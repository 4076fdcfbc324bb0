"""Rational approximations for the multishift solvers (the counterpart of the
reference's approximations.py).

The reference stores each approximation as one flat array: the first half the
residues alpha_i, the second half the shifts beta_i, used with shift 0 as
R(x) = sum_i alpha_i / (x + beta_i) (TfLeonardYMNDim.py:310-332 splits them and
builds dirac.RationalApproximation).  It ships tables for the heatbath, force and
Metropolis steps only (approximations.py:79-139).  This module adds x^(-1/2) on
[1e-4, 1] with 12 poles, generated here in closed form:

Zolotarev's optimal (n-1, n) rational approximation of 1/sqrt(x) on [1, b]
(Zolotarev 1877; in the form used for lattice fermions by e.g. van den Eshof et
al., Comput. Phys. Commun. 146 (2002) 203, and Chiu et al., Phys. Rev. D 66 (2002)
114502):
    R(x) = d0 prod_{l=1}^{n-1} (x + c_{2l}) / prod_{l=1}^{n} (x + c_{2l-1}),
    c_l = sn^2(l K / (2n); k) / cn^2(l K / (2n); k),   k^2 = 1 - 1/b,  K = K(k),
with sn, cn the Jacobi elliptic functions and d0 set so that the relative error
sqrt(x) R(x) - 1 oscillates between equal and opposite extremes.  On [lo, hi] the
variable is scaled by lo (b = hi / lo) and the result written in partial
fractions, so that every pole is a positive shift of the multishift solver.
"""
import numpy as np
import scipy.special


def zolotarev_inverse_sqrt(n, lo, hi=1.0, grid=200001):
    """alphas, betas (n each, betas ascending and positive) and the maximum relative
    error of sum_i alpha_i / (x + beta_i) against x^(-1/2) on [lo, hi]."""
    if n < 1 or not 0 < lo < hi:
        raise ValueError("need n >= 1 and 0 < lo < hi")
    b = hi / lo
    # k^2 = 1 - 1/b: K from ellipkm1 (accurate for k^2 near 1)
    m = 1.0 - 1.0 / b
    kk = scipy.special.ellipkm1(1.0 / b)
    sn, cn, _, _ = scipy.special.ellipj(np.arange(1, 2 * n) * kk / (2 * n), m)
    c = sn ** 2 / cn ** 2
    c_den, c_num = c[0::2], c[1::2]  # c_1, c_3, ..., c_{2n-1} and c_2, ..., c_{2n-2}
    # partial fractions of prod (x + c_num) / prod (x + c_den)
    a = np.array([np.prod(c_num - cd) / np.prod(np.delete(c_den, i) - cd) for i, cd in enumerate(c_den)])
    # equal-ripple scale on a logarithmic grid of [1, b]
    y = np.exp(np.linspace(0.0, np.log(b), grid))
    f = np.sqrt(y) * np.sum(a[:, None] / (y[None, :] + c_den[:, None]), axis=0)
    d0 = 2.0 / (f.max() + f.min())
    # back to [lo, hi]: 1/sqrt(x) = lo^(-1/2) R(x / lo)
    alphas = np.sqrt(lo) * d0 * a
    betas = lo * c_den
    order = np.argsort(betas)
    alphas, betas = alphas[order], betas[order]
    return alphas, betas, max_relative_error(alphas, betas, 0.0, lo, hi, grid)


def max_relative_error(alphas, betas, shift, lo, hi, grid=200001, power=-0.5):
    """max over a logarithmic grid of [lo, hi] of |R(x) / x^power - 1|, with
    R(x) = shift + sum_i alpha_i / (x + beta_i) (dirac.py:61-67, RationalApproximation.evaluate)."""
    x = np.exp(np.linspace(np.log(lo), np.log(hi), grid))
    r = shift + np.sum(np.asarray(alphas)[:, None] / (x[None, :] + np.asarray(betas)[:, None]), axis=0)
    return float(np.max(np.abs(r / x ** power - 1.0)))


def split(coefficients):
    """(alphas, betas) of a flat table in the reference's format (TfLeonardYMNDim.py:310-332)."""
    h = len(coefficients) // 2
    return coefficients[:h], coefficients[h:]


# x^(-1/2) on [1e-4, 1], 12 poles: [alpha_1..alpha_12, beta_1..beta_12], shift 0
_A12, _B12, INVERSE_SQRT_12_MAX_RELATIVE_ERROR = zolotarev_inverse_sqrt(12, 1e-4, 1.0)
inverse_sqrt_rational_approximation_coefficients = np.concatenate([_A12, _B12])
