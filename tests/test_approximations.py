"""The 12-pole x^(-1/2) rational approximation on [1e-4, 1] (no counterpart in the
reference's approximations.py, which ships heatbath / force / Metropolis tables
only): pinned by its maximum relative error, its equal ripple and its format."""
import numpy as np

from tfleonardym_b200 import approximations as A


def test_twelve_pole_inverse_sqrt_error_bound():
    coeffs = A.inverse_sqrt_rational_approximation_coefficients
    assert coeffs.shape == (24,)
    alphas, betas = A.split(coeffs)
    assert np.all(betas > 0) and np.all(np.diff(betas) > 0)  # positive shifts for the multishift CG
    assert np.all(alphas > 0)
    err = A.max_relative_error(alphas, betas, 0.0, 1e-4, 1.0, grid=400001)
    assert err < 1.1e-8, err
    assert abs(err - A.INVERSE_SQRT_12_MAX_RELATIVE_ERROR) < 1e-10


def test_equal_ripple():
    """Zolotarev's approximation is minimax: the relative error reaches its bound with
    alternating sign 2n + 1 times on [lo, hi] (Chebyshev alternation)."""
    n = 12
    alphas, betas, err = A.zolotarev_inverse_sqrt(n, 1e-4)
    x = np.exp(np.linspace(np.log(1e-4), 0.0, 400001))
    e = np.sqrt(x) * np.sum(alphas[:, None] / (x[None, :] + betas[:, None]), axis=0) - 1.0
    # local extrema of e with |e| within 1% of the bound, counted with their signs
    idx = np.where((np.abs(e[1:-1]) >= np.abs(e[:-2])) & (np.abs(e[1:-1]) >= np.abs(e[2:])))[0] + 1
    ext = [e[0]] + [e[i] for i in idx] + [e[-1]]
    signs = np.sign([v for v in ext if abs(v) > 0.99 * err])
    # rounding makes a flat extremum show up as several neighbouring maxima of one sign
    runs = 1 + int(np.count_nonzero(signs[1:] != signs[:-1]))
    assert runs >= 2 * n + 1, runs


def test_error_falls_with_poles_and_scales_with_the_interval():
    errs = [A.zolotarev_inverse_sqrt(n, 1e-4)[2] for n in (6, 9, 12)]
    assert errs[0] > errs[1] > errs[2]
    # scaling the interval scales the coefficients, not the relative error
    a1, b1, e1 = A.zolotarev_inverse_sqrt(8, 1e-4, 1.0)
    a2, b2, e2 = A.zolotarev_inverse_sqrt(8, 1e-2, 1e2)
    assert abs(e1 - e2) < 1e-3 * e1
    np.testing.assert_allclose(b2, 1e2 * b1, rtol=1e-9)
    np.testing.assert_allclose(a2, 1e1 * a1, rtol=1e-9)


def test_package_star_import_exports_every_listed_module():
    """Every name in the package's __all__ is a module that imports (a caller may
    `from tfleonardym_b200 import *` the way it imports the reference's modules)."""
    import importlib

    import tfleonardym_b200
    for name in tfleonardym_b200.__all__:
        importlib.import_module(f"tfleonardym_b200.{name}")
    ns = {}
    exec("from tfleonardym_b200 import *", ns)
    assert all(name in ns for name in tfleonardym_b200.__all__)
