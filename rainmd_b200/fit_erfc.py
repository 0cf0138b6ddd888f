"""Fit the f32 erfc used by the direct-space kernels, and print the coefficients.

The kernels evaluate   erfc(z) = t * P(t) * exp(-z*z),   t = 1 / (1 + z/2),
so that exp(-z*z), which the screened-Coulomb force needs anyway for its Gaussian term,
is computed once per pair. P is a degree-DEGREE polynomial in t fitted here by
iteratively reweighted least squares (Lawson's algorithm) towards the minimax RELATIVE
error of erfc over z in [0, Z_MAX]. Relative accuracy is what Ewald needs: erfc at the
cutoff is ~2e-4 of its value at contact, and the direct-space sum is a cancellation.

Z_MAX covers alpha*r for every cutoff with an Ewald tolerance down to 1e-10
(alpha*rc = sqrt(-ln(2*tol)) = 4.7); beyond it the product is below 2e-10 and the
kernels' result is a correctly tiny number.

Run:  python -m rainmd_b200.fit_erfc      (needs scipy; used only to regenerate)
"""
from __future__ import annotations

import numpy as np

DEGREE = 8
Z_MAX = 5.0


def fit(degree: int = DEGREE, z_max: float = Z_MAX, iterations: int = 60):
    from scipy.special import erfcx  # erfc(z) * exp(z^2), accurate for all z

    t_min = 1.0 / (1.0 + 0.5 * z_max)
    # Chebyshev nodes in t, densely
    k = np.arange(4000)
    t = 0.5 * (1 + t_min) + 0.5 * (1 - t_min) * np.cos(np.pi * (k + 0.5) / len(k))
    z = (1.0 / t - 1.0) * 2.0
    target = erfcx(z) / t
    # basis: Chebyshev in the mapped variable for conditioning
    x = (2 * t - (1 + t_min)) / (1 - t_min)
    basis = np.polynomial.chebyshev.chebvander(x, degree)
    weights = np.ones_like(t)
    for _ in range(iterations):
        w = np.sqrt(weights) / target
        coef, *_ = np.linalg.lstsq(basis * w[:, None], target * w, rcond=None)
        err = np.abs(basis @ coef - target) / target
        weights *= err / err.max() + 1e-12
        weights /= weights.sum()
    # convert Chebyshev(x) to a monomial in t
    cheb = np.polynomial.Chebyshev(coef, domain=[t_min, 1.0])
    mono = cheb.convert(kind=np.polynomial.Polynomial)
    return mono.coef, err.max()


def check(coefficients, z_max: float = Z_MAX):
    """Relative error of the f32 evaluation order the kernels use (Horner in t)."""
    from scipy.special import erfc

    z = np.linspace(0, z_max, 200001)
    t = 1.0 / (1.0 + 0.5 * z)
    p = np.zeros_like(z)
    for c in coefficients[::-1]:
        p = p * t + c
    approx = t * p * np.exp(-z * z)
    return np.max(np.abs(approx - erfc(z)) / erfc(z))


if __name__ == "__main__":
    coef, fitted = fit()
    print(f"// degree {DEGREE}, z in [0, {Z_MAX}], fitted max relative error {fitted:.3e}, "
          f"float64 check {check(coef):.3e}")
    for c in coef:
        print(f"  {c:.9e}f,")
