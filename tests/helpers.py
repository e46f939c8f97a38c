"""Shared helpers for the tests: seeded inputs, kernels, spectra, and the
reference's pass criteria (restated)."""
import numpy as np

from oracle import oracle as O


def kernel(KW, form="sigma", dx=1.0):
    """(Kx, Ky) float32.  form 'sigma': reference pixel form with R_w = 3 sigma
    = erosion (make_kernel, training/main_cd_training.cu:63-77); 'baseline':
    gamma = 1/30 nm, R_w = erosion*dx, dx in nm."""
    e = (KW - 1) // 2
    if form == "sigma":
        return O.make_kernel_sigma(KW, e / 3.0)
    return O.make_kernel(KW, dx, 1.0 / 30.0, e * dx)


def fields(N, n, seed, ell=8.0):
    return [O.grf(N, ell, seed + i) for i in range(n)]


def rel_max_err(a, b):
    """max|a-b| / max|b| — the forward criterion of adjoint/main_adjoint.cu:359-360."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pixel_violations(a, b, tol_abs=1e-5, tol_rel=1e-3):
    """Count pixels with |a-b| > max(tol_abs, tol_rel*max(|a|,|b|))
    (AdjointTester / TangentTester criterion, adjoint_tester.h:563-567)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    lim = np.maximum(tol_abs, tol_rel * np.maximum(np.abs(a), np.abs(b)))
    return int((np.abs(a - b) > lim).sum())
