"""Window checks of device outputs against the FP64 oracle.

At large N the whole-image oracle is out of reach, so each check crops from
the device inputs the part of the image that a square output window depends
on, runs the oracle on that crop, and compares the crop's outputs at the
window's position with the device outputs there.

Coordinates: images are [col, row] tensors (column-major memory).  A forward-
type output (R, dh: W x W) at W-coordinates (ox, oy) depends on the input
pixels [ox, ox + w + 2e); an adjoint-type output (N x N) at pixel (px, py)
depends on the W-sized arrays and the images within 2e + 2 pixels of it.  For
the adjoint-type outputs the crop is n = w + 4e + 4 pixels wide, placed at
x0 = clamp(px - 2e - 2, 0, N - n): its own valid region then holds every
contribution to the window, including the windows that touch the image edge
(there the crop edge is the image edge and both follow the same zero rule).

Errors are reported as max|d| / max|ref| over the window (the forward
criterion of adjoint/main_adjoint.cu:359-360) together with the per-pixel
criterion of adjoint_tester.h:563-567.
"""
import json
import os

import numpy as np

from oracle import oracle as O
from tests.helpers import pixel_violations, rel_max_err


def to_host(t, x0, y0, nx, ny=None):
    ny = nx if ny is None else ny
    return t[x0:x0 + nx, y0:y0 + ny].double().cpu().numpy()


def adj_crop(p, w, e, N):
    n = w + 4 * e + 4
    assert n <= N, "window too large for the image"
    return min(max(p - 2 * e - 2, 0), N - n), n


def forward_window(f, g, Kx, Ky, e, dx, R, ox, oy, w):
    """R = forward(E=g, I=f) on the W-window at (ox, oy)."""
    n = w + 2 * e
    ref = O.forward(to_host(g, ox, oy, n), to_host(f, ox, oy, n), Kx, Ky, e, dx)
    return to_host(R, ox, oy, w), ref


def tangent_window(f, g, df, dg, Kx, Ky, e, dx, dh, ox, oy, w):
    n = w + 2 * e
    c = [to_host(t, ox, oy, n) for t in (f, g, df, dg)]
    return to_host(dh, ox, oy, w), O.tangent(*c, Kx, Ky, e, dx)


def adjoint_window(v, ux, uy, I, Kx, Ky, e, dx, dLdI, dLdE, px, py, w, convention):
    """(dL/dI, dL/dE) of adjointSRK (v, ux, uy given) on the N-window at (px, py)."""
    N = I.shape[0]
    x0, n = adj_crop(px, w, e, N)
    y0, _ = adj_crop(py, w, e, N)
    m = n - 2 * e
    vh, uxh, uyh = (to_host(t, x0, y0, m) for t in (v, ux, uy))
    Ih = to_host(I, x0, y0, n)
    rI = O.adj_wrt_I(vh, uxh, uyh, n, e)
    rE = O.adj_wrt_E(vh, Ih, Kx, Ky, e, dx, convention)
    sx, sy = px - x0, py - y0
    return ((to_host(dLdI, px, py, w), rI[sx:sx + w, sy:sy + w]),
            (to_host(dLdE, px, py, w), rE[sx:sx + w, sy:sy + w]))


def tangent_adjoint_window(f, g, df, dg, lam, dlam, Kx, Ky, e, dx, dlf, dlg, px, py, w, convention):
    N = f.shape[0]
    x0, n = adj_crop(px, w, e, N)
    y0, _ = adj_crop(py, w, e, N)
    m = n - 2 * e
    c = [to_host(t, x0, y0, n) for t in (f, g, df, dg)]
    l = [to_host(t, x0, y0, m) for t in (lam, dlam)]
    rf, rg = O.tangent_adjoint(*c, *l, Kx, Ky, e, dx, convention)
    sx, sy = px - x0, py - y0
    return ((to_host(dlf, px, py, w), rf[sx:sx + w, sy:sy + w]),
            (to_host(dlg, px, py, w), rg[sx:sx + w, sy:sy + w]))


def windows(size, w, count, seed, corners=True):
    """`count` random window origins in [0, size - w], plus the two far corners."""
    rng = np.random.default_rng(seed)
    out = [(int(rng.integers(0, size - w + 1)), int(rng.integers(0, size - w + 1))) for _ in range(count)]
    if corners:
        out += [(0, 0), (size - w, size - w)]
    return out


class ErrorLog:
    """Max error over the windows of one (op, N, KW, dtype) case; appended as
    one JSON line to $SRK_ERROR_LOG when that variable is set."""

    def __init__(self, op, N, KW, dtype, **extra):
        self.case = dict(op=op, N=N, KW=KW, dtype=dtype, **extra)
        self.rel = 0.0
        self.viol = 0
        self.pixels = 0
        self.windows = 0

    def add(self, got, ref, tol_abs, tol_rel):
        self.rel = max(self.rel, rel_max_err(got, ref))
        self.viol += pixel_violations(got, ref, tol_abs=tol_abs, tol_rel=tol_rel)
        self.pixels += got.size
        self.windows += 1

    def write(self):
        path = os.environ.get("SRK_ERROR_LOG")
        if path:
            with open(path, "a") as fh:
                fh.write(json.dumps(dict(self.case, max_rel=self.rel, pixel_violations=self.viol,
                                         pixels=self.pixels, windows=self.windows)) + "\n")
        return self
