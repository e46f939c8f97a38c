"""FP64 CPU oracle for the resist-shrinkage operator — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference legs use this module, and only as the checker; the product
(shrinkage_full_tests_b200) never imports it.

Everything is column-major like the reference: an image array ``a`` of shape
(N, N) here is indexed ``a[col, row]`` and its memory is buf[col*N + row].
Kernels are (KW, KW) arrays indexed ``K[i, j]`` = column offset i - KW//2,
row offset j - KW//2, i.e. the reference's K[i*KW + j].

The C restatement (srk_oracle.c) cites the reference function each routine
follows.  The reference's own generators (GpGenerator, generate_pattern) are
available through oracle/_ref when the reference was compiled (oracle/build.py).
"""
import ctypes
import os

import numpy as np

from . import build as _build

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_ref_host = None

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


def nthreads_default():
    return int(os.environ.get("SRK_ORACLE_THREADS", os.cpu_count() or 1))


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "_build", "libsrk_oracle.so")
        if not os.path.exists(path):
            path = _build.build_oracle()
        L = ctypes.CDLL(path)
        i, d = ctypes.c_int, ctypes.c_double
        L.oracle_conv_window.argtypes = [_dp, i, _dp, _dp, i, i, d, i, i, i, i, _dp, _dp, i]
        L.oracle_forward_window.argtypes = [_dp, _dp, i, _dp, _dp, i, i, d, i, i, i, i, _dp, _dp, _dp, i]
        L.oracle_adj_wrt_I.argtypes = [_dp, _dp, i, i, i, _dp]
        L.oracle_adj_wrt_E.argtypes = [_dp, _dp, _dp, _dp, i, i, i, i, d, i, _dp, i]
        L.oracle_tangent.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, i, i, i, i, d, _dp, i]
        L.oracle_tangent_adjoint.argtypes = [_dp] * 8 + [i, i, i, i, d, i, _dp, _dp, i]
        L.oracle_make_kernel.argtypes = [i, ctypes.c_float, ctypes.c_float, ctypes.c_float, _fp, _fp]
        L.oracle_kernel_freq.argtypes = [_fp, i, i, _fp]
        L.oracle_grad.argtypes = [_dp, i, _dp, _dp]
        L.oracle_forward_f32_cols.argtypes = [_fp, _fp, i, _fp, _fp, i, i, ctypes.c_float, i, i, _fp]
        _lib = L
    return _lib


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _cm(a):
    """(N,N) [col,row] array -> its column-major memory is a C-contiguous copy."""
    return np.ascontiguousarray(a, dtype=np.float64)


def grad(I):
    """Central differences (dI/dx along columns, dI/dy along rows), zero outside."""
    I, pI = _d(I)
    N = I.shape[0]
    Ix = np.empty_like(I)
    Iy = np.empty_like(I)
    lib().oracle_grad(pI, N, Ix.ctypes.data_as(_dp), Iy.ctypes.data_as(_dp))
    return Ix, Iy


def conv_valid(E, Gx, Gy, erosion, dx, window=None, nthreads=None):
    """(ux, uy) = dx^2 * valid conv of E with Gx, Gy on the output window
    (ox0, oy0, wx, wy) (default: the whole W x W)."""
    E, pE = _d(E)
    Gx, pGx = _d(Gx)
    Gy, pGy = _d(Gy)
    N, KW = E.shape[0], Gx.shape[0]
    W = N - 2 * erosion
    ox0, oy0, wx, wy = window if window is not None else (0, 0, W, W)
    ux = np.empty((wx, wy))
    uy = np.empty((wx, wy))
    lib().oracle_conv_window(pE, N, pGx, pGy, KW, erosion, dx * dx, ox0, oy0, wx, wy, ux.ctypes.data_as(_dp),
                             uy.ctypes.data_as(_dp), nthreads or nthreads_default())
    return ux, uy


def forward(E, I, Gx, Gy, erosion, dx, window=None, nthreads=None, return_u=False):
    """R = ux*dI/dx + uy*dI/dy on the valid window (srkForwardOaS)."""
    E, pE = _d(E)
    I, pI = _d(I)
    Gx, pGx = _d(Gx)
    Gy, pGy = _d(Gy)
    N, KW = E.shape[0], Gx.shape[0]
    W = N - 2 * erosion
    ox0, oy0, wx, wy = window if window is not None else (0, 0, W, W)
    R = np.empty((wx, wy))
    ux = np.empty((wx, wy))
    uy = np.empty((wx, wy))
    lib().oracle_forward_window(pE, pI, N, pGx, pGy, KW, erosion, dx, ox0, oy0, wx, wy, R.ctypes.data_as(_dp),
                                ux.ctypes.data_as(_dp), uy.ctypes.data_as(_dp), nthreads or nthreads_default())
    return (R, ux, uy) if return_u else R


def forward_f32_cols(E, I, Gx, Gy, erosion, dx, ox0, wx):
    """Output columns [ox0, ox0+wx) of the forward in the reference CPU
    checker's own form (single-thread float, cpu_conv_valid's loop order):
    the timing row of the measurement, not the checker."""
    E = np.ascontiguousarray(E, np.float32)
    I = np.ascontiguousarray(I, np.float32)
    Gx = np.ascontiguousarray(Gx, np.float32)
    Gy = np.ascontiguousarray(Gy, np.float32)
    N, KW = E.shape[0], Gx.shape[0]
    W = N - 2 * erosion
    R = np.empty((wx, W), np.float32)
    lib().oracle_forward_f32_cols(E.ctypes.data_as(_fp), I.ctypes.data_as(_fp), N, Gx.ctypes.data_as(_fp),
                                  Gy.ctypes.data_as(_fp), KW, erosion, dx, ox0, wx, R.ctypes.data_as(_fp))
    return R


def adj_wrt_I(v, ux, uy, N, erosion):
    """dL/dI = Dx^T(ux v) + Dy^T(uy v) on N x N (adjointWrtI)."""
    wx, pwx = _d(np.asarray(ux) * np.asarray(v))
    wy, pwy = _d(np.asarray(uy) * np.asarray(v))
    W = wx.shape[0]
    out = np.empty((N, N))
    lib().oracle_adj_wrt_I(pwx, pwy, W, N, erosion, out.ctypes.data_as(_dp))
    return out


def adj_wrt_E(v, I, Gx, Gy, erosion, dx, convention="reference", nthreads=None):
    """dL/dE on N x N.  convention 'true' = exact adjoint (cpu_adj_wrtE);
    'reference' = the reference FFT path's convolution with G."""
    v, pv = _d(v)
    I, pI = _d(I)
    Gx, pGx = _d(Gx)
    Gy, pGy = _d(Gy)
    N, W, KW = I.shape[0], v.shape[0], Gx.shape[0]
    out = np.empty((N, N))
    lib().oracle_adj_wrt_E(pv, pI, pGx, pGy, KW, N, W, erosion, dx, 1 if convention == "reference" else 0,
                           out.ctypes.data_as(_dp), nthreads or nthreads_default())
    return out


def tangent(f, g, df, dg, Gx, Gy, erosion, dx, nthreads=None):
    arrs = [_d(a) for a in (f, g, df, dg, Gx, Gy)]
    N, KW = arrs[0][0].shape[0], arrs[4][0].shape[0]
    W = N - 2 * erosion
    dh = np.empty((W, W))
    lib().oracle_tangent(*[p for _, p in arrs], KW, N, W, erosion, dx, dh.ctypes.data_as(_dp),
                         nthreads or nthreads_default())
    return dh


def tangent_adjoint(f, g, df, dg, lam, dlam, Gx, Gy, erosion, dx, convention="reference", nthreads=None):
    arrs = [_d(a) for a in (f, g, df, dg, lam, dlam, Gx, Gy)]
    N, KW = arrs[0][0].shape[0], arrs[6][0].shape[0]
    W = N - 2 * erosion
    dlf = np.empty((N, N))
    dlg = np.empty((N, N))
    lib().oracle_tangent_adjoint(*[p for _, p in arrs], KW, N, W, erosion, dx,
                                 1 if convention == "reference" else 0, dlf.ctypes.data_as(_dp),
                                 dlg.ctypes.data_as(_dp), nthreads or nthreads_default())
    return dlf, dlg


def make_kernel(kw, dx, gamma, Rw):
    """(Kx, Ky) float32 (KW, KW) exactly as the reference generates them."""
    Kx = np.zeros((kw, kw), np.float32)
    Ky = np.zeros((kw, kw), np.float32)
    lib().oracle_make_kernel(kw, dx, gamma, Rw, Kx.ctypes.data_as(_fp), Ky.ctypes.data_as(_fp))
    return Kx, Ky


def make_kernel_sigma(kw, sigma_px):
    """Reference pixel-unit form: gamma = 1/sigma, R_w = 3 sigma, dx = 1
    (training/main_cd_training.cu:63-77)."""
    return make_kernel(kw, 1.0, 1.0 / sigma_px, 3.0 * sigma_px)


def kernel_freq(K, M):
    """Reference-layout spectrum (complex64 array of shape (M, M//2+1), [kx, ky])."""
    K = np.ascontiguousarray(K, np.float32)
    out = np.empty((M, M // 2 + 1), np.complex64)
    lib().oracle_kernel_freq(K.ctypes.data_as(_fp), K.shape[0], M, out.view(np.float32).ctypes.data_as(_fp))
    return out


def next_pow2(n):
    p = 1
    while p < n:
        p <<= 1
    return p


def grf_filter(noise, N, ell):
    """Filter white noise (Np, Np) [col, row] as GpGenerator::generate
    (third_party/include/stTestCore/gp_generator.h:119-147, filter :180-201):
    H = sqrt(max(0, Re FFT2(c))) of the periodic covariance
    c(dx, dy) = exp(-(dx^2 + dy^2) / (2 ell^2)) with nearest-image
    displacements d in (-Np/2, Np/2], x = Re IFFT2(H FFT2(w)), cropped to
    the top-left N x N.  FP64."""
    w = np.asarray(noise, np.float64)
    Np = w.shape[0]
    d = np.arange(Np)
    d = np.where(d <= Np // 2, d, d - Np).astype(np.float64)
    c = np.exp(-0.5 * (d[:, None] ** 2 + d[None, :] ** 2) / (ell * ell))
    H = np.sqrt(np.maximum(0.0, np.fft.fft2(c).real))
    x = np.fft.ifft2(H * np.fft.fft2(w)).real
    return x[:N, :N]


def minmax01(x):
    return (x - x.min()) / (x.max() - x.min())


def grf(N, ell, seed):
    """Seeded Gaussian random field, col-major (N, N) float32: white N(0,1)
    noise (numpy PCG64, this seed) on the padded grid, filtered as
    GpGenerator (grf_filter), then min-max scaled to [0, 1]."""
    Np = next_pow2(N)
    w = np.random.default_rng(seed).standard_normal((Np, Np))
    return minmax01(grf_filter(w, N, ell)).astype(np.float32)


# ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011), vectorised
_PH_M0, _PH_M1, _PH_W0, _PH_W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Counters c0..c3 (uint32 arrays or ints), key (k0, k1): the 4 output words."""
    m32 = np.uint64(0xFFFFFFFF)
    c = [np.asarray(v, np.uint64) & m32 for v in (c0, c1, c2, c3)]
    k = [np.uint64(k0 & 0xFFFFFFFF), np.uint64(k1 & 0xFFFFFFFF)]
    for r in range(10):
        if r:
            k = [(k[0] + np.uint64(_PH_W0)) & m32, (k[1] + np.uint64(_PH_W1)) & m32]
        p0 = np.uint64(_PH_M0) * c[0]
        p1 = np.uint64(_PH_M1) * c[2]
        c = [(p1 >> np.uint64(32)) ^ c[1] ^ k[0], p1 & m32, (p0 >> np.uint64(32)) ^ c[3] ^ k[1], p0 & m32]
    return [v.astype(np.uint32) for v in c]


def philox_noise(N, seed, b=0):
    """The white noise of the device generator for image b (key seed + b):
    (Np, Np) [col, row]; pixel p = col*Np + row takes word p mod 4 of the
    Philox block p // 4, pairs (0,1), (2,3) through Box-Muller, uniforms
    (bits + 0.5) 2^-32.  Float32 like the device."""
    Np = next_pow2(N)
    q = np.arange(Np * Np // 4, dtype=np.uint64)
    key = (seed + b) & 0xFFFFFFFFFFFFFFFF
    r = philox4x32_10(q & np.uint64(0xFFFFFFFF), q >> np.uint64(32), 0, 0, key & 0xFFFFFFFF, key >> 32)
    u = [((v.astype(np.float32) + np.float32(0.5)) * np.float32(2.0 ** -32)).astype(np.float64) for v in r]
    m0, m1 = np.sqrt(-2.0 * np.log(u[0])), np.sqrt(-2.0 * np.log(u[2]))
    a0, a1 = 2.0 * np.pi * u[1], 2.0 * np.pi * u[3]
    z = np.stack([m0 * np.cos(a0), m0 * np.sin(a0), m1 * np.cos(a1), m1 * np.sin(a1)], axis=1).ravel()
    return z.reshape(Np, Np)


def ref_host():
    """The reference's own host generators (None if not built here)."""
    global _ref_host
    if _ref_host is None:
        path = os.path.join(_HERE, "_ref", "libref_host.so")
        if not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        L.ref_gp_field.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_ulonglong, _fp]
        L.ref_lns.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, _fp]
        L.ref_gp_noise.argtypes = [ctypes.c_int, ctypes.c_ulonglong, _dp]
        _ref_host = L
    return _ref_host


def ref_gp_field(N, ell, seed):
    """GpGenerator(Covariance2D::isotropic(ell), N, N, seed).generate()."""
    out = np.empty((N, N), np.float32)
    ref_host().ref_gp_field(N, ell, seed, out.ctypes.data_as(_fp))
    return out


def ref_gp_noise(N, seed):
    """The white noise GpGenerator draws for this seed, (Np, Np) [col, row]."""
    Np = next_pow2(N)
    out = np.empty((Np, Np), np.float64)
    ref_host().ref_gp_noise(N, seed, out.ctypes.data_as(_dp))
    return out


def ref_lns(vertical, N, sigma_px, period_px=0.0):
    out = np.empty((N, N), np.float32)
    ref_host().ref_lns(0 if vertical else 1, N, sigma_px, period_px, out.ctypes.data_as(_fp))
    return out


def measure_cd(sig, L=16, A=8):
    """CD of each signal (rows of sig) in pixels, FP64 restatement of
    MeasureCD_Batched (third_party/src/metricUtil/cd_measure_util.cu:43-437):
    polyphase sinc x Blackman upsampling, linear zero crossings, nearest
    crossing left of / at-or-right of the centre.  Returns (left, right, cd)."""
    sig = np.atleast_2d(np.asarray(sig, np.float64))
    B, n = sig.shape
    taps = 2 * A + 1
    k = np.arange(-A, A + 1)
    h = np.zeros((L, taps))
    for r in range(L):
        t = k - r / L
        s = np.where(np.abs(t) < 1e-6, 1.0, np.sin(np.pi * t) / np.where(np.abs(t) < 1e-6, 1.0, np.pi * t))
        u = (t + A) / (2 * A)
        bw = 0.42 - 0.5 * np.cos(2 * np.pi * u) + 0.08 * np.cos(4 * np.pi * u)
        w = np.where(np.abs(t) > A + 1e-6, 0.0, s * bw)
        h[r] = w / w.sum()
    nup = n * L
    m = np.arange(nup)
    rr, kk = m % L, m // L
    idx = kk[:, None] + np.arange(taps)[None, :] - A
    valid = (idx >= 0) & (idx < n)
    idxc = np.clip(idx, 0, n - 1)
    centre = 0.5 * (nup - 1)
    left = np.full(B, -np.inf)
    right = np.full(B, np.inf)
    for b in range(B):
        up = (np.where(valid, sig[b][idxc], 0.0) * h[rr]).sum(axis=1)
        y0, y1 = up[:-1], up[1:]
        cross = ((y0 <= 0) & (y1 > 0)) | ((y0 > 0) & (y1 <= 0))
        i = np.nonzero(cross)[0]
        den = y1[i] - y0[i]
        x = np.where(np.abs(den) < 1e-30, i, i - y0[i] / np.where(np.abs(den) < 1e-30, 1.0, den))
        if np.any(x < centre):
            left[b] = x[x < centre].max()
        if np.any(x >= centre):
            right[b] = x[x >= centre].min()
    return left / L, right / L, (right - left) / L


def lns(vertical, N, sigma_px, period_px=0.0, nbrs=4):
    """Line/space pattern (Gaussian pulse train minus 0.5), col-major (N, N),
    restating gen_lns_vertical/_horizontal (third_party/src/patternUtil/test_pattern.cu:129-171)."""
    fwhm = 2.0 * np.sqrt(2.0 * np.log(2.0)) * sigma_px
    period = period_px if period_px > 0 else 4.0 * fwhm
    centre = 0.5 * (N - 1)
    x = np.arange(N, dtype=np.float64)
    val = sum(np.exp(-((x - (centre + k * period)) ** 2) / (2 * sigma_px ** 2)) for k in range(-nbrs, nbrs + 1)) - 0.5
    img = np.empty((N, N))
    if vertical:
        img[:, :] = val[:, None]   # value depends on the column
    else:
        img[:, :] = val[None, :]   # value depends on the row
    return img.astype(np.float32)
