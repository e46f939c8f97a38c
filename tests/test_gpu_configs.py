"""The derivative operators at their benchmark sizes, against the FP64 oracle
on output windows (tests/windows.py), in FP32 and in FP16 storage.

* adjoint grid: adjointSRK at N in {1k, 2k, 4k, 8k} x KW in {31, 61, 121}
  (the reference's large-N adjoint checks, adjoint/main_adjoint.cu:735-769,
  :846, :913), plus the dot-product identity <h(f,g), w> = <g, A_g* w> =
  <f, A_f* w> of the save-for-backward VJP at the same sizes;
* tangent grid: shrinkageTangentOaS and shrinkageTangentAdjointOaS at N in
  {4k, 8k, 16k} x KW in {31, 121} (tan_tanadj/main_tan_tanadj.cu:505-646);
* the reference's tangent and tangent-adjoint derivative protocols (every
  mode, 3 directions, the epsilon sweep, every pixel) at N = 4096, KW = 121,
  where the operators run on the 512-point tile path;
* one 32768 x 32768 image, KW = 121, Gaussian random fields of correlation
  length 32 px: all four operators on random windows.

Inputs are seeded Gaussian random fields (correlation length 8 px unless
stated, min-max scaled to [0, 1]) made on the device by the library's
generator; cotangents N(0, 1); tangent directions N(0, 1) x 1e-2.  FP16
storage is held to max|d|/max|ref| < 1e-2 and the per-pixel rule with
abs 1e-3 / rel 1e-2; FP32 to the reference's tolerances.  With
SRK_ERROR_LOG set, every case appends its maximum errors to that file."""
import os

import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from tests.gpu_util import spectra
from tests.helpers import kernel
from tests.windows import (ErrorLog, adjoint_window, forward_window, tangent_adjoint_window, tangent_window,
                           windows)

pytestmark = pytest.mark.gpu

SPECTRA_M = {True: 2048, False: 1024}  # the reference's OaS tile: 2048 for N >= 8k (adjoint/main_adjoint.cu:33)

# dtype -> (srk dtype, tolerances: forward/tangent rel, adjoint-type rel, pixel abs, pixel rel)
TOL = {"f32": (srk.SRK_F32, 1e-3, 1e-4, 1e-5, 1e-3),
       "f16": (srk.SRK_F16, 1e-2, 1e-2, 1e-3, 1e-2)}


def tdtype(torch, dt):
    return torch.float32 if dt == "f32" else torch.float16


def grf(torch, N, seed, ell=8.0):
    out = torch.empty((1, N, N), device="cuda")
    srk.grf(out, ell, seed)
    return out[0]


def make(torch, N, KW, dt, B=1):
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    Ms = SPECTRA_M[N >= 8192]
    GX, GY = spectra(Kx, Ky, Ms, torch)
    plan = srk.SrkPlan(N, W, e, 1.0, B, spectra_M=Ms, dtype=TOL[dt][0])
    return e, W, Kx, Ky, GX, GY, plan


def check(log, got, ref, rel_tol, tol_abs, tol_rel):
    log.add(got, ref, tol_abs, tol_rel)
    assert log.rel < rel_tol, log.case
    assert log.viol == 0, log.case


@pytest.mark.parametrize("dt", ["f32", "f16"])
@pytest.mark.parametrize("KW", [31, 61, 121])
@pytest.mark.parametrize("N", [1024, 2048, 4096, 8192])
def test_adjoint_grid_windows(torch_cuda, N, KW, dt):
    torch = torch_cuda
    T = tdtype(torch, dt)
    _, r_fwd, r_adj, t_abs, t_rel = TOL[dt]
    e, W, Kx, Ky, GX, GY, plan = make(torch, N, KW, dt)
    f = grf(torch, N, 10 + N + KW).to(T)
    g = grf(torch, N, 20 + N + KW).to(T)
    gen = torch.Generator(device="cuda").manual_seed(N + KW)
    v = torch.randn((W, W), device="cuda", generator=gen).to(T)
    R = torch.empty((W, W), device="cuda", dtype=T)
    ux, uy = torch.empty_like(R), torch.empty_like(R)
    srk.srkForwardOaS(g, f, GX, GY, N, W, e, 1.0, None, R, plan, ux, uy)
    dLdI = torch.empty((N, N), device="cuda", dtype=T)
    dLdE = torch.empty_like(dLdI)
    srk.adjointSRK(v, ux, uy, f, GX, GY, N, W, e, 1.0, None, dLdI, dLdE, plan)
    plan.sync()
    lf = ErrorLog("forward", N, KW, dt)
    li, le = ErrorLog("adjoint_dLdI", N, KW, dt), ErrorLog("adjoint_dLdE", N, KW, dt)
    w = 128
    for (ox, oy) in windows(W, w, 1, N + KW):
        got, ref = forward_window(f, g, Kx, Ky, e, 1.0, R, ox, oy, w)
        check(lf, got, ref, r_fwd, t_abs, t_rel)
    for (px, py) in windows(N, w, 2, 7 * N + KW):
        (gi, ri), (ge, re) = adjoint_window(v, ux, uy, f, Kx, Ky, e, 1.0, dLdI, dLdE, px, py, w, "reference")
        check(li, gi, ri, r_adj if dt == "f16" else 1e-5, t_abs, t_rel)
        check(le, ge, re, r_adj, t_abs, t_rel)
    for lg in (lf, li, le):
        lg.write()


@pytest.mark.parametrize("dt", ["f32", "f16"])
@pytest.mark.parametrize("KW", [31, 61, 121])
@pytest.mark.parametrize("N", [1024, 8192])
def test_vjp_dot_product_identity(torch_cuda, N, KW, dt):
    """<h(f, g), w> = <g, dL/dg> = <f, dL/df> for the exact adjoint (srk_vjp
    recomputes conv(g, G) from the saved f, g)."""
    torch = torch_cuda
    T = tdtype(torch, dt)
    e, W, Kx, Ky, GX, GY, plan = make(torch, N, KW, dt)
    plan.import_spectra(GX, GY)
    f = grf(torch, N, 30 + N).to(T)
    g = grf(torch, N, 40 + N).to(T)
    w = torch.randn((W, W), device="cuda", generator=torch.Generator(device="cuda").manual_seed(5)).to(T)
    h = torch.empty((1, W, W), device="cuda", dtype=T)
    srk.forward(f[None], g[None], 1, h, plan)
    dLdf = torch.empty((1, N, N), device="cuda", dtype=T)
    dLdg = torch.empty_like(dLdf)
    srk.vjp(w[None], f[None], g[None], 1, dLdf, dLdg, plan)
    plan.sync()
    d = lambda a, b: float((a.double() * b.double()).sum())
    lhs = d(h[0], w)
    scale = float(h.double().norm() * w.double().norm())
    tol = 1e-5 if dt == "f32" else 1e-3
    log = ErrorLog("vjp_dot_product", N, KW, dt)
    for rhs in (d(g, dLdg[0]), d(f, dLdf[0])):
        err = abs(lhs - rhs) / scale
        log.rel = max(log.rel, err)
        assert err < tol, (lhs, rhs, scale)
    log.write()


@pytest.mark.parametrize("dt", ["f32", "f16"])
@pytest.mark.parametrize("KW", [31, 121])
@pytest.mark.parametrize("N", [4096, 8192, 16384])
def test_tangent_grid_windows(torch_cuda, N, KW, dt):
    torch = torch_cuda
    T = tdtype(torch, dt)
    _, r_fwd, r_adj, t_abs, t_rel = TOL[dt]
    e, W, Kx, Ky, GX, GY, plan = make(torch, N, KW, dt)
    gen = torch.Generator(device="cuda").manual_seed(N * 3 + KW)
    f = grf(torch, N, 50 + N + KW).to(T)
    g = grf(torch, N, 60 + N + KW).to(T)
    df = (1e-2 * torch.randn((N, N), device="cuda", generator=gen)).to(T)
    dg = (1e-2 * torch.randn((N, N), device="cuda", generator=gen)).to(T)
    lam = torch.randn((W, W), device="cuda", generator=gen).to(T)
    dlam = torch.randn((W, W), device="cuda", generator=gen).to(T)
    dh = torch.empty((W, W), device="cuda", dtype=T)
    srk.shrinkageTangentOaS(f, g, df, dg, GX, GY, N, W, e, 1.0, None, dh, plan)
    dlf = torch.empty((N, N), device="cuda", dtype=T)
    dlg = torch.empty_like(dlf)
    srk.shrinkageTangentAdjointOaS(f, g, df, dg, lam, dlam, GX, GY, N, W, e, 1.0, None, dlf, dlg, plan)
    plan.sync()
    lt = ErrorLog("tangent", N, KW, dt)
    lf, lg = ErrorLog("tangent_adjoint_dLam_f", N, KW, dt), ErrorLog("tangent_adjoint_dLam_g", N, KW, dt)
    w = 128
    for (ox, oy) in windows(W, w, 1, N + 2 * KW):
        got, ref = tangent_window(f, g, df, dg, Kx, Ky, e, 1.0, dh, ox, oy, w)
        check(lt, got, ref, r_fwd, t_abs, t_rel)
    for (px, py) in windows(N, w, 1, 5 * N + KW):
        (a, ra), (b, rb) = tangent_adjoint_window(f, g, df, dg, lam, dlam, Kx, Ky, e, 1.0, dlf, dlg, px, py, w,
                                                  "reference")
        check(lf, a, ra, r_adj, t_abs, t_rel)
        check(lg, b, rb, r_adj, t_abs, t_rel)
    for l in (lt, lf, lg):
        l.write()


# ---- derivative protocols at N = 4096, KW = 121 (512-point tiles) -----------------
EPS_SWEEP = (1e-4, 1e-3, 1e-2, 1e-1)


def violations_dev(torch, a, b, tol_abs=1e-5, tol_rel=1e-3):
    """Per-pixel rule of adjoint_tester.h:563-567 on the device (float64)."""
    a, b = a.double(), b.double()
    lim = torch.clamp(tol_rel * torch.maximum(a.abs(), b.abs()), min=tol_abs)
    return int(((a - b).abs() > lim).sum())


def test_tangent_protocols_at_4096(torch_cuda):
    """TangentTester modes A (df), B (dg), C (both) and TangentAdjointTester
    modes D/E/G (dLam_f) and D/F/G (dLam_g), 3 directions each: a case passes
    if some epsilon of the sweep has no pixel outside the rule
    (tangent_tester.h:27-49), every pixel of the 4096^2 / 3976^2 outputs."""
    torch = torch_cuda
    N, KW = 4096, 121
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, 1024, torch)
    n2 = 2 * len(EPS_SWEEP)
    plan = srk.SrkPlan(N, W, e, 1.0, n2, spectra_M=1024)
    assert plan.info()["tile_M"] == 512
    plan.import_spectra(GX, GY)
    plan.set_adj_convention(srk.SRK_ADJ_TRUE)
    f, g = grf(torch, N, 42, 32.0), grf(torch, N, 43, 32.0)
    gen = torch.Generator(device="cuda").manual_seed(123)
    lam = torch.randn((W, W), device="cuda", generator=gen)
    failures = []

    def stack(x, d):
        return torch.stack([x + s * eps * d for eps in EPS_SWEEP for s in (1, -1)])

    def passes(ana, batched):
        return any(violations_dev(torch, ana, (batched[2 * i] - batched[2 * i + 1]) / (2 * eps)) == 0
                   for i, eps in enumerate(EPS_SWEEP))

    for d in range(3):
        dgen = torch.Generator(device="cuda").manual_seed(100 + d)
        df = 1e-2 * torch.randn((N, N), device="cuda", generator=dgen)
        dg = 1e-2 * torch.randn((N, N), device="cuda", generator=dgen)
        dlam = torch.randn((W, W), device="cuda", generator=dgen)
        z, zw = torch.zeros_like(f), torch.zeros_like(lam)
        for mode, (uf, ug) in {"A": (df, z), "B": (z, dg), "C": (df, dg)}.items():
            dh = torch.empty((1, W, W), device="cuda")
            srk.jvp(f[None], g[None], uf[None], ug[None], 1, dh, plan)
            h = torch.empty((n2, W, W), device="cuda")
            srk.forward(stack(f, uf), stack(g, ug), n2, h, plan)
            if not passes(dh[0], h):
                failures.append(("tangent", mode, d))
            del h
        for mode, (uf, ug, ul) in {"D": (z, z, dlam), "E": (z, dg, zw), "F": (df, z, zw),
                                   "G": (df, dg, dlam)}.items():
            dlf = torch.empty((N, N), device="cuda")
            dlg = torch.empty_like(dlf)
            srk.shrinkageTangentAdjointOaS(f, g, uf, ug, lam, ul, None, None, N, W, e, 1.0, None, dlf, dlg, plan)
            af = torch.empty((n2, N, N), device="cuda")
            ag = torch.empty_like(af)
            srk.vjp(stack(lam, ul), stack(f, uf), stack(g, ug), n2, af, ag, plan)
            if mode in "DEG" and not passes(dlf, af):
                failures.append(("tangent_adjoint_dLam_f", mode, d))
            if mode in "DFG" and not passes(dlg, ag):
                failures.append(("tangent_adjoint_dLam_g", mode, d))
            del af, ag
    assert not failures, failures


# ---- one 32768 x 32768 image, KW = 121 ------------------------------------------
@pytest.mark.parametrize("dt", ["f32", "f16"])
def test_large_image_all_ops_windows(torch_cuda, dt):
    torch = torch_cuda
    N, KW = 32768, 121
    T = tdtype(torch, dt)
    _, r_fwd, r_adj, t_abs, t_rel = TOL[dt]
    e, W, Kx, Ky, GX, GY, plan = make(torch, N, KW, dt)
    f = grf(torch, N, 1, 32.0).to(T)
    g = grf(torch, N, 2, 32.0).to(T)
    # default: a few 256 x 256 windows and the corners; SRK_FULL_WINDOWS=1: the
    # full protocol of 64 random 512 x 512 windows per operator (minutes of
    # FP64 oracle time on the host cores)
    full = os.environ.get("SRK_FULL_WINDOWS") == "1"
    w = 512 if full else 256
    wins_w = windows(W, w, 64 if full else 4, 11, corners=not full)
    wins_n = windows(N, w, 64 if full else 2, 12, corners=not full)
    R = torch.empty((W, W), device="cuda", dtype=T)
    ux, uy = torch.empty_like(R), torch.empty_like(R)
    srk.srkForwardOaS(g, f, GX, GY, N, W, e, 1.0, None, R, plan, ux, uy)
    plan.sync()
    log = ErrorLog("forward", N, KW, dt, ell=32)
    for ox, oy in wins_w:
        got, ref = forward_window(f, g, Kx, Ky, e, 1.0, R, ox, oy, w)
        check(log, got, ref, r_fwd, t_abs, t_rel)
    log.write()
    del R
    gen = torch.Generator(device="cuda").manual_seed(77)
    v = torch.randn((W, W), device="cuda", generator=gen).to(T)
    dLdI = torch.empty((N, N), device="cuda", dtype=T)
    dLdE = torch.empty_like(dLdI)
    srk.adjointSRK(v, ux, uy, f, GX, GY, N, W, e, 1.0, None, dLdI, dLdE, plan)
    plan.sync()
    li, le = ErrorLog("adjoint_dLdI", N, KW, dt, ell=32), ErrorLog("adjoint_dLdE", N, KW, dt, ell=32)
    for px, py in wins_n:
        (gi, ri), (ge, re) = adjoint_window(v, ux, uy, f, Kx, Ky, e, 1.0, dLdI, dLdE, px, py, w, "reference")
        check(li, gi, ri, r_adj if dt == "f16" else 1e-5, t_abs, t_rel)
        check(le, ge, re, r_adj, t_abs, t_rel)
    li.write(), le.write()
    del v, ux, uy, dLdI, dLdE
    torch.cuda.empty_cache()
    df = (1e-2 * torch.randn((N, N), device="cuda", generator=gen)).to(T)
    dg = (1e-2 * torch.randn((N, N), device="cuda", generator=gen)).to(T)
    dh = torch.empty((W, W), device="cuda", dtype=T)
    srk.shrinkageTangentOaS(f, g, df, dg, GX, GY, N, W, e, 1.0, None, dh, plan)
    plan.sync()
    lt = ErrorLog("tangent", N, KW, dt, ell=32)
    for ox, oy in wins_w:
        got, ref = tangent_window(f, g, df, dg, Kx, Ky, e, 1.0, dh, ox, oy, w)
        check(lt, got, ref, r_fwd, t_abs, t_rel)
    lt.write()
    del dh
    lam = torch.randn((W, W), device="cuda", generator=gen).to(T)
    dlam = torch.randn((W, W), device="cuda", generator=gen).to(T)
    dlf = torch.empty((N, N), device="cuda", dtype=T)
    dlg = torch.empty_like(dlf)
    srk.shrinkageTangentAdjointOaS(f, g, df, dg, lam, dlam, GX, GY, N, W, e, 1.0, None, dlf, dlg, plan)
    plan.sync()
    lf, lg = (ErrorLog("tangent_adjoint_dLam_f", N, KW, dt, ell=32),
              ErrorLog("tangent_adjoint_dLam_g", N, KW, dt, ell=32))
    for px, py in wins_n:
        (a, ra), (b, rb) = tangent_adjoint_window(f, g, df, dg, lam, dlam, Kx, Ky, e, 1.0, dlf, dlg, px, py, w,
                                                  "reference")
        check(lf, a, ra, r_adj, t_abs, t_rel)
        check(lg, b, rb, r_adj, t_abs, t_rel)
    lf.write(), lg.write()
