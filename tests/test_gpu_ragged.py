"""Ragged batches: images of different N in one call (one launch sequence).

Each image of a ragged call must agree with the FP64 oracle and with the
same operator called on that image alone.  Work tiles pair tiles of
different images, and a packed complex transform rounds differently with a
different partner, so the comparison with the single-image calls is to
rounding (per-pixel criterion of adjoint_tester.h:563-567), not bitwise."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from oracle import oracle as O
from tests.helpers import fields, kernel, pixel_violations, rel_max_err
from tests.gpu_util import dev, host, spectra
from tests.windows import adjoint_window, windows

pytestmark = pytest.mark.gpu

SPECTRA_M = 1024  # the reference's OaS tile size for N < 8k (adjoint/main_adjoint.cu:33)


def concat(arrs, torch):
    return dev(np.concatenate([np.ascontiguousarray(a, np.float32).ravel() for a in arrs]), torch)


def split(t, sizes):
    h = host(t)
    out, o = [], 0
    for n in sizes:
        out.append(h[o:o + n * n].reshape(n, n))
        o += n * n
    return out


def setup(KW, Ns, tile, torch):
    e = (KW - 1) // 2
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, SPECTRA_M, torch)
    Nmax = max(Ns)
    plan = srk.SrkPlan(Nmax, Nmax - 2 * e, e, 1.0, len(Ns), spectra_M=SPECTRA_M, tile_M=tile)
    return e, Kx, Ky, GX, GY, plan


def single_plan(N, e, tile):
    return srk.SrkPlan(N, N - 2 * e, e, 1.0, 1, spectra_M=SPECTRA_M, tile_M=tile)


def test_ragged_forward(torch_cuda):
    torch = torch_cuda
    KW, Ns, tile = 31, [300, 257, 128, 200, 31], 128
    e, Kx, Ky, GX, GY, plan = setup(KW, Ns, tile, torch)
    Ws = [n - 2 * e for n in Ns]
    imgs = [fields(n, 2, 40 + n) for n in Ns]  # (f, g) per image
    f = concat([a for a, _ in imgs], torch)
    g = concat([b for _, b in imgs], torch)
    R = torch.zeros(sum(w * w for w in Ws), device="cuda")
    srk.srkForwardOaSRagged(g, f, GX, GY, Ns, e, 1.0, None, R, plan)
    plan.sync()
    got = split(R, Ws)
    for b, n in enumerate(Ns):
        fb, gb = imgs[b]
        ref = O.forward(gb, fb, Kx, Ky, e, 1.0)
        assert rel_max_err(got[b], ref) < 1e-3, b
        one = torch.zeros((Ws[b], Ws[b]), device="cuda")
        srk.srkForwardOaS(dev(gb, torch), dev(fb, torch), GX, GY, n, Ws[b], e, 1.0, None, one, single_plan(n, e, tile))
        torch.cuda.synchronize()
        assert pixel_violations(got[b], host(one), tol_abs=1e-6, tol_rel=1e-5) == 0, b


@pytest.mark.parametrize("conv", ["reference", "true"])
def test_ragged_adjoint(torch_cuda, conv):
    torch = torch_cuda
    KW, Ns, tile = 31, [200, 300, 129], 256
    e, Kx, Ky, GX, GY, plan = setup(KW, Ns, tile, torch)
    plan.set_adj_convention(srk.SRK_ADJ_REFERENCE if conv == "reference" else srk.SRK_ADJ_TRUE)
    Ws = [n - 2 * e for n in Ns]
    rng = np.random.default_rng(5)
    per = []
    for n, w in zip(Ns, Ws):
        f, g = fields(n, 2, 70 + n)
        _, ux, uy = O.forward(g, f, Kx, Ky, e, 1.0, return_u=True)
        v = rng.standard_normal((w, w)).astype(np.float32)
        per.append((f, v, ux.astype(np.float32), uy.astype(np.float32)))
    f = concat([p[0] for p in per], torch)
    v = concat([p[1] for p in per], torch)
    ux = concat([p[2] for p in per], torch)
    uy = concat([p[3] for p in per], torch)
    nn = sum(n * n for n in Ns)
    dLdI = torch.zeros(nn, device="cuda")
    dLdE = torch.zeros(nn, device="cuda")
    srk.adjointSRKRagged(v, ux, uy, f, GX, GY, Ns, e, 1.0, None, dLdI, dLdE, plan)
    plan.sync()
    gI, gE = split(dLdI, Ns), split(dLdE, Ns)
    for b, n in enumerate(Ns):
        fb, vb, uxb, uyb = per[b]
        oI = O.adj_wrt_I(vb, uxb, uyb, n, e)
        oE = O.adj_wrt_E(vb, fb, Kx, Ky, e, 1.0, conv)
        assert rel_max_err(gI[b], oI) < 1e-5, b
        assert rel_max_err(gE[b], oE) < 1e-4, b
        assert pixel_violations(gE[b], oE) == 0, b


def test_ragged_tangent_and_tangent_adjoint(torch_cuda):
    torch = torch_cuda
    KW, Ns, tile = 31, [160, 230, 96], 128
    e, Kx, Ky, GX, GY, plan = setup(KW, Ns, tile, torch)
    Ws = [n - 2 * e for n in Ns]
    rng = np.random.default_rng(9)
    per = []
    for n, w in zip(Ns, Ws):
        f, g = fields(n, 2, 90 + n)
        df, dg = [(1e-2 * rng.standard_normal((n, n))).astype(np.float32) for _ in range(2)]
        lam, dlam = [rng.standard_normal((w, w)).astype(np.float32) for _ in range(2)]
        per.append((f, g, df, dg, lam, dlam))
    T = [concat([p[k] for p in per], torch) for k in range(6)]
    ww = sum(w * w for w in Ws)
    nn = sum(n * n for n in Ns)
    dh = torch.zeros(ww, device="cuda")
    srk.shrinkageTangentOaSRagged(T[0], T[1], T[2], T[3], GX, GY, Ns, e, 1.0, None, dh, plan)
    dlf = torch.zeros(nn, device="cuda")
    dlg = torch.zeros(nn, device="cuda")
    srk.shrinkageTangentAdjointOaSRagged(T[0], T[1], T[2], T[3], T[4], T[5], GX, GY, Ns, e, 1.0, None, dlf, dlg,
                                         plan)
    plan.sync()
    gh, gf, gg = split(dh, Ws), split(dlf, Ns), split(dlg, Ns)
    for b, n in enumerate(Ns):
        f, g, df, dg, lam, dlam = per[b]
        oh = O.tangent(f, g, df, dg, Kx, Ky, e, 1.0)
        assert rel_max_err(gh[b], oh) < 1e-3, b
        of, og = O.tangent_adjoint(f, g, df, dg, lam, dlam, Kx, Ky, e, 1.0)
        assert rel_max_err(gf[b], of) < 1e-4, b
        assert rel_max_err(gg[b], og) < 1e-4, b


def test_ragged_adjoint_sixteen_large_images(torch_cuda):
    """Sixteen images with N drawn from {1k, 2k, 4k, 8k}, KW = 61, one ragged
    adjoint call, against the single-image calls and, for every distinct
    size, the FP64 oracle on two 128 x 128 output windows (one at the image's
    last pixels)."""
    torch = torch_cuda
    KW, tile = 61, 512
    Ns = [int(n) for n in np.random.default_rng(2026).choice([1024, 2048, 4096, 8192], 16)]
    e, Kx, Ky, GX, GY, plan = setup(KW, Ns, tile, torch)
    Ws = [n - 2 * e for n in Ns]
    gen = torch.Generator(device="cuda").manual_seed(3)
    nn, ww = sum(n * n for n in Ns), sum(w * w for w in Ws)
    f = torch.rand(nn, device="cuda", generator=gen)
    v = torch.randn(ww, device="cuda", generator=gen)
    ux = torch.randn(ww, device="cuda", generator=gen) * 0.1
    uy = torch.randn(ww, device="cuda", generator=gen) * 0.1
    dLdI = torch.zeros(nn, device="cuda")
    dLdE = torch.zeros(nn, device="cuda")
    srk.adjointSRKRagged(v, ux, uy, f, GX, GY, Ns, e, 1.0, None, dLdI, dLdE, plan)
    plan.sync()
    on = ow = 0
    checked = set()
    for b, n in enumerate(Ns):
        w = Ws[b]
        if n not in checked:  # one single-image call per distinct size
            checked.add(n)
            p1 = single_plan(n, e, tile)
            sI = torch.zeros((n, n), device="cuda")
            sE = torch.zeros((n, n), device="cuda")
            srk.adjointSRK(v[ow:ow + w * w], ux[ow:ow + w * w], uy[ow:ow + w * w], f[on:on + n * n], GX, GY, n, w, e,
                           1.0, None, sI, sE, p1)
            p1.sync()
            assert torch.equal(dLdI[on:on + n * n].view(n, n), sI), b
            a, r = host(dLdE[on:on + n * n]).reshape(n, n), host(sE)
            assert pixel_violations(a, r, tol_abs=1e-6, tol_rel=1e-4) == 0, b
            del p1, sI, sE
            img = lambda t, o, m: t[o:o + m * m].view(m, m)
            for px, py in windows(n, 128, 1, n, corners=False) + [(n - 128, n - 128)]:
                (gi, ri), (ge, re) = adjoint_window(img(v, ow, w), img(ux, ow, w), img(uy, ow, w), img(f, on, n),
                                                    Kx, Ky, e, 1.0, img(dLdI, on, n), img(dLdE, on, n), px, py,
                                                    128, "reference")
                assert rel_max_err(gi, ri) < 1e-5, (b, px, py)
                assert rel_max_err(ge, re) < 1e-4, (b, px, py)
                assert pixel_violations(ge, re) == 0, (b, px, py)
        on += n * n
        ow += w * w


def test_ragged_rejects_oversize_image(torch_cuda):
    torch = torch_cuda
    e, Kx, Ky, GX, GY, plan = setup(31, [128, 200], 128, torch)
    R = torch.zeros(10, device="cuda")
    E = torch.zeros(10, device="cuda")
    with pytest.raises(srk.SrkError) as ei:
        srk.srkForwardOaSRagged(E, E, GX, GY, [128, 256], e, 1.0, None, R, plan)
    assert ei.value.status == srk.SRK_ERR_INVALID_ARG
    with pytest.raises(srk.SrkError) as ei:
        srk.srkForwardOaSRagged(E, E, GX, GY, [20], e, 1.0, None, R, plan)
    assert ei.value.status == srk.SRK_ERR_INVALID_ARG
