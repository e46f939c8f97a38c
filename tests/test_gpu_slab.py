"""One image split by column slabs (srk_forward_oas_slab, srk_tangent_slab,
srk_adjoint_slab, srk_tangent_adjoint_slab), the per-GPU step of the
multi-GPU split of a single large image.  The slabs of every rank are computed here one after another on one
GPU from buffers that hold exactly the halo'd columns the C declarations
name, between guard columns of NaN: a read outside the halo turns an output
NaN.  The stitched slabs must match the whole-image call to rounding (work
tiles pair differently) and the FP64 oracle."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from oracle import oracle as O
from shrinkage_full_tests_b200.shard import slab_bounds, ta_wrange
from tests.helpers import fields, kernel, pixel_violations, rel_max_err
from tests.gpu_util import dev, host, spectra

pytestmark = pytest.mark.gpu


def guarded(full, lo, hi, c0, guard, torch):
    """Columns [lo, hi) of `full` ([cols, rows] CUDA tensor) between `guard`
    NaN columns on each side; returns the view whose row 0 is column c0."""
    rows = full.shape[1]
    buf = torch.full((hi - lo + 2 * guard, rows), float("nan"), device="cuda")
    buf[guard:guard + hi - lo] = full[lo:hi]
    return buf[guard + c0 - lo:]


def setup(N, KW, tile, torch):
    e = (KW - 1) // 2
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, 1024, torch)
    plan = srk.SrkPlan(N, N - 2 * e, e, 1.0, 1, spectra_M=1024, tile_M=tile)
    plan.set_adj_convention(srk.SRK_ADJ_TRUE)
    return e, Kx, Ky, GX, GY, plan


@pytest.mark.parametrize("N,KW,tile,world", [(300, 31, 128, 3), (4096, 61, 512, 4)])
def test_slabs_forward_tangent_adjoint(torch_cuda, N, KW, tile, world):
    torch = torch_cuda
    e, Kx, Ky, GX, GY, plan = setup(N, KW, tile, torch)
    W = N - 2 * e
    S = plan.info()["tile_stride"]
    gen = torch.Generator(device="cuda").manual_seed(11)
    f, g, df, dg = (torch.rand((N, N), device="cuda", generator=gen) for _ in range(4))
    v, ux, uy = (torch.randn((W, W), device="cuda", generator=gen) for _ in range(3))
    # whole-image calls
    R = torch.zeros((W, W), device="cuda")
    srk.srkForwardOaS(g, f, GX, GY, N, W, e, 1.0, None, R, plan)
    dh = torch.zeros((W, W), device="cuda")
    srk.shrinkageTangentOaS(f, g, df, dg, GX, GY, N, W, e, 1.0, None, dh, plan)
    dI = torch.zeros((N, N), device="cuda")
    dE = torch.zeros((N, N), device="cuda")
    srk.adjointSRK(v, ux, uy, f, GX, GY, N, W, e, 1.0, None, dI, dE, plan)
    lam, dlam = (torch.randn((W, W), device="cuda", generator=gen) for _ in range(2))
    tf = torch.zeros((N, N), device="cuda")
    tg = torch.zeros((N, N), device="cuda")
    srk.shrinkageTangentAdjointOaS(f, g, df, dg, lam, dlam, GX, GY, N, W, e, 1.0, None, tf, tg, plan)
    # slabs
    sR, sdh, sdI, sdE, stf, stg = (torch.zeros_like(t) for t in (R, dh, dI, dE, tf, tg))
    guard = tile
    for lo, hi in slab_bounds(N, e, S, world):
        if lo == hi:
            continue
        c1 = min(hi, W)
        ins = [guarded(t, lo, min(c1 + 2 * e, N), lo, guard, torch) for t in (f, g, df, dg)]
        srk.srkForwardOaSSlab(ins[1], ins[0], GX, GY, N, e, 1.0, lo, c1, None, sR[lo:], plan)
        srk.shrinkageTangentOaSSlab(*ins, GX, GY, N, e, 1.0, lo, c1, None, sdh[lo:], plan)
        vs = [guarded(t, max(lo - 2 * e, 0), min(hi, W), lo, guard, torch) for t in (v, ux, uy)]
        fs = guarded(f, max(lo - e - 1, 0), min(hi + e + 1, N), lo, guard, torch)
        srk.adjointSRKSlab(*vs, fs, GX, GY, N, e, 1.0, lo, hi, None, sdI[lo:], sdE[lo:], plan)
        # tangent-adjoint: the halos of srk_tangent_adjoint_slab
        r0, rE = ta_wrange(lo, hi, N, e, S)
        fd = [guarded(t, max(lo - e - 1, 0), min(hi + e + 1, N), lo, guard, torch) for t in (f, df)]
        gd = [guarded(t, r0, max(min(rE + 2 * e, N), lo + 1), lo, guard, torch) for t in (g, dg)]
        ld = [guarded(t, min(max(lo - 2 * e, 0), r0), max(min(hi, W), rE, lo + 1), lo, guard, torch)
              for t in (lam, dlam)]
        srk.shrinkageTangentAdjointOaSSlab(fd[0], gd[0], fd[1], gd[1], ld[0], ld[1], GX, GY, N, e, 1.0, lo, hi, None,
                                           stf[lo:], stg[lo:], plan)
    torch.cuda.synchronize()
    for got, ref in ((sR, R), (sdh, dh), (sdE, dE), (stf, tf), (stg, tg)):
        a, b = host(got), host(ref)
        assert np.isfinite(a).all()
        assert pixel_violations(a, b, tol_abs=1e-6, tol_rel=1e-4) == 0
    assert torch.equal(sdI, dI)  # the stencil does not depend on the tiling
    if N <= 512:
        fh, gh = host(f), host(g)
        assert rel_max_err(host(sR), O.forward(gh, fh, Kx, Ky, e, 1.0)) < 1e-3
        oE = O.adj_wrt_E(host(v), fh, Kx, Ky, e, 1.0, "true")
        assert rel_max_err(host(sdE), oE) < 1e-4


def test_slab_rejects_partial_tiles(torch_cuda):
    torch = torch_cuda
    N, KW, tile = 300, 31, 128
    e, Kx, Ky, GX, GY, plan = setup(N, KW, tile, torch)
    W = N - 2 * e
    S = plan.info()["tile_stride"]
    x = torch.zeros((N, N), device="cuda")
    for c0, c1 in ((0, S + 1), (0, W + 1), (5, 5), (-1, S - 1)):
        with pytest.raises(srk.SrkError) as ei:
            srk.srkForwardOaSSlab(x, x, GX, GY, N, e, 1.0, c0, c1, None, x, plan)
        assert ei.value.status == srk.SRK_ERR_INVALID_ARG
    with pytest.raises(srk.SrkError) as ei:
        srk.adjointSRKSlab(x, x, x, x, GX, GY, N, e, 1.0, 0, S + 3, None, x, x, plan)
    assert ei.value.status == srk.SRK_ERR_INVALID_ARG
