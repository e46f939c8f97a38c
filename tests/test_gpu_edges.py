"""Smallest halos: erosion 0 (KW = 1, W = N: the central differences reach
the image border and take the zero-padding rule of srk_grad_x / srk_grad_y,
srk_forward.cuh:429-445) and erosion 1 (KW = 3, the smallest halo of the
staged gradient windows), with asymmetric random kernels so that the two
adjoint conventions differ.  Every operator against the FP64 oracle."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from oracle import oracle as O
from tests.helpers import fields, pixel_violations, rel_max_err
from tests.gpu_util import dev, host, spectra

pytestmark = pytest.mark.gpu


def setup(N, KW, tile, seed, torch):
    e = (KW - 1) // 2
    W = N - 2 * e
    rng = np.random.default_rng(seed)
    Kx, Ky = (0.1 * rng.standard_normal((KW, KW)) for _ in range(2))
    M = 128
    GX, GY = spectra(Kx, Ky, M, torch)
    plan = srk.SrkPlan(N, W, e, 1.0, 1, spectra_M=M, tile_M=tile)
    return e, W, Kx, Ky, GX, GY, plan, rng


@pytest.mark.parametrize("N,KW", [(100, 1), (300, 1), (100, 3), (300, 3)])
def test_forward_and_tangent_small_halo(torch_cuda, N, KW):
    torch = torch_cuda
    e, W, Kx, Ky, GX, GY, plan, rng = setup(N, KW, 128, N + KW, torch)
    f, g = fields(N, 2, 900 + N)
    R = torch.zeros((W, W), device="cuda")
    srk.srkForwardOaS(dev(g, torch), dev(f, torch), GX, GY, N, W, e, 1.0, None, R, plan)
    df, dg = [(1e-2 * rng.standard_normal((N, N))).astype(np.float32) for _ in range(2)]
    dh = torch.zeros((W, W), device="cuda")
    srk.shrinkageTangentOaS(*[dev(a, torch) for a in (f, g, df, dg)], GX, GY, N, W, e, 1.0, None, dh, plan)
    torch.cuda.synchronize()
    oR = O.forward(g, f, Kx, Ky, e, 1.0)
    assert rel_max_err(host(R), oR) < 1e-4
    assert pixel_violations(host(R), oR) == 0
    oh = O.tangent(f, g, df, dg, Kx, Ky, e, 1.0)
    assert rel_max_err(host(dh), oh) < 1e-4


@pytest.mark.parametrize("N,KW", [(100, 1), (300, 1), (100, 3), (300, 3)])
@pytest.mark.parametrize("conv", ["reference", "true"])
def test_adjoint_and_tangent_adjoint_small_halo(torch_cuda, N, KW, conv):
    torch = torch_cuda
    e, W, Kx, Ky, GX, GY, plan, rng = setup(N, KW, 128, 2 * N + KW, torch)
    plan.set_adj_convention(srk.SRK_ADJ_REFERENCE if conv == "reference" else srk.SRK_ADJ_TRUE)
    f, g = fields(N, 2, 950 + N)
    v = rng.standard_normal((W, W)).astype(np.float32)
    _, uxo, uyo = O.forward(g, f, Kx, Ky, e, 1.0, return_u=True)
    ux, uy = (a.astype(np.float32) for a in (uxo, uyo))
    dLdI = torch.zeros((N, N), device="cuda")
    dLdE = torch.zeros((N, N), device="cuda")
    srk.adjointSRK(*[dev(a, torch) for a in (v, ux, uy, f)], GX, GY, N, W, e, 1.0, None, dLdI, dLdE, plan)
    df, dg = [(1e-2 * rng.standard_normal((N, N))).astype(np.float32) for _ in range(2)]
    lam, dlam = [rng.standard_normal((W, W)).astype(np.float32) for _ in range(2)]
    dlf = torch.zeros((N, N), device="cuda")
    dlg = torch.zeros((N, N), device="cuda")
    srk.shrinkageTangentAdjointOaS(*[dev(a, torch) for a in (f, g, df, dg, lam, dlam)], GX, GY, N, W, e, 1.0,
                                   None, dlf, dlg, plan)
    torch.cuda.synchronize()
    assert rel_max_err(host(dLdI), O.adj_wrt_I(v, ux, uy, N, e)) < 1e-5
    oE = O.adj_wrt_E(v, f, Kx, Ky, e, 1.0, conv)
    assert rel_max_err(host(dLdE), oE) < 1e-4
    of, og = O.tangent_adjoint(f, g, df, dg, lam, dlam, Kx, Ky, e, 1.0, conv)
    assert rel_max_err(host(dlf), of) < 1e-4
    assert rel_max_err(host(dlg), og) < 1e-4
