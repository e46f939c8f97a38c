"""Large-image scale: one 32768 x 32768 image, KW = 121 (W = 32648), spectra at
the reference's large-image tile size M_TILE = 2048 (adjoint/main_adjoint.cu:33).
Errors are measured against the FP64 oracle on random output windows, as the
full-image oracle is out of reach at this size."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from oracle import oracle as O
from tests.gpu_util import spectra
from tests.helpers import kernel, rel_max_err

pytestmark = pytest.mark.gpu

N, KW = 32768, 121
E_ = (KW - 1) // 2
W = N - 2 * E_


def smooth_field(torch, seed):
    """Smooth deterministic field in [0, 1] (a few random plane waves), built
    on the device column-major as [col, row]."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.arange(N, device="cuda", dtype=torch.float32)
    out = torch.zeros((N, N), device="cuda")
    for _ in range(6):
        k = (torch.rand(2, generator=g, device="cuda") - 0.5) * 0.2
        ph = torch.rand(1, generator=g, device="cuda") * 6.283
        out += torch.cos(k[0] * x[:, None] + k[1] * x[None, :] + ph)
    return (out - out.min()) / (out.max() - out.min())


def crop(t, x0, y0, w):
    return t[x0:x0 + w, y0:y0 + w].double().cpu().numpy()


def test_large_image_forward_and_tangent_windows(torch_cuda):
    torch = torch_cuda
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, 2048, torch)
    plan = srk.SrkPlan(N, W, E_, 1.0, 1, spectra_M=2048)
    f = smooth_field(torch, 1)
    g = smooth_field(torch, 2)
    R = torch.empty((W, W), device="cuda")
    srk.srkForwardOaS(g, f, GX, GY, N, W, E_, 1.0, None, R, plan)
    plan.sync()
    rng = np.random.default_rng(7)
    wins = [(int(rng.integers(0, W - 128)), int(rng.integers(0, W - 128))) for _ in range(6)]
    wins.append((W - 128, W - 128))  # the last tiles
    for ox, oy in wins:
        # outputs [o, o+128) need image [o, o+128+2e)
        ff = crop(f, ox, oy, 128 + 2 * E_)
        gg = crop(g, ox, oy, 128 + 2 * E_)
        ref = O.forward(gg, ff, Kx, Ky, E_, 1.0)
        got = R[ox:ox + 128, oy:oy + 128].double().cpu().numpy()
        assert rel_max_err(got, ref) < 1e-3, (ox, oy)
    del R
    df = (smooth_field(torch, 3) - 0.5) * 0.02
    dg = (smooth_field(torch, 4) - 0.5) * 0.02
    dh = torch.empty((W, W), device="cuda")
    srk.shrinkageTangentOaS(f, g, df, dg, GX, GY, N, W, E_, 1.0, None, dh, plan)
    plan.sync()
    for ox, oy in wins[:4]:
        ff, gg = crop(f, ox, oy, 128 + 2 * E_), crop(g, ox, oy, 128 + 2 * E_)
        dff, dgg = crop(df, ox, oy, 128 + 2 * E_), crop(dg, ox, oy, 128 + 2 * E_)
        ref = O.tangent(ff, gg, dff, dgg, Kx, Ky, E_, 1.0)
        got = dh[ox:ox + 128, oy:oy + 128].double().cpu().numpy()
        assert rel_max_err(got, ref) < 1e-3, (ox, oy)
