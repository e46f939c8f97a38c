"""The window checks of the large-N GPU tests are exact: for every operator,
the oracle run on a crop reproduces the whole-image oracle at the window,
including windows at the image's first and last pixels.  CPU only (torch CPU
tensors stand in for the device arrays)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.helpers import fields, kernel
from tests.windows import adjoint_window, forward_window, tangent_adjoint_window, tangent_window


N, KW, w = 120, 15, 24
e = (KW - 1) // 2
W = N - 2 * e


@pytest.fixture(scope="module")
def case():
    Kx, Ky = kernel(KW)
    f, g = fields(N, 2, 5)
    rng = np.random.default_rng(3)
    df, dg = (1e-2 * rng.standard_normal((N, N)) for _ in range(2))
    v, ux, uy, lam, dlam = (rng.standard_normal((W, W)) for _ in range(5))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a))
    return Kx, Ky, {k: t(a) for k, a in dict(f=f, g=g, df=df, dg=dg, v=v, ux=ux, uy=uy, lam=lam, dlam=dlam).items()}


OUT_W = [(0, 0), (W - w, W - w), (37, 5), (W - w, 0)]
OUT_N = [(0, 0), (N - w, N - w), (3, 61), (50, N - w), (N // 2, N // 2)]


def test_forward_and_tangent_windows(case):
    Kx, Ky, a = case
    R = O.forward(a["g"].numpy(), a["f"].numpy(), Kx, Ky, e, 1.0)
    dh = O.tangent(*(a[k].numpy() for k in ("f", "g", "df", "dg")), Kx, Ky, e, 1.0)
    for ox, oy in OUT_W:
        got, ref = forward_window(a["f"], a["g"], Kx, Ky, e, 1.0, torch.from_numpy(R), ox, oy, w)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
        got, ref = tangent_window(a["f"], a["g"], a["df"], a["dg"], Kx, Ky, e, 1.0, torch.from_numpy(dh), ox, oy, w)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("conv", ["reference", "true"])
def test_adjoint_type_windows(case, conv):
    Kx, Ky, a = case
    h = {k: a[k].numpy() for k in a}
    dI = O.adj_wrt_I(h["v"], h["ux"], h["uy"], N, e)
    dE = O.adj_wrt_E(h["v"], h["f"], Kx, Ky, e, 1.0, conv)
    tf, tg = O.tangent_adjoint(h["f"], h["g"], h["df"], h["dg"], h["lam"], h["dlam"], Kx, Ky, e, 1.0, conv)
    T = torch.from_numpy
    for px, py in OUT_N:
        for got, ref in adjoint_window(a["v"], a["ux"], a["uy"], a["f"], Kx, Ky, e, 1.0, T(dI), T(dE), px, py, w,
                                       conv):
            assert np.abs(got - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1e-30), (px, py)
        for got, ref in tangent_adjoint_window(a["f"], a["g"], a["df"], a["dg"], a["lam"], a["dlam"], Kx, Ky, e, 1.0,
                                               T(tf), T(tg), px, py, w, conv):
            assert np.abs(got - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1e-30), (px, py)
