"""The oracle against independent restatements (scipy / numpy FFT) and the
algebraic identities the reference's tests rely on.  CPU only."""
import numpy as np
import pytest
import scipy.signal
import scipy.special

from oracle import oracle as O
from tests.helpers import kernel, fields


@pytest.mark.parametrize("N,KW", [(48, 7), (64, 15), (90, 31)])
def test_conv_matches_scipy(N, KW):
    e = (KW - 1) // 2
    E = fields(N, 1, 5)[0].astype(np.float64)
    Kx, Ky = kernel(KW)
    ux, uy = O.conv_valid(E, Kx, Ky, e, 2.0)
    assert np.allclose(ux, 4.0 * scipy.signal.convolve2d(E, Kx.astype(np.float64), mode="valid"), atol=1e-14)
    assert np.allclose(uy, 4.0 * scipy.signal.convolve2d(E, Ky.astype(np.float64), mode="valid"), atol=1e-14)


def test_kernel_symmetry_and_support():
    for KW in (31, 61, 121):
        Kx, Ky = kernel(KW)
        assert np.array_equal(Kx, -Kx[::-1, :])      # odd in x
        assert np.array_equal(Kx, Kx[:, ::-1])       # even in y
        assert np.array_equal(Ky, Kx.T)
        c = KW // 2
        assert Kx[c, c] == 0.0 and Ky[c, c] == 0.0  # r = 0 set to zero


def test_reference_k1_polynomials_accuracy():
    """The float A&S K1 in the restated make_kernel is ~1e-6 relative to K1."""
    KW = 61
    e = 30
    Kx, _ = kernel(KW)
    sigma = e / 3.0
    x = (np.arange(KW) - KW // 2).astype(np.float64)
    X, Y = np.meshgrid(x, x, indexing="ij")
    r = np.hypot(X, Y)
    m = (r > 0) & (r <= 3 * sigma)
    t = r / (3 * sigma)
    w = 0.42 + 0.5 * np.cos(np.pi * t) + 0.08 * np.cos(2 * np.pi * t)
    exact = np.where(m, (1 / sigma) / (2 * np.pi) * scipy.special.k1(r / sigma) * w * X / np.where(m, r, 1), 0)
    assert np.abs(Kx - exact).max() <= 2e-6 * np.abs(exact).max()


@pytest.mark.parametrize("M", [32, 64])
def test_kernel_freq_matches_numpy(M):
    KW = 15
    Kx, _ = kernel(KW)
    c = KW // 2
    pad = np.zeros((M, M))
    for i in range(KW):
        for j in range(KW):
            pad[(i - c) % M, (j - c) % M] = Kx[i, j]
    ref = np.fft.rfft2(pad)  # [kx, ky<=M/2]
    got = O.kernel_freq(Kx, M)
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


def test_adjoint_conventions_and_dot_products():
    N, KW = 70, 21
    e = 10
    W = N - 2 * e
    E, I = [a.astype(np.float64) for a in fields(N, 2, 11)]
    v = np.random.default_rng(3).standard_normal((W, W))
    Kx, Ky = kernel(KW)
    R, ux, uy = O.forward(E, I, Kx, Ky, e, 1.0, return_u=True)
    # <A_I(E), v> = <E, A_I^*(v)> with the exact adjoint
    at = O.adj_wrt_E(v, I, Kx, Ky, e, 1.0, "true")
    assert abs((R * v).sum() - (E * at).sum()) < 1e-12 * np.abs(R * v).sum()
    # R is linear in I too: <R, v> = <I, adjWrtI(v)>
    aI = O.adj_wrt_I(v, ux, uy, N, e)
    assert abs((R * v).sum() - (I * aI).sum()) < 1e-12 * np.abs(R * v).sum()
    # the reference FFT path convolves (not correlates): negative for the odd tensor
    ar = O.adj_wrt_E(v, I, Kx, Ky, e, 1.0, "reference")
    assert np.abs(ar + at).max() < 1e-15 * max(1.0, np.abs(at).max()) * 10
    # ... and identical for an even kernel (the reference's Gaussian adjoint test)
    G = np.exp(-((np.arange(KW) - KW // 2) ** 2)[:, None] / 20.0 - ((np.arange(KW) - KW // 2) ** 2)[None, :] / 20.0)
    assert np.allclose(O.adj_wrt_E(v, I, G, G, e, 1.0, "true"), O.adj_wrt_E(v, I, G, G, e, 1.0, "reference"))


def test_tangent_is_derivative_of_forward():
    N, KW = 60, 15
    e = 7
    f, g, df, dg = [a.astype(np.float64) for a in fields(N, 4, 21)]
    Kx, Ky = kernel(KW)
    dh = O.tangent(f, g, df, dg, Kx, Ky, e, 1.0)
    eps = 1e-3
    num = (O.forward(g + eps * dg, f + eps * df, Kx, Ky, e, 1.0) -
           O.forward(g - eps * dg, f - eps * df, Kx, Ky, e, 1.0)) / (2 * eps)
    assert np.abs(dh - num).max() < 1e-9 * max(1.0, np.abs(dh).max())


@pytest.mark.parametrize("conv", ["true", "reference"])
def test_tangent_adjoint_is_derivative_of_adjoint(conv):
    N, KW = 50, 11
    e = 5
    W = N - 2 * e
    f, g, df, dg = [a.astype(np.float64) for a in fields(N, 4, 31)]
    rng = np.random.default_rng(9)
    lam, dlam = rng.standard_normal((W, W)), rng.standard_normal((W, W))
    Kx, Ky = kernel(KW)

    def adj(f_, g_, l_):
        _, ux, uy = O.forward(g_, f_, Kx, Ky, e, 1.0, return_u=True)
        return O.adj_wrt_I(l_, ux, uy, N, e), O.adj_wrt_E(l_, f_, Kx, Ky, e, 1.0, conv)

    dlf, dlg = O.tangent_adjoint(f, g, df, dg, lam, dlam, Kx, Ky, e, 1.0, conv)
    eps = 1e-3
    p = adj(f + eps * df, g + eps * dg, lam + eps * dlam)
    m = adj(f - eps * df, g - eps * dg, lam - eps * dlam)
    assert np.abs(dlf - (p[0] - m[0]) / (2 * eps)).max() < 1e-9 * max(1.0, np.abs(dlf).max())
    assert np.abs(dlg - (p[1] - m[1]) / (2 * eps)).max() < 1e-9 * max(1.0, np.abs(dlg).max())


def test_windowed_forward_matches_full():
    N, KW = 80, 15
    e = 7
    E, I = [a.astype(np.float64) for a in fields(N, 2, 41)]
    Kx, Ky = kernel(KW)
    full = O.forward(E, I, Kx, Ky, e, 1.0)
    win = O.forward(E, I, Kx, Ky, e, 1.0, window=(5, 9, 20, 13))
    assert np.array_equal(win, full[5:25, 9:22])


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors of the published algorithm
    (Salmon et al., SC 2011; Random123 test vectors)."""
    m = 0xFFFFFFFF
    cases = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
             ((m, m, m, m), (m, m), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
             ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
              (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for c, k, want in cases:
        got = O.philox4x32_10(*c, *k)
        assert tuple(int(v) for v in got) == want


def test_philox_noise_is_standard_normal():
    z = O.philox_noise(256, 1234)
    assert abs(z.mean()) < 0.01 and abs(z.var() - 1.0) < 0.01
    # neighbouring pixels uncorrelated
    assert abs(np.mean(z[:, 1:] * z[:, :-1])) < 0.01
    assert abs(np.mean(z[1:, :] * z[:-1, :])) < 0.01


@pytest.mark.skipif(O.ref_host() is None, reason="reference generators not built")
@pytest.mark.parametrize("N,ell,seed", [(64, 8.0, 7), (50, 8.0, 11), (96, 3.0, 5)])
def test_grf_filter_reproduces_reference_generator(N, ell, seed):
    """Given GpGenerator's own noise, the oracle's filter reproduces its field
    (gp_generator.h:119-147) to the float rounding of its output."""
    ref = O.ref_gp_field(N, ell, seed).astype(np.float64)
    ours = O.grf_filter(O.ref_gp_noise(N, seed), N, ell)
    assert np.abs(ours - ref).max() < 1e-6 * np.abs(ref).max()


def test_reference_checker_form_matches_oracle():
    """The single-thread float restatement of cpu_conv_valid + combine (the
    timing row of the reference arm) agrees with the FP64 oracle."""
    N, KW = 64, 15
    e = (KW - 1) // 2
    Kx, Ky = O.make_kernel_sigma(KW, e / 3.0)
    f = O.grf(N, 8.0, 77)
    R64 = O.forward(f, f, Kx, Ky, e, 1.0)
    R32 = O.forward_f32_cols(f, f, Kx, Ky, e, 1.0, 3, 9)
    ref = R64[3:12]
    assert np.abs(R32 - ref).max() < 1e-4 * np.abs(R64).max()
