"""Synthetic inputs generated on the device (srk_grf, srk_grf_filter,
srk_lns) against the oracle and the reference's own host generators
(GpGenerator, generate_pattern) compiled from its sources."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from oracle import oracle as O
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

need_ref = pytest.mark.skipif(O.ref_host() is None, reason="reference generators not built")


@need_ref
@pytest.mark.parametrize("N,ell,seed", [(64, 8.0, 7), (50, 8.0, 11), (256, 8.0, 3), (128, 32.0, 9)])
def test_grf_filter_matches_reference_generator(torch_cuda, N, ell, seed):
    """The device filter applied to GpGenerator's own noise reproduces its field."""
    torch = torch_cuda
    noise = O.ref_gp_noise(N, seed).astype(np.float32)
    ref = O.ref_gp_field(N, ell, seed).astype(np.float64)
    out = torch.zeros((1, N, N), device="cuda")
    srk.grf_filter(dev(noise[None], torch), out, ell)
    torch.cuda.synchronize()
    assert np.abs(host(out)[0] - ref).max() < 2e-5 * np.abs(ref).max()


def test_grf_noise_and_filter_match_oracle(torch_cuda):
    torch = torch_cuda
    N, ell, seed, B = 200, 8.0, 42, 3
    out = torch.zeros((B, N, N), device="cuda")
    srk.grf(out, ell, seed, minmax=False)
    torch.cuda.synchronize()
    got = host(out)
    for b in range(B):
        ref = O.grf_filter(O.philox_noise(N, seed, b), N, ell)
        assert np.abs(got[b] - ref).max() < 2e-4 * np.abs(ref).max(), b


def test_grf_batch_independent_and_scaled(torch_cuda):
    torch = torch_cuda
    N, ell, seed = 512, 8.0, 1000
    big = torch.zeros((6, N, N), device="cuda")
    srk.grf(big, ell, seed)
    one = torch.zeros((1, N, N), device="cuda")
    srk.grf(one, ell, seed + 4)
    torch.cuda.synchronize()
    assert torch.equal(big[4], one[0])  # image b depends on seed + b only
    h = host(big)
    assert np.allclose(h.min(axis=(1, 2)), 0.0) and np.allclose(h.max(axis=(1, 2)), 1.0)
    # correlation length: c(d) = exp(-d^2 / (2 ell^2)) for the unscaled field
    raw = torch.zeros((4, N, N), device="cuda")
    srk.grf(raw, ell, 7, minmax=False)
    r = host(raw)
    r = (r - r.mean()) / r.std()
    for d in (4, 8, 16):
        emp = np.mean(r[:, d:, :] * r[:, :-d, :])
        assert abs(emp - np.exp(-d * d / (2 * ell * ell))) < 0.06, d


@need_ref
def test_lns_matches_reference_generator(torch_cuda):
    torch = torch_cuda
    N, sigma = 160, 6.0
    kinds = [0, 1, 1, 0]
    out = torch.zeros((len(kinds), N, N), device="cuda")
    srk.lns(out, kinds, sigma)
    torch.cuda.synchronize()
    got = host(out)
    for b, k in enumerate(kinds):
        ref = O.ref_lns(k == 0, N, sigma)
        assert np.abs(got[b] - ref).max() < 2e-6, b


def test_grf_large_image_covariance(torch_cuda):
    """Large periods (the filter spectrum's rounding-level negatives are zeros)."""
    torch = torch_cuda
    N, ell = 4096, 8.0
    raw = torch.zeros((1, N, N), device="cuda")
    srk.grf(raw, ell, 5, minmax=False)
    torch.cuda.synchronize()
    r = host(raw)[0]
    r = (r - r.mean()) / r.std()
    for d in (8, 16):
        emp = np.mean(r[d:, :] * r[:-d, :])
        assert abs(emp - np.exp(-d * d / (2 * ell * ell))) < 0.03, d
