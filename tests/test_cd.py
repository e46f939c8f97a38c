"""CD measurement: the oracle restatement against the reference's own pattern
generator (CPU), and the fused GPU kernel against the oracle and the
reference's MeasureCD_Batched built from its sources (GPU)."""
import numpy as np
import pytest

from oracle import oracle as O


def test_oracle_lns_matches_reference_generator():
    if O.ref_host() is None:
        pytest.skip("reference host generators not built")
    for vertical in (True, False):
        ours = O.lns(vertical, 96, 6.0)
        ref = O.ref_lns(vertical, 96, 6.0)
        assert np.abs(ours - ref).max() < 2e-6


def test_oracle_cd_of_analytic_pulse():
    # a single Gaussian pulse minus 0.5 crosses zero at +-sigma*sqrt(2 ln 2)
    n, sigma = 200, 10.0
    x = np.arange(n)
    sig = np.exp(-((x - (n - 1) / 2) ** 2) / (2 * sigma ** 2)) - 0.5
    left, right, cd = O.measure_cd(sig[None, :])
    fwhm = 2 * sigma * np.sqrt(2 * np.log(2))
    assert abs(cd[0] - fwhm) < 1e-3


@pytest.mark.gpu
def test_gpu_cd_matches_oracle_and_reference(torch_cuda):
    torch = torch_cuda
    import shrinkage_full_tests_b200 as srk
    from tests.gpu_util import ref_gpu
    rng = np.random.default_rng(0)
    B, n = 24, 300
    sigs = np.stack([O.lns(True, n, s, 0.0)[:, 0] + 0.01 * rng.standard_normal(n).astype(np.float32)
                     for s in np.linspace(6.0, 12.0, B)]).astype(np.float32)
    d = torch.from_numpy(sigs).cuda()
    l, r, cd = [t.cpu().numpy() for t in srk.measure_cd(d)]
    ol, orr, ocd = O.measure_cd(sigs)
    assert np.abs(cd - ocd).max() < 1e-4
    assert np.abs(l - ol).max() < 1e-4
    L = ref_gpu()
    if L is not None:
        import ctypes
        fp = ctypes.POINTER(ctypes.c_float)
        rl, rr, rc = [np.zeros(B, np.float32) for _ in range(3)]
        assert L.ref_measure_cd(d.data_ptr(), B, n, 16, 8, torch.cuda.current_stream().cuda_stream,
                                rl.ctypes.data_as(fp), rr.ctypes.data_as(fp), rc.ctypes.data_as(fp)) == 0
        assert np.abs(cd - rc).max() < 1e-3   # the reference's pass bar is 0.01 px


@pytest.mark.gpu
def test_gpu_cd_after_training_forward(torch_cuda):
    """CD of E + c*R on line/space patterns: fused GPU pipeline vs the oracle
    forward + oracle CD (max CD diff < 0.01 px, README.md:36)."""
    torch = torch_cuda
    import shrinkage_full_tests_b200 as srk
    from tests.helpers import kernel
    from tests.gpu_util import spectra
    N, KW, B = 256, 61, 6
    e = 30
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, N, torch)
    for axis, vertical in ((0, True), (1, False)):
        imgs = [O.lns(vertical, N, s) for s in np.linspace(5.6, 11.2, B)]
        E = torch.from_numpy(np.stack(imgs)).cuda()
        R = torch.zeros((B, W, W), device="cuda")
        plan = srk.SrkPlan(N, W, e, 1.0, B)
        srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R, plan)
        _, _, cd = srk.cd_after_shrinkage(E, R, N, W, e, 1.0, axis)
        cd = cd.cpu().numpy()
        sig = []
        for b in range(B):
            Ro = O.forward(imgs[b], imgs[b], Kx, Ky, e, 1.0)
            Ec = imgs[b].astype(np.float64)[e:e + W, e:e + W]
            s = Ec + 1.0 * Ro
            sig.append(s[:, W // 2] if axis == 0 else s[W // 2, :])
        _, _, ocd = O.measure_cd(np.stack(sig))
        assert np.all(np.isfinite(cd))
        assert np.abs(cd - ocd).max() < 0.01


@pytest.mark.gpu
def test_gpu_cd_strip_matches_full_pipeline(torch_cuda):
    """CD from R on the measured line only (direct convolution) against the
    full operator + CD, and against the FP64 oracle."""
    torch = torch_cuda
    import shrinkage_full_tests_b200 as srk
    from tests.helpers import kernel
    from tests.gpu_util import dev, spectra
    for N, KW, B in ((256, 61, 6), (512, 121, 4)):
        e = (KW - 1) // 2
        W = N - 2 * e
        Kx, Ky = kernel(KW, "baseline", 4.0)
        GX, GY = spectra(Kx, Ky, N, torch)
        for axis, vertical in ((0, True), (1, False)):
            imgs = [O.lns(vertical, N, s) for s in np.linspace(5.6, 11.2, B)]
            E = torch.from_numpy(np.stack(imgs)).cuda()
            R = torch.zeros((B, W, W), device="cuda")
            plan = srk.SrkPlan(N, W, e, 4.0, B)
            srk.srkTrainingForward(E, E, GX, GY, N, W, e, 4.0, B, None, R, plan)
            _, _, cd_full = srk.cd_after_shrinkage(E, R, N, W, e, 0.3, axis)
            _, _, cd_strip = srk.cd_strip(E, E, dev(Kx, torch), dev(Ky, torch), N, W, e, 4.0, 0.3, axis)
            cd_full, cd_strip = cd_full.cpu().numpy(), cd_strip.cpu().numpy()
            assert np.all(np.isfinite(cd_strip))
            assert np.abs(cd_strip - cd_full).max() < 1e-3, (N, KW, axis)
            sig = []
            for b in range(B):
                Ro = O.forward(imgs[b], imgs[b], Kx, Ky, e, 4.0)
                s = imgs[b].astype(np.float64)[e:e + W, e:e + W] + 0.3 * Ro
                sig.append(s[:, W // 2] if axis == 0 else s[W // 2, :])
            _, _, ocd = O.measure_cd(np.stack(sig))
            assert np.abs(cd_strip - ocd).max() < 0.01
