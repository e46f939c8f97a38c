"""Parity of the CUDA path (through the C ABI) with the FP64 oracle and with
the reference's own srkTrainingForward built from its sources.  Tolerances are
the reference's: forward max|d|/max|ref| < 1e-3 (adjoint/main_adjoint.cu:359-360),
per-pixel |d| <= max(1e-5, 1e-3 max(|a|,|b|)) for derivatives
(adjoint_tester.h:563-567), training vs cuDNN 5e-3 (main_forward_training.cu:593-599)."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from oracle import oracle as O
from tests.helpers import fields, kernel, pixel_violations, rel_max_err
from tests.gpu_util import dev, host, ref_gpu, spectra

pytestmark = pytest.mark.gpu

FWD_CASES = [
    # N, KW, tile (0 = auto), spectra size, kernel form
    (64, 15, 128, 64, "sigma"),
    (256, 31, 0, 256, "baseline"),
    (300, 31, 128, 1024, "sigma"),      # several tiles; spectra at the OaS M_TILE
    (512, 121, 0, 512, "baseline"),
    (700, 61, 256, 1024, "sigma"),
    (257, 21, 256, 258, "sigma"),       # odd N, ragged last tile
]


@pytest.mark.parametrize("N,KW,tile,Ms,form", FWD_CASES)
def test_forward_oas_matches_oracle(torch_cuda, N, KW, tile, Ms, form):
    torch = torch_cuda
    e = (KW - 1) // 2
    W = N - 2 * e
    dx = 4.0 if form == "baseline" else 1.0
    f, g = fields(N, 2, 100 + N)
    Kx, Ky = kernel(KW, form, dx)
    GX, GY = spectra(Kx, Ky, Ms, torch)
    plan = srk.SrkPlan(N, W, e, dx, 1, spectra_M=Ms, tile_M=tile)
    R = torch.zeros((W, W), device="cuda")
    ux = torch.zeros_like(R)
    uy = torch.zeros_like(R)
    srk.srkForwardOaS(dev(g, torch), dev(f, torch), GX, GY, N, W, e, dx, None, R, plan, ux, uy)
    torch.cuda.synchronize()
    Ro, uxo, uyo = O.forward(g, f, Kx, Ky, e, dx, return_u=True)
    assert rel_max_err(host(ux), uxo) < 1e-4
    assert rel_max_err(host(uy), uyo) < 1e-4
    assert rel_max_err(host(R), Ro) < 1e-3
    assert pixel_violations(host(R), Ro) == 0


@pytest.mark.parametrize("N,KW,B", [(256, 31, 5), (256, 121, 4), (512, 61, 3), (192, 61, 2)])
def test_training_forward_matches_oracle_and_reference(torch_cuda, N, KW, B):
    torch = torch_cuda
    e = (KW - 1) // 2
    W = N - 2 * e
    imgs = fields(N, B, 7 * N + KW)
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, N, torch)
    E = dev(np.stack(imgs), torch)
    plan = srk.SrkPlan(N, W, e, 1.0, B)
    R = torch.zeros((B, W, W), device="cuda")
    srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R, plan)
    torch.cuda.synchronize()
    Rh = host(R)
    for b in range(B):
        Ro = O.forward(imgs[b], imgs[b], Kx, Ky, e, 1.0)
        assert rel_max_err(Rh[b], Ro) < 1e-3
        assert pixel_violations(Rh[b], Ro) == 0
    L = ref_gpu()
    if L is not None:
        s = torch.cuda.current_stream().cuda_stream
        ws = L.ref_train_ws_create(N, B, s)
        Rr = torch.zeros_like(R)
        assert L.ref_train_forward(E.data_ptr(), E.data_ptr(), GX.data_ptr(), GY.data_ptr(), N, W, e, 1.0, B, s,
                                   Rr.data_ptr(), ws) == 0
        torch.cuda.synchronize()
        L.ref_train_ws_destroy(ws, s)
        Rrh = host(Rr)
        for b in range(B):
            assert rel_max_err(Rh[b], Rrh[b]) < 1e-3
            assert np.abs(Rh[b] - Rrh[b]).max() < 5e-3


@pytest.mark.parametrize("N,KW,tile", [(96, 15, 128), (300, 31, 128), (512, 61, 0)])
@pytest.mark.parametrize("conv", ["reference", "true"])
def test_adjoint_srk_matches_oracle(torch_cuda, N, KW, tile, conv):
    torch = torch_cuda
    e = (KW - 1) // 2
    W = N - 2 * e
    f, g = fields(N, 2, 300 + N)
    v = np.random.default_rng(N).standard_normal((W, W)).astype(np.float32)
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, N + (N & 1), torch)
    plan = srk.SrkPlan(N, W, e, 1.0, 1, spectra_M=N + (N & 1), tile_M=tile)
    plan.set_adj_convention(srk.SRK_ADJ_REFERENCE if conv == "reference" else srk.SRK_ADJ_TRUE)
    _, uxo, uyo = O.forward(g, f, Kx, Ky, e, 1.0, return_u=True)
    ux, uy = dev(uxo.astype(np.float32), torch), dev(uyo.astype(np.float32), torch)
    dLdI = torch.zeros((N, N), device="cuda")
    dLdE = torch.zeros((N, N), device="cuda")
    srk.adjointSRK(dev(v, torch), ux, uy, dev(f, torch), GX, GY, N, W, e, 1.0, None, dLdI, dLdE, plan)
    torch.cuda.synchronize()
    oI = O.adj_wrt_I(v, uxo.astype(np.float32), uyo.astype(np.float32), N, e)
    oE = O.adj_wrt_E(v, f, Kx, Ky, e, 1.0, conv)
    assert rel_max_err(host(dLdI), oI) < 1e-5
    assert rel_max_err(host(dLdE), oE) < 1e-4
    assert pixel_violations(host(dLdE), oE) == 0


@pytest.mark.parametrize("N,KW,tile", [(128, 31, 128), (400, 61, 256)])
def test_tangent_matches_oracle(torch_cuda, N, KW, tile):
    torch = torch_cuda
    e = (KW - 1) // 2
    W = N - 2 * e
    f, g = fields(N, 2, 500 + N)
    rng = np.random.default_rng(7)
    df, dg = [(1e-2 * rng.standard_normal((N, N))).astype(np.float32) for _ in range(2)]
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, 1024, torch)
    plan = srk.SrkPlan(N, W, e, 1.0, 1, spectra_M=1024, tile_M=tile)
    dh = torch.zeros((W, W), device="cuda")
    srk.shrinkageTangentOaS(*[dev(a, torch) for a in (f, g, df, dg)], GX, GY, N, W, e, 1.0, None, dh, plan)
    torch.cuda.synchronize()
    o = O.tangent(f, g, df, dg, Kx, Ky, e, 1.0)
    assert rel_max_err(host(dh), o) < 1e-4
    assert pixel_violations(host(dh), o) == 0


@pytest.mark.parametrize("N,KW,tile", [(128, 31, 128), (400, 61, 256)])
@pytest.mark.parametrize("conv", ["reference", "true"])
def test_tangent_adjoint_matches_oracle(torch_cuda, N, KW, tile, conv):
    torch = torch_cuda
    e = (KW - 1) // 2
    W = N - 2 * e
    f, g = fields(N, 2, 600 + N)
    rng = np.random.default_rng(8)
    df, dg = [(1e-2 * rng.standard_normal((N, N))).astype(np.float32) for _ in range(2)]
    lam, dlam = [rng.standard_normal((W, W)).astype(np.float32) for _ in range(2)]
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, 1024, torch)
    plan = srk.SrkPlan(N, W, e, 1.0, 1, spectra_M=1024, tile_M=tile)
    plan.set_adj_convention(srk.SRK_ADJ_REFERENCE if conv == "reference" else srk.SRK_ADJ_TRUE)
    dlf = torch.zeros((N, N), device="cuda")
    dlg = torch.zeros((N, N), device="cuda")
    srk.shrinkageTangentAdjointOaS(*[dev(a, torch) for a in (f, g, df, dg, lam, dlam)], GX, GY, N, W, e, 1.0,
                                   None, dlf, dlg, plan)
    torch.cuda.synchronize()
    of, og = O.tangent_adjoint(f, g, df, dg, lam, dlam, Kx, Ky, e, 1.0, conv)
    assert rel_max_err(host(dlf), of) < 1e-4
    assert rel_max_err(host(dlg), og) < 1e-4
    assert pixel_violations(host(dlf), of) == 0
    assert pixel_violations(host(dlg), og) == 0


def test_green_tensor_and_spectrum_fp64(torch_cuda):
    import scipy.special
    torch = torch_cuda
    KW, dx = 61, 4.0
    e = 30
    gamma, Rw = 1.0 / 30.0, e * dx
    Kx = torch.zeros((KW, KW), device="cuda")
    Ky = torch.zeros_like(Kx)
    srk.green_tensor(Kx, Ky, gamma, Rw, dx)
    torch.cuda.synchronize()
    x = (np.arange(KW) - KW // 2) * dx
    X, Y = np.meshgrid(x, x, indexing="ij")
    r = np.hypot(X, Y)
    m = (r >= 1e-6 * dx) & (r <= Rw)
    rs = np.where(m, r, 1.0)
    t = rs / Rw
    w = 0.42 + 0.5 * np.cos(np.pi * t) + 0.08 * np.cos(2 * np.pi * t)
    base = np.where(m, gamma / (2 * np.pi) * scipy.special.k1(gamma * rs) * w, 0.0)
    assert np.abs(host(Kx) - base * X / rs).max() <= 1e-6 * np.abs(base).max()
    assert np.abs(host(Ky) - base * Y / rs).max() <= 1e-6 * np.abs(base).max()
    M = 256
    F = torch.zeros((M, M // 2 + 1), dtype=torch.complex64, device="cuda")
    srk.srkPrecomputeKernelFreq(Kx, KW, KW, M, F)
    torch.cuda.synchronize()
    ref = O.kernel_freq(host(Kx).astype(np.float32), M)
    assert np.abs(F.cpu().numpy() - ref).max() <= 1e-6 * np.abs(ref).max()


def test_vjp_jvp_dot_products(torch_cuda):
    """Save-for-backward contract: <J t, v> = <t, J^T v> for the full
    (f, g) -> h map, with J from srk_jvp and J^T from srk_vjp."""
    torch = torch_cuda
    N, KW, B = 200, 31, 3
    e = 15
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    plan = srk.SrkPlan(N, W, e, 1.0, B, tile_M=128)
    plan.set_kernel(dev(Kx, torch), dev(Ky, torch))
    f = dev(np.stack(fields(N, B, 900)), torch)
    g = dev(np.stack(fields(N, B, 950)), torch)
    rng = np.random.default_rng(1)
    df = dev(rng.standard_normal((B, N, N)).astype(np.float32), torch)
    dg = dev(rng.standard_normal((B, N, N)).astype(np.float32), torch)
    v = dev(rng.standard_normal((B, W, W)).astype(np.float32), torch)
    dh = torch.zeros((B, W, W), device="cuda")
    srk.jvp(f, g, df, dg, B, dh, plan)
    a_f = torch.zeros((B, N, N), device="cuda")
    a_g = torch.zeros((B, N, N), device="cuda")
    srk.vjp(v, f, g, B, a_f, a_g, plan)
    torch.cuda.synchronize()
    lhs = (dh.double() * v.double()).sum().item()
    rhs = (df.double() * a_f.double()).sum().item() + (dg.double() * a_g.double()).sum().item()
    assert abs(lhs - rhs) <= 1e-4 * (abs(lhs) + abs(rhs))
    # per image, against the oracle
    fh, gh, vh = host(f), host(g), host(v)
    for b in range(B):
        _, ux, uy = O.forward(gh[b], fh[b], Kx, Ky, e, 1.0, return_u=True)
        assert rel_max_err(host(a_f)[b], O.adj_wrt_I(vh[b], ux, uy, N, e)) < 1e-4
        assert rel_max_err(host(a_g)[b], O.adj_wrt_E(vh[b], fh[b], Kx, Ky, e, 1.0, "true")) < 1e-4
    h = torch.zeros((B, W, W), device="cuda")
    srk.forward(f, g, B, h, plan)
    torch.cuda.synchronize()
    for b in range(B):
        assert rel_max_err(host(h)[b], O.forward(gh[b], fh[b], Kx, Ky, e, 1.0)) < 1e-3


def test_error_paths_on_device(torch_cuda):
    torch = torch_cuda
    plan = srk.SrkPlan(128, 98, 15, 1.0, 2)
    E = torch.zeros((3, 128, 128), device="cuda")
    R = torch.zeros((3, 98, 98), device="cuda")
    with pytest.raises(srk.SrkError) as ei:   # B > B_max
        srk.srkTrainingForward(E, E, None, None, 128, 98, 15, 1.0, 3, None, R, plan)
    assert ei.value.status == srk.SRK_ERR_INVALID_ARG
    with pytest.raises(srk.SrkError) as ei:   # no spectra anywhere
        srk.srkTrainingForward(E, E, None, None, 128, 98, 15, 1.0, 2, None, R, plan)
    assert ei.value.status == srk.SRK_ERR_INVALID_ARG
    with pytest.raises(srk.SrkError) as ei:   # size mismatch with the plan
        srk.srkTrainingForward(E, E, None, None, 128, 96, 16, 1.0, 2, None, R, plan)
    assert ei.value.status == srk.SRK_ERR_INVALID_ARG


@pytest.mark.parametrize("N,KW,B,tile", [(256, 31, 7, 0), (512, 121, 3, 0), (300, 31, 2, 128)])
def test_persistent_and_three_pass_schedules_agree(torch_cuda, N, KW, B, tile):
    """Both kernel schedules run the same phases on the same work tiles: the
    results must be bit-identical, and match the oracle."""
    torch = torch_cuda
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, N, torch)
    E = dev(np.stack(fields(N, B, 40 + N)), torch)
    out = []
    for sch in (srk.SRK_SCHEDULE_PERSISTENT, srk.SRK_SCHEDULE_THREE_PASS):
        plan = srk.SrkPlan(N, W, e, 1.0, B, tile_M=tile)
        plan.set_schedule(sch)
        R = torch.zeros((B, W, W), device="cuda")
        srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R, plan)
        plan.sync()
        launches = plan.info()["last_launches"]
        assert launches == 1 if sch == srk.SRK_SCHEDULE_PERSISTENT else launches % 3 == 0
        out.append(host(R))
    assert np.array_equal(out[0], out[1])
    Eh = host(E)
    for b in range(B):
        assert rel_max_err(out[0][b], O.forward(Eh[b], Eh[b], Kx, Ky, e, 1.0)) < 1e-3


def test_bounded_wait_gives_up_and_context_survives(torch_cuda):
    torch = torch_cuda
    plan = srk.SrkPlan(128, 98, 15, 1.0, 2)
    assert plan.wait_selftest(1 << 12) == srk.SRK_ERR_TIMEOUT
    assert b"bounded" in srk.lib().srk_last_error()
    # the context is still usable: a normal call afterwards succeeds
    Kx, Ky = kernel(31)
    GX, GY = spectra(Kx, Ky, 128, torch)
    E = dev(np.stack(fields(128, 2, 5)), torch)
    R = torch.zeros((2, 98, 98), device="cuda")
    srk.srkTrainingForward(E, E, GX, GY, 128, 98, 15, 1.0, 2, None, R, plan)
    plan.sync()
    assert rel_max_err(host(R)[0], O.forward(host(E)[0], host(E)[0], Kx, Ky, 15, 1.0)) < 1e-3


def test_failed_allocation_reports_alloc_and_context_survives(torch_cuda):
    """A plan whose scratch cannot be allocated (65535 work tiles of a 512
    tile, ~350 GB) fails with SRK_ERR_ALLOC; nothing is left half-built and
    the device keeps working."""
    torch = torch_cuda
    with pytest.raises(srk.SrkError) as ei:
        srk.SrkPlan(512, 392, 60, 1.0, 1_000_000, tile_M=512, scratch_budget=1 << 40)
    assert ei.value.status == srk.SRK_ERR_ALLOC
    plan = srk.SrkPlan(128, 98, 15, 1.0, 2)
    Kx, Ky = kernel(31)
    GX, GY = spectra(Kx, Ky, 128, torch)
    E = dev(np.stack(fields(128, 2, 6)), torch)
    R = torch.zeros((2, 98, 98), device="cuda")
    srk.srkTrainingForward(E, E, GX, GY, 128, 98, 15, 1.0, 2, None, R, plan)
    plan.sync()
    assert rel_max_err(host(R)[1], O.forward(host(E)[1], host(E)[1], Kx, Ky, 15, 1.0)) < 1e-3


@pytest.mark.parametrize("dtype", ["f16", "bf16"])
@pytest.mark.parametrize("N,KW,B", [(256, 31, 3), (512, 121, 2)])
def test_half_storage_training_forward(torch_cuda, dtype, N, KW, B):
    """FP16/BF16 storage, FP32 arithmetic: within rel 1e-2 / abs 1e-3 of the
    FP64 oracle on the same (rounded) inputs."""
    torch = torch_cuda
    tdt = torch.float16 if dtype == "f16" else torch.bfloat16
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW, "baseline", 4.0)
    GX, GY = spectra(Kx, Ky, N, torch)
    E = dev(np.stack(fields(N, B, 70 + N)), torch).to(tdt)
    plan = srk.SrkPlan(N, W, e, 4.0, B, dtype=srk.SRK_F16 if dtype == "f16" else srk.SRK_BF16)
    R = torch.zeros((B, W, W), device="cuda", dtype=tdt)
    srk.srkTrainingForward(E, E, GX, GY, N, W, e, 4.0, B, None, R, plan)
    plan.sync()
    Eh = E.float().cpu().numpy().astype(np.float64)
    Rh = R.float().cpu().numpy().astype(np.float64)
    for b in range(B):
        ref = O.forward(Eh[b], Eh[b], Kx, Ky, e, 4.0)
        assert rel_max_err(Rh[b], ref) < 1e-2
        assert pixel_violations(Rh[b], ref, tol_abs=1e-3, tol_rel=1e-2) == 0


@pytest.mark.parametrize("dtype", ["f16", "bf16"])
def test_half_storage_derivatives(torch_cuda, dtype):
    torch = torch_cuda
    tdt = torch.float16 if dtype == "f16" else torch.bfloat16
    N, KW = 300, 31
    e = 15
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, 1024, torch)
    f, g = fields(N, 2, 801)
    rng = np.random.default_rng(5)
    df, dg = [(1e-2 * rng.standard_normal((N, N))).astype(np.float32) for _ in range(2)]
    lam, dlam = [rng.standard_normal((W, W)).astype(np.float32) for _ in range(2)]
    hp = lambda a: dev(a, torch).to(tdt)
    back = lambda t: t.float().cpu().numpy().astype(np.float64)
    F, G, DF, DG, LAM, DLAM = [hp(a) for a in (f, g, df, dg, lam, dlam)]
    fh, gh, dfh, dgh, lamh, dlamh = [back(t) for t in (F, G, DF, DG, LAM, DLAM)]
    plan = srk.SrkPlan(N, W, e, 1.0, 1, spectra_M=1024, tile_M=128,
                       dtype=srk.SRK_F16 if dtype == "f16" else srk.SRK_BF16)
    dh = torch.zeros((W, W), device="cuda", dtype=tdt)
    srk.shrinkageTangentOaS(F, G, DF, DG, GX, GY, N, W, e, 1.0, None, dh, plan)
    dlf = torch.zeros((N, N), device="cuda", dtype=tdt)
    dlg = torch.zeros((N, N), device="cuda", dtype=tdt)
    srk.shrinkageTangentAdjointOaS(F, G, DF, DG, LAM, DLAM, GX, GY, N, W, e, 1.0, None, dlf, dlg, plan)
    plan.sync()
    assert rel_max_err(back(dh), O.tangent(fh, gh, dfh, dgh, Kx, Ky, e, 1.0)) < 1e-2
    of, og = O.tangent_adjoint(fh, gh, dfh, dgh, lamh, dlamh, Kx, Ky, e, 1.0, "reference")
    assert rel_max_err(back(dlf), of) < 1e-2
    assert rel_max_err(back(dlg), og) < 1e-2
    # the adjoint (reference contract: v, ux, uy given) in the same storage
    _, uxo, uyo = O.forward(gh, fh, Kx, Ky, e, 1.0, return_u=True)
    UX, UY = hp(uxo.astype(np.float32)), hp(uyo.astype(np.float32))
    dI = torch.zeros((N, N), device="cuda", dtype=tdt)
    dE = torch.zeros((N, N), device="cuda", dtype=tdt)
    srk.adjointSRK(LAM, UX, UY, F, GX, GY, N, W, e, 1.0, None, dI, dE, plan)
    plan.sync()
    uxh, uyh = back(UX), back(UY)
    assert rel_max_err(back(dI), O.adj_wrt_I(lamh, uxh, uyh, N, e)) < 1e-2
    assert rel_max_err(back(dE), O.adj_wrt_E(lamh, fh, Kx, Ky, e, 1.0, "reference")) < 1e-2


def test_autotuned_plan_is_correct_and_cached(torch_cuda, tmp_path, monkeypatch):
    torch = torch_cuda
    monkeypatch.setenv("SRK_TUNE_CACHE", str(tmp_path / "tune.txt"))
    N, KW, B = 256, 31, 4
    e = 15
    W = N - 2 * e
    M, sch = srk.autotune(N, W, e, 1.0, B)
    assert M in (128, 256, 512) and sch in (0, 1)
    lines = (tmp_path / "tune.txt").read_text().split("\n")
    assert any(l.endswith(" %d %d" % (M, sch)) for l in lines)
    assert srk.autotune(N, W, e, 1.0, B) == (M, sch)  # from the cache
    plan = srk.SrkPlan(N, W, e, 1.0, B, tile_M=srk.SRK_TILE_AUTOTUNE)
    assert plan.info()["tile_M"] == M and plan.info()["schedule"] == sch
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, N, torch)
    E = dev(np.stack(fields(N, B, 3)), torch)
    R = torch.zeros((B, W, W), device="cuda")
    srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R, plan)
    plan.sync()
    assert rel_max_err(host(R)[1], O.forward(host(E)[1], host(E)[1], Kx, Ky, e, 1.0)) < 1e-3
