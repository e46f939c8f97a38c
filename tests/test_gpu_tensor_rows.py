"""The tensor-core row schedule (SRK_SCHEDULE_TENSOR_ROWS, FP16/BF16 storage
at tile 512): after the column transform (a DFT on the tensor cores where
its TMA boxes apply, else the column FFT) the convolution along x runs per
frequency row as a banded complex matrix product on tcgen05 with FP16
column spectra.  It serves the pair ops (training forward, OaS forward,
VJP); the tangent and tangent-adjoint run the FFT schedule on such a plan.
Checked against the FP64 oracle (storage tolerance rel 1e-2 / abs 1e-3)
and against the FFT row pass on the same inputs."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from oracle import oracle as O
from tests.gpu_util import dev, spectra
from tests.helpers import fields, kernel, pixel_violations, rel_max_err
from tests.windows import forward_window, tangent_adjoint_window, tangent_window, windows

pytestmark = pytest.mark.gpu

DT = {"f16": (srk.SRK_F16, "float16"), "bf16": (srk.SRK_BF16, "bfloat16")}


@pytest.mark.parametrize("dt", ["f16", "bf16"])
@pytest.mark.parametrize("N,KW,B,budget", [(512, 121, 5, 0), (512, 121, 40, 64 << 20), (512, 61, 3, 0)])
def test_tensor_rows_training_forward(torch_cuda, dt, N, KW, B, budget):
    torch = torch_cuda
    sdt, tname = DT[dt]
    tdt = getattr(torch, tname)
    e = (KW - 1) // 2
    W = N - 2 * e
    dx = 4.0
    Kx, Ky = kernel(KW, "baseline", dx)
    GX, GY = spectra(Kx, Ky, N, torch)
    E = dev(np.stack(fields(N, B, 70 + KW)), torch).to(tdt)
    I = dev(np.stack(fields(N, B, 90 + KW)), torch).to(tdt)
    out = {}
    for sch in (srk.SRK_SCHEDULE_TENSOR_ROWS, srk.SRK_SCHEDULE_THREE_PASS):
        plan = srk.SrkPlan(N, W, e, dx, B, dtype=sdt, tile_M=512, scratch_budget=budget)
        plan.set_schedule(sch)
        R = torch.full((B, W, W), float("nan"), device="cuda", dtype=tdt)
        srk.srkTrainingForward(E, I, GX, GY, N, W, e, dx, B, None, R, plan)
        plan.sync()
        out[sch] = R.double().cpu().numpy()
    Rt, Rf = out[srk.SRK_SCHEDULE_TENSOR_ROWS], out[srk.SRK_SCHEDULE_THREE_PASS]
    assert np.isfinite(Rt).all()
    Eh, Ih = E.double().cpu().numpy(), I.double().cpu().numpy()
    for b in sorted({0, B // 2, B - 1}):
        ref = O.forward(Eh[b], Ih[b], Kx, Ky, e, dx)
        assert rel_max_err(Rt[b], ref) < 1e-2, b
        assert pixel_violations(Rt[b], ref, tol_abs=1e-3, tol_rel=1e-2) == 0, b
        assert rel_max_err(Rt[b], Rf[b]) < 1e-2, b


@pytest.mark.parametrize("dt,amp", [("f16", 1e4), ("bf16", 1e8), ("bf16", 1e-20)])
def test_tensor_rows_input_range(torch_cuda, dt, amp):
    """Inputs far from [0, 1]: column spectra of an FP16 image scaled to 1e4
    (or a BF16 one to 1e8) exceed FP16's range, those of a BF16 image scaled
    to 1e-20 fall below it; the per-chunk plane scale keeps both within the
    storage tolerance of the oracle (R is linear in E: the absolute floor
    scales with amp)."""
    torch = torch_cuda
    sdt, tname = DT[dt]
    tdt = getattr(torch, tname)
    N, KW, B, dx = 512, 121, 2, 4.0
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW, "baseline", dx)
    GX, GY = spectra(Kx, Ky, N, torch)
    E = (dev(np.stack(fields(N, B, 70 + KW)), torch) * amp).to(tdt)
    I = dev(np.stack(fields(N, B, 90 + KW)), torch).to(tdt)
    out = {}
    for sch in (srk.SRK_SCHEDULE_TENSOR_ROWS, srk.SRK_SCHEDULE_THREE_PASS):
        plan = srk.SrkPlan(N, W, e, dx, B, dtype=sdt, tile_M=512)
        plan.set_schedule(sch)
        R = torch.full((B, W, W), float("nan"), device="cuda", dtype=tdt)
        srk.srkTrainingForward(E, I, GX, GY, N, W, e, dx, B, None, R, plan)
        plan.sync()
        out[sch] = R.double().cpu().numpy()
    Rt, Rf = out[srk.SRK_SCHEDULE_TENSOR_ROWS], out[srk.SRK_SCHEDULE_THREE_PASS]
    assert np.isfinite(Rt).all()
    Eh, Ih = E.double().cpu().numpy(), I.double().cpu().numpy()
    for b in range(B):
        ref = O.forward(Eh[b], Ih[b], Kx, Ky, e, dx)
        assert rel_max_err(Rt[b], ref) < 1e-2, b
        assert pixel_violations(Rt[b], ref, tol_abs=1e-3 * amp, tol_rel=1e-2) == 0, b
        assert rel_max_err(Rt[b], Rf[b]) < 1e-2, b


def test_tensor_rows_mixed_amplitudes_ring(torch_cuda):
    """B = 600 (300 work tiles: three chunks through the two-slot pipeline,
    the third reusing the first slot's planes and largest-|Z| words) with
    the amplitude changing per image pair from 1e-3 to 1e4, so that work
    tiles at scale 1 and refitted ones sit side by side in every chunk.
    Every image against the FFT row pass; the extremes against the oracle."""
    torch = torch_cuda
    N, KW, B, dx = 512, 121, 600, 4.0
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW, "baseline", dx)
    GX, GY = spectra(Kx, Ky, N, torch)
    amp = np.array([10.0 ** (((b // 2) * 3) % 8 - 3) for b in range(B)])
    base = np.stack(fields(N, 16, 17))
    E = (dev(base[np.arange(B) % 16], torch) * torch.from_numpy(amp).float().cuda()[:, None, None]).half()
    I = dev(np.stack(fields(N, 16, 19))[np.arange(B)[::-1] % 16], torch).half()
    out = {}
    for sch in (srk.SRK_SCHEDULE_TENSOR_ROWS, srk.SRK_SCHEDULE_THREE_PASS):
        plan = srk.SrkPlan(N, W, e, dx, B, dtype=srk.SRK_F16, tile_M=512)
        plan.set_schedule(sch)
        R = torch.full((B, W, W), float("nan"), device="cuda", dtype=torch.float16)
        srk.srkTrainingForward(E, I, GX, GY, N, W, e, dx, B, None, R, plan)
        plan.sync()
        out[sch] = R.float().cpu().numpy()
        if sch == srk.SRK_SCHEDULE_TENSOR_ROWS:
            assert plan.info()["last_launches"] == 12  # three chunks of four launches
    Rt, Rf = out[srk.SRK_SCHEDULE_TENSOR_ROWS], out[srk.SRK_SCHEDULE_THREE_PASS]
    assert np.isfinite(Rt).all()
    for b in range(B):
        assert rel_max_err(Rt[b], Rf[b]) < 1e-2, (b, amp[b])
    for b in (int(np.argmin(amp)), int(np.argmax(amp))):
        ref = O.forward(E[b].double().cpu().numpy(), I[b].double().cpu().numpy(), Kx, Ky, e, dx)
        assert rel_max_err(Rt[b], ref) < 1e-2, (b, amp[b])
        assert pixel_violations(Rt[b], ref, tol_abs=1e-3 * amp[b], tol_rel=1e-2) == 0, (b, amp[b])


@pytest.mark.parametrize("dt", ["f16", "bf16"])
@pytest.mark.parametrize("N,KW", [(4096, 61), (1024, 121)])
def test_tensor_rows_single_image_ops(torch_cuda, dt, N, KW):
    """One image of several tiles of 512: the OaS forward with ux / uy, the
    tangent and the tangent-adjoint (the FFT schedule on this plan) on oracle
    windows; the VJP against the same VJP on the FFT row pass.  At N = 4096,
    KW = 61 the tile stride (452) is not a multiple of 8 and the column FFT
    runs; at N = 1024, KW = 121 (stride 392) the column DFT on the tensor
    cores."""
    torch = torch_cuda
    sdt, tname = DT[dt]
    tdt = getattr(torch, tname)
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, 1024, torch)
    gen = torch.Generator(device="cuda").manual_seed(4)
    f = torch.rand((N, N), device="cuda", generator=gen).to(tdt)
    g = torch.rand((N, N), device="cuda", generator=gen).to(tdt)
    df = (1e-2 * torch.randn((N, N), device="cuda", generator=gen)).to(tdt)
    dg = (1e-2 * torch.randn((N, N), device="cuda", generator=gen)).to(tdt)
    lam = torch.randn((W, W), device="cuda", generator=gen).to(tdt)
    dlam = torch.randn((W, W), device="cuda", generator=gen).to(tdt)
    plan = srk.SrkPlan(N, W, e, 1.0, 1, spectra_M=1024, dtype=sdt, tile_M=512)
    plan.set_adj_convention(srk.SRK_ADJ_TRUE)
    plan.import_spectra(GX, GY)
    plan.set_schedule(srk.SRK_SCHEDULE_TENSOR_ROWS)
    R = torch.empty((W, W), device="cuda", dtype=tdt)
    ux, uy = torch.empty_like(R), torch.empty_like(R)
    srk.srkForwardOaS(g, f, GX, GY, N, W, e, 1.0, None, R, plan, ux, uy)
    dh = torch.empty_like(R)
    srk.shrinkageTangentOaS(f, g, df, dg, GX, GY, N, W, e, 1.0, None, dh, plan)
    dlf = torch.empty((N, N), device="cuda", dtype=tdt)
    dlg = torch.empty_like(dlf)
    srk.shrinkageTangentAdjointOaS(f, g, df, dg, lam, dlam, GX, GY, N, W, e, 1.0, None, dlf, dlg, plan)
    vf = torch.empty((1, N, N), device="cuda", dtype=tdt)
    vg = torch.empty_like(vf)
    srk.vjp(lam[None], f[None], g[None], 1, vf, vg, plan)
    plan.sync()
    for ox, oy in windows(W, 128, 2, 3):
        got, ref = forward_window(f, g, Kx, Ky, e, 1.0, R, ox, oy, 128)
        assert rel_max_err(got, ref) < 1e-2 and pixel_violations(got, ref, 1e-3, 1e-2) == 0
        _, uxo, _ = O.forward(*(t[ox:ox + 128 + 2 * e, oy:oy + 128 + 2 * e].double().cpu().numpy() for t in (g, f)),
                              Kx, Ky, e, 1.0, return_u=True)
        assert rel_max_err(ux[ox:ox + 128, oy:oy + 128].double().cpu().numpy(), uxo) < 1e-2
        got, ref = tangent_window(f, g, df, dg, Kx, Ky, e, 1.0, dh, ox, oy, 128)
        assert rel_max_err(got, ref) < 1e-2 and pixel_violations(got, ref, 1e-3, 1e-2) == 0
    for px, py in windows(N, 128, 1, 5):
        for got, ref in tangent_adjoint_window(f, g, df, dg, lam, dlam, Kx, Ky, e, 1.0, dlf, dlg, px, py, 128,
                                               "true"):
            assert rel_max_err(got, ref) < 1e-2 and pixel_violations(got, ref, 1e-3, 1e-2) == 0
    # the VJP's dL/df (row pass on the tensor cores) against the FFT row pass
    plan.set_schedule(srk.SRK_SCHEDULE_THREE_PASS)
    wf = torch.empty_like(vf)
    wg = torch.empty_like(vg)
    srk.vjp(lam[None], f[None], g[None], 1, wf, wg, plan)
    plan.sync()
    a, b = vf[0].double().cpu().numpy(), wf[0].double().cpu().numpy()
    assert rel_max_err(a, b) < 1e-2


def test_tensor_rows_rejects_unsupported(torch_cuda):
    plan = srk.SrkPlan(512, 392, 60, 1.0, 1)  # FP32 storage
    with pytest.raises(srk.SrkError) as ei:
        plan.set_schedule(srk.SRK_SCHEDULE_TENSOR_ROWS)
    assert ei.value.status == srk.SRK_ERR_UNSUPPORTED
    plan = srk.SrkPlan(512, 312, 100, 1.0, 1, dtype=srk.SRK_F16, tile_M=512)  # erosion > 64
    with pytest.raises(srk.SrkError) as ei:
        plan.set_schedule(srk.SRK_SCHEDULE_TENSOR_ROWS)
    assert ei.value.status == srk.SRK_ERR_UNSUPPORTED
