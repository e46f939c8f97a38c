"""The tensor-core direct schedule of the forward (SRK_SCHEDULE_DIRECT:
tcgen05.mma over the image window staged by TMA, the kernel as a banded
Toeplitz operand), against the FP64 oracle and against the FFT schedule on
the same inputs, in FP32 (three-pass FP16 split), FP16 and BF16 storage.
Tolerances: FP32 the reference's forward criterion (max|d|/max|ref| < 1e-3,
adjoint/main_adjoint.cu:359-360, and the per-pixel rule of
adjoint_tester.h:563-567); FP16/BF16 storage rel 1e-2 / abs 1e-3."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from oracle import oracle as O
from tests.gpu_util import dev, spectra
from tests.helpers import fields, kernel, pixel_violations, rel_max_err

pytestmark = pytest.mark.gpu

DT = {"f32": (srk.SRK_F32, "float32", 1e-3, 1e-5, 1e-3),
      "f16": (srk.SRK_F16, "float16", 1e-2, 1e-3, 1e-2),
      "bf16": (srk.SRK_BF16, "bfloat16", 1e-2, 1e-3, 1e-2)}


def run(torch, N, KW, B, dt, sched, E, I, GX, GY, dx):
    sdt, tname, *_ = DT[dt]
    e = (KW - 1) // 2
    W = N - 2 * e
    plan = srk.SrkPlan(N, W, e, dx, B, dtype=sdt)
    plan.set_schedule(sched)
    R = torch.full((B, W, W), float("nan"), device="cuda", dtype=getattr(torch, tname))
    srk.srkTrainingForward(E, I, GX, GY, N, W, e, dx, B, None, R, plan)
    plan.sync()
    return R.double().cpu().numpy(), plan


@pytest.mark.parametrize("dt", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("N,KW,B", [(256, 31, 3), (128, 15, 2), (200, 9, 2), (264, 61, 1)])
def test_direct_forward_matches_oracle_and_fft(torch_cuda, N, KW, B, dt):
    torch = torch_cuda
    _, tname, r_tol, t_abs, t_rel = DT[dt]
    e = (KW - 1) // 2
    dx = 4.0
    Kx, Ky = kernel(KW, "baseline", dx)
    GX, GY = spectra(Kx, Ky, N, torch)
    Eh = np.stack(fields(N, B, 500 + N + KW))
    Ih = np.stack(fields(N, B, 900 + N + KW))
    E = dev(Eh, torch).to(getattr(torch, tname))
    I = dev(Ih, torch).to(getattr(torch, tname))
    Rd, plan = run(torch, N, KW, B, dt, srk.SRK_SCHEDULE_DIRECT, E, I, GX, GY, dx)
    assert plan.info()["schedule"] == srk.SRK_SCHEDULE_DIRECT
    assert np.isfinite(Rd).all(), "outputs left unwritten"
    Rf, _ = run(torch, N, KW, B, dt, srk.SRK_SCHEDULE_THREE_PASS, E, I, GX, GY, dx)
    Eq, Iq = E.double().cpu().numpy(), I.double().cpu().numpy()
    for b in range(B):
        ref = O.forward(Eq[b], Iq[b], Kx, Ky, e, dx)
        assert rel_max_err(Rd[b], ref) < r_tol, b
        assert pixel_violations(Rd[b], ref, tol_abs=t_abs, tol_rel=t_rel) == 0, b
        # the FFT schedule on the same inputs
        assert rel_max_err(Rd[b], Rf[b]) < r_tol, b


def test_direct_save_for_backward_forward_and_repeat(torch_cuda):
    """srk_forward (f != g) on the direct schedule, spectra bound by
    srk_plan_set_kernel; a second call gives the same bits."""
    torch = torch_cuda
    N, KW, B = 256, 21, 4
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    plan = srk.SrkPlan(N, W, e, 1.0, B, dtype=srk.SRK_F16)
    plan.set_kernel(dev(Kx, torch), dev(Ky, torch))
    plan.set_schedule(srk.SRK_SCHEDULE_DIRECT)
    f = dev(np.stack(fields(N, B, 31)), torch).half()
    g = dev(np.stack(fields(N, B, 37)), torch).half()
    h1 = torch.empty((B, W, W), device="cuda", dtype=torch.float16)
    h2 = torch.empty_like(h1)
    srk.forward(f, g, B, h1, plan)
    srk.forward(f, g, B, h2, plan)
    plan.sync()
    assert torch.equal(h1, h2)
    fh, gh = f.double().cpu().numpy(), g.double().cpu().numpy()
    for b in (0, B - 1):
        ref = O.forward(gh[b], fh[b], Kx, Ky, e, 1.0)
        assert rel_max_err(h1[b].double().cpu().numpy(), ref) < 1e-2


def test_direct_rejects_unsupported(torch_cuda):
    for N, KW in ((512, 121), (262, 31)):
        e = (KW - 1) // 2
        plan = srk.SrkPlan(N, N - 2 * e, e, 1.0, 1)
        with pytest.raises(srk.SrkError) as ei:
            plan.set_schedule(srk.SRK_SCHEDULE_DIRECT)
        assert ei.value.status == srk.SRK_ERR_UNSUPPORTED
