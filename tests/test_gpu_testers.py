"""The reference's own derivative test protocols (stTestCore testers),
restated on the device operators.

* AdjointTester (adjoint_tester.h:107-122, pass rule :563-567): q = sum R^2;
  the analytic dq/dA = adjoint(2R) against per-pixel central differences
  (q(A + eps e_p) - q(A - eps e_p)) / (2 eps) at every pixel; a pixel passes
  if |a - n| <= max(tol_abs, tol_rel max(|a|, |n|)).  Configurations wrtI
  {eps 0.1, 1e-5, 1e-3} and wrtE {eps 0.5, 1e-5, 1e-3}
  (adjoint/main_adjoint.cu:633, :718).
* TangentTester (tangent_tester.h:27-49): the analytic JVP against
  (F(x + eps d) - F(x - eps d)) / (2 eps) over eps in {1e-4, 1e-3, 1e-2,
  1e-1}; a case passes if some eps has no violations (tol_abs 1e-5,
  tol_rel 1e-3).  Modes A (df), B (dg), C (both), 3 directions
  (tan_tanadj/main_tan_tanadj.cu:336-349, :505-534).
* TangentAdjointTester: dLam_f modes D (dlam), E (dg), G (all); dLam_g
  modes D, F (df), G (main_tan_tanadj.cu:588-646).

Every central difference is one image of a single batched call of the
operator.  The adjoint with respect to the convolved field is checked in the
exact convention (srk_vjp); the reference's own convention agrees with it for
even kernels only (see the adjoint convention of srk_b200.h)."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from tests.helpers import fields, kernel, pixel_violations
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

EPS_SWEEP = (1e-4, 1e-3, 1e-2, 1e-1)


def setup(N, KW, B_max, torch):
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    plan = srk.SrkPlan(N, W, e, 1.0, B_max, tile_M=128)
    plan.set_kernel(dev(Kx, torch), dev(Ky, torch))
    plan.set_adj_convention(srk.SRK_ADJ_TRUE)
    return e, W, plan


def batched_forward(plan, f, g, W):
    B = f.shape[0]
    import torch
    h = torch.zeros((B, W, W), device="cuda")
    srk.forward(f, g, B, h, plan)
    return h


@pytest.mark.parametrize("wrt,eps", [("I", 0.1), ("E", 0.5)])
def test_adjoint_tester_gradient_check(torch_cuda, wrt, eps):
    torch = torch_cuda
    N, KW = 48, 15
    B = 2 * N * N
    e, W, plan = setup(N, KW, B, torch)
    f0, g0 = (dev(a, torch) for a in fields(N, 2, 42))
    R0 = batched_forward(plan, f0[None], g0[None], W)
    # analytic: dq/dA = adjoint(2 R)
    af = torch.zeros((1, N, N), device="cuda")
    ag = torch.zeros((1, N, N), device="cuda")
    srk.vjp(2.0 * R0, f0[None], g0[None], 1, af, ag, plan)
    ana = host(af if wrt == "I" else ag)[0]
    # numeric: every pixel +-eps, one batched forward
    base = f0 if wrt == "I" else g0
    pert = base.reshape(1, N * N).repeat(B, 1)
    idx = torch.arange(N * N, device="cuda")
    pert[2 * idx, idx] += eps
    pert[2 * idx + 1, idx] -= eps
    pert = pert.reshape(B, N, N)
    other = (g0 if wrt == "I" else f0)[None].expand(B, N, N).contiguous()
    h = batched_forward(plan, pert, other, W) if wrt == "I" else batched_forward(plan, other, pert, W)
    q = (h.double() ** 2).sum(dim=(1, 2))
    num = ((q[0::2] - q[1::2]) / (2 * eps)).reshape(N, N).cpu().numpy()
    assert pixel_violations(ana, num, tol_abs=1e-5, tol_rel=1e-3) == 0


def direction(N, d, torch, seed_off):
    # GP directions with seeds 100 + 3d + {0, 1} (main_tan_tanadj.cu:336-349), scaled by 1e-2
    return dev((1e-2 * (fields(N, 1, 100 + 3 * d + seed_off)[0] - 0.5) * 2).astype(np.float32), torch)


def passes_some_eps(ana, nums):
    return any(pixel_violations(ana, n, tol_abs=1e-5, tol_rel=1e-3) == 0 for n in nums)


@pytest.mark.parametrize("mode", ["A", "B", "C"])
def test_tangent_tester_modes(torch_cuda, mode):
    torch = torch_cuda
    N, KW = 96, 15
    e, W, plan = setup(N, KW, 2 * len(EPS_SWEEP), torch)
    f, g = (dev(a, torch) for a in fields(N, 2, 60))
    for d in range(3):
        df = direction(N, d, torch, 0) if mode in "AC" else torch.zeros_like(f)
        dg = direction(N, d, torch, 1) if mode in "BC" else torch.zeros_like(g)
        dh = torch.zeros((1, W, W), device="cuda")
        srk.jvp(f[None], g[None], df[None], dg[None], 1, dh, plan)
        fs = torch.stack([f + s * eps * df for eps in EPS_SWEEP for s in (1, -1)])
        gs = torch.stack([g + s * eps * dg for eps in EPS_SWEEP for s in (1, -1)])
        h = batched_forward(plan, fs, gs, W)
        nums = [host((h[2 * i] - h[2 * i + 1]) / (2 * eps)) for i, eps in enumerate(EPS_SWEEP)]
        assert passes_some_eps(host(dh)[0], nums), (mode, d)


@pytest.mark.parametrize("out,mode", [("f", "D"), ("f", "E"), ("f", "G"), ("g", "D"), ("g", "F"), ("g", "G")])
def test_tangent_adjoint_tester_modes(torch_cuda, out, mode):
    torch = torch_cuda
    N, KW = 96, 15
    e, W, plan = setup(N, KW, 2 * len(EPS_SWEEP), torch)
    f, g = (dev(a, torch) for a in fields(N, 2, 61))
    rng = np.random.default_rng(7)
    lam = dev(rng.standard_normal((W, W)).astype(np.float32), torch)
    for d in range(3):
        df = direction(N, d, torch, 0) if mode in "FG" else torch.zeros_like(f)
        dg = direction(N, d, torch, 1) if mode in "EG" else torch.zeros_like(g)
        dlam = (dev(np.random.default_rng(200 + d).standard_normal((W, W)).astype(np.float32), torch)
                if mode in "DG" else torch.zeros_like(lam))
        dlf = torch.zeros((N, N), device="cuda")
        dlg = torch.zeros((N, N), device="cuda")
        srk.shrinkageTangentAdjointOaS(f, g, df, dg, lam, dlam, None, None, N, W, e, 1.0, None, dlf, dlg, plan)
        n2 = 2 * len(EPS_SWEEP)
        fs = torch.stack([f + s * eps * df for eps in EPS_SWEEP for s in (1, -1)])
        gs = torch.stack([g + s * eps * dg for eps in EPS_SWEEP for s in (1, -1)])
        ls = torch.stack([lam + s * eps * dlam for eps in EPS_SWEEP for s in (1, -1)])
        af = torch.zeros((n2, N, N), device="cuda")
        ag = torch.zeros((n2, N, N), device="cuda")
        srk.vjp(ls, fs, gs, n2, af, ag, plan)
        a = af if out == "f" else ag
        nums = [host((a[2 * i] - a[2 * i + 1]) / (2 * eps)) for i, eps in enumerate(EPS_SWEEP)]
        assert passes_some_eps(host(dlf if out == "f" else dlg), nums), (out, mode, d)
