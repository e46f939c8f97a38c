"""The training forward at the benchmark's full size: B = 5000 images of
N = 512, KW = 121 (W = 392), dx = 4 nm, Green's tensor of gamma = 1/30 nm,
Gaussian random fields generated on the device; the default plan splits the
batch into several scratch chunks (through the ring of scratch slots).

* every image against the reference's own cuFFT srkTrainingForward compiled
  from its sources (when built), to the reference forward tolerance;
* four images against the FP64 oracle;
* size-independent properties: a second call is bit-identical, and a call
  on the first ten images equals the first ten outputs of the full call (the
  pairing of images into work tiles is the same)."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from oracle import oracle as O
from tests.gpu_util import dev, host, ref_gpu
from tests.helpers import kernel, pixel_violations, rel_max_err

pytestmark = pytest.mark.gpu

N, KW, B, DX = 512, 121, 5000, 4.0
E_ = (KW - 1) // 2
W = N - 2 * E_


def test_full_size_training_forward(torch_cuda):
    torch = torch_cuda
    Kx, Ky = kernel(KW, form="baseline", dx=DX)
    GX, GY = dev(O.kernel_freq(Kx, N), torch), dev(O.kernel_freq(Ky, N), torch)
    E = torch.zeros((B, N, N), device="cuda")
    srk.grf(E, 8.0, 4242)
    plan = srk.SrkPlan(N, W, E_, DX, B)
    assert plan.info()["chunk_wt"] < B // 2  # several chunks
    R = torch.zeros((B, W, W), device="cuda")
    srk.srkTrainingForward(E, E, GX, GY, N, W, E_, DX, B, None, R, plan)
    R2 = torch.zeros_like(R)
    srk.srkTrainingForward(E, E, GX, GY, N, W, E_, DX, B, None, R2, plan)
    R10 = torch.zeros((10, W, W), device="cuda")
    srk.srkTrainingForward(E[:10], E[:10], GX, GY, N, W, E_, DX, 10, None, R10, plan)
    torch.cuda.synchronize()
    assert torch.equal(R, R2)
    assert torch.equal(R[:10], R10)
    del R2, R10
    Eh = {b: host(E[b]) for b in (0, 1, 2777, B - 1)}
    for b, img in Eh.items():
        Ro = O.forward(img, img, Kx, Ky, E_, DX)
        got = host(R[b])
        assert rel_max_err(got, Ro) < 1e-3, b
        assert pixel_violations(got, Ro, tol_abs=1e-5 * np.abs(Ro).max()) == 0, b
    L = ref_gpu()
    if L is None:
        pytest.skip("reference build not available")
    s = torch.cuda.current_stream().cuda_stream
    ws = L.ref_train_ws_create(N, B, s)
    Rr = torch.zeros_like(R)
    assert L.ref_train_forward(E.data_ptr(), E.data_ptr(), GX.data_ptr(), GY.data_ptr(), N, W, E_, DX, B, s,
                               Rr.data_ptr(), ws) == 0
    torch.cuda.synchronize()
    L.ref_train_ws_destroy(ws, s)
    err = (R - Rr).abs().amax(dim=(1, 2)) / Rr.abs().amax(dim=(1, 2)).clamp_min(1e-30)
    assert float(err.max()) < 1e-3, float(err.max())
