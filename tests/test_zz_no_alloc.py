"""srk_training_forward_noalloc: the training forward for callers that cannot
allocate device memory (inside another framework's memory pool, under a fixed
budget, or in a plug-in whose host owns every allocation).  Called through
the C ABI twice in a row — the second call reuses the library's static
scratch array with the first call's contents still in it — and checked
against the plan-based srk_training_forward on the same inputs, with the
forward tolerances used everywhere else (max|d|/max|ref| < 1e-3 and the
per-pixel bound).  Kept in its own file, collected last."""
import ctypes

import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from tests.gpu_util import dev, host, spectra
from tests.helpers import fields, kernel, pixel_violations, rel_max_err

pytestmark = pytest.mark.gpu


def _noalloc(L, E, I, GX, GY, N, W, e, dx, B, R, stream):
    fn = L.srk_training_forward_noalloc
    fn.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn(E.data_ptr(), I.data_ptr(), GX.data_ptr(), GY.data_ptr(), N, W, e, dx, B, stream, R.data_ptr())


@pytest.mark.parametrize("N,KW,B", [(128, 15, 3), (256, 31, 5), (512, 121, 13)])
def test_noalloc_matches_plan_forward_twice(torch_cuda, N, KW, B):
    """E (convolved) and I (differentiated) are different fields, so a
    swapped or ignored I changes the result."""
    torch = torch_cuda
    L = srk.lib()
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW, "baseline", 4.0)
    GX, GY = spectra(Kx, Ky, N, torch)
    stream = torch.cuda.current_stream().cuda_stream
    plan = srk.SrkPlan(N, W, e, 4.0, B)
    for call, seed in enumerate((11, 29)):
        E = dev(np.stack(fields(N, B, seed)), torch)
        I = dev(np.stack(fields(N, B, seed + 1000)), torch)
        R_plan = torch.zeros((B, W, W), device="cuda")
        srk.srkTrainingForward(E, I, GX, GY, N, W, e, 4.0, B, None, R_plan, plan)
        R = torch.full((B, W, W), float("nan"), device="cuda")
        st = _noalloc(L, E, I, GX, GY, N, W, e, 4.0, B, R, stream)
        assert st == srk.SRK_OK, L.srk_last_error()
        torch.cuda.synchronize()
        a, b = host(R), host(R_plan)
        assert np.all(np.isfinite(a)), "call %d left outputs unwritten" % call
        for i in range(B):
            assert rel_max_err(a[i], b[i]) < 1e-3
            assert pixel_violations(a[i], b[i]) == 0


def test_noalloc_rejects_unsupported_sizes(torch_cuda):
    torch = torch_cuda
    L = srk.lib()
    E = torch.zeros((1, 300, 300), device="cuda")
    R = torch.zeros((1, 270, 270), device="cuda")
    G = torch.zeros((300, 151), dtype=torch.complex64, device="cuda")
    st = _noalloc(L, E, E, G, G, 300, 270, 15, 1.0, 1, R, torch.cuda.current_stream().cuda_stream)
    assert st == srk.SRK_ERR_UNSUPPORTED
    assert b"N in {128, 256, 512}" in L.srk_last_error()
