"""Makes the golden fixtures of tests/test_golden.py from the reference's own
code, compiled from its sources into oracle/_ref by oracle/build.py (the
reference sources are needed only to build those libraries).

    python tests/golden/make_golden.py --host [--out DIR]   # CPU: GpGenerator, generate_pattern
    python tests/golden/make_golden.py --gpu  [--out DIR]   # a GPU: srkTrainingForward (cuFFT), MeasureCD_Batched

--host writes ref_host.npz: GpGenerator's white noise and field for three
(N, ell, seed) cases (gp_generator.h:95-147) and line/space patterns
(test_pattern.cu:83-109).  --gpu writes ref_gpu.npz: seeded inputs, kernel
spectra and the reference srkTrainingForward output
(training/srk_training_forward.cuh:175-241) for two configurations, and
seeded line/space signals with their MeasureCD_Batched result
(cd_measure_util.cu:310-437)."""
import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

GP_CASES = [(64, 8.0, 7), (50, 8.0, 11), (96, 3.0, 5)]
LNS_CASES = [(True, 96, 6.0, 0.0), (False, 96, 6.0, 0.0), (True, 128, 4.0, 40.0)]
TRAIN_CASES = [(64, 15, 2, 101), (128, 31, 2, 202)]  # N, KW, B, seed


def make_host(out):
    d = {}
    for i, (N, ell, seed) in enumerate(GP_CASES):
        d[f"gp{i}_noise"] = O.ref_gp_noise(N, seed)
        d[f"gp{i}_field"] = O.ref_gp_field(N, ell, seed)
        d[f"gp{i}_case"] = np.array([N, ell, seed], np.float64)
    for i, (vert, N, sigma, period) in enumerate(LNS_CASES):
        d[f"lns{i}"] = O.ref_lns(vert, N, sigma, period)
        d[f"lns{i}_case"] = np.array([1.0 if vert else 0.0, N, sigma, period], np.float64)
    path = os.path.join(out, "ref_host.npz")
    np.savez_compressed(path, **d)
    print(path)


def make_gpu(out):
    import torch
    from tests.gpu_util import ref_gpu
    L = ref_gpu()
    if L is None:
        raise SystemExit("oracle/_ref/libref_gpu.so is not built")
    s = torch.cuda.current_stream().cuda_stream
    d = {}
    for i, (N, KW, B, seed) in enumerate(TRAIN_CASES):
        e = (KW - 1) // 2
        W = N - 2 * e
        Kx, Ky = O.make_kernel_sigma(KW, e / 3.0)
        E = np.stack([O.grf(N, 8.0, seed + b) for b in range(B)])
        GXh, GYh = O.kernel_freq(Kx, N), O.kernel_freq(Ky, N)
        Ed = torch.from_numpy(np.ascontiguousarray(E)).cuda()
        GX, GY = torch.from_numpy(GXh).cuda(), torch.from_numpy(GYh).cuda()
        R = torch.zeros((B, W, W), device="cuda")
        ws = L.ref_train_ws_create(N, B, s)
        assert L.ref_train_forward(Ed.data_ptr(), Ed.data_ptr(), GX.data_ptr(), GY.data_ptr(), N, W, e, 1.0, B, s,
                                   R.data_ptr(), ws) == 0
        torch.cuda.synchronize()
        L.ref_train_ws_destroy(ws, s)
        d[f"train{i}_case"] = np.array([N, KW, B], np.int64)
        d[f"train{i}_E"] = E.astype(np.float32)
        d[f"train{i}_Kx"], d[f"train{i}_Ky"] = Kx, Ky
        d[f"train{i}_R"] = R.cpu().numpy()
    rng = np.random.default_rng(31)
    n, B = 200, 6
    sig = np.stack([O.lns(True, n, sg, 0.0)[:, 0] + 0.01 * rng.standard_normal(n).astype(np.float32)
                    for sg in np.linspace(4.0, 9.0, B)]).astype(np.float32)
    ds = torch.from_numpy(sig).cuda()
    fp = ctypes.POINTER(ctypes.c_float)
    rl, rr, rc = [np.zeros(B, np.float32) for _ in range(3)]
    assert L.ref_measure_cd(ds.data_ptr(), B, n, 16, 8, s, rl.ctypes.data_as(fp), rr.ctypes.data_as(fp),
                            rc.ctypes.data_as(fp)) == 0
    d["cd_signals"], d["cd_left"], d["cd_right"], d["cd"] = sig, rl, rr, rc
    path = os.path.join(out, "ref_gpu.npz")
    np.savez_compressed(path, **d)
    print(path)


if __name__ == "__main__":
    p = argparse.ArgumentParser()
    p.add_argument("--host", action="store_true")
    p.add_argument("--gpu", action="store_true")
    p.add_argument("--out", default=HERE)
    a = p.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.host:
        make_host(a.out)
    if a.gpu:
        make_gpu(a.out)
