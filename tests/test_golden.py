"""The oracle pinned against golden outputs of the reference's own code
(tests/golden/make_golden.py): GpGenerator and generate_pattern (host),
srkTrainingForward (cuFFT) and MeasureCD_Batched (run on a B200).  These run
on the CPU without the reference or a GPU."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_max_err

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_golden_gp_generator():
    g = load("ref_host.npz")
    i = 0
    while f"gp{i}_case" in g:
        N, ell, _ = g[f"gp{i}_case"]
        ref = g[f"gp{i}_field"].astype(np.float64)
        ours = O.grf_filter(g[f"gp{i}_noise"], int(N), float(ell))
        assert np.abs(ours - ref).max() < 1e-6 * np.abs(ref).max(), i
        i += 1
    assert i == 3


def test_golden_line_space_patterns():
    g = load("ref_host.npz")
    for i in range(3):
        vert, N, sigma, period = g[f"lns{i}_case"]
        ours = O.lns(bool(vert), int(N), float(sigma), float(period))
        assert np.abs(ours - g[f"lns{i}"]).max() < 2e-6, i


@pytest.mark.parametrize("i", [0, 1])
def test_golden_training_forward(i):
    """srkTrainingForward (cuFFT, float) against the FP64 oracle: the
    reference's own forward tolerance is 1e-3 (adjoint/main_adjoint.cu:359-360);
    the measured agreement is ~1e-6."""
    g = load("ref_gpu.npz")
    N, KW, B = (int(v) for v in g[f"train{i}_case"])
    e = (KW - 1) // 2
    E, Kx, Ky, R = g[f"train{i}_E"], g[f"train{i}_Kx"], g[f"train{i}_Ky"], g[f"train{i}_R"]
    for b in range(B):
        ours = O.forward(E[b].astype(np.float64), E[b].astype(np.float64), Kx, Ky, e, 1.0)
        assert rel_max_err(R[b], ours) < 2e-5, b


def test_golden_measure_cd():
    g = load("ref_gpu.npz")
    left, right, cd = O.measure_cd(g["cd_signals"])
    assert np.abs(cd - g["cd"]).max() < 1e-3   # the reference's pass bar is 0.01 px (README.md:36)
    assert np.abs(left - g["cd_left"]).max() < 1e-3
    assert np.abs(right - g["cd_right"]).max() < 1e-3
