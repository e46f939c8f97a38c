"""The batched training forward captured in a CUDA graph and replayed.

A training loop replays the same launch sequence every step: capturing it
once removes the per-call host work.  Both kernel schedules are captured
(the persistent one includes its control-block reset and mailbox copy) and
a replay on new input data must give bit-identical results to a direct call,
and match the FP64 oracle."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from oracle import oracle as O
from tests.helpers import fields, kernel, rel_max_err
from tests.gpu_util import dev, host, spectra

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("schedule", ["persistent", "three_pass"])
def test_training_forward_replays_from_cuda_graph(torch_cuda, schedule):
    torch = torch_cuda
    N, KW, B = 256, 31, 6
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, N, torch)
    plan = srk.SrkPlan(N, W, e, 1.0, B)
    plan.set_schedule(srk.SRK_SCHEDULE_PERSISTENT if schedule == "persistent" else srk.SRK_SCHEDULE_THREE_PASS)
    E = dev(np.stack(fields(N, B, 11)), torch)
    R = torch.zeros((B, W, W), device="cuda")
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        # first call outside the capture: binds the spectra to the plan
        srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R, plan)
    plan.sync(stream)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R, plan)
    new = np.stack(fields(N, B, 12))
    for _ in range(2):
        E.copy_(dev(new, torch))
        R.zero_()
        graph.replay()
        torch.cuda.synchronize()
        plan.sync()
        got = host(R)
        R2 = torch.zeros_like(R)
        srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R2, plan)
        plan.sync()
        assert np.array_equal(got, host(R2))
        for b in (0, B - 1):
            assert rel_max_err(got[b], O.forward(new[b], new[b], Kx, Ky, e, 1.0)) < 1e-3
        new = np.stack(fields(N, B, 13))
    del graph
