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


def test_alternating_slab_ops_replay_from_cuda_graph(torch_cuda):
    """A forward slab and an adjoint slab of one image on one plan (two
    different tile-table keys), called once each, then captured together and
    replayed: every key keeps its own tables, so the replay uploads nothing
    and equals direct calls."""
    torch = torch_cuda
    N, KW, tile = 300, 31, 128
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, 1024, torch)
    plan = srk.SrkPlan(N, W, e, 1.0, 1, spectra_M=1024, tile_M=tile)
    plan.set_adj_convention(srk.SRK_ADJ_TRUE)
    S = plan.info()["tile_stride"]
    c0, c1 = S, 2 * S  # one interior slab of whole tiles
    gen = torch.Generator(device="cuda").manual_seed(3)
    f, g = (torch.rand((N, N), device="cuda", generator=gen) for _ in range(2))
    v, ux, uy = (torch.randn((W, W), device="cuda", generator=gen) for _ in range(3))
    R = torch.zeros((W, W), device="cuda")
    dI, dE = (torch.zeros((N, N), device="cuda") for _ in range(2))

    def step():
        # every pointer addresses column c0 of its (column-major) array
        srk.srkForwardOaSSlab(g[c0:], f[c0:], GX, GY, N, e, 1.0, c0, c1, None, R[c0:], plan)
        srk.adjointSRKSlab(v[c0:], ux[c0:], uy[c0:], f[c0:], GX, GY, N, e, 1.0, c0, c1, None, dI[c0:], dE[c0:],
                           plan)

    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        step()  # builds both keys' tables outside the capture
    stream.synchronize()
    ref = [host(t).copy() for t in (R, dI, dE)]
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        step()
    for _ in range(2):
        for t in (R, dI, dE):
            t.zero_()
        graph.replay()
        torch.cuda.synchronize()
        for t, r in zip((R, dI, dE), ref):
            assert np.array_equal(host(t), r)
    del graph
