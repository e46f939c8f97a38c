"""Work tiles in several scratch chunks.  A small scratch budget splits a
batch into chunks that cycle through a ring of scratch slots, P1 and P3 on
the plan's own streams and P2 on the caller's, so the passes of neighbouring
chunks overlap.  Results must be bit-identical to a single-chunk plan (the
work tiles and their pairing do not depend on the chunking), directly and
replayed from a CUDA graph."""
import numpy as np
import pytest

import shrinkage_full_tests_b200 as srk
from oracle import oracle as O
from tests.helpers import fields, kernel, rel_max_err
from tests.gpu_util import dev, host, spectra

pytestmark = pytest.mark.gpu


def test_chunked_training_forward_bit_identical_and_capturable(torch_cuda):
    torch = torch_cuda
    N, KW, B = 256, 31, 22
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    GX, GY = spectra(Kx, Ky, N, torch)
    one = srk.SrkPlan(N, W, e, 1.0, B, tile_M=256)
    one.set_schedule(srk.SRK_SCHEDULE_THREE_PASS)
    assert one.info()["chunk_wt"] >= B // 2
    per_wt = one.info()["scratch_bytes"] // one.info()["chunk_wt"]
    many = srk.SrkPlan(N, W, e, 1.0, B, tile_M=256, scratch_budget=6 * per_wt)
    many.set_schedule(srk.SRK_SCHEDULE_THREE_PASS)
    assert many.info()["chunk_wt"] == 6  # a ring of three slots of two work tiles
    E = dev(np.stack(fields(N, B, 70)), torch)
    R1 = torch.zeros((B, W, W), device="cuda")
    R2 = torch.zeros((B, W, W), device="cuda")
    srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R1, one)
    srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R2, many)
    torch.cuda.synchronize()
    assert many.info()["last_launches"] == 3 * 6  # 11 work tiles in chunks of 2
    assert torch.equal(R1, R2)
    # captured: the side stream forks from and joins the capturing stream
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    graph = torch.cuda.CUDAGraph()
    R3 = torch.zeros_like(R2)
    with torch.cuda.graph(graph, stream=stream):
        srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R3, many)
    new = np.stack(fields(N, B, 71))
    E.copy_(dev(new, torch))
    graph.replay()
    torch.cuda.synchronize()
    srk.srkTrainingForward(E, E, GX, GY, N, W, e, 1.0, B, None, R1, one)
    torch.cuda.synchronize()
    assert torch.equal(R3, R1)
    for b in (0, B - 1):
        assert rel_max_err(host(R3[b]), O.forward(new[b], new[b], Kx, Ky, e, 1.0)) < 1e-3
    del graph
