"""Multi-rank host logic of the data-parallel path, on CPU with gloo
(world_size 2 and 3): shards tile the batch exactly once and the step time
reported is the max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from shrinkage_full_tests_b200.shard import batch_shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, B, q):
    import torch
    import torch.distributed as dist
    from shrinkage_full_tests_b200.shard import batch_shard, max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    start, count = batch_shard(B, rank, world)
    mine = torch.zeros(B, dtype=torch.int64)
    mine[start:start + count] = 1
    dist.all_reduce(mine)
    t = max_over_ranks(1.0 + rank, dist)
    q.put((rank, mine.tolist(), t))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,B", [(2, 5000), (3, 7)])
def test_batch_shards_cover_once_and_time_is_max(world, B):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, B, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, cover, t in res:
        assert cover == [1] * B
        assert t == float(world)


def test_batch_shard_edges():
    assert batch_shard(10, 0, 3) == (0, 4)
    assert batch_shard(10, 2, 3) == (7, 3)
    assert batch_shard(0, 0, 2) == (0, 0)
    with pytest.raises(ValueError):
        batch_shard(5, 2, 2)


# ---- one image split by column slabs --------------------------------------
# Each rank computes its own output columns after the halo exchange; the
# local compute here is the FP64 oracle on an image that is zero outside the
# rank's halo'd columns, so any missing halo column changes the result and
# the stitched slabs must equal the whole-image oracle exactly.
SLAB_N, SLAB_KW, SLAB_STRIDE = 64, 11, 12


def _embed(h, lo, n_cols, rows):
    import numpy as np
    full = np.zeros((n_cols, rows))
    full[lo:lo + h.shape[0]] = h
    return full


def _slab_worker(rank, world, port, q):
    import numpy as np
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    from shrinkage_full_tests_b200 import shard
    from tests.helpers import fields, kernel
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    N, KW, S = SLAB_N, SLAB_KW, SLAB_STRIDE
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    f, g, df, dg = fields(N, 4, 300)
    rng = np.random.default_rng(3)
    v, ux, uy = (rng.standard_normal((W, W)) for _ in range(3))
    owns = shard.slab_bounds(N, e, S, world)
    lo, hi = owns[rank]
    wlo, whi = min(lo, W), min(hi, W)
    T = lambda a, a0, a1: torch.from_numpy(np.ascontiguousarray(a[a0:a1], np.float64))

    def fwd_op(E_h, I_h, c0, c1, R):
        Ef = _embed(E_h.numpy(), c0, N, N)
        If = _embed(I_h.numpy(), c0, N, N)
        R.copy_(torch.from_numpy(O.forward(Ef, If, Kx, Ky, e, 1.0, window=(c0, 0, c1 - c0, W))))

    def tan_op(f_h, g_h, df_h, dg_h, c0, c1, dh):
        emb = [_embed(t.numpy(), c0, N, N) for t in (f_h, g_h, df_h, dg_h)]
        dh.copy_(torch.from_numpy(O.tangent(*emb, Kx, Ky, e, 1.0)[c0:c1]))

    def adj_op(v_h, ux_h, uy_h, I_h, c0, c1, dLdI, dLdE):
        # the views start at column c0; their halo lies before them in storage
        vb = [t._base if t._base is not None else t for t in (v_h, ux_h, uy_h, I_h)]
        k = [t.storage_offset() // t.shape[1] for t in (v_h, ux_h, uy_h, I_h)]
        ve, uxe, uye = (_embed(b.numpy(), c0 - kk, W, W) for b, kk in zip(vb[:3], k[:3]))
        Ie = _embed(vb[3].numpy(), c0 - k[3], N, N)
        dLdI.copy_(torch.from_numpy(O.adj_wrt_I(ve, uxe, uye, N, e)[c0:c1]))
        dLdE.copy_(torch.from_numpy(O.adj_wrt_E(ve, Ie, Kx, Ky, e, 1.0, "true")[c0:c1]))

    def ta_op(f_h, g_h, df_h, dg_h, lam_h, dlam_h, c0, c1, dlf, dlg):
        emb = []
        for t, n_cols, rows in ((f_h, N, N), (g_h, N, N), (df_h, N, N), (dg_h, N, N), (lam_h, W, W), (dlam_h, W, W)):
            b = t._base if t._base is not None else t
            emb.append(_embed(b.numpy(), c0 - t.storage_offset() // t.shape[1], n_cols, rows))
        of, og = O.tangent_adjoint(*emb, Kx, Ky, e, 1.0, "true")
        dlf.copy_(torch.from_numpy(of[c0:c1]))
        dlg.copy_(torch.from_numpy(og[c0:c1]))

    R = shard.forward_slabs(T(g, lo, hi), T(f, lo, hi), N, e, S, rank, world, dist, fwd_op)
    dh = shard.tangent_slabs(T(f, lo, hi), T(g, lo, hi), T(df, lo, hi), T(dg, lo, hi), N, e, S, rank, world, dist,
                             tan_op)
    dI, dE = shard.adjoint_slabs(T(v, wlo, whi), T(ux, wlo, whi), T(uy, wlo, whi), T(f, lo, hi), N, e, S, rank,
                                 world, dist, adj_op)
    lam, dlam = (rng.standard_normal((W, W)) for _ in range(2))
    tf, tg = shard.tangent_adjoint_slabs(T(f, lo, hi), T(g, lo, hi), T(df, lo, hi), T(dg, lo, hi), T(lam, wlo, whi),
                                         T(dlam, wlo, whi), N, e, S, rank, world, dist, ta_op)
    q.put((rank, (lo, hi), R.numpy(), dh.numpy(), dI.numpy(), dE.numpy(), tf.numpy(), tg.numpy()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_column_slabs_with_halo_exchange_match_whole_image(world):
    import numpy as np
    from oracle import oracle as O
    from tests.helpers import fields, kernel
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(world)], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    N, KW = SLAB_N, SLAB_KW
    e = (KW - 1) // 2
    W = N - 2 * e
    Kx, Ky = kernel(KW)
    f, g, df, dg = fields(N, 4, 300)
    rng = np.random.default_rng(3)
    v, ux, uy = (rng.standard_normal((W, W)) for _ in range(3))
    assert [r[1] for r in res][0][0] == 0 and res[-1][1][1] == N
    assert all(res[i][1][1] == res[i + 1][1][0] for i in range(world - 1))
    assert np.array_equal(np.concatenate([r[2] for r in res]), O.forward(g, f, Kx, Ky, e, 1.0))
    assert np.array_equal(np.concatenate([r[3] for r in res]), O.tangent(f, g, df, dg, Kx, Ky, e, 1.0))
    assert np.array_equal(np.concatenate([r[4] for r in res]), O.adj_wrt_I(v, ux, uy, N, e))
    assert np.array_equal(np.concatenate([r[5] for r in res]), O.adj_wrt_E(v, f, Kx, Ky, e, 1.0, "true"))
    lam, dlam = (rng.standard_normal((W, W)) for _ in range(2))
    of, og = O.tangent_adjoint(f, g, df, dg, lam, dlam, Kx, Ky, e, 1.0, "true")
    assert np.array_equal(np.concatenate([r[6] for r in res]), of)
    assert np.array_equal(np.concatenate([r[7] for r in res]), og)


def test_slab_bounds_whole_tiles():
    from shrinkage_full_tests_b200.shard import slab_bounds
    b = slab_bounds(32768, 60, 392, 8)
    assert b[0][0] == 0 and b[-1][1] == 32768
    assert all(lo % 392 == 0 for lo, _ in b) and all(b[i][1] == b[i + 1][0] for i in range(7))
    assert slab_bounds(100, 10, 40, 4)[0] == (0, 0)  # two tile columns over four ranks
