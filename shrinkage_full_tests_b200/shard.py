"""Data-parallel sharding of the batched training forward.

The B images of srkTrainingForward are independent, so N GPUs split the batch
into contiguous shards and run with no data-path collective
(training/srk_training_forward.cuh:148-155 batches the same way on one GPU).
Timing across ranks is the max of the per-rank device times.
"""


def batch_shard(B, rank, world):
    """Contiguous shard [start, start+count) of a batch of B images for `rank`
    of `world`; the first B % world ranks take one extra image."""
    if world < 1 or not (0 <= rank < world) or B < 0:
        raise ValueError("bad shard request B=%d rank=%d world=%d" % (B, rank, world))
    base, extra = divmod(B, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def max_over_ranks(value, dist=None, device=None):
    """Max of a per-rank float over the process group (identity without one)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---- one image split by columns across ranks ------------------------------
# Column-major images are column slabs in memory: rank r owns the image
# columns [lo_r, hi_r) of every N-sized array and the columns
# [lo_r, min(hi_r, W)) of every W-sized one.  Each op is output-partitioned:
# a rank computes the output columns it owns after one halo exchange IN
# (point-to-point sends of the neighbouring ranks' columns, over NCCL or
# gloo), so no output is reduced across ranks.  Halos (in columns):
#   forward, tangent: N-sized inputs [lo, hi + 2e)
#   adjoint: W-sized v, ux, uy [lo - 2e, hi); I [lo - e - 1, hi + e + 1)
# The interior boundaries are multiples of the plan's tile stride, so every
# slab spans whole tiles (srk_forward_oas_slab and friends).


def slab_bounds(N, erosion, stride, world):
    """Image-column ownership [lo, hi) of every rank for one N x N image:
    the tile columns of the W x W output split as evenly as possible
    (ranks past the tile count own nothing)."""
    W = N - 2 * erosion
    if world < 1 or stride < 1 or W < 1:
        raise ValueError("bad slab request N=%d erosion=%d stride=%d world=%d" % (N, erosion, stride, world))
    T = -(-W // stride)
    cuts = [0] + [(r * T // world) * stride for r in range(1, world)] + [N]
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def _clip(lo, hi, n):
    lo, hi = max(lo, 0), min(hi, n)
    return (lo, hi) if lo < hi else (lo, lo)


def exchange_columns(x, own, need, owns, needs, rank, dist):
    """Columns need = [a, b) of an array whose columns are spread over the
    ranks (rank q owns owns[q]); x holds this rank's own columns as a
    [cols, rows] tensor.  Every rank sends each other rank the part of its
    own columns that the other needs (needs[q]), in one batch of
    point-to-point operations."""
    if tuple(need) == tuple(own) and all(tuple(n) == tuple(o) for n, o in zip(needs, owns)):
        return x  # nothing crosses ranks (one rank)
    rows = x.shape[1]
    out = x.new_zeros((need[1] - need[0], rows))
    lo, hi = max(own[0], need[0]), min(own[1], need[1])
    if lo < hi:
        out[lo - need[0]:hi - need[0]] = x[lo - own[0]:hi - own[0]]
    ops, keep = [], []  # keep: send buffers alive until the waits
    for q in range(len(owns)):
        if q == rank:
            continue
        lo, hi = max(own[0], needs[q][0]), min(own[1], needs[q][1])
        if lo < hi:
            t = x[lo - own[0]:hi - own[0]].contiguous()
            keep.append(t)
            ops.append(dist.P2POp(dist.isend, t, q))
        lo, hi = max(owns[q][0], need[0]), min(owns[q][1], need[1])
        if lo < hi:
            ops.append(dist.P2POp(dist.irecv, out[lo - need[0]:hi - need[0]], q))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    return out


def _w_owns(owns, W):
    return [_clip(lo, hi, W) for lo, hi in owns]


def forward_slabs(E, I, N, erosion, stride, rank, world, dist, op):
    """Output columns [lo, min(hi, W)) of srkForwardOaS for this rank's slab.
    E, I: this rank's own image columns ([hi - lo, N] tensors; I may be E).
    op(E_h, I_h, c0, c1, R) computes the slab from halo'd inputs whose row 0
    is column c0 (srk_forward_oas_slab on the device)."""
    W = N - 2 * erosion
    owns = slab_bounds(N, erosion, stride, world)
    needs = [_clip(lo, hi + 2 * erosion, N) if lo < hi else (lo, lo) for lo, hi in owns]
    E_h = exchange_columns(E, owns[rank], needs[rank], owns, needs, rank, dist)
    I_h = E_h if I is E else exchange_columns(I, owns[rank], needs[rank], owns, needs, rank, dist)
    c0, c1 = _w_owns(owns, W)[rank]
    R = E.new_zeros((c1 - c0, W))
    if c0 < c1:
        op(E_h, I_h, c0, c1, R)
    return R


def tangent_slabs(f, g, df, dg, N, erosion, stride, rank, world, dist, op):
    """Output columns [lo, min(hi, W)) of shrinkageTangentOaS;
    op(f_h, g_h, df_h, dg_h, c0, c1, dh) as in forward_slabs."""
    W = N - 2 * erosion
    owns = slab_bounds(N, erosion, stride, world)
    needs = [_clip(lo, hi + 2 * erosion, N) if lo < hi else (lo, lo) for lo, hi in owns]
    hal = [exchange_columns(x, owns[rank], needs[rank], owns, needs, rank, dist) for x in (f, g, df, dg)]
    c0, c1 = _w_owns(owns, W)[rank]
    dh = f.new_zeros((c1 - c0, W))
    if c0 < c1:
        op(*hal, c0, c1, dh)
    return dh


def adjoint_slabs(v, ux, uy, I, N, erosion, stride, rank, world, dist, op):
    """Columns [lo, hi) of adjointSRK's dL/dI and dL/dE for this rank.  v, ux,
    uy: own W-sized columns [lo, min(hi, W)); I: own image columns.
    op(v_h, ux_h, uy_h, I_h, c0, c1, dLdI, dLdE) gets halo'd tensors whose
    row 0 is column c0 (the halo before it is at negative offsets, as
    srk_adjoint_slab reads it)."""
    e = erosion
    W = N - 2 * e
    owns = slab_bounds(N, e, stride, world)
    wowns = _w_owns(owns, W)
    vneeds = [_clip(lo - 2 * e, min(hi, W), W) if lo < hi else (0, 0) for lo, hi in owns]
    ineeds = [_clip(lo - e - 1, hi + e + 1, N) if lo < hi else (lo, lo) for lo, hi in owns]
    vh = [exchange_columns(x, wowns[rank], vneeds[rank], wowns, vneeds, rank, dist) for x in (v, ux, uy)]
    Ih = exchange_columns(I, owns[rank], ineeds[rank], owns, ineeds, rank, dist)
    lo, hi = owns[rank]
    dLdI = I.new_zeros((hi - lo, N))
    dLdE = I.new_zeros((hi - lo, N))
    if lo < hi:
        kv, ki = lo - vneeds[rank][0], lo - ineeds[rank][0]
        op(*[t[kv:] for t in vh], Ih[ki:], lo, hi, dLdI, dLdE)
    return dLdI, dLdE


def ta_wrange(lo, hi, N, erosion, stride):
    """W-columns [r0, rE) of the tangent-adjoint's intermediate that its slab
    [lo, hi) computes by whole tiles (srk_tangent_adjoint_slab)."""
    e = erosion
    W = N - 2 * e
    r0, r1 = max(lo - e - 1, 0), min(hi - e + 1, W)
    if r1 <= r0:
        return r0, r0
    T = -(-(r1 - r0) // stride)
    return r0, min(r0 + T * stride, W)


def tangent_adjoint_slabs(f, g, df, dg, lam, dlam, N, erosion, stride, rank, world, dist, op):
    """Columns [lo, hi) of shrinkageTangentAdjointOaS's dLam_f and dLam_g.
    f, g, df, dg: own image columns; lam, dlam: own W-sized columns.
    op(f_h, g_h, df_h, dg_h, lam_h, dlam_h, c0, c1, dLam_f, dLam_g) gets views
    whose row 0 is column c0 (the halos of srk_tangent_adjoint_slab around
    them)."""
    e = erosion
    W = N - 2 * e
    owns = slab_bounds(N, e, stride, world)
    wowns = _w_owns(owns, W)
    fneeds, gneeds, lneeds = [], [], []
    for lo, hi in owns:
        if lo == hi:
            fneeds.append((lo, lo))
            gneeds.append((lo, lo))
            lneeds.append((0, 0))
            continue
        r0, rE = ta_wrange(lo, hi, N, e, stride)
        fneeds.append(_clip(lo - e - 1, hi + e + 1, N))
        gneeds.append(_clip(min(r0, lo), max(rE + 2 * e, lo + 1), N))
        lneeds.append(_clip(min(lo - 2 * e, r0), max(min(hi, W), rE, lo + 1), W))
    fh = [exchange_columns(x, owns[rank], fneeds[rank], owns, fneeds, rank, dist) for x in (f, df)]
    gh = [exchange_columns(x, owns[rank], gneeds[rank], owns, gneeds, rank, dist) for x in (g, dg)]
    lh = [exchange_columns(x, wowns[rank], lneeds[rank], wowns, lneeds, rank, dist) for x in (lam, dlam)]
    lo, hi = owns[rank]
    dlf = f.new_zeros((hi - lo, N))
    dlg = f.new_zeros((hi - lo, N))
    if lo < hi:
        kf, kg, kl = lo - fneeds[rank][0], lo - gneeds[rank][0], lo - lneeds[rank][0]
        op(fh[0][kf:], gh[0][kg:], fh[1][kf:], gh[1][kg:], lh[0][kl:], lh[1][kl:], lo, hi, dlf, dlg)
    return dlf, dlg


def device_slab_ops(plan, Gx, Gy, N, erosion, dx, stream=None):
    """The device ops for forward_slabs / tangent_slabs / adjoint_slabs
    (tangent_adjoint_slabs: device_tangent_adjoint_slab_op)."""
    from . import srkForwardOaSSlab, shrinkageTangentOaSSlab, adjointSRKSlab

    def fwd(E_h, I_h, c0, c1, R):
        srkForwardOaSSlab(E_h, I_h, Gx, Gy, N, erosion, dx, c0, c1, stream, R, plan)

    def tan(f_h, g_h, df_h, dg_h, c0, c1, dh):
        shrinkageTangentOaSSlab(f_h, g_h, df_h, dg_h, Gx, Gy, N, erosion, dx, c0, c1, stream, dh, plan)

    def adj(v_h, ux_h, uy_h, I_h, c0, c1, dLdI, dLdE):
        adjointSRKSlab(v_h, ux_h, uy_h, I_h, Gx, Gy, N, erosion, dx, c0, c1, stream, dLdI, dLdE, plan)

    return fwd, tan, adj


def device_tangent_adjoint_slab_op(plan, Gx, Gy, N, erosion, dx, stream=None):
    """The device op for tangent_adjoint_slabs."""
    from . import shrinkageTangentAdjointOaSSlab

    def tadj(f_h, g_h, df_h, dg_h, lam_h, dlam_h, c0, c1, dlf, dlg):
        shrinkageTangentAdjointOaSSlab(f_h, g_h, df_h, dg_h, lam_h, dlam_h, Gx, Gy, N, erosion, dx, c0, c1, stream,
                                       dlf, dlg, plan)

    return tadj
