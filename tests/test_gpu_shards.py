"""Edge-sharded counting on the GPU: the shards of one graph's schedule
(xt_count_shard_async, xt_count_edges_shard_async) sum to the whole count,
per-vertex counts and per-edge supports, checked against the oracle, for
every tier alone and mixed, both orientations and the cluster tier. One GPU
runs the shards one after another: the same kernels each rank of
xxtric_b200.shards runs on its own GPU before the all-reduce."""
import numpy as np
import pytest

import oracle
import xxtric_b200 as xt
from xxtric_b200 import shards

pytestmark = pytest.mark.gpu

ORIENTS = [xt.ORIENT_ID, xt.ORIENT_DEGREE]
# (lane_work, warp_work): every head on one tier, then the automatic mix
TIERS = [(1 << 40, 0), (0, 1 << 40), (0, 0), (-1, -1)]


@pytest.fixture(scope="module")
def ctx():
    c = xt.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


def _graph_edges(ctx, torch, kind):
    if kind == "rmat":
        n, m = 1 << 14, 16 << 14
        s = torch.empty(m, dtype=torch.int32, device="cuda")
        d = torch.empty_like(s)
        ctx.gen_rmat(14, m, 7, s, d)
    else:
        n = 1 << 15
        cdf, m = xt.chunglu_cdf(n, 2.1, 24.0, 8192.0)
        s = torch.empty(m, dtype=torch.int32, device="cuda")
        d = torch.empty_like(s)
        ctx.gen_chunglu(cdf, m, 9, s, d)
    torch.cuda.synchronize()
    return n, m, s, d


def _shard_sums(g, torch, nshards, nv, ne):
    """Sums over the nshards shards of (global, per-vertex, per-edge)."""
    tot, pv, sup = 0, np.zeros(nv, np.int64), np.zeros(ne, np.int64)
    dg = torch.zeros(1, dtype=torch.int64, device="cuda")
    dp = torch.full((nv,), -1, dtype=torch.int64, device="cuda")
    ds = torch.full((max(ne, 1),), -1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    for k in range(nshards):
        g.count_shard_async(k, nshards, dg, dp)
        g.ctx.synchronize()
        tot += int(dg.item())
        pv += dp.cpu().numpy()
        g.count_edges_shard_async(k, nshards, dg, ds)
        g.ctx.synchronize()
        sup += ds.cpu().numpy()[:ne]
    return tot, pv, sup


@pytest.mark.parametrize("kind", ["rmat", "chunglu"])
def test_shards_sum_to_whole(ctx, torch_cuda, kind):
    torch = torch_cuda
    n, m, s, d = _graph_edges(ctx, torch, kind)
    off, tails = oracle.canon_csr(n, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    expect, opv = oracle.count_merge(off, tails, per_vertex=True)
    for orient in ORIENTS:
        g = ctx.graph_from_device_edges(n, m, s, d, orient)
        try:
            ne = g.info()["n_edges"]
            for lane_work, warp_work in TIERS:
                g.set_tiers(lane_work, warp_work)
                whole_t, whole_sup = g.count_edges()
                assert whole_t == expect
                for nshards in (1, 2, 3, 8):
                    t, pv, sup = _shard_sums(g, torch, nshards, n, ne)
                    assert t == expect, (orient, lane_work, warp_work, nshards)
                    assert (pv == opv).all(), (orient, lane_work, warp_work, nshards)
                    assert (sup == whole_sup).all(), (orient, lane_work, warp_work, nshards)
            # a shard may hold no task of a short list: more shards than tasks
            g.set_tiers(-1, -1)
            t, pv, _ = _shard_sums(g, torch, 64, n, ne)
            assert t == expect and (pv == opv).all()
        finally:
            g.free()


def test_shards_with_cluster_tier(ctx, torch_cuda):
    # under the id orientation the Chung-Lu hubs outgrow a CTA's member set:
    # the cluster tier's task list is sharded like the others
    torch = torch_cuda
    n, m, s, d = _graph_edges(ctx, torch, "chunglu")
    off, tails = oracle.canon_csr(n, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    expect = oracle.count_merge(off, tails)
    g = ctx.graph_from_device_edges(n, m, s, d, xt.ORIENT_ID)
    try:
        g.set_cluster(True)
        assert g.count() == expect
        dg = torch.zeros(1, dtype=torch.int64, device="cuda")
        for nshards in (2, 5):
            tot = 0
            for k in range(nshards):
                g.count_shard_async(k, nshards, dg)
                g.ctx.synchronize()
                tot += int(dg.item())
            assert tot == expect, nshards
    finally:
        g.free()


def test_count_sharded_one_rank(ctx, torch_cuda):
    # without a process group the sharded count is the whole count
    torch = torch_cuda
    n, m, s, d = _graph_edges(ctx, torch, "rmat")
    off, tails = oracle.canon_csr(n, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    expect, opv = oracle.count_merge(off, tails, per_vertex=True)
    with xt.Context(0) as c2:
        # the library on torch's stream, so the all-reduce (none at one rank) follows the count
        c2.set_stream(torch.cuda.current_stream().cuda_stream)
        g = c2.graph_from_device_edges(n, m, s, d, xt.ORIENT_DEGREE)
        try:
            t, pv = shards.count_sharded(g, per_vertex=True)
            assert t == expect and (pv.cpu().numpy() == opv).all()
            t2, sup = shards.count_edges_sharded(g)
            assert t2 == expect and int(sup.sum().item()) == 3 * expect
        finally:
            g.free()


def test_shard_arguments_checked(ctx, torch_cuda):
    torch = torch_cuda
    n, m, s, d = _graph_edges(ctx, torch, "rmat")
    g = ctx.graph_from_device_edges(n, m, s, d, xt.ORIENT_DEGREE)
    try:
        dg = torch.zeros(1, dtype=torch.int64, device="cuda")
        for shard, nshards in ((2, 2), (-1, 2), (0, 0)):
            with pytest.raises(xt.XtError):
                g.count_shard_async(shard, nshards, dg)
        assert g.count() > 0  # the context is still usable
    finally:
        g.free()
