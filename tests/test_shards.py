"""The N>1 path of the edge-sharded count (xxtric_b200.shards) on CPU: two
gloo ranks each count a shard of one graph and the all-reduce sums the
parts. A CPU stand-in takes the GPU's place for each rank's part: it owns the
triangles whose lowest vertex is the rank modulo the world size (any split
of the triangles into disjoint shards sums the same way), credits them to
the global count and to all three corners, and the test checks the reduced
sums against the oracle's whole-graph counts."""
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

from conftest import load_fixtures, load_golden


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class _CpuShardGraph:
    """Stands in for a DeviceGraph: count_shard_async writes the shard's part
    into the given (CPU) tensors, as the GPU kernel does into device memory."""

    def __init__(self, off, tails):
        self.off, self.tails = off, tails

    @property
    def nv(self):
        return len(self.off) - 1

    def count_shard_async(self, shard, nshards, d_global, d_per_vertex=None):
        off, tails = self.off, self.tails
        tot = 0
        pv = np.zeros(self.nv, np.int64)
        for u in range(shard, self.nv, nshards):
            nu = tails[off[u]:off[u + 1]]
            nu = nu[nu > u]
            su = set(nu.tolist())
            for v in nu:
                for w in tails[off[v]:off[v + 1]]:
                    if w > v and w in su:
                        tot += 1
                        pv[u] += 1
                        pv[v] += 1
                        pv[w] += 1
        d_global[0] = tot
        if d_per_vertex is not None:
            d_per_vertex.copy_(torch.from_numpy(pv))


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import oracle
    from xxtric_b200 import replicas, shards
    replicas.init(backend="gloo", timeout_s=60)
    assert shards.world() == (rank, world)
    gold, fix = load_golden(), load_fixtures()
    res = {}
    for name in ("k64", "rmat10", "er0"):
        f = gold[name]
        off, tails = oracle.canon_csr(f["nv"], fix[name + "_src"].astype(np.int64), fix[name + "_dst"].astype(np.int64))
        g = _CpuShardGraph(off, tails)
        out = torch.zeros(1 + g.nv, dtype=torch.int64)
        t, pv = shards.count_sharded(g, per_vertex=True, out=out)
        res[name] = (t, pv.numpy().copy())
    # int64 parts stay exact past 2^53 through the collective
    big = torch.tensor([(1 << 61) + rank, -(1 << 60) + 3 * rank], dtype=torch.int64)
    shards.reduce_parts(big)
    q.put((rank, res, big.tolist()))
    replicas.finish()


def test_two_rank_sharded_count_sums_to_oracle():
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(180)
        assert p.exitcode == 0
    out = [q.get(timeout=10) for _ in range(2)]
    gold, fix = load_golden(), load_fixtures()
    for rank, res, big in out:
        assert big == [(1 << 62) + 1, -(1 << 61) + 3]
        for name, (t, pv) in res.items():
            f = gold[name]
            off, tails = oracle.canon_csr(f["nv"], fix[name + "_src"].astype(np.int64),
                                          fix[name + "_dst"].astype(np.int64))
            want, wpv = oracle.count_merge(off, tails, per_vertex=True)
            assert t == want == f["triangles"], (rank, name)
            assert (pv == wpv).all(), (rank, name)


def test_one_process_reduce_is_identity():
    from xxtric_b200 import shards
    x = torch.tensor([5, 1 << 62], dtype=torch.int64)
    assert shards.reduce_parts(x).tolist() == [5, 1 << 62]
    assert shards.world() == (0, 1)
