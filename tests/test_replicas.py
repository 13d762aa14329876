"""The N>1 path of bench.py (independent replicas, max-over-ranks timing) on
CPU with the gloo backend and two ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from xxtric_b200 import replicas
    r, w, _ = replicas.init(backend="gloo", timeout_s=60)
    assert (r, w) == (rank, world)
    replicas.barrier()
    # rank k processed 100*(k+1) units in (k+1) seconds
    value, total, tmax = replicas.aggregate(100.0 * (rank + 1), 1.0 + rank)
    q.put((rank, value, total, tmax))
    replicas.finish()


def test_two_rank_aggregate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for _, value, total, tmax in res:
        assert total == 300.0 and tmax == 2.0 and value == 150.0


def test_single_process_is_identity():
    from xxtric_b200 import replicas
    assert replicas.aggregate(10.0, 2.0) == (5.0, 10.0, 2.0)
