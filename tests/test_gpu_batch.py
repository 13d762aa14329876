"""The batching form: many graphs built as one and counted in one launch.

Per-graph counts must equal the oracle's count of each graph (small batch)
and the plain single-graph path's count (the full 4,096-graph workload), for
the direct launch, the captured CUDA-graph replay and after autotuning.
"""
import numpy as np
import pytest

import oracle
import xxtric_b200 as xt

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = xt.Context(0)
    yield c
    c.close()


def take(spec, idx):
    return {k: np.ascontiguousarray(v[idx]) for k, v in spec.items()}


def host_edges(torch, eoff, d_src, d_dst):
    s = torch.as_tensor(d_src, device="cuda").cpu().numpy() if eoff[-1] else np.zeros(0, np.int32)
    d = torch.as_tensor(d_dst, device="cuda").cpu().numpy() if eoff[-1] else np.zeros(0, np.int32)
    return s, d


def test_small_batch_generators_and_counts_vs_oracle(ctx):
    import torch
    full = xt.batch_spec(4096, 7)
    idx = np.arange(48)
    idx = idx[full["n"][idx] <= 20000][:24]  # a mixed handful the oracle counts quickly
    spec = take(full, idx)
    eoff, d_src, d_dst = ctx.gen_batch(spec)
    s, d = host_edges(torch, eoff, d_src, d_dst)
    voff = np.concatenate([[0], np.cumsum(spec["n"])])
    expect = []
    for g in range(len(idx)):
        os_, od_ = oracle.batch_graph(spec["kind"][g], spec["n"][g], spec["mean_deg"][g], spec["graph_seed"][g])
        gs, gd = s[eoff[g]:eoff[g + 1]].astype(np.int64), d[eoff[g]:eoff[g + 1]].astype(np.int64)
        n = int(spec["n"][g])
        # the same edge set as the oracle's twin generator
        a = oracle.canon_csr(n, gs, gd)
        b = oracle.canon_csr(n, os_, od_)
        assert (a[0] == b[0]).all() and (a[1] == b[1]).all(), g
        expect.append(oracle.count_merge(*b))
    for orient in (xt.ORIENT_ID, xt.ORIENT_DEGREE):
        bg = ctx.graph_from_batch(voff, eoff, d_src, d_dst, orient, device=True)
        assert bg.groups == len(idx)
        total, per = bg.count_groups()
        assert per.tolist() == expect
        assert total == sum(expect)
        bg.capture()
        for _ in range(2):
            t2, per2 = bg.count_groups()
            assert t2 == total and (per2 == per).all()
        bg.free()
    # host-buffer entry points: the graph object and the one-call count
    bg = ctx.graph_from_batch(voff, eoff, s, d)
    assert bg.count_groups()[1].tolist() == expect
    bg.free()
    total1, per1 = ctx.batch_count(voff, eoff, s, d)
    assert per1.tolist() == expect and total1 == sum(expect)
    # capture while the context runs on the legacy default stream (handle 0),
    # which cannot itself be captured; replays still count on it
    c0 = xt.Context(0)
    c0.set_stream(0)
    bg = c0.graph_from_batch(voff, eoff, s, d)
    bg.capture()
    l0 = c0.launches
    for _ in range(2):
        assert bg.count_groups()[1].tolist() == expect
    assert c0.launches > l0  # replayed kernels are counted
    bg.free()
    c0.close()
    d_src.free()
    d_dst.free()


def test_full_batch_matches_plain_path(ctx):
    import torch
    spec = xt.batch_spec(4096, 1)
    eoff, d_src, d_dst = ctx.gen_batch(spec)
    voff = np.concatenate([[0], np.cumsum(spec["n"])])
    bg = ctx.graph_from_batch(voff, eoff, d_src, d_dst, device=True)
    total, per = bg.count_groups()
    assert total == per.sum()
    bg.capture()
    t2, per2 = bg.count_groups()
    assert t2 == total and (per2 == per).all()
    report = bg.autotune(reps=1)
    assert "best" in report or report.get("cached")
    t3, per3 = bg.count_groups()
    assert t3 == total and (per3 == per).all()
    bg.free()
    # the plain single-graph path on a sample of the graphs
    ts = torch.as_tensor(d_src, device="cuda")
    td = torch.as_tensor(d_dst, device="cuda")
    rng = np.random.default_rng(0)
    sample = np.concatenate([rng.choice(4096, 40, replace=False), [int(np.argmax(spec["n"]))]])
    for g in sample:
        e0, e1 = int(eoff[g]), int(eoff[g + 1])
        pg = ctx.graph_from_device_edges(int(spec["n"][g]), e1 - e0, ts[e0:e1], td[e0:e1])
        assert pg.count() == per[g], g
        pg.free()
    d_src.free()
    d_dst.free()


def test_batch_rejects_bad_tables(ctx):
    with pytest.raises(xt.XtError) as e:
        ctx.graph_from_batch(np.array([0, 3, 2]), np.array([0, 1, 1]), np.array([0], np.int32),
                             np.array([1], np.int32))
    assert e.value.status == xt.XT_ERR_INVALID
    with pytest.raises(xt.XtError) as e:  # vertex 3 is outside graph 0's three vertices
        ctx.graph_from_batch(np.array([0, 3, 5]), np.array([0, 1, 1]), np.array([3], np.int32),
                             np.array([1], np.int32))
    assert e.value.status == xt.XT_ERR_INVALID
    g = ctx.graph_from_batch(np.array([0, 3, 6]), np.array([0, 3, 4]), np.array([0, 1, 2, 0], np.int32),
                             np.array([1, 2, 0, 1], np.int32))
    total, per = g.count_groups()
    assert total == 1 and per.tolist() == [1, 0]
    g.free()
