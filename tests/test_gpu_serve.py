"""The serving form: queries admitted under a memory budget, batched as slots
free up, each result identical to counting its graph alone.

Counts are integers: every comparison is exact. The oracle counts the small
graphs; the plain single-graph path (xt_graph_from_edges + xt_count) is the
solo result for the rest.
"""
import threading

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


def rmat_host(ctx, scale, seed, ef=16):
    import torch
    ne = ef << scale
    s = torch.empty(ne, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    ctx.gen_rmat(scale, ne, seed, s, d)
    return 1 << scale, s.cpu().numpy(), d.cpu().numpy()


def er_host(ctx, n, ne, seed):
    import torch
    s = torch.empty(ne, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    ctx.gen_er(n, ne, seed, s, d)
    return n, s.cpu().numpy(), d.cpu().numpy()


@pytest.fixture(scope="module")
def queries(ctx):
    """A mix of small R-MAT and Erdos-Renyi queries with their oracle counts."""
    qs = []
    for i in range(40):
        if i % 3 == 2:
            n, s, d = er_host(ctx, 200 + 37 * i, 8 * (200 + 37 * i), 100 + i)
        else:
            n, s, d = rmat_host(ctx, 6 + i % 8, 1000 + i)
        off, tails = oracle.canon_csr(n, s.astype(np.int64), d.astype(np.int64))
        qs.append((n, s, d, oracle.count_merge(off, tails)))
    return qs


def test_results_equal_solo_counts_alone_and_in_the_mix(ctx, queries):
    # solo: each graph through the plain path
    for n, s, d, expect in queries[:8]:
        g = ctx.graph_from_edges(n, s, d)
        assert g.count() == expect
        g.free()
    with xt.Server(0, slots=3) as srv:
        # alone: one query in flight at a time
        for n, s, d, expect in queries[:5]:
            assert srv.wait(srv.submit(n, s, d))[0] == expect
        assert srv.stats()["max_batch"] == 1
        # in the mix: two threads submit bursts while earlier batches run
        tickets = {}
        lock = threading.Lock()

        def feed(part):
            for k in part:
                n, s, d, _ = queries[k]
                t = srv.submit(n, s, d)
                with lock:
                    tickets[t] = k

        th = [threading.Thread(target=feed, args=(list(range(j, len(queries), 2)),)) for j in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        for t, k in tickets.items():
            count, lat = srv.wait(t, 60000)
            assert count == queries[k][3], k
            assert lat > 0
        st = srv.stats()
        assert st["completed"] == 5 + len(queries) and st["failed"] == 0
        assert st["max_batch"] > 1  # bursts were batched
        assert st["in_flight"] == 0 and st["queued"] == 0 and st["budget_used"] == 0
        assert st["launches"] > 0


def test_bad_query_fails_alone(ctx, queries):
    with xt.Server(0, slots=1) as srv:
        n, s, d, _ = queries[3]
        big_n, bs, bd = rmat_host(ctx, 15, 7)
        # a large query first keeps the only slot busy so the rest queue up and batch
        t0 = srv.submit(big_n, bs, bd)
        good = [srv.submit(*q[:3]) for q in queries[:6]]
        bad_s = s.copy()
        bad_s[len(bad_s) // 2] = n + 5  # an id outside [0, nv)
        bad = srv.submit(n, bad_s, d)
        good += [srv.submit(*q[:3]) for q in queries[6:12]]
        assert srv.wait(t0)[0] > 0
        for t, q in zip(good, queries[:6] + queries[6:12]):
            assert srv.wait(t)[0] == q[3]
        with pytest.raises(xt.XtError) as e:
            srv.wait(bad)
        assert e.value.status == xt.XT_ERR_INVALID
        st = srv.stats()
        assert st["failed"] == 1 and st["max_batch"] > 1
        # a result is handed out once
        with pytest.raises(xt.XtError) as e:
            srv.poll(good[0])
        assert e.value.status == xt.XT_ERR_INVALID


def test_admission_under_a_small_budget(ctx, queries):
    n18, s18, d18 = rmat_host(ctx, 16, 3)
    big = xt.serve_estimate(n18, len(s18))
    small_max = max(xt.serve_estimate(q[0], len(q[1])) for q in queries)
    budget = big + 2 * small_max  # the big query plus at most two small ones at a time
    with xt.Server(0, budget_bytes=budget, slots=3) as srv:
        assert srv.stats()["budget_bytes"] == budget
        n19, s19, d19 = rmat_host(ctx, 17, 4)
        with pytest.raises(xt.XtError) as e:  # can never fit
            srv.submit(n19, s19, d19)
        assert e.value.status == xt.XT_ERR_ADMISSION
        ts = [srv.submit(n18, s18, d18)] + [srv.submit(*q[:3]) for q in queries]
        t_big2 = srv.submit(n18, s18, d18)
        res = [srv.wait(t, 120000)[0] for t in ts]
        assert res[1:] == [q[3] for q in queries]
        assert srv.wait(t_big2)[0] == res[0]
        g = ctx.graph_from_edges(n18, s18, d18)
        assert g.count() == res[0]
        g.free()
        st = srv.stats()
        assert st["rejected"] == 1
        assert st["budget_peak"] <= budget
        # what the slots' allocations really held stays inside the budget
        assert 0 < st["device_peak"] <= budget


@pytest.mark.parametrize("scale", [10, 14, 18])
def test_estimate_bounds_measured_peak(ctx, scale):
    n, s, d = rmat_host(ctx, scale, 11)
    for orient in (xt.ORIENT_ID, xt.ORIENT_DEGREE):
        ctx.synchronize()
        live0, _ = ctx.mem_stats(reset_peak=True)
        g = ctx.graph_from_edges(n, s, d, orient)
        g.count()
        _, peak = ctx.mem_stats()
        g.free()
        assert ctx.mem_stats()[0] == live0  # everything released
        assert peak - live0 <= xt.serve_estimate(n, len(s)), (scale, orient, peak - live0)
    # a batch of graphs holds at most the sum of their estimates
    parts = [rmat_host(ctx, scale - k, 20 + k) for k in range(3)]
    voff = np.cumsum([0] + [p[0] for p in parts])
    eoff = np.cumsum([0] + [len(p[1]) for p in parts])
    ctx.synchronize()
    live0, _ = ctx.mem_stats(reset_peak=True)
    bg = ctx.graph_from_batch(voff, eoff, np.concatenate([p[1] for p in parts]), np.concatenate([p[2] for p in parts]))
    bg.count_groups()
    _, peak = ctx.mem_stats()
    bg.free()
    assert peak - live0 <= sum(xt.serve_estimate(p[0], len(p[1])) for p in parts)


def test_wait_timeout_and_close_with_queued_queries(ctx, queries):
    n, s, d = rmat_host(ctx, 17, 9)
    srv = xt.Server(0, slots=1)
    t = srv.submit(n, s, d)
    if srv.poll(t) is None:
        with pytest.raises(xt.XtError) as e:
            srv.wait(t, 0)
        assert e.value.status == xt.XT_ERR_TIMEOUT
    assert srv.wait(t)[0] > 0
    for q in queries:
        srv.submit(*q[:3])
    srv.close()  # fails what is still queued, finishes what runs, returns
    with xt.Server(0, slots=2) as srv2:  # the device is fine afterwards
        assert srv2.wait(srv2.submit(*queries[0][:3]))[0] == queries[0][3]
