"""Parity at the benchmark's sizes.

The oracle cannot count scale 24 in test time, so the full-size graphs were
counted ahead of time on the CPU (tests/golden/make_golden_large.py: the
oracle's merge counter and its restatement of the reference's loop, on the
oracle's bit-exact twins of the device generators) and their totals and
per-vertex digests are golden values here. Beside them, size-independent
properties every correct count satisfies: the same total under both
orientations and under any relabelling of the vertices, per-vertex counts
summing to three times the total, and per-vertex counts of sampled vertices
(hubs included) equal to the oracle's count of edges among their neighbours.
"""
import hashlib

import numpy as np
import pytest

import oracle
import xxtric_b200 as xt
from conftest import load_golden_large

pytestmark = pytest.mark.gpu

LARGE = load_golden_large()


def digest(pv: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(pv, "<i8").tobytes()).hexdigest()


def check_large(name: str, t: int, pv: np.ndarray, n_edges: int) -> None:
    """Total, per-vertex digest and edge count against the CPU-pinned values."""
    f = LARGE[name]
    assert t == f["triangles"]
    assert n_edges == f["undirected"]
    assert int(pv.sum()) == f["per_vertex_sum"]
    assert digest(pv) == f["per_vertex_sha256"]


@pytest.fixture(scope="module")
def ctx():
    c = xt.Context(0)
    yield c
    c.close()


def rmat_device(ctx, scale, seed=1):
    import torch
    ne = 16 << scale
    s = torch.empty(ne, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    ctx.gen_rmat(scale, ne, seed, s, d)
    return s, d


def test_scale22_orientations_and_sampled_vertices(ctx):
    scale = 22
    n = 1 << scale
    s, d = rmat_device(ctx, scale)
    g_deg = ctx.graph_from_device_edges(n, len(s), s, d, xt.ORIENT_DEGREE)
    t_deg, pv = g_deg.count(per_vertex=True)
    g_deg_info = g_deg.info()
    g_deg.free()
    g_id = ctx.graph_from_device_edges(n, len(s), s, d, xt.ORIENT_ID)
    t_id = g_id.count()
    g_id.free()
    assert t_deg == t_id
    assert pv.sum() == 3 * t_deg
    check_large("rmat22", t_deg, pv, g_deg_info["n_edges"])
    off, tails = oracle.canon_csr(n, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    deg = np.diff(off)
    rng = np.random.default_rng(22)
    sel = np.concatenate([np.argsort(deg)[-32:], rng.choice(n, 2000, replace=False)])
    assert (oracle.local_counts(off, tails, sel) == pv[sel]).all()


def test_scale24_properties(ctx):
    import torch
    scale = 24
    n = 1 << scale
    s, d = rmat_device(ctx, scale)
    g = ctx.graph_from_device_edges(n, len(s), s, d, xt.ORIENT_DEGREE)
    inf = g.info()
    t, pv = g.count(per_vertex=True)
    assert g.count() == t  # global-only kernel agrees with the per-vertex one
    g.free()
    assert pv.sum() == 3 * t
    assert inf["n_edges"] == 260453894
    check_large("rmat24", t, pv, inf["n_edges"])
    # the reference's own precedence (u < v < w by input id, xxtric.hpp:165):
    # hubs keep up to ~200k higher neighbours, counted as CTA parts
    gi = ctx.graph_from_device_edges(n, len(s), s, d, xt.ORIENT_ID)
    assert gi.count() == t
    gi.free()
    # relabel every vertex by a random permutation: same total, permuted counts
    perm = torch.randperm(n, device="cuda", dtype=torch.int64).to(torch.int32)
    ps, pd = perm[s.long()], perm[d.long()]
    torch.cuda.synchronize()  # produced on torch's stream, read on the library's
    g2 = ctx.graph_from_device_edges(n, len(s), ps, pd, xt.ORIENT_DEGREE)
    t2, pv2 = g2.count(per_vertex=True)
    g2.free()
    assert t2 == t
    p = perm.cpu().numpy()
    assert (pv2[p] == pv).all()


def test_scale24_reference_layout_entry(ctx):
    """xt_count_device on the reference's own device CSR (int64 offsets and
    tails, symmetric) of the scale-22 graph equals the edge-list path."""
    import torch
    scale = 22
    n = 1 << scale
    s, d = rmat_device(ctx, scale, seed=5)
    g = ctx.graph_from_device_edges(n, len(s), s, d)
    t = g.count()
    g.free()
    assert t == LARGE["rmat22_seed5"]["triangles"]
    off, tails = oracle.canon_csr(n, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    d_off = torch.from_numpy(off).cuda()
    d_t = torch.from_numpy(tails).cuda()
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    xt.count_device(n, d_off, d_t, out, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(out.item()) == t


def test_size_limits(ctx):
    with pytest.raises(xt.XtError) as e:
        ctx.graph_from_edges(1 << 31, np.zeros(1, np.int32), np.zeros(1, np.int32))
    assert e.value.status == xt.XT_ERR_OVERFLOW


def test_chunglu_config_properties(ctx):
    """The heavy-skew workload at full size: Chung-Lu, n = 4,194,304, degree
    exponent 2.1, mean degree 64, expected maximum 131,072. Both orientations
    (the id order puts hubs on the part-split CTA tier), global and
    per-vertex counts, and the hubs' local counts against the oracle."""
    import torch
    n = 4194304
    cdf, m = xt.chunglu_cdf(n, 2.1, 64.0, 131072.0)
    s = torch.empty(m, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    ctx.gen_chunglu(cdf, m, 1, s, d)
    g = ctx.graph_from_device_edges(n, m, s, d, xt.ORIENT_DEGREE)
    t, pv = g.count(per_vertex=True)
    assert g.count() == t
    inf = g.info()
    g.free()
    assert pv.sum() == 3 * t
    g_id = ctx.graph_from_device_edges(n, m, s, d, xt.ORIENT_ID)
    t_id, pv_id = g_id.count(per_vertex=True)
    g_id.free()
    assert t_id == t and (pv_id == pv).all()
    check_large("chunglu_full", t, pv, inf["n_edges"])
    off, tails = oracle.canon_csr(n, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    deg = np.diff(off)
    assert inf["max_degree"] == deg.max() and inf["n_edges"] * 2 == len(tails)
    rng = np.random.default_rng(3)
    sel = np.concatenate([np.argsort(deg)[-32:], rng.choice(n, 2000, replace=False)])
    assert (oracle.local_counts(off, tails, sel) == pv[sel]).all()
