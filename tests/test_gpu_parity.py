"""Parity of the CUDA path with the oracle and the reference's golden counts.

Every test here runs the product through the C ABI (libxtb200.so) on the
GPU and checks it against golden vectors from the reference binary or the
oracle on the same seeded inputs. Integer counts: bit-exact, no tolerance.
"""
import numpy as np
import pytest

import oracle
import xxtric_b200 as xt
from conftest import load_fixtures, load_golden

pytestmark = pytest.mark.gpu

GOLDEN = load_golden()
FIX = load_fixtures()
EDGE_NAMES = [n for n in GOLDEN if n + "_src" in FIX]
ORIENTS = [xt.ORIENT_ID, xt.ORIENT_DEGREE]


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


def canon(name):
    f = GOLDEN[name]
    return oracle.canon_csr(f["nv"], FIX[name + "_src"].astype(np.int64), FIX[name + "_dst"].astype(np.int64))


@pytest.mark.parametrize("orient", ORIENTS)
@pytest.mark.parametrize("name", EDGE_NAMES)
def test_golden_from_edges(ctx, name, orient):
    f = GOLDEN[name]
    g = ctx.graph_from_edges(f["nv"], FIX[name + "_src"], FIX[name + "_dst"], orient)
    try:
        t, pv = g.count(per_vertex=True)
        assert t == f["triangles"]
        off, tails = canon(name)
        _, opv = oracle.count_merge(off, tails, per_vertex=True)
        assert (pv == opv).all()
        assert g.info()["n_edges"] == f["undirected"]
    finally:
        g.free()


@pytest.mark.parametrize("canonical", [True, False])
@pytest.mark.parametrize("name", ["k4", "iso_tail", "k64", "star_path", "er0", "rmat14", "chunglu14", "amazon0302"])
def test_golden_from_reference_csr(ctx, name, canonical):
    # the vite-layout CSR the reference engine takes (xxtric-gpu.hpp:116-121)
    off, tails = canon(name)
    for orient in ORIENTS:
        g = ctx.graph_from_csr(off, tails, canonical=canonical, orient=orient)
        try:
            assert g.count() == GOLDEN[name]["triangles"]
        finally:
            g.free()


def test_noncanonical_input_is_canonicalised(ctx):
    # repeated pairs, one-directional rows and self loops: the builder
    # dedups, so the count equals the reference's on the canonical file
    s = np.array([0, 0, 0, 1, 1, 2, 0, 1, 2, 3, 3], np.int32)
    d = np.array([1, 2, 3, 2, 3, 3, 1, 0, 2, 3, 0], np.int32)
    for orient in ORIENTS:
        g = ctx.graph_from_edges(4, s, d, orient)
        assert g.count() == 4
        g.free()
    # a raw (unsorted, duplicated) CSR through the non-canonical path
    off = np.array([0, 4, 6, 8, 10], np.int64)
    tails = np.array([3, 1, 2, 1, 0, 2, 0, 1, 0, 2], np.int64)
    g = ctx.graph_from_csr(off, tails, canonical=False)
    assert g.count() == 2  # edges 01 02 03 12 23: triangles 012 and 023
    g.free()


@pytest.mark.parametrize("orient", ORIENTS)
def test_canonical_flag_checks_its_promise(ctx, orient):
    """XT_CSR_CANONICAL skips the sort, so rows that break the promise (out of
    order, a repeated id, the row's own id, an edge listed from one end only)
    are rejected on the device before any build or count kernel uses them,
    and the context stays usable."""
    bad = [
        ([0, 2, 4, 6], [2, 1, 0, 2, 0, 1]),      # row 0 out of order
        ([0, 3, 5, 7], [1, 1, 2, 0, 2, 0, 1]),   # row 0 repeats 1
        ([0, 3, 5, 7], [0, 1, 2, 0, 2, 0, 1]),   # row 0 holds 0
        ([0, 2, 3, 5], [1, 2, 2, 0, 1]),         # row 0 lists 1, row 1 lacks 0
        ([0, 1, 3, 5], [2, 0, 2, 0, 1]),         # row 1 lists 0, row 0 lacks 1
    ]
    for o, t in bad:
        with pytest.raises(xt.XtError) as e:
            ctx.graph_from_csr(np.array(o, np.int64), np.array(t, np.int64), canonical=True, orient=orient)
        assert e.value.status == xt.XT_ERR_INVALID, (o, t)
        # the same rows through the sorting path are canonicalised and counted
        g = ctx.graph_from_csr(np.array(o, np.int64), np.array(t, np.int64), canonical=False, orient=orient)
        assert g.count() == 1
        g.free()
    off, tails = canon("k64")
    g = ctx.graph_from_csr(off, tails, canonical=True, orient=orient)
    assert g.count() == GOLDEN["k64"]["triangles"]
    g.free()


def test_count_device_rejects_broken_rows(torch_cuda):
    """The reference-layout launcher (xt_count_device) takes the canonical
    path too: a row out of order is rejected and the counter keeps its value."""
    torch = torch_cuda
    out = torch.full((1,), 5, dtype=torch.int64, device="cuda")
    with pytest.raises(xt.XtError) as e:
        xt.count_device(3, torch.tensor([0, 2, 4, 6], dtype=torch.int64, device="cuda"),
                        torch.tensor([2, 1, 0, 2, 0, 1], dtype=torch.int64, device="cuda"), out,
                        stream=torch.cuda.current_stream().cuda_stream)
    assert e.value.status == xt.XT_ERR_INVALID
    torch.cuda.synchronize()
    assert int(out.item()) == 5


@pytest.mark.parametrize("n", [1024, 4096, 16384, 65536])
def test_reference_rgg_counts(ctx, n):
    off, tails = xt.generate_rgg(n, 1)
    f = GOLDEN[f"rgg{n}"]
    assert len(tails) == f["directed_entries"]
    for orient in ORIENTS:
        g = ctx.graph_from_csr(off, tails, canonical=True, orient=orient)
        assert g.count() == f["triangles"]
        g.free()


@pytest.mark.parametrize("elem", [8, 4])
@pytest.mark.parametrize("name", ["k4", "iso_tail", "k64", "er0", "rmat14", "chunglu14", "amazon0302"])
def test_vite_file_through_the_device(ctx, tmp_path, name, elem):
    """xt_graph_from_vite: the reference's vite file streamed to the device and
    parsed there counts the same as the golden count, canonical or not, and
    a file whose size or offsets contradict its header is XT_ERR_IO."""
    off, tails = canon(name)
    p = str(tmp_path / f"{name}_{elem}.bin")
    xt.write_vite(p, off, tails, elem)
    for canonical in (True, False):
        for orient in ORIENTS:
            g = ctx.graph_from_vite(p, elem, canonical=canonical, orient=orient)
            assert g.count() == GOLDEN[name]["triangles"]
            assert g.info()["n_input"] == len(tails)
            g.free()
    raw = open(p, "rb").read()
    with open(p, "wb") as f:  # one record short of its header
        f.write(raw[:-2 * elem])
    with pytest.raises(xt.XtError) as e:
        ctx.graph_from_vite(p, elem)
    assert e.value.status == xt.XT_ERR_IO
    if len(tails) > 1:  # the header and the size agree, but offsets[nv] says fewer records
        o2 = off.copy()
        o2[-1] -= 1
        hdr = np.array([len(off) - 1, len(tails)], np.int64 if elem == 8 else np.int32).tobytes()
        body = o2.astype(np.int64 if elem == 8 else np.int32).tobytes()
        with open(p, "wb") as f:
            f.write(hdr + body + raw[len(hdr) + len(body):])
        with pytest.raises(xt.XtError) as e:
            ctx.graph_from_vite(p, elem)
        assert e.value.status == xt.XT_ERR_IO
    # the context stays usable
    g = ctx.graph_from_csr(off, tails, canonical=True)
    assert g.count() == GOLDEN[name]["triangles"]
    g.free()


@pytest.mark.parametrize("n,nprocs,config_radius", [(1024, 1, False), (4096, 1, False), (16384, 1, False),
                                                     (65536, 1, False), (65536, 2, False), (65536, 2, True),
                                                     (65536, 4, True), (1 << 20, 2, True)])
def test_device_rgg_is_the_reference_graph(ctx, n, nprocs, config_radius):
    """xt_gen_rgg builds the reference's random geometric graph on the device:
    its edge set equals the host restatement's (itself pinned to the
    reference binary's rgg fixtures) edge for edge, and its count equals the
    golden count where the reference ran it (one rank, the reference's r)."""
    radius = float(np.sqrt(16.0 / (np.pi * n))) if config_radius else 0.0
    m, s, d = ctx.gen_rgg(n, nprocs, radius)
    off_h, tails_h = xt.generate_rgg(n, nprocs, radius)
    assert 2 * m == len(tails_h)
    s_np, d_np = s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64)
    assert (s_np < d_np).all()
    off_d, tails_d = oracle.canon_csr(n, s_np, d_np)
    assert (off_d == off_h).all() and (tails_d == tails_h).all()
    g = ctx.graph_from_device_edges(n, m, s, d)
    t = g.count()
    g.free()
    g = ctx.graph_from_rgg(n, nprocs, radius)  # generated and built in one call
    assert g.count() == t and g.info()["n_input"] == len(tails_h)
    g.free()
    if nprocs == 1 and not config_radius:
        assert t == GOLDEN[f"rgg{n}"]["triangles"]
    elif n <= 65536:
        assert t == oracle.count_merge(off_h, tails_h)


def test_rgg_two_ranks_and_config_radius(ctx):
    # mpiexec -n 2 graph and the r = sqrt(16/(pi n)) variant: oracle counts
    n = 65536
    for radius in (0.0, float(np.sqrt(16.0 / (np.pi * n)))):
        off, tails = xt.generate_rgg(n, 2, radius)
        expect = oracle.count_merge(off, tails)
        g = ctx.graph_from_csr(off, tails, canonical=True)
        assert g.count() == expect
        g.free()


def test_generators_bit_exact(ctx, torch_cuda):
    torch = torch_cuda
    ne = 1 << 18
    s = torch.empty(ne, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    ctx.gen_rmat(16, ne, 5, s, d)
    so, do = oracle.rmat_edges(16, ne, 5)
    assert (s.cpu().numpy() == so).all() and (d.cpu().numpy() == do).all()
    ctx.gen_rmat(12, ne, 5, s, d, noise_pct=0, permute=False)
    so, do = oracle.rmat_edges(12, ne, 5, noise_pct=0, permute=False)
    assert (s.cpu().numpy() == so).all() and (d.cpu().numpy() == do).all()
    cdf, _ = xt.chunglu_cdf(1 << 16, 2.1, 64.0, 4096.0)
    ctx.gen_chunglu(cdf, ne, 9, s, d)
    so, do = oracle.chunglu_edges(cdf, ne, 9)
    assert (s.cpu().numpy() == so).all() and (d.cpu().numpy() == do).all()
    ctx.gen_er(100000, ne, 11, s, d)
    so, do = oracle.er_edges(100000, ne, 11)
    assert (s.cpu().numpy() == so).all() and (d.cpu().numpy() == do).all()


@pytest.mark.parametrize("scale", [12, 16, 18])
def test_rmat_counts_vs_oracle(ctx, torch_cuda, scale):
    torch = torch_cuda
    ne = 16 << scale
    s = torch.empty(ne, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    ctx.gen_rmat(scale, ne, 1, s, d)
    off, tails = oracle.canon_csr(1 << scale, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    expect, opv = oracle.count_merge(off, tails, per_vertex=True)
    for orient in ORIENTS:
        g = ctx.graph_from_device_edges(1 << scale, ne, s, d, orient)
        t, pv = g.count(per_vertex=True)
        assert t == expect
        assert (pv == opv).all()
        g.free()


def test_chunglu_skewed_counts_vs_oracle(ctx, torch_cuda):
    # heavy skew: hub lists exceed the warp and block hash bins under the id
    # orientation (the part bin) and exercise every bin under degree order
    torch = torch_cuda
    n = 1 << 17
    cdf, m = xt.chunglu_cdf(n, 2.1, 32.0, 16384.0)
    s = torch.empty(m, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    ctx.gen_chunglu(cdf, m, 21, s, d)
    off, tails = oracle.canon_csr(n, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    expect, opv = oracle.count_merge(off, tails, per_vertex=True)
    for orient in ORIENTS:
        g = ctx.graph_from_device_edges(n, m, s, d, orient)
        inf = g.info()
        t, pv = g.count(per_vertex=True)
        assert t == expect, (orient, inf)
        assert (pv == opv).all()
        g.free()


def test_builder_rows_of_every_tier(ctx):
    # Rows of 1 to ~70,000 entries, each edge repeated in either direction
    # one time in five, and self loops: under the id orientation the hub's
    # row (69,999 entries) takes the device-sort tier, the long random rows
    # the CTA tier, the rest the warp (K = 1..32) and thread tiers. The
    # emitted out-CSR must be the oracle's canonical edge set, each row
    # ascending and above its own id.
    rng = np.random.default_rng(7)
    n = 70000
    src = [np.zeros(n - 1, np.int64)]
    dst = [np.arange(1, n, dtype=np.int64)]
    lens = np.exp(rng.uniform(0, np.log(3000), 4000)).astype(np.int64)
    for i, L in enumerate(lens, start=1):
        src.append(np.full(L, i, np.int64))
        dst.append(rng.integers(0, n, L))
    src.append(rng.integers(0, n, 200000))
    dst.append(rng.integers(0, n, 200000))
    s, d = np.concatenate(src), np.concatenate(dst)
    rep = rng.random(len(s)) < 0.2
    flip = rng.random(int(rep.sum())) < 0.5
    rs, rd = s[rep], d[rep]
    loops = rng.integers(0, n, 1000)
    s = np.concatenate([s, np.where(flip, rd, rs), loops])
    d = np.concatenate([d, np.where(flip, rs, rd), loops])
    off, tails = oracle.canon_csr(n, s, d)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
    up = tails > rows
    expect = rows[up] * n + tails[up]
    expect_t = oracle.count_merge(off, tails)
    for orient in ORIENTS:
        g = ctx.graph_from_edges(n, s.astype(np.int32), d.astype(np.int32), orient)
        goff, gcol = g.csr()
        perm = g.perm().astype(np.int64)
        grow = np.repeat(np.arange(n, dtype=np.int64), np.diff(goff))
        assert (gcol > grow).all(), orient
        same = grow[1:] == grow[:-1]
        assert (np.diff(gcol.astype(np.int64))[same] > 0).all(), orient
        a, b = perm[grow], perm[gcol.astype(np.int64)]
        assert np.array_equal(np.sort(np.minimum(a, b) * n + np.maximum(a, b)), expect), orient
        assert g.count() == expect_t, orient
        g.free()


def test_cluster_tier_vs_cta_parts(ctx, torch_cuda):
    # Under the id orientation the hubs of a skewed graph have more
    # out-neighbours than one CTA's member set holds (2,048): by default
    # every count runs them as CTA tasks over parts of 2,048 members; with
    # the cluster tier on, the global count runs them on thread-block
    # clusters (members spread over 8 CTAs' shared memories, up to 16,384 a
    # part). Default, on, off, on again, and a captured replay: every count
    # the oracle's.
    torch = torch_cuda
    n = 1 << 17
    cdf, m = xt.chunglu_cdf(n, 2.1, 32.0, 65536.0)
    s = torch.empty(m, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    ctx.gen_chunglu(cdf, m, 5, s, d)
    off, tails = oracle.canon_csr(n, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    expect, opv = oracle.count_merge(off, tails, per_vertex=True)
    g = ctx.graph_from_device_edges(n, m, s, d, xt.ORIENT_ID)
    assert g.info()["cluster_tasks"] == 0  # CTA parts by default
    assert g.count() == expect
    g.set_cluster(True)
    inf = g.info()
    assert inf["max_out_degree"] > 16384, inf  # some hub spans two cluster parts
    assert inf["cluster_tasks"] > 0, inf
    assert g.count() == expect
    t, pv = g.count(per_vertex=True)
    assert t == expect and (pv == opv).all()
    g.set_cluster(False)
    assert g.info()["cluster_tasks"] == 0
    assert g.count() == expect
    g.set_cluster(True)
    assert g.info()["cluster_tasks"] == inf["cluster_tasks"]
    g.capture()
    assert g.count() == expect
    assert g.count() == expect
    g.free()


def test_count_device_reference_layout(ctx, torch_cuda):
    torch = torch_cuda
    off, tails = canon("amazon0302")
    d_off = torch.from_numpy(off).cuda()
    d_t = torch.from_numpy(tails).cuda()
    out = torch.full((1,), 123, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    xt.count_device(len(off) - 1, d_off, d_t, out, accumulate=False, stream=stream)
    torch.cuda.synchronize()
    assert int(out.item()) == GOLDEN["amazon0302"]["triangles"]
    xt.count_device(len(off) - 1, d_off, d_t, out, accumulate=True, stream=stream)
    torch.cuda.synchronize()
    assert int(out.item()) == 2 * GOLDEN["amazon0302"]["triangles"]


def test_edge_cases(ctx):
    # one vertex, no edges; a single edge; only self loops; isolated tail
    g = ctx.graph_from_edges(1, np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert g.count() == 0
    g.free()
    g = ctx.graph_from_edges(2, np.array([0], np.int32), np.array([1], np.int32))
    assert g.count(per_vertex=True)[0] == 0
    g.free()
    g = ctx.graph_from_edges(3, np.array([0, 1, 2], np.int32), np.array([0, 1, 2], np.int32))
    assert g.count() == 0 and g.info()["n_edges"] == 0
    g.free()
    g = ctx.graph_from_edges(10, np.array([7, 8, 7], np.int32), np.array([8, 9, 9], np.int32))
    t, pv = g.count(per_vertex=True)
    assert t == 1 and pv.tolist() == [0] * 7 + [1, 1, 1]
    g.free()


def test_errors_leave_context_usable(ctx):
    with pytest.raises(xt.XtError) as e:
        ctx.graph_from_edges(4, np.array([0, 5], np.int32), np.array([1, 2], np.int32))
    assert e.value.status == xt.XT_ERR_INVALID
    with pytest.raises(xt.XtError) as e:
        ctx.graph_from_edges(4, np.array([0, -1], np.int32), np.array([1, 2], np.int32))
    assert e.value.status == xt.XT_ERR_INVALID
    with pytest.raises(xt.XtError) as e:
        ctx.graph_from_csr(np.array([0, 2, 1], np.int64), np.array([1, 0], np.int64))
    assert e.value.status == xt.XT_ERR_INVALID
    # an allocation failure injected on the host side of the allocator
    for k in range(1, 12):
        ctx.fail_alloc_after(k)
        try:
            g = ctx.graph_from_edges(GOLDEN["k64"]["nv"], FIX["k64_src"], FIX["k64_dst"])
        except xt.XtError as err:
            assert err.status == xt.XT_ERR_OOM
            continue
        g.free()
        break
    ctx.fail_alloc_after(0)
    g = ctx.graph_from_edges(GOLDEN["k64"]["nv"], FIX["k64_src"], FIX["k64_dst"])
    assert g.count() == GOLDEN["k64"]["triangles"]
    g.free()


def test_cli_on_gpu(tmp_path):
    import subprocess
    from conftest import ROOT
    import os
    cli = os.path.join(ROOT, "xxtric_b200", "xtric")
    r = subprocess.run([cli, "-n", "4096", "-l"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert f"Number of triangles: {GOLDEN['rgg4096']['triangles']}" in r.stdout
    off, tails = xt.generate_rgg(16384, 1)
    p = str(tmp_path / "g.bin")
    xt.write_vite(p, off, tails)
    pvf = str(tmp_path / "pv.txt")
    r = subprocess.run([cli, "-f", p, "--orient", "id", "--per-vertex", pvf], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert f"Number of triangles: {GOLDEN['rgg16384']['triangles']}" in r.stdout
    pv = np.loadtxt(pvf, dtype=np.int64)
    assert pv.sum() == 3 * GOLDEN["rgg16384"]["triangles"]


def test_mirror_class(ctx):
    off, tails = canon("rmat10")
    tc = xt.TriangleCountingSingle(off, tails)
    assert tc.count() == GOLDEN["rmat10"]["triangles"]
    assert tc.count() == GOLDEN["rmat10"]["triangles"]  # counting twice is idempotent
    tc.clear()


# (lane_work, warp_work): every head on one tier, and the automatic choice
TIERS = [(1 << 40, 0), (0, 1 << 40), (0, 0), (64, 4096), (-1, -1)]


@pytest.mark.parametrize("kind", ["rmat", "chunglu"])
def test_each_tier_alone_vs_oracle(ctx, torch_cuda, kind):
    # Lane tasks (binary search in the row, or a two-pointer merge), warp
    # tasks and CTA tasks each count the whole graph alone, then mixed;
    # totals, per-vertex counts and a captured replay after a re-plan all
    # equal the oracle's.
    torch = torch_cuda
    if kind == "rmat":
        n, m = 1 << 14, 16 << 14
        s = torch.empty(m, dtype=torch.int32, device="cuda")
        d = torch.empty_like(s)
        ctx.gen_rmat(14, m, 3, s, d)
    else:
        n = 1 << 15
        cdf, m = xt.chunglu_cdf(n, 2.1, 24.0, 8192.0)
        s = torch.empty(m, dtype=torch.int32, device="cuda")
        d = torch.empty_like(s)
        ctx.gen_chunglu(cdf, m, 5, s, d)
    off, tails = oracle.canon_csr(n, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    expect, opv = oracle.count_merge(off, tails, per_vertex=True)
    for orient in ORIENTS:
        g = ctx.graph_from_device_edges(n, m, s, d, orient)
        try:
            for lane_work, warp_work in TIERS:
                g.set_tiers(lane_work, warp_work)
                t, pv = g.count(per_vertex=True)
                assert t == expect, (orient, lane_work, warp_work)
                assert (pv == opv).all(), (orient, lane_work, warp_work)
                # the lane tier's two-pointer merge instead of its binary search
                g.set_lane_intersect(xt.LANE_MERGE)
                t, pv = g.count(per_vertex=True)
                assert t == expect and (pv == opv).all(), (orient, lane_work, warp_work, "merge")
                assert g.count() == expect, (orient, lane_work, warp_work, "merge")
                g.set_lane_intersect(xt.LANE_BSEARCH)
                # the global-count kernel: cuckoo member sets, their linear-
                # probing fallback (chains capped at 0 and 1 evictions) and
                # the bulk suffix prefetch
                for iters, pf in ((-1, False), (-1, True), (0, False), (1, True)):
                    g.debug_cuckoo_iters(iters)
                    g.set_prefetch(pf)
                    assert g.count() == expect, (orient, lane_work, warp_work, iters, pf)
                g.debug_cuckoo_iters(-1)
                g.set_prefetch(False)
            g.set_tiers(1 << 40, 0)
            g.capture()
            assert g.count_groups()[0] == expect  # the captured replay
            g.set_tiers(0, 1 << 40)  # re-plans and re-captures
            assert g.count_groups()[0] == expect
        finally:
            g.free()


@pytest.mark.parametrize("kind", ["rmat", "chunglu"])
def test_claim_blocks_vs_oracle(ctx, torch_cuda, kind):
    # warp tasks (and groups of 32 lane heads) taken 1, 3, 4, 16 or 64 per
    # atomic on their cursor: the same counts on every tier, in every mode,
    # with shards (strided lists) and through a captured replay
    torch = torch_cuda
    if kind == "rmat":
        n, m = 1 << 14, 16 << 14
        s = torch.empty(m, dtype=torch.int32, device="cuda")
        d = torch.empty_like(s)
        ctx.gen_rmat(14, m, 11, s, d)
    else:
        n = 1 << 15
        cdf, m = xt.chunglu_cdf(n, 2.1, 24.0, 8192.0)
        s = torch.empty(m, dtype=torch.int32, device="cuda")
        d = torch.empty_like(s)
        ctx.gen_chunglu(cdf, m, 13, s, d)
    off, tails = oracle.canon_csr(n, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    expect, opv = oracle.count_merge(off, tails, per_vertex=True)
    g = ctx.graph_from_device_edges(n, m, s, d, xt.ORIENT_DEGREE)
    try:
        _, ref_sup = g.count_edges()
        dg = torch.zeros(1, dtype=torch.int64, device="cuda")
        for lane_work, warp_work in ((1 << 40, 0), (0, 1 << 40), (-1, -1)):
            g.set_tiers(lane_work, warp_work)
            for claim in (1, 3, 4, 16, 64):
                g.set_claim(claim)
                t, pv = g.count(per_vertex=True)
                assert t == expect and (pv == opv).all(), (lane_work, warp_work, claim)
                t2, sup = g.count_edges()
                assert t2 == expect and (sup == ref_sup).all(), (lane_work, warp_work, claim)
                tot = 0
                for k in range(3):
                    g.count_shard_async(k, 3, dg)
                    ctx.synchronize()
                    tot += int(dg.item())
                assert tot == expect, (lane_work, warp_work, claim, "shards")
        g.set_claim(0)
        g.capture()
        g.set_claim(16)  # re-captures
        assert g.count_groups()[0] == expect
        with pytest.raises(xt.XtError):
            g.set_claim(65)
    finally:
        g.free()


def oracle_support_of(off, tails, a, b):
    """The oracle's support of undirected edges (a[i], b[i]), a < b."""
    es = oracle.edge_support(off, tails)
    nv = len(off) - 1
    keys = np.repeat(np.arange(nv, dtype=np.int64), np.diff(off)) * nv + tails  # sorted: rows ascend
    pos = np.searchsorted(keys, a.astype(np.int64) * nv + b)
    assert (tails[pos] == b).all()
    return es[pos]


@pytest.mark.parametrize("name", ["k4", "k64", "iso_tail", "star_path", "er0", "rmat14", "chunglu14", "amazon0302"])
def test_edge_support_and_clustering_vs_oracle(ctx, name):
    f = GOLDEN[name]
    off, tails = canon(name)
    _, opv = oracle.count_merge(off, tails, per_vertex=True)
    deg = np.diff(off)
    for orient in ORIENTS:
        g = ctx.graph_from_edges(f["nv"], FIX[name + "_src"], FIX[name + "_dst"], orient)
        try:
            t, sup = g.count_edges()
            assert t == f["triangles"] and sup.sum() == 3 * t
            a, b, s = g.edge_support()
            assert (s == oracle_support_of(off, tails, a, b)).all()
            assert (g.degrees() == deg).all()
            c = g.clustering()
            want = np.where(deg >= 2, 2.0 * opv / np.maximum(deg * (deg - 1.0), 1.0), 0.0)
            assert np.allclose(c, want, rtol=0, atol=1e-12)
        finally:
            g.free()


def test_edge_support_every_tier(ctx, torch_cuda):
    # lane, warp and CTA tasks (hash member sets with parts on the hubs)
    torch = torch_cuda
    n = 1 << 15
    cdf, m = xt.chunglu_cdf(n, 2.1, 24.0, 8192.0)
    s = torch.empty(m, dtype=torch.int32, device="cuda")
    d = torch.empty_like(s)
    ctx.gen_chunglu(cdf, m, 5, s, d)
    off, tails = oracle.canon_csr(n, s.cpu().numpy().astype(np.int64), d.cpu().numpy().astype(np.int64))
    for orient in ORIENTS:
        g = ctx.graph_from_device_edges(n, m, s, d, orient)
        try:
            ref = None
            for lane_work, warp_work in TIERS:
                g.set_tiers(lane_work, warp_work)
                a, b, sup = g.edge_support()
                if ref is None:
                    ref = oracle_support_of(off, tails, a, b)
                assert (sup == ref).all(), (orient, lane_work, warp_work)
                g.set_lane_intersect(xt.LANE_MERGE)
                assert (g.edge_support()[2] == ref).all(), (orient, lane_work, warp_work, "merge")
                g.set_lane_intersect(xt.LANE_BSEARCH)
            # the device-output form gives the same supports, in csr() order
            t, host = g.count_edges()
            dg = torch.zeros(1, dtype=torch.int64, device="cuda")
            ds = torch.full((len(host),), -1, dtype=torch.int64, device="cuda")
            torch.cuda.synchronize()
            g.count_edges_async(dg.data_ptr(), ds.data_ptr())
            ctx.synchronize()
            assert int(dg.item()) == t and (ds.cpu().numpy() == host).all()
        finally:
            g.free()


@pytest.mark.parametrize("orient", ORIENTS)
def test_graph_statistics(ctx, orient):
    # the plan's statistics against the same sums taken on the host from
    # the oriented CSR the library exposes
    name = "chunglu14"
    f = GOLDEN[name]
    g = ctx.graph_from_edges(f["nv"], FIX[name + "_src"], FIX[name + "_dst"], orient)
    try:
        inf = g.info()
        off, col = g.csr()
        dout = np.diff(off)
        din = np.bincount(col, minlength=len(dout))
        assert inf["max_out_degree"] == dout.max() and inf["max_in_degree"] == din.max()
        assert inf["max_degree"] == (dout + din).max()
        assert inf["wedge_work"] == int(dout[col].sum())
        assert inf["stream_work"] == int((dout * (dout - 1) // 2).sum())
    finally:
        g.free()


def test_cpp_mirror_batch_edges_and_server(tmp_path):
    # the C++ host mirror's batch count, per-edge count and server on the GPU
    import subprocess
    from test_host import compile_mirror_check
    exe = compile_mirror_check(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.split("\n")[:3] == ["batch 5 4 1", "edges 4 6 12", "served 4 1"], r.stdout
