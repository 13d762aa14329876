"""The oracle is pinned before it is trusted: its restatement of the
reference's count (xxtric.hpp:60-80, 150-207, 516-588) and the independent
merge counter must reproduce every count the reference's own binary printed
for the golden fixtures, and its restatement of the reference's generator
must reproduce the reference's graphs."""
import numpy as np
import pytest

import oracle
from conftest import load_fixtures, load_golden

GOLDEN = load_golden()
FIX = load_fixtures()
EDGE_NAMES = [n for n in GOLDEN if n + "_src" in FIX]


def canon(name):
    f = GOLDEN[name]
    return oracle.canon_csr(f["nv"], FIX[name + "_src"].astype(np.int64), FIX[name + "_dst"].astype(np.int64))


@pytest.mark.parametrize("name", EDGE_NAMES)
def test_oracle_counts_match_reference(name):
    off, tails = canon(name)
    f = GOLDEN[name]
    assert len(tails) == f["directed_entries"]
    assert oracle.count_xxtric(off, tails) == f["triangles"]
    t, pv = oracle.count_merge(off, tails, per_vertex=True)
    assert t == f["triangles"]
    assert pv.sum() == 3 * t


@pytest.mark.parametrize("n", [1024, 4096, 16384])
def test_oracle_rgg_restatement_matches_reference(n):
    off, tails = oracle.ref_rgg(n, 1)
    f = GOLDEN[f"rgg{n}"]
    assert len(tails) == f["directed_entries"]
    assert oracle.count_xxtric(off, tails) == f["triangles"]


def test_seed_seq_restatement():
    # std::seed_seq({s}).generate() of one word, checked against libstdc++
    # (the reference's reseeder, utils.hpp:37-44)
    assert oracle.lib().xo_seed_seq1(1) == 1967017404
    assert oracle.lib().xo_seed_seq1(7) == 992434658
    assert oracle.lib().xo_seed_seq1(12345) == 2956583348


def test_local_counts_match_per_vertex():
    off, tails = canon("rmat14")
    _, pv = oracle.count_merge(off, tails, per_vertex=True)
    rng = np.random.default_rng(0)
    sel = rng.choice(len(off) - 1, 500, replace=False)
    assert (oracle.local_counts(off, tails, sel) == pv[sel]).all()


def test_reference_over_counts_duplicates():
    # the reference trusts its input: a repeated pair over-counts (graph.hpp
    # reads rows verbatim); canonical input gives the true count
    f = GOLDEN["k4dup"]
    assert f["triangles"] == 4
    assert f["reference_on_raw_file"] > 4


def test_generators_deterministic():
    a = oracle.rmat_edges(10, 1000, seed=3)
    b = oracle.rmat_edges(10, 1000, seed=3)
    c = oracle.rmat_edges(10, 1000, seed=4)
    assert (a[0] == b[0]).all() and (a[1] == b[1]).all()
    assert not (a[0] == c[0]).all()
    # chunks generate the same edges as one pass
    s1, d1 = oracle.rmat_edges(10, 500, seed=3, e0=500)
    assert (s1 == a[0][500:]).all() and (d1 == a[1][500:]).all()
    # permutation is a bijection
    s, _ = oracle.rmat_edges(12, 1 << 16, seed=1, noise_pct=0)
    assert s.min() >= 0 and s.max() < (1 << 12)


@pytest.mark.skipif(not oracle.os.path.exists(oracle.REF_TRIC), reason="reference binary not built here")
def test_reference_binary_on_rgg_matches_golden():
    r = oracle.run_ref(["-n", "4096", "-l"])
    assert r["rc"] == 0
    assert r["triangles"] == GOLDEN["rgg4096"]["triangles"]
    assert r["edges"] == GOLDEN["rgg4096"]["directed_entries"]


def test_local_counts_equal_per_vertex_merge_counts():
    # the sampled-vertex checker of the full-size GPU tests against the
    # independent merge counter, every vertex of a skewed graph
    n = 1 << 13
    cdf, m = oracle.chunglu_cdf(n, 2.1, 16.0, 2048.0)
    s, d = oracle.chunglu_edges(cdf, m, 4)
    off, tails = oracle.canon_csr(n, s, d)
    _, pv = oracle.count_merge(off, tails, per_vertex=True)
    assert (oracle.local_counts(off, tails, np.arange(n)) == pv).all()


def test_edge_support_consistent_with_vertex_counts():
    # every triangle puts 1 on each of its 3 edges (2 CSR entries each) and
    # 2 on the CSR entries around each of its corners
    n = 1 << 12
    s, d = oracle.rmat_edges(12, 16 << 12, 3)
    off, tails = oracle.canon_csr(n, s, d)
    total, pv = oracle.count_merge(off, tails, per_vertex=True)
    es = oracle.edge_support(off, tails)
    assert es.sum() == 6 * total
    at_v = np.zeros(n, np.int64)
    np.add.at(at_v, np.repeat(np.arange(n), np.diff(off)), es)
    assert (at_v == 2 * pv).all()


def test_full_size_pins_are_consistent():
    """The full-size pins (tests/golden/make_golden_large.py): every entry was
    counted by both oracle counters, its per-vertex counts sum to three times
    its total, and where the reference's own binary counted it, its printed
    total agrees: exactly for the single-threaded build, modulo 2^32 (read as
    a signed 32-bit int) for the OpenMP build, whose total is summed by
    std::accumulate with an int initial value (xxtric.hpp:147)."""
    import json
    import os
    from conftest import GOLDEN_DIR
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        large = json.load(f)["large"]
    assert {"rmat24", "rmat22", "rmat22_seed5", "chunglu_full"} <= set(large)
    for name, f in large.items():
        assert f["per_vertex_sum"] == 3 * f["triangles"], name
        assert set(f["counted_by"]) == {"oracle xo_count_merge", "oracle xo_count_xxtric"}, name
        for key, r in f.items():
            if not key.startswith("reference_") or not r.get("finished"):
                continue
            if r["binary"] == "tric":
                assert r["triangles"] == f["triangles"], (name, key)
            else:
                wrapped = ((f["triangles"] + (1 << 31)) % (1 << 32)) - (1 << 31)
                assert r["triangles"] == wrapped, (name, key)
    # the headline: the reference's own serial build gave the same count
    assert large["rmat24"]["reference_degree_relabelled_serial"]["triangles"] == 10182539214
    assert large["rmat24"]["triangles"] == 10182539214
