"""Regenerate the golden fixtures in this directory from the reference's own
CPU binary (oracle/_ref/tric, built from the read-only reference tree by
oracle/Makefile). Run where the reference tree exists:

    python tests/golden/make_golden.py

Writes golden.json (counts printed by the reference for every fixture) and
fixtures.npz (each fixture's undirected edge list, u < v, int32), so the GPU
tests need neither the reference tree nor its binary.
"""
from __future__ import annotations

import itertools
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

AMAZON_TSV = os.path.join(oracle.REFERENCE_TREE, "cugraph", "example-inputs", "amazon0302_adj.tsv")


def write_bin(path, nv, src, dst, canonical=True):
    """vite layout; canonical -> symmetric sorted deduped rows."""
    if canonical:
        off, tails = oracle.canon_csr(nv, src, dst)
    else:  # rows exactly as given (sorted by row, then column), both directions
        s = np.concatenate([src, dst])
        d = np.concatenate([dst, src])
        order = np.lexsort((d, s))
        s, d = s[order], d[order]
        off = np.zeros(nv + 1, np.int64)
        np.add.at(off, s + 1, 1)
        off = np.cumsum(off)
        tails = d.astype(np.int64)
    rec = np.zeros(len(tails), dtype=[("t", "<i8"), ("w", "<f8")])
    rec["t"] = tails
    rec["w"] = 1.0
    with open(path, "wb") as f:
        np.array([nv, len(tails)], np.int64).tofile(f)
        off.astype(np.int64).tofile(f)
        rec.tofile(f)
    return off, tails


def undirected(off, tails):
    deg = np.diff(off)
    src = np.repeat(np.arange(len(off) - 1, dtype=np.int64), deg)
    m = src < tails
    return src[m].astype(np.int32), tails[m].astype(np.int32)


def main():
    oracle.build(ref=True)
    if not os.path.exists(oracle.REF_TRIC):
        sys.exit("oracle/_ref/tric is not built: the reference tree is required to regenerate fixtures")
    golden = {"source": "oracle/_ref/tric (reference main.cpp + xxtric.hpp, 1 rank)", "fixtures": {}}
    arrays = {}
    tmp = tempfile.mkdtemp()

    def file_fixture(name, nv, src, dst, note, canonical=True, ref_may_fail=False):
        path = os.path.join(tmp, name + ".bin")
        off, tails = write_bin(path, nv, np.asarray(src, np.int64), np.asarray(dst, np.int64), canonical)
        r = oracle.run_ref(["-f", path])
        if ref_may_fail and r["rc"] != 0:
            # no count printed: record the exit status and the defined answer
            r.setdefault("edges", int(len(tails)))
            r["triangles"] = 0
            note += f" (the reference exits with status {r['rc']} on it; 0 is the count by definition)"
        else:
            assert r["rc"] == 0, r["stdout"]
        cs, cd = undirected(*oracle.canon_csr(nv, np.asarray(src, np.int64), np.asarray(dst, np.int64)))
        arrays[name + "_src"], arrays[name + "_dst"] = cs, cd
        golden["fixtures"][name] = {"nv": nv, "directed_entries": r["edges"], "undirected": int(len(cs)),
                                    "triangles": r["triangles"], "canonical_input": canonical, "note": note}
        print(name, golden["fixtures"][name])

    k4 = list(itertools.combinations(range(4), 2))
    file_fixture("k4", 4, [a for a, _ in k4], [b for _, b in k4], "complete graph K4")
    k5 = list(itertools.combinations(range(5), 2))
    file_fixture("k5", 5, [a for a, _ in k5], [b for _, b in k5], "complete graph K5")
    file_fixture("iso_tail", 6, [0, 1, 0, 2], [1, 2, 2, 3], "one triangle, a pendant vertex and an isolated tail "
                 "(the reference reads past its edge array for vertex 5, xxtric.hpp:67-74)")
    k64 = list(itertools.combinations(range(64), 2))
    file_fixture("k64", 64, [a for a, _ in k64], [b for _, b in k64], "complete graph K64")
    star_s = [0] * 1000 + list(range(1, 999))
    star_d = list(range(1, 1001)) + list(range(2, 1000))
    file_fixture("star_path", 1001, star_s, star_d, "hub joined to a path of 1000: 998 triangles")
    file_fixture("empty", 5, [], [], "five vertices, no edges", ref_may_fail=True)
    # duplicated pair: the raw file over-counts in the reference (it trusts
    # its input); the canonical file is what the device builder makes of it
    dup_s = [a for a, _ in k4] + [0]
    dup_d = [b for _, b in k4] + [1]
    path = os.path.join(tmp, "k4dup_raw.bin")
    write_bin(path, 4, np.asarray(dup_s), np.asarray(dup_d), canonical=False)
    raw = oracle.run_ref(["-f", path])
    file_fixture("k4dup", 4, dup_s + [2, 3], dup_d + [2, 3],
                 "K4 with a repeated pair and self loops; canonicalised")
    golden["fixtures"]["k4dup"]["reference_on_raw_file"] = raw["triangles"]
    for seed in range(3):
        rng = np.random.default_rng(seed)
        n = 2000
        pairs = rng.integers(0, n, size=(30000, 2))
        file_fixture(f"er{seed}", n, pairs[:, 0], pairs[:, 1], "30000 random pairs on 2000 vertices")
    # this library's R-MAT generator (oracle twin), counted by the reference
    for scale in (10, 14):
        s, d = oracle.rmat_edges(scale, 16 << scale, seed=7)
        file_fixture(f"rmat{scale}", 1 << scale, s, d, f"R-MAT scale {scale}, edge factor 16, seed 7, noise 10%")
    cdf, m = oracle.chunglu_cdf(1 << 14, 2.1, 16.0, 1024.0)
    s, d = oracle.chunglu_edges(cdf, m, seed=3)
    file_fixture("chunglu14", 1 << 14, s, d, "Chung-Lu n=16384, gamma 2.1, mean 16, max 1024, seed 3")
    # the reference's own LCG geometric graphs (-n N -l, one rank)
    for n in (1024, 4096, 16384, 65536):
        r = oracle.run_ref(["-n", str(n), "-l"])
        assert r["rc"] == 0
        golden["fixtures"][f"rgg{n}"] = {"nv": n, "directed_entries": r["edges"], "triangles": r["triangles"],
                                         "args": ["-n", str(n), "-l"], "nprocs": 1}
        print(f"rgg{n}", golden["fixtures"][f"rgg{n}"])
    if os.path.exists(AMAZON_TSV):
        a = np.loadtxt(AMAZON_TSV, dtype=np.int64, usecols=(0, 1))
        n = int(a.max()) + 1
        file_fixture("amazon0302", n, a[:, 0], a[:, 1], "cugraph/example-inputs/amazon0302_adj.tsv (ids as given)")
    np.savez_compressed(os.path.join(HERE, "fixtures.npz"), **arrays)
    path = os.path.join(HERE, "golden.json")
    if os.path.exists(path):  # keep the full-size pins of make_golden_large.py
        with open(path) as f:
            old = json.load(f)
        if "large" in old:
            golden["large"] = old["large"]
    with open(path, "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
