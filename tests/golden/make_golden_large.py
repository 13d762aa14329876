"""Pin the counts of the full-size benchmark graphs on the CPU.

The GPU tests at full size (tests/test_gpu_large.py) compare their counts with
the numbers this script writes under the "large" key of golden.json:

* rmat24 - R-MAT scale 24, edge factor 16, seed 1 (noise 10%, ids permuted):
  the headline workload;
* rmat22 - the same generator at scale 22, seeds 1 and 5;
* chunglu_full - Chung-Lu n = 4,194,304, exponent 2.1, mean degree 64,
  maximum expected degree 131,072, seed 1.

Each graph comes from the oracle's generator twins (bit-exact to the device
generators, tests/test_gpu_parity.py::test_generators_bit_exact), is
canonicalised by the oracle, relabelled by (degree, id) rank - a relabelling
leaves every count unchanged and bounds the out-degrees, so the CPU counters
finish in minutes - and counted twice:

* ``xo_count_merge`` (sorted-list merge, per-vertex credits), and
* ``xo_count_xxtric`` (the restatement of the reference's loop,
  xxtric.hpp:60-80, 150-207, 516-588).

The per-vertex counts, mapped back to the generated ids, are stored as their
sum and a SHA-256 digest of the little-endian int64 array, so a GPU test can
compare every vertex without a multi-GB fixture.

With ``--reference`` the reference's own binary (built from the read-only
reference tree by oracle/Makefile) also counts each graph from a vite file:
the degree-relabelled file and, with ``--reference-id-order HOURS``, the file
in the generated ids under a wall cap (the reference's own orientation; "did
not finish" when capped). By default that binary is the OpenMP build
(oracle/_ref/tric_omp), whose total is the true count modulo 2^32: its
OpenMP branch sums the per-vertex counts with std::accumulate(tcount,
tcount + lnv, 0) (xxtric.hpp:147), an int initial value, so the sum is
carried in 32 bits; the record then checks that congruence. With
``--reference-serial`` the single-threaded build (oracle/_ref/tric, a 64-bit
sum) runs instead and must equal the count exactly. Run where the reference
tree exists:

    python tests/golden/make_golden_large.py [--reference] [--reference-serial]
        [--reference-id-order 3] [--threads 6] [--bin-dir DIR] [--only rmat24,chunglu_full]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import platform
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

GOLDEN = os.path.join(HERE, "golden.json")


def graphs():
    """name -> (description, nv, edge generator)."""
    def rmat(scale, seed):
        return lambda: oracle.rmat_edges(scale, 16 << scale, seed)

    def chunglu():
        cdf, m = oracle.chunglu_cdf(4194304, 2.1, 64.0, 131072.0)
        return oracle.chunglu_edges(cdf, m, 1)

    return {
        "rmat24": ("R-MAT scale 24, edge factor 16, seed 1, noise 10%, ids permuted", 1 << 24, rmat(24, 1)),
        "rmat22": ("R-MAT scale 22, edge factor 16, seed 1, noise 10%, ids permuted", 1 << 22, rmat(22, 1)),
        "rmat22_seed5": ("R-MAT scale 22, edge factor 16, seed 5, noise 10%, ids permuted", 1 << 22, rmat(22, 5)),
        "chunglu_full": ("Chung-Lu n=4194304, exponent 2.1, mean degree 64, max expected 131072, seed 1",
                         4194304, chunglu),
    }


def digest(pv: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(pv, "<i8").tobytes()).hexdigest()


def degree_rank(off: np.ndarray) -> np.ndarray:
    """rank[x] = position of vertex x in ascending (degree, id) order."""
    n = len(off) - 1
    deg = np.diff(off)
    order = np.lexsort((np.arange(n, dtype=np.int64), deg))
    rank = np.empty(n, np.int64)
    rank[order] = np.arange(n, dtype=np.int64)
    return rank


def upper_pairs(off: np.ndarray, tails: np.ndarray):
    n = len(off) - 1
    u = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
    m = u < tails
    return u[m], tails[m]


def write_vite(path: str, off: np.ndarray, tails: np.ndarray) -> None:
    """The reference's 8-byte vite layout (graph.hpp:294-395): nv, ne, offsets,
    then ne records {int64 tail, double weight}."""
    nv = len(off) - 1
    with open(path, "wb") as f:
        np.array([nv, len(tails)], np.int64).tofile(f)
        off.astype(np.int64).tofile(f)
        step = 1 << 24
        for a in range(0, len(tails), step):
            rec = np.zeros(min(step, len(tails) - a), dtype=[("t", "<i8"), ("w", "<f8")])
            rec["t"] = tails[a:a + step]
            rec["w"] = 1.0
            rec.tofile(f)


def int32_wrap(t: int) -> int:
    """t as a 32-bit two's-complement int holds it (std::accumulate with an
    int initial value)."""
    return ((t + (1 << 31)) % (1 << 32)) - (1 << 31)


def run_reference(path: str, threads: int, cap_s: float, serial: bool = False) -> dict:
    exe = oracle.REF_TRIC if serial else oracle.REF_TRIC_OMP
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    t0 = time.time()
    try:
        r = subprocess.run(["nice", "-n", "10", exe, "-f", path], capture_output=True, text=True,
                           timeout=cap_s, env=env)
    except subprocess.TimeoutExpired:
        return {"finished": False, "wall_s": round(time.time() - t0, 1), "binary": os.path.basename(exe),
                "note": f"did not finish in {cap_s / 3600:.2f} h on {1 if serial else threads} thread(s)"}
    out = {"finished": r.returncode == 0, "rc": r.returncode, "wall_s": round(time.time() - t0, 1),
           "binary": os.path.basename(exe), "threads": 1 if serial else threads}
    for line in r.stdout.splitlines():
        if line.startswith("Number of triangles:"):
            out["triangles"] = int(line.split(":")[1])
        elif line.startswith("Number of edges:"):
            out["directed_entries"] = int(line.split(":")[1])
        elif line.startswith("Avg/Min/Max times for local counting"):
            out["t_local_s"] = float(line.split(":")[1].split(",")[2])
        elif line.startswith("Avg/Min/Max execution time"):
            out["t_count_s"] = float(line.split(":")[1].split(",")[2])
    return out


def check_reference(name: str, r: dict, t: int, serial: bool) -> None:
    """The reference binary's total against the oracle's: equal for the
    serial build, equal modulo 2^32 for the OpenMP build (xxtric.hpp:147)."""
    if not r.get("finished"):
        return
    if serial:
        assert r["triangles"] == t, (name, r, t)
        r["agrees_with_oracle"] = "exactly"
    else:
        assert r["triangles"] == int32_wrap(t), (name, r, t)
        r["agrees_with_oracle"] = ("modulo 2^32: the OpenMP branch sums with std::accumulate(..., 0), an int "
                                   "initial value (xxtric.hpp:147)" + ("; exactly" if r["triangles"] == t else ""))


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def load_golden() -> dict:
    with open(GOLDEN) as f:
        return json.load(f)


def save_golden(g: dict) -> None:
    with open(GOLDEN, "w") as f:
        json.dump(g, f, indent=1, sort_keys=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--reference", action="store_true", help="also count with oracle/_ref/tric_omp")
    ap.add_argument("--reference-serial", action="store_true",
                    help="use the single-threaded reference binary (an exact 64-bit total)")
    ap.add_argument("--skip-oracle", action="store_true",
                    help="keep the recorded oracle counts and only run the reference")
    ap.add_argument("--reference-id-order", type=float, default=0.0,
                    help="wall cap in hours for the reference on the generated ids (0: skip)")
    ap.add_argument("--bin-dir", default="/tmp")
    args = ap.parse_args()
    os.environ["OMP_NUM_THREADS"] = str(args.threads)
    oracle.build(ref=args.reference)
    sel = [s for s in args.only.split(",") if s]
    for name, (desc, nv, gen) in graphs().items():
        if sel and name not in sel:
            continue
        t0 = time.time()
        src, dst = gen()
        off, tails = oracle.canon_csr(nv, src, dst)
        del src, dst
        rank = degree_rank(off)
        u, v = upper_pairs(off, tails)
        off_r, tails_r = oracle.canon_csr(nv, rank[u], rank[v])
        del u, v
        t_gen = time.time() - t0
        if args.skip_oracle and name in load_golden().get("large", {}):
            t_merge = load_golden()["large"][name]["triangles"]
            print(name, "oracle counts kept:", t_merge, flush=True)
        else:
            t0 = time.time()
            t_merge, pv_r = oracle.count_merge(off_r, tails_r, per_vertex=True)
            t_m = time.time() - t0
            t0 = time.time()
            t_restated = oracle.count_xxtric(off_r, tails_r)
            t_x = time.time() - t0
            assert t_merge == t_restated, (name, t_merge, t_restated)
            pv = pv_r[rank]
            assert int(pv.sum()) == 3 * t_merge
            deg = np.diff(off)
            hubs = np.argsort(deg, kind="stable")[-8:][::-1]
            rec = {
                "description": desc, "nv": nv, "undirected": int(len(tails) // 2), "triangles": int(t_merge),
                "max_degree": int(deg.max()), "per_vertex_sum": int(pv.sum()), "per_vertex_sha256": digest(pv),
                "hubs": [[int(h), int(deg[h]), int(pv[h])] for h in hubs],
                "counted_by": ["oracle xo_count_merge", "oracle xo_count_xxtric"],
                "cpu_seconds": {"generate_canonicalise_relabel": round(t_gen, 1), "merge": round(t_m, 1),
                                "restated_reference_loop": round(t_x, 1)},
                "cpu": {"model": cpu_model(), "threads": args.threads},
            }
            print(name, {k: rec[k] for k in ("nv", "undirected", "triangles", "max_degree")}, rec["cpu_seconds"],
                  flush=True)
            g = load_golden()
            g.setdefault("large", {})[name] = dict(g.get("large", {}).get(name, {}), **rec)
            save_golden(g)
        if args.reference and os.path.exists(oracle.REF_TRIC_OMP):
            path = os.path.join(args.bin_dir, f"xt_golden_{name}_degree.bin")
            write_vite(path, off_r, tails_r)
            del off_r, tails_r
            r = run_reference(path, args.threads, 12 * 3600, args.reference_serial)
            os.remove(path)
            r["file"] = "degree-relabelled vite file"
            print(name, "reference (degree-relabelled):", r, flush=True)
            check_reference(name, r, t_merge, args.reference_serial)
            g = load_golden()
            g["large"][name]["reference_degree_relabelled" + ("_serial" if args.reference_serial else "")] = r
            save_golden(g)
            if args.reference_id_order > 0:
                path = os.path.join(args.bin_dir, f"xt_golden_{name}_ids.bin")
                write_vite(path, off, tails)
                del off, tails
                r = run_reference(path, args.threads, args.reference_id_order * 3600, args.reference_serial)
                os.remove(path)
                r["file"] = "vite file in the generated ids (the reference's own orientation)"
                print(name, "reference (generated ids):", r, flush=True)
                check_reference(name, r, t_merge, args.reference_serial)
                g = load_golden()
                g["large"][name]["reference_generated_ids"] = r
                save_golden(g)


if __name__ == "__main__":
    main()
