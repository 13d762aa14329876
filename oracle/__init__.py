"""The oracle: a CPU restatement of sg0/xxtric's counting path and of this
library's deterministic generators (xtoracle.c), plus the reference's own
binaries built from its sources (oracle/_ref/, see the Makefile): its CPU
count and its single-GPU engine.

TEST INFRASTRUCTURE ONLY. It is loaded by tests/, by __graft_entry__.smoke()
and by bench.py's CPU-baseline leg, always as the checker or the timed CPU
baseline, never as part of the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_TRIC = os.path.join(REF_DIR, "tric")
REF_TRIC_OMP = os.path.join(REF_DIR, "tric_omp")
REF_TRIC_GPU = os.path.join(REF_DIR, "tric_gpu")
# the read-only reference checkout the recipe compiles from (override: XT_REFERENCE_TREE)
REFERENCE_TREE = os.environ.get("XT_REFERENCE_TREE", "/root/reference")

_i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C")
_L = None


def build(ref: bool = True) -> None:
    """Compile liboracle.so, and oracle/_ref/ when the reference tree exists
    (the CPU binaries, and the single-GPU binary when nvcc is present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref and os.path.isdir(REFERENCE_TREE):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REFERENCE_TREE}"], check=True)
        if os.path.exists("/usr/local/cuda/bin/nvcc"):
            subprocess.run(["make", "-s", "-C", HERE, "refgpu", f"REF={REFERENCE_TREE}"], check=True)


def lib() -> ctypes.CDLL:
    global _L
    if _L is None:
        if not os.path.exists(LIB):
            build(ref=False)
        L = ctypes.CDLL(LIB)
        c = ctypes
        for name, res, args in [
            ("xo_count_xxtric", c.c_int64, [c.c_int64, _i64p, _i64p]),
            ("xo_count_merge", c.c_int64, [c.c_int64, _i64p, _i64p, c.c_void_p]),
            ("xo_local_counts", None, [c.c_int64, _i64p, _i64p, c.c_int64, _i64p, _i64p]),
            ("xo_edge_support", None, [c.c_int64, _i64p, _i64p, _i64p]),
            ("xo_canon_csr", c.c_int64, [c.c_int64, c.c_int64, _i64p, _i64p, _i64p, _i64p]),
            ("xo_rmat_edges", None, [c.c_int, c.c_uint64, c.c_int, c.c_int, c.c_int, c.c_int, c.c_int, c.c_int64,
                                     c.c_int64, _i64p, _i64p]),
            ("xo_chunglu_edges", None, [c.c_int64, _u64p, c.c_uint64, c.c_int, c.c_int64, c.c_int64, _i64p, _i64p]),
            ("xo_chunglu_cdf", c.c_int64, [c.c_int64, c.c_double, c.c_double, c.c_double, _u64p]),
            ("xo_er_edges", None, [c.c_int64, c.c_uint64, c.c_int64, c.c_int64, _i64p, _i64p]),
            ("xo_rgg_edges", c.c_int64, [c.c_int64, c.c_uint64, c.c_double, c.c_int64, _i64p, _i64p]),
            ("xo_ref_rgg", c.c_int64, [c.c_int64, c.c_int, c.c_double, c.c_int64, _i64p, _i64p]),
            ("xo_seed_seq1", c.c_uint32, [c.c_uint32]),
            ("xo_batch_spec", None, [c.c_int64, c.c_uint64, np.ctypeslib.ndpointer(np.int32, flags="C"), _i64p,
                                     np.ctypeslib.ndpointer(np.float64, flags="C"), _u64p]),
            ("xo_batch_graph", c.c_int64, [c.c_int32, c.c_int64, c.c_double, c.c_uint64, c.c_int64, _i64p, _i64p]),
        ]:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _L = L
    return _L


def count_xxtric(off: np.ndarray, tails: np.ndarray) -> int:
    """The reference's single-rank count (xxtric.hpp:60-80, 150-207, 516-588)."""
    off = np.ascontiguousarray(off, np.int64)
    tails = np.ascontiguousarray(tails, np.int64)
    return int(lib().xo_count_xxtric(len(off) - 1, off, tails))


def count_merge(off: np.ndarray, tails: np.ndarray, per_vertex: bool = False):
    off = np.ascontiguousarray(off, np.int64)
    tails = np.ascontiguousarray(tails, np.int64)
    pv = np.zeros(len(off) - 1, np.int64) if per_vertex else None
    t = int(lib().xo_count_merge(len(off) - 1, off, tails, pv.ctypes.data if per_vertex else None))
    return (t, pv) if per_vertex else t


def local_counts(off: np.ndarray, tails: np.ndarray, sel: np.ndarray) -> np.ndarray:
    off = np.ascontiguousarray(off, np.int64)
    tails = np.ascontiguousarray(tails, np.int64)
    sel = np.ascontiguousarray(sel, np.int64)
    out = np.zeros(len(sel), np.int64)
    lib().xo_local_counts(len(off) - 1, off, tails, len(sel), sel, out)
    return out


def edge_support(off: np.ndarray, tails: np.ndarray) -> np.ndarray:
    """Triangles on every CSR entry (a, b): |N(a) and N(b)|."""
    off = np.ascontiguousarray(off, np.int64)
    tails = np.ascontiguousarray(tails, np.int64)
    out = np.zeros(len(tails), np.int64)
    lib().xo_edge_support(len(off) - 1, off, tails, out)
    return out


def canon_csr(nv: int, src: np.ndarray, dst: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    src = np.ascontiguousarray(src, np.int64)
    dst = np.ascontiguousarray(dst, np.int64)
    off = np.zeros(nv + 1, np.int64)
    tails = np.zeros(2 * len(src), np.int64)
    m = int(lib().xo_canon_csr(nv, len(src), src, dst, off, tails))
    if m < 0:
        raise ValueError("vertex id outside [0, nv)")
    return off, tails[:m].copy()


def rmat_edges(scale: int, ne: int, seed: int, noise_pct: int = 10, permute: bool = True,
               a16: int = 37355, b16: int = 12452, c16: int = 12452, e0: int = 0):
    src = np.empty(ne, np.int64)
    dst = np.empty(ne, np.int64)
    lib().xo_rmat_edges(scale, seed, a16, b16, c16, noise_pct, int(permute), e0, e0 + ne, src, dst)
    return src, dst


def chunglu_cdf(n: int, gamma: float = 2.1, mean_deg: float = 64.0, max_deg: float = 131072.0):
    cdf = np.empty(n + 1, np.uint64)
    m = int(lib().xo_chunglu_cdf(n, gamma, mean_deg, max_deg, cdf))
    return cdf, m


def chunglu_edges(cdf: np.ndarray, ne: int, seed: int, permute: bool = True, e0: int = 0):
    src = np.empty(ne, np.int64)
    dst = np.empty(ne, np.int64)
    lib().xo_chunglu_edges(len(cdf) - 1, np.ascontiguousarray(cdf, np.uint64), seed, int(permute), e0, e0 + ne,
                           src, dst)
    return src, dst


def er_edges(n: int, ne: int, seed: int, e0: int = 0):
    src = np.empty(ne, np.int64)
    dst = np.empty(ne, np.int64)
    lib().xo_er_edges(n, seed, e0, e0 + ne, src, dst)
    return src, dst


def rgg_edges(n: int, seed: int, r2: float):
    cap = max(1024, int(n * 40))
    while True:
        src = np.empty(cap, np.int64)
        dst = np.empty(cap, np.int64)
        m = int(lib().xo_rgg_edges(n, seed, r2, cap, src, dst))
        if m >= 0:
            return src[:m].copy(), dst[:m].copy()
        cap = -m


def batch_spec(n_graphs: int, seed: int) -> dict:
    kind = np.zeros(n_graphs, np.int32)
    n = np.zeros(n_graphs, np.int64)
    deg = np.zeros(n_graphs, np.float64)
    gseed = np.zeros(n_graphs, np.uint64)
    lib().xo_batch_spec(n_graphs, seed, kind, n, deg, gseed)
    return {"kind": kind, "n": n, "mean_deg": deg, "graph_seed": gseed}


def batch_graph(kind: int, n: int, mean_deg: float, gseed: int):
    """One graph of the batch workload: (src, dst) local ids."""
    cap = max(1024, int(n * mean_deg))
    while True:
        src = np.empty(cap, np.int64)
        dst = np.empty(cap, np.int64)
        m = int(lib().xo_batch_graph(int(kind), int(n), float(mean_deg), int(gseed), cap, src, dst))
        if m >= 0:
            return src[:m].copy(), dst[:m].copy()
        cap = -m


def ref_rgg(nv: int, nprocs: int = 1, radius: float = 0.0):
    """The reference's RGG + LCG (graph.hpp:745-1364) for nprocs strip ranks, literal all-pairs form."""
    cap = nv * 64
    while True:
        off = np.zeros(nv + 1, np.int64)
        tails = np.zeros(cap, np.int64)
        m = int(lib().xo_ref_rgg(nv, nprocs, radius, cap, off, tails))
        if m == -1:
            raise ValueError("invalid RGG arguments")
        if m >= 0:
            return off, tails[:m].copy()
        cap = -m


def run_ref(args: list[str], omp: bool = False, threads: int | None = None, timeout: float = 3600,
            gpu: bool = False) -> dict:
    """Run the reference's own binary (CPU, or its single-GPU engine with
    gpu=True) and parse its output lines (main.cpp:129-190)."""
    exe = REF_TRIC_GPU if gpu else (REF_TRIC_OMP if omp else REF_TRIC)
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    if gpu:
        # modules load with the context (in the constructor), so the timed
        # count() holds the kernel, its synchronisation and the 8-byte read
        env["CUDA_MODULE_LOADING"] = "EAGER"
    r = subprocess.run([exe] + args, capture_output=True, text=True, timeout=timeout, env=env)
    out = {"rc": r.returncode, "stdout": r.stdout}
    for line in r.stdout.splitlines():
        if line.startswith("Number of triangles:"):
            out["triangles"] = int(line.split(":")[1])
        elif line.startswith("Number of edges:"):
            out["edges"] = int(line.split(":")[1])
        elif line.startswith("Number of vertices:"):
            out["vertices"] = int(line.split(":")[1])
        elif line.startswith("Avg/Min/Max times for local counting"):
            out["t_local"] = float(line.split(":")[1].split(",")[2])
        elif line.startswith("Avg/Min/Max execution time"):
            out["t_count"] = float(line.split(":")[1].split(",")[2])
    return out
