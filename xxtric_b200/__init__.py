"""xxtric_b200 — B200-native exact triangle counting (sm_100a CUDA behind a C ABI).

Python host mirror of the reference's single-device surface (sg0/xxtric):
``read_vite`` (BinaryEdgeList::read, graph.hpp:294-395), ``generate_rgg``
(GenerateRGG::generate, graph.hpp:745-1364), ``TriangleCountingSingle``
(xxtric-gpu.hpp:22-298: constructor builds, ``count()`` counts, ``clear()``
frees). Everything calls libxtb200.so through ctypes; there is no CPU
fallback — importing the package fails if the library is missing.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libxtb200.so")

XT_OK, XT_ERR_INVALID, XT_ERR_CUDA, XT_ERR_OOM, XT_ERR_IO, XT_ERR_OVERFLOW = 0, 1, 2, 3, 4, 5
XT_ERR_TIMEOUT, XT_ERR_ADMISSION, XT_ERR_NOT_READY, XT_ERR_NO_DEVICE, XT_ERR_CLOSED = 6, 7, 8, 9, 10
ORIENT_ID, ORIENT_DEGREE = 0, 1
LANE_BSEARCH, LANE_MERGE = 0, 1
CSR_CANONICAL = 1

# R-MAT quadrant weights a, b, c (d = rest) in 1/65536 units: .57/.19/.19/.05
RMAT_A16, RMAT_B16, RMAT_C16 = 37355, 12452, 12452


class XtError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python xxtric_b200/build.py` "
                          "(the CUDA library is required: there is no CPU fallback)")
    return ctypes.CDLL(LIB_PATH)


_L = _load()
_i64, _i32, _u64, _int, _dbl, _vp = (ctypes.c_int64, ctypes.c_int32, ctypes.c_uint64, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_void_p)
_P = ctypes.POINTER


class GraphInfo(ctypes.Structure):
    _fields_ = [("nv", _i64), ("n_input", _i64), ("n_edges", _i64), ("max_degree", _i64),
                ("max_out_degree", _i64), ("max_in_degree", _i64), ("wedge_work", _i64),
                ("stream_work", _i64), ("alg_bytes", _i64), ("tail_alg_bytes", _i64),
                ("orient", _i32), ("reserved", _i32), ("footprint_bytes", _i64), ("cluster_tasks", _i64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


def _proto(name, res, *args):
    f = getattr(_L, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_proto("xt_strerror", ctypes.c_char_p, _int)
_proto("xt_last_error", ctypes.c_char_p, _vp)
_proto("xt_open", _int, _int, _P(_vp))
_proto("xt_close", _int, _vp)
_proto("xt_set_stream", _int, _vp, _vp)
_proto("xt_debug_fail_alloc", _int, _vp, _i64)
_proto("xt_launch_count", _i64, _vp)
_proto("xt_synchronize", _int, _vp)
_proto("xt_graph_get_perm", _int, _vp, _vp)
_proto("xt_graph_from_csr", _int, _vp, _i64, _vp, _vp, _int, _int, _P(_vp))
_proto("xt_graph_from_edges", _int, _vp, _i64, _i64, _vp, _vp, _int, _P(_vp))
_proto("xt_graph_from_device_edges", _int, _vp, _i64, _i64, _vp, _vp, _int, _P(_vp))
_proto("xt_graph_get_info", _int, _vp, _P(GraphInfo))
_proto("xt_graph_get_csr", _int, _vp, _vp, _vp)
_proto("xt_graph_free", _int, _vp)
_proto("xt_count", _int, _vp, _vp, _vp)
_proto("xt_count_async", _int, _vp, _vp, _vp)
_proto("xt_count_edges", _int, _vp, _vp, _vp)
_proto("xt_count_edges_async", _int, _vp, _vp, _vp)
_proto("xt_count_shard_async", _int, _vp, _int, _int, _vp, _vp)
_proto("xt_count_edges_shard_async", _int, _vp, _int, _int, _vp, _vp)
_proto("xt_count_device", _int, _i64, _vp, _vp, _vp, _int, _vp)
_proto("xt_count_device_static", _int, _i64, _vp, _vp, _vp, _int, _vp)
_proto("xt_graph_from_batch", _int, _vp, _i64, _vp, _vp, _vp, _vp, _int, _P(_vp))
_proto("xt_graph_from_device_batch", _int, _vp, _i64, _vp, _vp, _vp, _vp, _int, _P(_vp))
_proto("xt_graph_groups", _i64, _vp)
_proto("xt_count_groups", _int, _vp, _vp, _vp)
_proto("xt_batch_count", _int, _vp, _i64, _vp, _vp, _vp, _vp, _int, _P(_i64), _vp)
_proto("xt_count_groups_async", _int, _vp, _vp, _vp)
_proto("xt_graph_capture", _int, _vp)
_proto("xt_graph_set_tuning", _int, _vp, _i64, _i64, _i64)
_proto("xt_graph_set_tiers", _int, _vp, _i64, _i64)
_proto("xt_graph_set_prefetch", _int, _vp, _int)
_proto("xt_graph_set_cluster", _int, _vp, _int)
_proto("xt_graph_set_lane_intersect", _int, _vp, _int)
_proto("xt_graph_set_claim", _int, _vp, _int)
_proto("xt_gen_rgg", _int, _vp, _i64, _int, _dbl, _i64, _P(_i64), _vp, _vp)
_proto("xt_graph_from_vite", _int, _vp, ctypes.c_char_p, _int, _int, _int, _P(_vp))
_proto("xt_graph_from_rgg", _int, _vp, _i64, _int, _dbl, _int, _P(_vp))
_proto("xt_graph_debug_cuckoo_iters", _int, _vp, _int)
_proto("xt_mem_stats", _int, _vp, _P(_i64), _P(_i64), _int)
_proto("xt_serve_estimate", _i64, _i64, _i64)
_proto("xt_serve_open", _int, _int, _vp, _P(_vp))
_proto("xt_serve_submit", _int, _vp, _i64, _i64, _vp, _vp, _P(_i64))
_proto("xt_serve_poll", _int, _vp, _i64, _P(_i64), _P(_dbl))
_proto("xt_serve_wait", _int, _vp, _i64, _i64, _P(_i64), _P(_dbl))
_proto("xt_serve_get_stats", _int, _vp, _vp)
_proto("xt_serve_close", _int, _vp)
_proto("xt_serve_batches", _i64, _vp, _vp, _i64)
_proto("xt_tsv_read", _int, ctypes.c_char_p, _P(_i64), _P(_i64), _vp, _vp, _i64)
_proto("xt_tsv_write", _int, ctypes.c_char_p, _i64, _vp, _vp)
_proto("xt_graph_autotune", _int, _vp, _int, ctypes.c_char_p, _vp, _i64)
_proto("xt_batch_spec", _int, _i64, _u64, _vp, _vp, _vp, _vp)
_proto("xt_gen_batch", _int, _vp, _i64, _vp, _vp, _vp, _vp, _vp, _P(_vp), _P(_vp))
_proto("xt_device_free", _int, _vp, _vp)
_proto("xt_gen_rmat", _int, _vp, _int, _i64, _u64, _int, _int, _int, _int, _int, _vp, _vp)
_proto("xt_gen_chunglu", _int, _vp, _i64, _vp, _i64, _u64, _int, _vp, _vp)
_proto("xt_chunglu_cdf", _i64, _i64, _dbl, _dbl, _dbl, _vp)
_proto("xt_gen_er", _int, _vp, _i64, _i64, _u64, _vp, _vp)
_proto("xt_vite_read", _int, ctypes.c_char_p, _int, _P(_i64), _P(_i64), _vp, _vp)
_proto("xt_vite_write", _int, ctypes.c_char_p, _int, _i64, _vp, _vp)
_proto("xt_rgg_generate", _int, _i64, _int, _dbl, _dbl, _u64, _i64, _P(_i64), _vp, _vp)

EXPORTED = ["xt_strerror", "xt_last_error", "xt_open", "xt_close", "xt_set_stream", "xt_debug_fail_alloc",
            "xt_launch_count", "xt_synchronize", "xt_graph_get_perm",
            "xt_graph_from_csr", "xt_graph_from_edges", "xt_graph_from_device_edges", "xt_graph_get_info",
            "xt_graph_get_csr", "xt_graph_free", "xt_count", "xt_count_async", "xt_count_edges", "xt_count_edges_async",
            "xt_count_shard_async", "xt_count_edges_shard_async", "xt_count_device",
            "xt_count_device_static", "xt_graph_from_batch", "xt_graph_from_device_batch", "xt_graph_groups",
            "xt_count_groups", "xt_count_groups_async", "xt_batch_count", "xt_graph_capture", "xt_graph_set_tuning", "xt_graph_set_tiers", "xt_graph_set_prefetch", "xt_graph_set_cluster", "xt_graph_set_lane_intersect", "xt_graph_set_claim",
            "xt_graph_debug_cuckoo_iters",
            "xt_mem_stats", "xt_serve_estimate", "xt_serve_open", "xt_serve_submit", "xt_serve_poll",
            "xt_serve_wait", "xt_serve_get_stats", "xt_serve_close", "xt_serve_batches", "xt_tsv_read", "xt_tsv_write",
            "xt_graph_autotune", "xt_batch_spec", "xt_gen_batch", "xt_device_free",
            "xt_gen_rmat", "xt_gen_chunglu", "xt_chunglu_cdf", "xt_gen_er", "xt_gen_rgg", "xt_graph_from_vite",
            "xt_graph_from_rgg", "xt_vite_read", "xt_vite_write",
            "xt_rgg_generate"]


def lib() -> ctypes.CDLL:
    return _L


def strerror(s: int) -> str:
    return _L.xt_strerror(s).decode()


def _check(s: int, what: str, ctx: Optional["Context"] = None) -> None:
    if s != XT_OK:
        detail = ""
        if ctx is not None and ctx._h:
            detail = _L.xt_last_error(ctx._h).decode()
        raise XtError(s, f"{what}: {strerror(s)}" + (f" ({detail})" if detail else ""))


def _ptr(a) -> int:
    """Device or host address of a numpy array, torch tensor or int."""
    if a is None:
        return 0
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())  # torch.Tensor


# ---------------------------------------------------------------------------
# host-side input: vite files and the reference's RGG generator
# ---------------------------------------------------------------------------

def read_vite(path: str, elem_bytes: int = 8) -> tuple[np.ndarray, np.ndarray]:
    """BinaryEdgeList::read for one process: (offsets int64[nv+1], tails int64[ne])."""
    nv, ne = _i64(0), _i64(0)
    _check(_L.xt_vite_read(path.encode(), elem_bytes, ctypes.byref(nv), ctypes.byref(ne), None, None),
           f"reading {path}")
    off = np.empty(nv.value + 1, np.int64)
    tails = np.empty(ne.value, np.int64)
    _check(_L.xt_vite_read(path.encode(), elem_bytes, ctypes.byref(nv), ctypes.byref(ne), _ptr(off), _ptr(tails)),
           f"reading {path}")
    return off, tails


def write_vite(path: str, offsets: np.ndarray, tails: np.ndarray, elem_bytes: int = 8) -> None:
    off = np.ascontiguousarray(offsets, np.int64)
    t = np.ascontiguousarray(tails, np.int64)
    _check(_L.xt_vite_write(path.encode(), elem_bytes, len(off) - 1, _ptr(off), _ptr(t)), f"writing {path}")


def read_tsv(path: str) -> tuple[int, np.ndarray, np.ndarray]:
    """Tab-separated edge list (src, dst[, weight]) with ids as given:
    (nv = largest id + 1, src int32, dst int32)."""
    nv, ne = _i64(0), _i64(0)
    _check(_L.xt_tsv_read(path.encode(), ctypes.byref(nv), ctypes.byref(ne), None, None, 0), f"reading {path}")
    src = np.empty(ne.value, np.int32)
    dst = np.empty(ne.value, np.int32)
    _check(_L.xt_tsv_read(path.encode(), ctypes.byref(nv), ctypes.byref(ne), _ptr(src), _ptr(dst), len(src)),
           f"reading {path}")
    return nv.value, src, dst


def write_tsv(path: str, src: np.ndarray, dst: np.ndarray) -> None:
    s = np.ascontiguousarray(src, np.int32)
    d = np.ascontiguousarray(dst, np.int32)
    _check(_L.xt_tsv_write(path.encode(), len(s), _ptr(s), _ptr(d)), f"writing {path}")


def generate_rgg(nv: int, nprocs: int = 1, radius: float = 0.0, random_edge_pct: float = 0.0,
                 seed: int = 1) -> tuple[np.ndarray, np.ndarray]:
    """GenerateRGG(nv).generate(LCG, unit weights, pct) as `nprocs` strip ranks build it."""
    ne = _i64(0)
    _check(_L.xt_rgg_generate(nv, nprocs, radius, random_edge_pct, seed, 0, ctypes.byref(ne), None, None),
           "generate_rgg")
    off = np.empty(nv + 1, np.int64)
    tails = np.empty(ne.value, np.int64)
    _check(_L.xt_rgg_generate(nv, nprocs, radius, random_edge_pct, seed, ne.value, ctypes.byref(ne), _ptr(off),
                              _ptr(tails)), "generate_rgg")
    return off, tails


def batch_spec(n_graphs: int, seed: int) -> dict:
    """The batch workload's per-graph parameters (xt_batch_spec)."""
    kind = np.zeros(n_graphs, np.int32)
    n = np.zeros(n_graphs, np.int64)
    deg = np.zeros(n_graphs, np.float64)
    gseed = np.zeros(n_graphs, np.uint64)
    _check(_L.xt_batch_spec(n_graphs, seed, _ptr(kind), _ptr(n), _ptr(deg), _ptr(gseed)), "xt_batch_spec")
    return {"kind": kind, "n": n, "mean_deg": deg, "graph_seed": gseed}


class DeviceArray:
    """A library-owned device array (released with the context's allocator);
    torch.as_tensor(arr, device='cuda') views it without a copy."""

    def __init__(self, ctx: "Context", ptr: int, n: int, typestr: str, itemsize: int):
        self.ctx, self.ptr, self.n, self.typestr, self.itemsize = ctx, ptr, n, typestr, itemsize

    @property
    def __cuda_array_interface__(self):
        return {"shape": (self.n,), "typestr": self.typestr, "data": (self.ptr, False), "version": 3}

    def data_ptr(self) -> int:
        return self.ptr

    def free(self) -> None:
        if self.ptr and self.ctx._h:
            _check(_L.xt_device_free(self.ctx._h, self.ptr), "xt_device_free", self.ctx)
        self.ptr = 0


def chunglu_cdf(n: int, gamma: float = 2.1, mean_deg: float = 64.0, max_deg: float = 131072.0):
    cdf = np.empty(n + 1, np.uint64)
    m = _L.xt_chunglu_cdf(n, gamma, mean_deg, max_deg, _ptr(cdf))
    if m < 0:
        raise XtError(XT_ERR_INVALID, "chunglu_cdf: bad arguments")
    return cdf, int(m)


# ---------------------------------------------------------------------------
# device: context, graphs, counting, generators
# ---------------------------------------------------------------------------

class Context:
    """One device + one CUDA stream (xt_open)."""

    def __init__(self, device: int = 0):
        h = _vp()
        s = _L.xt_open(device, ctypes.byref(h))
        if s != XT_OK:
            raise XtError(s, f"xt_open({device}): {strerror(s)}")
        self._h = h.value
        self.device = device

    def close(self) -> None:
        if self._h:
            _L.xt_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int) -> None:
        _check(_L.xt_set_stream(self._h, stream_ptr), "xt_set_stream", self)

    def fail_alloc_after(self, k: int) -> None:
        _check(_L.xt_debug_fail_alloc(self._h, k), "xt_debug_fail_alloc", self)

    @property
    def last_error(self) -> str:
        return _L.xt_last_error(self._h).decode()

    @property
    def launches(self) -> int:
        """This library's kernels launched on the context so far."""
        return int(_L.xt_launch_count(self._h))

    def mem_stats(self, reset_peak: bool = False) -> tuple[int, int]:
        """(live, peak) device bytes of this context's own allocations."""
        live, peak = _i64(0), _i64(0)
        _check(_L.xt_mem_stats(self._h, ctypes.byref(live), ctypes.byref(peak), int(reset_peak)), "xt_mem_stats",
               self)
        return live.value, peak.value

    # -- graphs --
    def graph_from_vite(self, path: str, elem_bytes: int = 8, canonical: bool = False,
                        orient: int = ORIENT_DEGREE) -> "DeviceGraph":
        """A vite binary file read through the device (xt_graph_from_vite)."""
        h = _vp()
        _check(_L.xt_graph_from_vite(self._h, path.encode(), elem_bytes, CSR_CANONICAL if canonical else 0, orient,
                                     ctypes.byref(h)), "xt_graph_from_vite", self)
        return DeviceGraph(self, h.value)

    def graph_from_rgg(self, nv: int, nprocs: int = 1, radius: float = 0.0,
                       orient: int = ORIENT_DEGREE) -> "DeviceGraph":
        """The reference's random geometric graph generated and built on the device."""
        h = _vp()
        _check(_L.xt_graph_from_rgg(self._h, nv, nprocs, radius, orient, ctypes.byref(h)), "xt_graph_from_rgg", self)
        return DeviceGraph(self, h.value)

    def graph_from_csr(self, offsets: np.ndarray, tails: np.ndarray, canonical: bool = False,
                       orient: int = ORIENT_DEGREE) -> "DeviceGraph":
        off = np.ascontiguousarray(offsets, np.int64)
        t = np.ascontiguousarray(tails, np.int64)
        h = _vp()
        _check(_L.xt_graph_from_csr(self._h, len(off) - 1, _ptr(off), _ptr(t), CSR_CANONICAL if canonical else 0,
                                    orient, ctypes.byref(h)), "xt_graph_from_csr", self)
        return DeviceGraph(self, h.value)

    def graph_from_edges(self, nv: int, src: np.ndarray, dst: np.ndarray,
                         orient: int = ORIENT_DEGREE) -> "DeviceGraph":
        s = np.ascontiguousarray(src, np.int32)
        d = np.ascontiguousarray(dst, np.int32)
        h = _vp()
        _check(_L.xt_graph_from_edges(self._h, nv, len(s), _ptr(s), _ptr(d), orient, ctypes.byref(h)),
               "xt_graph_from_edges", self)
        return DeviceGraph(self, h.value)

    def graph_from_device_edges(self, nv: int, ne: int, d_src, d_dst, orient: int = ORIENT_DEGREE) -> "DeviceGraph":
        h = _vp()
        _check(_L.xt_graph_from_device_edges(self._h, nv, ne, _ptr(d_src), _ptr(d_dst), orient, ctypes.byref(h)),
               "xt_graph_from_device_edges", self)
        return DeviceGraph(self, h.value)

    def synchronize(self) -> None:
        _check(_L.xt_synchronize(self._h), "xt_synchronize", self)

    # -- batching form --
    def gen_batch(self, spec: dict):
        """Generate the batch's graphs on the device: (edge_offsets, src, dst)
        with local ids; src/dst are DeviceArray (free them when done)."""
        ng = len(spec["n"])
        kind = np.ascontiguousarray(spec["kind"], np.int32)
        n = np.ascontiguousarray(spec["n"], np.int64)
        deg = np.ascontiguousarray(spec["mean_deg"], np.float64)
        seed = np.ascontiguousarray(spec["graph_seed"], np.uint64)
        eoff = np.zeros(ng + 1, np.int64)
        ps, pd = _vp(), _vp()
        _check(_L.xt_gen_batch(self._h, ng, _ptr(kind), _ptr(n), _ptr(deg), _ptr(seed), _ptr(eoff),
                               ctypes.byref(ps), ctypes.byref(pd)), "xt_gen_batch", self)
        ne = int(eoff[-1])
        return eoff, DeviceArray(self, ps.value or 0, ne, "<i4", 4), DeviceArray(self, pd.value or 0, ne, "<i4", 4)

    def batch_count(self, vertex_offsets, edge_offsets, src, dst, orient: int = ORIENT_DEGREE):
        """Build, count and free a batch in one call (xt_batch_count): (total, per-graph counts)."""
        voff = np.ascontiguousarray(vertex_offsets, np.int64)
        eoff = np.ascontiguousarray(edge_offsets, np.int64)
        s_ = np.ascontiguousarray(src, np.int32)
        d_ = np.ascontiguousarray(dst, np.int32)
        per = np.zeros(len(voff) - 1, np.int64)
        t = _i64(0)
        _check(_L.xt_batch_count(self._h, len(voff) - 1, _ptr(voff), _ptr(eoff), _ptr(s_), _ptr(d_), orient,
                                 ctypes.byref(t), _ptr(per)), "xt_batch_count", self)
        return t.value, per

    def graph_from_batch(self, vertex_offsets, edge_offsets, src, dst, orient: int = ORIENT_DEGREE,
                         device: bool = False) -> "DeviceGraph":
        """Many graphs as one (local ids per graph); device=True when src/dst are device arrays."""
        voff = np.ascontiguousarray(vertex_offsets, np.int64)
        eoff = np.ascontiguousarray(edge_offsets, np.int64)
        h = _vp()
        if device:
            s = _L.xt_graph_from_device_batch(self._h, len(voff) - 1, _ptr(voff), _ptr(eoff), _ptr(src), _ptr(dst),
                                              orient, ctypes.byref(h))
        else:
            s_ = np.ascontiguousarray(src, np.int32)
            d_ = np.ascontiguousarray(dst, np.int32)
            s = _L.xt_graph_from_batch(self._h, len(voff) - 1, _ptr(voff), _ptr(eoff), _ptr(s_), _ptr(d_), orient,
                                       ctypes.byref(h))
        _check(s, "xt_graph_from_batch", self)
        return DeviceGraph(self, h.value)

    # -- generators (device int32 outputs: torch tensors or raw pointers). They
    # run on the context stream; sync=True waits for them, so the outputs can
    # be read from any other stream right away.
    def gen_rmat(self, scale: int, ne: int, seed: int, d_src, d_dst, noise_pct: int = 10, permute: bool = True,
                 a16: int = RMAT_A16, b16: int = RMAT_B16, c16: int = RMAT_C16, sync: bool = True) -> None:
        _check(_L.xt_gen_rmat(self._h, scale, ne, seed, a16, b16, c16, noise_pct, int(permute), _ptr(d_src),
                              _ptr(d_dst)), "xt_gen_rmat", self)
        if sync:
            self.synchronize()

    def gen_chunglu(self, cdf: np.ndarray, ne: int, seed: int, d_src, d_dst, permute: bool = True,
                    sync: bool = True) -> None:
        c = np.ascontiguousarray(cdf, np.uint64)
        _check(_L.xt_gen_chunglu(self._h, len(c) - 1, _ptr(c), ne, seed, int(permute), _ptr(d_src), _ptr(d_dst)),
               "xt_gen_chunglu", self)
        if sync:
            self.synchronize()

    def gen_rgg(self, nv: int, nprocs: int = 1, radius: float = 0.0):
        """The reference's random geometric graph (as nprocs strip ranks build
        it) generated on the device: (n_pairs, src, dst), int32 torch tensors
        on this context's device holding each undirected edge once (a < b)."""
        import torch
        n = ctypes.c_int64(0)
        _check(_L.xt_gen_rgg(self._h, nv, nprocs, radius, 0, ctypes.byref(n), None, None), "xt_gen_rgg", self)
        src = torch.empty(max(1, n.value), dtype=torch.int32, device=f"cuda:{self.device}")
        dst = torch.empty_like(src)
        _check(_L.xt_gen_rgg(self._h, nv, nprocs, radius, n.value, ctypes.byref(n), _ptr(src), _ptr(dst)),
               "xt_gen_rgg", self)
        self.synchronize()
        return n.value, src[:n.value], dst[:n.value]

    def gen_er(self, n: int, ne: int, seed: int, d_src, d_dst, sync: bool = True) -> None:
        _check(_L.xt_gen_er(self._h, n, ne, seed, _ptr(d_src), _ptr(d_dst)), "xt_gen_er", self)
        if sync:
            self.synchronize()


class DeviceGraph:
    """Oriented device CSR (+ its transpose and schedule) owned by the library."""

    def __init__(self, ctx: Context, handle: int):
        self.ctx = ctx
        self._h = handle

    def info(self) -> dict:
        i = GraphInfo()
        _check(_L.xt_graph_get_info(self._h, ctypes.byref(i)), "xt_graph_get_info", self.ctx)
        return i.as_dict()

    @property
    def nv(self) -> int:
        return self.info()["nv"]

    def perm(self) -> np.ndarray:
        """internal id -> input id."""
        p = np.empty(self.nv, np.int32)
        _check(_L.xt_graph_get_perm(self._h, _ptr(p)), "xt_graph_get_perm", self.ctx)
        return p

    def csr(self) -> tuple[np.ndarray, np.ndarray]:
        """The oriented CSR in internal numbering (see perm())."""
        inf = self.info()
        off = np.empty(inf["nv"] + 1, np.int64)
        col = np.empty(inf["n_edges"], np.int32)
        _check(_L.xt_graph_get_csr(self._h, _ptr(off), _ptr(col)), "xt_graph_get_csr", self.ctx)
        return off, col

    def count(self, per_vertex: bool = False):
        g = _i64(0)
        pv = np.empty(self.nv, np.int64) if per_vertex else None
        _check(_L.xt_count(self._h, ctypes.byref(g), _ptr(pv)), "xt_count", self.ctx)
        return (g.value, pv) if per_vertex else g.value

    def count_edges(self):
        """(total, support): triangles on every oriented edge, in the order of
        csr() (internal numbering)."""
        g = _i64(0)
        sup = np.empty(self.info()["n_edges"], np.int64)
        _check(_L.xt_count_edges(self._h, ctypes.byref(g), _ptr(sup)), "xt_count_edges", self.ctx)
        return g.value, sup

    def edge_support(self):
        """(src, dst, support) per undirected edge in INPUT ids, src < dst."""
        off, col = self.csr()
        _, sup = self.count_edges()
        p = self.perm()
        a = p[np.repeat(np.arange(len(off) - 1), np.diff(off))].astype(np.int64)
        b = p[col].astype(np.int64)
        return np.minimum(a, b), np.maximum(a, b), sup

    def degrees(self) -> np.ndarray:
        """Undirected degree of every vertex, input ids."""
        off, col = self.csr()
        d = np.diff(off) + np.bincount(col, minlength=len(off) - 1)
        out = np.empty_like(d)
        out[self.perm()] = d
        return out

    def clustering(self) -> np.ndarray:
        """Local clustering coefficient 2 T(v) / (d(v) (d(v) - 1)) per vertex
        (0 below degree 2), from the per-vertex counts."""
        _, pv = self.count(per_vertex=True)
        d = self.degrees().astype(np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            c = np.where(d >= 2, 2.0 * pv / (d * (d - 1.0)), 0.0)
        return c

    def count_async(self, d_global, d_per_vertex=None) -> None:
        _check(_L.xt_count_async(self._h, _ptr(d_global), _ptr(d_per_vertex)), "xt_count_async", self.ctx)

    def count_edges_async(self, d_global, d_support) -> None:
        """Global count and per-edge supports into device memory (d_support:
        n_edges int64 entries), queued on the context stream."""
        _check(_L.xt_count_edges_async(self._h, _ptr(d_global), _ptr(d_support)), "xt_count_edges_async", self.ctx)

    def count_shard_async(self, shard: int, nshards: int, d_global, d_per_vertex=None) -> None:
        """Shard `shard` of `nshards` of the count (every nshards-th task of the
        schedule) into device memory, queued on the context stream; the
        shards' outputs sum to count_async's."""
        _check(_L.xt_count_shard_async(self._h, int(shard), int(nshards), _ptr(d_global), _ptr(d_per_vertex)),
               "xt_count_shard_async", self.ctx)

    def count_edges_shard_async(self, shard: int, nshards: int, d_global, d_support) -> None:
        """Shard `shard` of `nshards` of the per-edge count (see count_shard_async)."""
        _check(_L.xt_count_edges_shard_async(self._h, int(shard), int(nshards), _ptr(d_global), _ptr(d_support)),
               "xt_count_edges_shard_async", self.ctx)

    @property
    def groups(self) -> int:
        return int(_L.xt_graph_groups(self._h))

    def count_groups(self):
        """(total, per-graph counts) of a batch."""
        t = _i64(0)
        per = np.zeros(max(self.groups, 0), np.int64)
        _check(_L.xt_count_groups(self._h, ctypes.byref(t), _ptr(per) if len(per) else None), "xt_count_groups",
               self.ctx)
        return t.value, per

    def count_groups_async(self, d_total, d_per_group=None) -> None:
        _check(_L.xt_count_groups_async(self._h, _ptr(d_total), _ptr(d_per_group)), "xt_count_groups_async",
               self.ctx)

    def capture(self) -> None:
        _check(_L.xt_graph_capture(self._h), "xt_graph_capture", self.ctx)

    def set_tuning(self, block_work: int = 0, warp_work: int = 0, bitmap_bits: int = 0) -> None:
        _check(_L.xt_graph_set_tuning(self._h, block_work, warp_work, bitmap_bits), "xt_graph_set_tuning", self.ctx)

    def set_prefetch(self, on: bool) -> None:
        """Bulk L2 prefetch of each in-record's suffix one batch ahead (global count)."""
        _check(_L.xt_graph_set_prefetch(self._h, int(on)), "xt_graph_set_prefetch", self.ctx)

    def set_lane_intersect(self, kind: int) -> None:
        """Lane tier: members found by binary search (LANE_BSEARCH, default) or a two-pointer merge (LANE_MERGE)."""
        _check(_L.xt_graph_set_lane_intersect(self._h, int(kind)), "xt_graph_set_lane_intersect", self.ctx)

    def set_claim(self, claim: int) -> None:
        """Warp tasks (and groups of 32 lane tasks) taken per atomic on their cursor: 1..64, 0 automatic."""
        _check(_L.xt_graph_set_claim(self._h, int(claim)), "xt_graph_set_claim", self.ctx)

    def set_cluster(self, on: bool) -> None:
        """Global count: heads over a CTA's member set on thread-block clusters, or CTA parts (default)."""
        _check(_L.xt_graph_set_cluster(self._h, int(on)), "xt_graph_set_cluster", self.ctx)

    def debug_cuckoo_iters(self, iters: int) -> None:
        """Test hook: cap the cuckoo member sets' eviction chains (-1: default)."""
        _check(_L.xt_graph_debug_cuckoo_iters(self._h, iters), "xt_graph_debug_cuckoo_iters", self.ctx)

    def set_tiers(self, lane_work: int = -1, warp_work: int = -1) -> None:
        """Tier limits of the schedule: heads with at most lane_work candidates
        go one per lane, then heads with at most warp_work candidates (and at
        most 256 members) one per warp, the rest to CTA tasks. -1 = automatic,
        0 = tier off."""
        _check(_L.xt_graph_set_tiers(self._h, lane_work, warp_work), "xt_graph_set_tiers", self.ctx)

    def autotune(self, reps: int = 3, cache_path: Optional[str] = None) -> dict:
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        _check(_L.xt_graph_autotune(self._h, reps, cache_path.encode() if cache_path else None, buf, len(buf)),
               "xt_graph_autotune", self.ctx)
        return json.loads(buf.value.decode() or "{}")

    def free(self) -> None:
        if self._h:
            _L.xt_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            if self.ctx._h:
                self.free()
        except Exception:
            pass


def count_device(nv: int, d_indices, d_edge_list, d_count, accumulate: bool = False, stream: int = 0) -> None:
    """single_gpu_count replacement on the reference's device CSR layout (int64 offsets and tails)."""
    s = _L.xt_count_device(nv, _ptr(d_indices), _ptr(d_edge_list), _ptr(d_count), int(accumulate), stream)
    _check(s, "xt_count_device")


def count_device_static(nv: int, d_indices, d_edge_list, d_count, accumulate: bool = False,
                        stream: int = 0) -> None:
    """Like count_device, for callers that must not allocate device memory: all
    scratch lives in a fixed array inside the library (8 bytes per vertex, at
    most 8,389,088 vertices); calls on one device must not overlap."""
    s = _L.xt_count_device_static(nv, _ptr(d_indices), _ptr(d_edge_list), _ptr(d_count), int(accumulate), stream)
    _check(s, "xt_count_device_static")


class TriangleCountingSingle:
    """Mirror of TriangleCountingSingle (xxtric-gpu.hpp:22-298) over a host CSR."""

    def __init__(self, offsets: np.ndarray, tails: np.ndarray, orient: int = ORIENT_DEGREE, device: int = 0):
        self.ctx = Context(device)
        self.graph = self.ctx.graph_from_csr(offsets, tails, canonical=False, orient=orient)

    def count(self) -> int:
        return self.graph.count()

    def clear(self) -> None:
        if self.graph is not None:
            self.graph.free()
            self.graph = None
        if self.ctx is not None:
            self.ctx.close()
            self.ctx = None


# ---------------------------------------------------------------------------
# serving form
# ---------------------------------------------------------------------------

class ServeConfig(ctypes.Structure):
    _fields_ = [("budget_bytes", _i64), ("max_batch_graphs", _i64), ("max_batch_edges", _i64),
                ("slots", _i32), ("orient", _i32)]


class ServeStats(ctypes.Structure):
    _fields_ = [(k, _i64) for k in ("budget_bytes", "submitted", "completed", "failed", "rejected", "queued",
                                    "in_flight", "batches", "max_batch", "budget_used", "budget_peak",
                                    "device_peak", "launches")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServeBatch(ctypes.Structure):
    _fields_ = [("t_take_ns", _i64), ("t_built_ns", _i64), ("t_done_ns", _i64), ("graphs", _i64),
                ("edge_rows", _i64), ("slot", _i32), ("status", _i32)]


def serve_estimate(nv: int, ne: int) -> int:
    """Device bytes one query of nv vertices and ne edge rows may hold (admission figure)."""
    return int(_L.xt_serve_estimate(nv, ne))


class Server:
    """Count queries admitted under a device-memory budget and batched as slots
    free up (xt_serve_*). submit() returns a ticket; poll()/wait() return
    (count, latency seconds) once, raising XtError for a failed query."""

    def __init__(self, device: int = 0, budget_bytes: int = 0, slots: int = 0, orient: int = ORIENT_DEGREE,
                 max_batch_graphs: int = 0, max_batch_edges: int = 0):
        cfg = ServeConfig(budget_bytes, max_batch_graphs, max_batch_edges, slots, orient)
        h = _vp()
        s = _L.xt_serve_open(device, ctypes.byref(cfg), ctypes.byref(h))
        if s != XT_OK:
            raise XtError(s, f"xt_serve_open({device}): {strerror(s)}")
        self._h = h.value
        self._keep = {}  # ticket -> the host arrays the query reads until it finishes

    def submit(self, nv: int, src: np.ndarray, dst: np.ndarray) -> int:
        s_ = np.ascontiguousarray(src, np.int32)
        d_ = np.ascontiguousarray(dst, np.int32)
        if len(s_) != len(d_):
            raise XtError(XT_ERR_INVALID, "src and dst differ in length")
        t = _i64(0)
        _check(_L.xt_serve_submit(self._h, nv, len(s_), _ptr(s_), _ptr(d_), ctypes.byref(t)), "xt_serve_submit")
        self._keep[t.value] = (s_, d_)
        return t.value

    def _result(self, s: int, ticket: int, c, lat):
        if s == XT_ERR_NOT_READY:
            return None
        self._keep.pop(ticket, None)
        _check(s, f"query {ticket}")
        return c.value, lat.value

    def poll(self, ticket: int):
        """(count, latency_s), or None while the query runs."""
        c, lat = _i64(0), _dbl(0)
        return self._result(_L.xt_serve_poll(self._h, ticket, ctypes.byref(c), ctypes.byref(lat)), ticket, c, lat)

    def wait(self, ticket: int, timeout_ms: int = -1):
        c, lat = _i64(0), _dbl(0)
        s = _L.xt_serve_wait(self._h, ticket, timeout_ms, ctypes.byref(c), ctypes.byref(lat))
        if s == XT_ERR_TIMEOUT:
            raise XtError(s, f"query {ticket}: no result within {timeout_ms} ms")
        return self._result(s, ticket, c, lat)

    def stats(self) -> dict:
        st = ServeStats()
        _check(_L.xt_serve_get_stats(self._h, ctypes.byref(st)), "xt_serve_get_stats")
        return st.as_dict()

    def batches(self, max_n: int = 65536) -> list[dict]:
        """The most recent batches: times (s since open), graphs, edge rows, slot, status."""
        buf = (ServeBatch * max_n)()
        n = _L.xt_serve_batches(self._h, buf, max_n)
        if n < 0:
            raise XtError(XT_ERR_INVALID, "xt_serve_batches")
        return [{"take": b.t_take_ns * 1e-9, "built": b.t_built_ns * 1e-9, "done": b.t_done_ns * 1e-9,
                 "graphs": b.graphs, "edge_rows": b.edge_rows, "slot": b.slot, "status": b.status}
                for b in buf[:n]]

    def close(self) -> None:
        if self._h:
            _L.xt_serve_close(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
