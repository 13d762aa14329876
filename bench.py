#!/usr/bin/env python
"""Headline benchmark: exact triangle count of the scale-24 R-MAT graph on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl xtric|reference]
                    [--workload rmat24|chunglu|rgg|batch|serve]

Workload (one step, default rmat24): one exact count of R-MAT scale 24
(16,777,216 vertices, edge factor 16 -> 268,435,456 generated edges;
quadrants .57/.19/.19/.05 with 10% per-level noise; ids permuted;
symmetrised, deduplicated, self loops dropped; degree-oriented int32 columns
/ int64 offsets), graph resident in HBM. Metric: oriented edges counted per
second (|E+| per step / step time).

  value : device time of the count kernel over K steps (CUDA events on the
          launching stream), graph already in HBM. The graph (2.1 GB of CSR
          + transpose) is far larger than L2 (126 MB), so no flush is needed.
  e2e   : the same metric through the public C ABI with host buffers: the
          int32 edge list copied from pinned host memory, built into the
          oriented CSR on the device, counted, the count read back.
N > 1 GPUs (torchrun): independent replicas, one graph per GPU, no data-path
collective; value = all ranks' edges / the slowest rank's time. With
--shard, the GPUs count ONE graph together instead: every rank holds the
graph and counts its shard of the schedule (xxtric_b200.shards), and an NCCL
all-reduce of the count closes each step; value = the graph's edges / the
slowest rank's time (strong scaling).

Other single-graph workloads, same line: chunglu (the heavy-skew Chung-Lu
graph, n = 4,194,304, exponent 2.1, mean degree 64, max expected 131,072;
also times the per-vertex kernel and the id orientation) and rgg (the
reference's own random geometric graph, n = 65,536, r = sqrt(16/(pi n)), as
two strip ranks build it). batch and serve are the batching and serving
forms (graphs/s; see run_batch and run_serve).

--impl reference times the reference's own CPU counting path
(oracle/_ref/tric_omp: main.cpp + xxtric.hpp built with USE_OPENMP against a
one-rank MPI shim) on this host's cores, on a bounded sample of the same
workload: for rmat24 the R-MAT graph of the same generator at scale 18; for
chunglu a Chung-Lu graph of n = 131,072; for rgg the workload graph itself.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "oriented edges/s"
UNIT = "edges/s"
SCALE = 24
EDGE_FACTOR = 16
SEED = 1
SAMPLE_SCALE = 18



def env_ranks() -> tuple[int, int, int]:
    """(rank, world, local rank) from torchrun's environment, without joining
    a process group or loading the product library."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return rank, world, int(os.environ.get("LOCAL_RANK", str(rank)))


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled_value(name: str, key: str):
    """A `key: value` line of the committed ncu summary profiles/<name> (the
    figures the roofline takes from a capture: DRAM bytes per launch, issue
    utilisation), or None when there is no such summary."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "100"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[4:]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        smax = max(r[1] for r in rows)
        loaded = [r for r in rows if r[2] > 250.0] or rows
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in loaded:
            for n, v in zip(names, r[3][1:]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": smax,
                "power_w_max": max(r[2] for r in rows), "samples": len(rows), "samples_under_load": len(loaded),
                "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# single-graph workloads
# ---------------------------------------------------------------------------

CHUNGLU_N, CHUNGLU_GAMMA, CHUNGLU_MEAN, CHUNGLU_MAX = 4194304, 2.1, 64.0, 131072.0
RGG_N, RGG_RANKS = 65536, 2


class Workload:
    """One graph counted per step: how to make it on the device, what it is
    called, and the bounded sample the CPU reference is timed on."""

    def __init__(self, key: str, scale: int = SCALE):
        self.key = key
        self.scale = scale
        if key == "rmat24":
            self.name = workload_name(scale)
            self.extra = {"scale": scale, "edge_factor": EDGE_FACTOR}
        elif key == "chunglu":
            self.name = (f"Chung-Lu, n={CHUNGLU_N:,}, degree exponent {CHUNGLU_GAMMA}, mean degree {CHUNGLU_MEAN:g}, "
                         f"max expected degree {CHUNGLU_MAX:,.0f}, ids permuted; symmetrised + deduped, "
                         "degree-oriented, int32 cols / int64 offsets")
            self.extra = {"n": CHUNGLU_N, "gamma": CHUNGLU_GAMMA, "mean_degree": CHUNGLU_MEAN,
                          "max_expected_degree": CHUNGLU_MAX}
        elif key == "rgg":
            self.radius = float(np.sqrt(16.0 / (np.pi * RGG_N)))
            self.name = (f"random geometric graph of the reference's generator (LCG seed 1, -l), n={RGG_N:,} in the "
                         f"unit square, r=sqrt(16/(pi n))={self.radius:.5f}, -p 0, as mpiexec -n {RGG_RANKS} builds "
                         "it; degree-oriented")
            self.extra = {"n": RGG_N, "radius": self.radius, "strip_ranks": RGG_RANKS}
        else:
            raise ValueError(key)

    def device_edges(self, ctx, torch):
        """(nv, src, dst): int32 edge rows in device memory."""
        import xxtric_b200 as xt
        if self.key == "rmat24":
            n, ne = 1 << self.scale, EDGE_FACTOR << self.scale
            src = torch.empty(ne, dtype=torch.int32, device="cuda")
            dst = torch.empty_like(src)
            ctx.gen_rmat(self.scale, ne, SEED, src, dst)
            return n, src, dst
        if self.key == "chunglu":
            cdf, ne = xt.chunglu_cdf(CHUNGLU_N, CHUNGLU_GAMMA, CHUNGLU_MEAN, CHUNGLU_MAX)
            src = torch.empty(ne, dtype=torch.int32, device="cuda")
            dst = torch.empty_like(src)
            ctx.gen_chunglu(cdf, ne, SEED, src, dst)
            return CHUNGLU_N, src, dst
        off, tails = xt.generate_rgg(RGG_N, RGG_RANKS, self.radius)
        src = torch.from_numpy(np.repeat(np.arange(RGG_N, dtype=np.int32), np.diff(off))).cuda()
        dst = torch.from_numpy(tails.astype(np.int32)).cuda()
        return RGG_N, src, dst

    def cpu_sample(self):
        """(canonical CSR, description, config) of the graph the CPU reference
        counts: the workload itself where it finishes in seconds, else a
        smaller graph of the same generator. Built by the oracle alone (the
        reference arm loads nothing of the product)."""
        import oracle
        if self.key == "rmat24":
            sc = min(self.scale, SAMPLE_SCALE)
            n = 1 << sc
            src, dst = oracle.rmat_edges(sc, EDGE_FACTOR << sc, SEED)
            cfg = {"workload": workload_name(sc), "scale": sc, "edge_factor": EDGE_FACTOR}
            return oracle.canon_csr(n, src, dst), f"R-MAT scale {sc} of the same generator", cfg
        if self.key == "chunglu":
            n = 1 << 17
            mx = CHUNGLU_MAX * n / CHUNGLU_N
            cdf, ne = oracle.chunglu_cdf(n, CHUNGLU_GAMMA, CHUNGLU_MEAN, mx)
            src, dst = oracle.chunglu_edges(cdf, ne, SEED)
            what = (f"Chung-Lu n={n:,} of the same generator (exponent {CHUNGLU_GAMMA}, mean {CHUNGLU_MEAN:g}, "
                    f"max expected degree {mx:,.0f})")
            cfg = {"workload": what + ", ids permuted; symmetrised + deduped", "n": n, "gamma": CHUNGLU_GAMMA,
                   "mean_degree": CHUNGLU_MEAN, "max_expected_degree": mx}
            return oracle.canon_csr(n, src, dst), what, cfg
        # the reference's own generator restated by the oracle (literal all-pairs form)
        cfg = {"workload": self.name, **self.extra}
        return oracle.ref_rgg(RGG_N, RGG_RANKS, self.radius), "the workload graph itself", cfg

    def config(self, world: int, info: dict | None, shard: bool = False) -> dict:
        par = (f"edge-sharded x{world} (NCCL all-reduce)" if shard else f"replicas x{world}") if world > 1 \
            else "single GPU"
        c = {"workload": self.name, **self.extra, "seed": SEED, "orient": "degree",
             "parallelism": par,
             "l2": ("inputs larger than L2 (CSR + transpose > 126 MB), no flush" if self.key != "rgg" else
                    "graph (~10 MB) fits in L2: back-to-back counts, no flush (launch-bound size)")}
        if info:
            c.update({"nv": info["nv"], "oriented_edges": info["n_edges"], "max_degree": info["max_degree"],
                      "max_out_degree": info["max_out_degree"]})
        return c


def workload_name(scale: int) -> str:
    return (f"R-MAT scale {scale}, edge factor 16 (a=.57 b=.19 c=.19 d=.05, 10% per-level noise, ids permuted), "
            "symmetrised + deduped + loops dropped, degree-oriented, int32 cols / int64 offsets")


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own CPU path on a sample of the workload
# ---------------------------------------------------------------------------

def write_vite(off, tails) -> str:
    path = os.path.join(tempfile.gettempdir(), f"xtric_sample_{os.getpid()}.bin")
    rec = np.zeros(len(tails), dtype=[("t", "<i8"), ("w", "<f8")])
    rec["t"] = tails
    rec["w"] = 1.0
    with open(path, "wb") as f:
        np.array([len(off) - 1, len(tails)], np.int64).tofile(f)
        np.asarray(off, np.int64).tofile(f)
        rec.tofile(f)
    return path


def time_reference_once(path: str, off, tails, cores: int) -> tuple[float, str, int]:
    """Seconds of one reference count. Prefers the reference's own binary;
    falls back to the oracle's restatement when it is not built."""
    import oracle
    if os.path.exists(oracle.REF_TRIC_OMP):
        r = oracle.run_ref(["-f", path], omp=True, threads=cores, timeout=1800)
        if r["rc"] != 0 or "t_local" not in r:
            raise RuntimeError("reference binary failed:\n" + r["stdout"][-2000:])
        # the count runs inside the constructor on one rank (xxtric.hpp:150-223);
        # main times only count() (main.cpp:158-183): report both phases
        return r["t_local"] + r.get("t_count", 0.0), "reference", r.get("triangles", -1)
    os.environ["OMP_NUM_THREADS"] = str(cores)
    t0 = time.perf_counter()
    t = oracle.count_xxtric(off, tails)
    return time.perf_counter() - t0, "port", t


def cpu_baseline(wl: Workload, cores: int, steps: int = 1, warmup: int = 0) -> dict:
    (off, tails), what, cfg = wl.cpu_sample()
    n_edges = len(tails) // 2
    path = write_vite(off, tails)
    try:
        ts = []
        kind = "reference"
        tri = -1
        i = 0
        # at least `steps` timed runs, more while they add up to under ~10 s
        while i < warmup + steps or (sum(ts) < 10.0 and len(ts) < 200):
            t, kind, tri = time_reference_once(path, off, tails, cores)
            if i >= warmup:
                ts.append(t)
            i += 1
    finally:
        os.unlink(path)
    total = sum(ts)
    return {"value": n_edges * len(ts) / total, "unit": UNIT, "cores": cores, "cpu_model": cpu_model(),
            "kind": kind,
            "sample": f"{what} ({n_edges} oriented edges, {tri} triangles), reference OpenMP CPU count, "
                      f"{len(ts)} run(s), {total / len(ts):.4f} s per run",
            "seconds_per_run": total / len(ts), "n_edges": n_edges, "triangles": tri, "config": cfg,
            "csr": (off, tails)}


def run_reference_arm(args) -> None:
    rank, world, _ = env_ranks()
    if rank != 0:
        return  # rank 0 alone times the CPU reference
    if args.workload in ("batch", "serve"):
        print(json.dumps({"impl": "reference", "unavailable": f"the {args.workload} form has no counterpart in the "
                          "reference (it counts one graph per run); its CPU baseline is the rmat24 line"}))
        return
    wl = Workload(args.workload, args.scale)
    cores = os.cpu_count() or 1
    try:
        cb = cpu_baseline(wl, cores, steps=args.steps, warmup=args.warmup)
    except Exception as e:  # report, never fake a number
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU path failed: {e}"[:300]}))
        return
    # the config names the graph actually timed (a bounded sample of the
    # workload where the workload itself would take minutes per step)
    cfg = dict(cb["config"], seed=SEED, orient="the reference's vertex-id precedence (xxtric.hpp:165)",
               parallelism=f"{cores} OpenMP threads on the host, one rank", sample_of=wl.name,
               oriented_edges=cb["n_edges"], triangles=cb["triangles"])
    # the sample is the same graph; the reference orients it by vertex id
    cfg["workload"] = cfg["workload"].replace("degree-oriented", "oriented by vertex id")
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * cb["seconds_per_run"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "cpu_model", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# the product arm
# ---------------------------------------------------------------------------

def time_counts(g, stream, torch, steps: int, per_vertex=None, support=None) -> float:
    """Mean device seconds of one count (CUDA events on the launching stream):
    the global count, or with per-vertex (per_vertex) or per-edge (support)
    counts into the given device arrays."""
    d = torch.zeros(1, dtype=torch.int64, device="cuda")
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def one():
        if support is not None:
            g.count_edges_async(d, support)
        else:
            g.count_async(d, per_vertex)
    one()  # warm
    a.record(stream)
    for _ in range(steps):
        one()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / 1e3 / steps


def run_xtric(args) -> None:
    import torch

    import xxtric_b200 as xt
    from xxtric_b200 import replicas

    wl = Workload(args.workload, args.scale)
    rank, world, local = replicas.init(backend="nccl")
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    ctx = xt.Context(local)
    ctx.set_stream(stream.cuda_stream)
    n, src, dst = wl.device_edges(ctx, torch)
    ne = len(src)
    torch.cuda.synchronize()
    g = ctx.graph_from_device_edges(n, ne, src, dst, xt.ORIENT_DEGREE)
    info = g.info()
    d_count = torch.zeros(1, dtype=torch.int64, device="cuda")
    # --mode per-vertex / per-edge: the timed step is the count with those
    # outputs (the kernels k_count<1> / k_count<2>), for profiling them
    d_pv = torch.zeros(n, dtype=torch.int64, device="cuda") if args.mode == "per-vertex" else None
    d_sup = torch.zeros(max(1, info["n_edges"]), dtype=torch.int64, device="cuda") if args.mode == "per-edge" else None
    d_shard = None
    if args.shard:
        from xxtric_b200 import shards
        d_shard = torch.zeros(1 + (n if d_pv is not None else info["n_edges"] if d_sup is not None else 0),
                              dtype=torch.int64, device="cuda")

    def count_step():
        if args.shard:  # this rank's shard, then the all-reduce of the parts
            if d_sup is not None:
                shards.count_edges_sharded(g, out=d_shard)
            else:
                shards.count_sharded(g, per_vertex=d_pv is not None, out=d_shard)
            d_count.copy_(d_shard[:1])
        elif d_sup is not None:
            g.count_edges_async(d_count, d_sup)
        else:
            g.count_async(d_count, d_pv)

    counts = []
    for _ in range(args.warmup):
        count_step()
        counts.append(int(d_count.item()))

    replicas.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if sampler:
        sampler.start()
    l0 = ctx.launches
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for k in range(args.steps):
        ev[k][0].record(stream)
        count_step()
        ev[k][1].record(stream)
    end.record(stream)
    torch.cuda.synchronize()
    launches = ctx.launches - l0
    clocks = sampler.stop() if sampler else None
    replicas.barrier()
    t_total = start.elapsed_time(end) / 1e3
    t_kernel = statistics.mean(a.elapsed_time(b) for a, b in ev) / 1e3
    counts.append(int(d_count.item()))
    if len(set(counts)) != 1:
        raise RuntimeError(f"count changed between steps: {counts}")
    if args.shard:  # one graph counted by all ranks together
        t_max = replicas.reduce_max(t_total)
        value = info["n_edges"] * args.steps / t_max
    else:
        value, total_edges, t_max = replicas.aggregate(info["n_edges"] * args.steps, t_total)

    extra = {"mode": args.mode}
    if args.shard:
        extra["sharding"] = {"shards": world, "collective": "NCCL all-reduce of the int64 parts" if world > 1 else None}
    del d_pv, d_sup, d_shard
    if args.workload == "rmat24" and args.mode == "global" and not args.no_forms:
        # the per-vertex and per-edge kernels on the same graph
        pv = torch.zeros(n, dtype=torch.int64, device="cuda")
        extra["per_vertex_ms"] = 1e3 * time_counts(g, stream, torch, 3, pv)
        del pv
        sup = torch.zeros(max(1, info["n_edges"]), dtype=torch.int64, device="cuda")
        extra["per_edge_ms"] = 1e3 * time_counts(g, stream, torch, 3, support=sup)
        del sup
        # the reference's own precedence (vertex ids) on the same graph
        gi = ctx.graph_from_device_edges(n, ne, src, dst, xt.ORIENT_ID)
        if gi.count() != counts[0]:
            raise RuntimeError("the id orientation's count differs from the degree orientation's")
        extra["id_orientation_ms"] = 1e3 * time_counts(gi, stream, torch, 1)
        ii = gi.info()
        extra["id_orientation_max_out_degree"] = ii["max_out_degree"]
        extra["candidates"] = info["stream_work"]
        extra["id_orientation_candidates"] = ii["stream_work"]
        gi.free()
    if args.workload == "chunglu":
        # the per-vertex kernel and the reference's id orientation on the same graph
        pv = torch.zeros(n, dtype=torch.int64, device="cuda")
        extra["per_vertex_ms"] = 1e3 * time_counts(g, stream, torch, 3, pv)
        del pv
        gi = ctx.graph_from_device_edges(n, ne, src, dst, xt.ORIENT_ID)
        extra["id_orientation_ms"] = 1e3 * time_counts(gi, stream, torch, 3)
        ii = gi.info()
        extra["id_orientation_max_out_degree"] = ii["max_out_degree"]
        # candidates streamed: sum over u of C(d+(u), 2), the work the orientation sets
        extra["candidates"] = info["stream_work"]
        extra["id_orientation_candidates"] = ii["stream_work"]
        gi.free()

    # ---- end to end through the C ABI with host buffers ----
    e2e = run_e2e(args, ctx, stream, torch, n, ne, src, dst, g, counts, info) if not args.no_e2e else None
    del src, dst
    g.free()
    roofline = roofline_fields(args, info, t_kernel)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
        "scaling": "strong" if args.shard else "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": wl.config(world, info, args.shard), "triangles": counts[0],
        "triangles_per_s": counts[0] * args.steps * (1 if args.shard else world) / t_max,
        "roofline": roofline, "e2e": e2e, "gpu_launches": launches, "clocks": clocks, **extra,
    }

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = cpu_baseline(wl, os.cpu_count() or 1)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "cpu_model", "kind", "sample")}
            line["cpu_sample_on_gpu"] = sample_on_gpu(ctx, stream, torch, cb)
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)[:200]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "rmat24":
        try:
            line["reference_gpu"] = reference_gpu_leg(ctx, stream, torch)
        except Exception as e:
            line["reference_gpu"] = {"unavailable": str(e)[:200]}
    if not args.no_forms and args.workload == "rmat24":
        # the batching and serving forms, summarised (the full lines: --workload batch|serve)
        line["batch"] = measure_batch(ctx, stream, torch, steps=5, warmup=3, e2e_steps=2)["summary"]
        line["serve"] = measure_serve(ctx, local, torch, SERVE_RATES_DEFAULT, max_queries=400)["summary"]
    del ctx
    replicas.finish()
    if rank == 0:
        print(json.dumps(line))


def run_e2e(args, ctx, stream, torch, n, ne, src, dst, g, counts, info) -> dict:
    """The same metric through the C ABI with host buffers: per step the
    int32 edge list is copied in from pinned memory, built into the oriented
    CSR, planned, counted, and the count read back. Frees the resident graph
    first (its memory goes to the builder)."""
    import xxtric_b200 as xt
    from xxtric_b200 import replicas
    h_src = torch.empty(ne, dtype=torch.int32, pin_memory=True)
    h_dst = torch.empty(ne, dtype=torch.int32, pin_memory=True)
    h_src.copy_(src)
    h_dst.copy_(dst)
    g.free()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    hs, hd = h_src.numpy(), h_dst.numpy()
    e2e_counts = []
    d_part = torch.zeros(1, dtype=torch.int64, device="cuda") if args.shard else None

    def count_of(g2):
        if args.shard:  # this rank's shard + the all-reduce, the sum read back
            from xxtric_b200 import shards
            return shards.count_sharded(g2, out=d_part)[0]
        return g2.count()

    # untimed builds first: the stream-ordered pool grows over the first few
    # builds of a size (two warm-up builds left the next two at 172 and 125 ms
    # of build against 81-83 ms steady)
    for _ in range(4):
        g2 = ctx.graph_from_edges(n, hs, hd, xt.ORIENT_DEGREE)
        e2e_counts.append(count_of(g2))
        g2.free()
    replicas.barrier()
    torch.cuda.synchronize()
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(args.e2e_steps + 1)]
    host = []  # per step, host wall ms of the build call, the count call and the free
    marks[0].record(stream)
    for i in range(args.e2e_steps):
        h0 = time.perf_counter()
        g2 = ctx.graph_from_edges(n, hs, hd, xt.ORIENT_DEGREE)  # H2D + build + orient + plan
        h1 = time.perf_counter()
        e2e_counts.append(count_of(g2))                        # count + D2H of the result
        h2 = time.perf_counter()
        g2.free()
        marks[i + 1].record(stream)
        h3 = time.perf_counter()
        host.append([round(1e3 * (h1 - h0), 2), round(1e3 * (h2 - h1), 2), round(1e3 * (h3 - h2), 2)])
    torch.cuda.synchronize()
    t_e2e = marks[0].elapsed_time(marks[-1]) / 1e3
    e2e_step_ms = [marks[i].elapsed_time(marks[i + 1]) for i in range(args.e2e_steps)]
    if set(e2e_counts) != set(counts):
        raise RuntimeError(f"end-to-end count {e2e_counts} differs from {counts}")
    if args.shard:
        e2e_value = info["n_edges"] * args.e2e_steps / replicas.reduce_max(t_e2e)
    else:
        e2e_value, _, _ = replicas.aggregate(info["n_edges"] * args.e2e_steps, t_e2e)

    return {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * 4 * ne, "d2h_bytes_per_step": 8,
            "ms_per_step": 1e3 * t_e2e / args.e2e_steps, "steps": args.e2e_steps,
            "step_ms": [round(x, 2) for x in e2e_step_ms],
            "median_step_ms": round(statistics.median(e2e_step_ms), 2),
            "host_build_count_free_ms": host}


def roofline_fields(args, info: dict, t_kernel: float) -> dict:
    """The count kernel's roofline. `achieved` is DRAM bytes per launch over
    the kernel's CUDA-event time in this run, the DRAM bytes taken from the
    committed ncu capture of one launch of this workload (`traffic_source`);
    without a capture it falls back to the bytes the schedule's loads request
    (`basis` says which). Beside it: the requested (logical) bytes, the
    compulsory footprint (each array read once), the tail-grouped formula's
    bytes, and the issue-slot utilisation of the small-case capture."""
    peaks = measured_peaks()
    peak = peaks["hbm_gbs"]
    name = {"rmat24": "k_count_rmat_s24.md", "chunglu": "k_count_chunglu.md"}.get(args.workload)
    if getattr(args, "mode", "global") != "global":
        name = None  # the committed DRAM capture is the global count's
    dram = profiled_value(name, "dram_bytes_per_launch_full_size") if name and args.scale == SCALE else None
    logical = info["alg_bytes"] / t_kernel / 1e9
    r = {"bound": "hbm", "peak": peak, "unit": "GB/s", "peak_source": peaks["source"],
         "kernel": {"global": "k_count<0>", "per-vertex": "k_count<1>",
                    "per-edge": "k_count<2>"}[getattr(args, "mode", "global")], "kernel_ms": 1e3 * t_kernel}
    if dram:
        a = dram / t_kernel / 1e9
        r.update({"achieved": a, "frac": a / peak, "traffic": int(dram),
                  "basis": "DRAM bytes per launch (ncu capture of one full-size launch) / kernel time in this run",
                  "traffic_source": f"profiles/{name} (dram__bytes_read.sum + dram__bytes_write.sum)"})
    else:
        r.update({"achieved": logical, "frac": logical / peak, "traffic": None,
                  "basis": "bytes the schedule's loads request (no ncu capture of this workload committed)",
                  "traffic_source": None})
    r.update({"logical_bytes": info["alg_bytes"], "logical_achieved": logical, "logical_frac": logical / peak,
              "footprint_bytes": info["footprint_bytes"],
              "footprint_frac": info["footprint_bytes"] / t_kernel / 1e9 / peak,
              "tail_grouped_alg_bytes": info["tail_alg_bytes"],
              "tail_grouped_frac": info["tail_alg_bytes"] / t_kernel / 1e9 / peak})
    small = {"rmat24": "k_count_rmat_s22.md"}.get(args.workload)
    if small:
        iss = profiled_value(small, "issue_slots_busy_frac")
        if iss is not None:
            r["issue_frac"] = iss
            r["issue_source"] = f"profiles/{small} (ncu --set full, R-MAT scale 22: sm__inst_issued / issue slots)"
    return r


def reference_gpu_leg(ctx, stream, torch) -> dict:
    """The reference's own single-GPU engine (oracle/_ref/tric_gpu:
    TriangleCountingSingle over single_gpu_count, xxtric-gpu.hpp:27-270,
    counting.cu:537-638, built for sm_100a) and this library's count on the
    same graphs, on this GPU: R-MAT scales 16 and 18 of the workload's
    generator and the reference's random geometric graph of config 1. The
    reference's time is its main()'s timing of count() (the kernel, its
    synchronisation and the 8-byte read), best of 3 runs; this library's is
    the count kernel's CUDA-event time. Larger R-MAT scales are left out: the
    reference's warp-per-vertex loop over a hub's neighbour pairs runs for
    minutes there."""
    import oracle
    if not os.path.exists(oracle.REF_TRIC_GPU):
        return {"unavailable": "oracle/_ref/tric_gpu is not built (it is built where the reference tree exists)"}
    graphs = []
    for sc in (16, 18):
        src, dst = oracle.rmat_edges(sc, EDGE_FACTOR << sc, SEED)
        graphs.append((f"R-MAT scale {sc} of the workload's generator", oracle.canon_csr(1 << sc, src, dst)))
    rgg = Workload("rgg")
    graphs.append(("the reference's random geometric graph, n=65,536, r=sqrt(16/(pi n)), two strip ranks",
                   oracle.ref_rgg(RGG_N, RGG_RANKS, rgg.radius)))
    out = []
    for name, (off, tails) in graphs:
        path = write_vite(off, tails)
        try:
            runs = [oracle.run_ref(["-f", path], gpu=True, timeout=300) for _ in range(3)]
        finally:
            os.unlink(path)
        bad = [r for r in runs if r["rc"] != 0 or "t_count" not in r]
        if bad:
            out.append({"graph": name, "unavailable": "reference GPU run failed: " + bad[0]["stdout"][-200:]})
            continue
        t_ref = min(r["t_count"] for r in runs)
        g = ctx.graph_from_csr(off, tails, canonical=True)
        d = torch.zeros(1, dtype=torch.int64, device="cuda")
        g.count_async(d)
        torch.cuda.synchronize()
        tri = int(d.item())
        t = time_counts(g, stream, torch, 20)
        ne = g.info()["n_edges"]
        g.free()
        out.append({"graph": name, "oriented_edges": ne, "triangles": tri,
                    "reference_triangles": runs[0].get("triangles"),
                    "reference_ms": 1e3 * t_ref, "xtric_ms": 1e3 * t, "speedup": t_ref / t})
    return {"binary": "oracle/_ref/tric_gpu (reference main.cpp + xxtric-gpu.hpp + counting.cu, "
                      "-DUSE_CUDA -DUSE_SINGLE_DEVICE, sm_100a)", "graphs": out}


def sample_on_gpu(ctx, stream, torch, cb: dict) -> dict:
    """The CPU baseline's sample graph counted on the GPU: the same graph on
    both sides (built from the same canonical CSR), device time of the count."""
    import xxtric_b200 as xt
    off, tails = cb["csr"]
    g = ctx.graph_from_csr(off, tails, canonical=True)
    d = torch.zeros(1, dtype=torch.int64, device="cuda")
    g.count_async(d)
    torch.cuda.synchronize()
    tri = int(d.item())
    t = time_counts(g, stream, torch, 20)
    ne = g.info()["n_edges"]
    g.free()
    if tri != cb["triangles"]:
        raise RuntimeError(f"sample graph: GPU {tri} triangles, reference {cb['triangles']}")
    return {"graph": cb["sample"].split(" (")[0], "oriented_edges": ne, "triangles": tri,
            "gpu_count_ms": 1e3 * t, "gpu_value": ne / t, "cpu_value": cb["value"],
            "gpu_over_cpu": (ne / t) / cb["value"], "unit": UNIT}


BATCH_GRAPHS = 4096
BATCH_WORKLOAD = ("4,096 graphs: half unit-square random geometric, half Erdos-Renyi G(n,m); n log-uniform in "
                  "[256, 65536), mean degree log-uniform in [8, 64); int32 local ids, one concatenated CSR with "
                  "per-graph offset tables, degree-oriented")


def measure_batch(ctx, stream, torch, steps: int, warmup: int, e2e_steps: int) -> dict:
    """Batching form on one GPU: the 4,096 graphs built as one union, counted
    in one persistent launch (captured CUDA graph, autotuned schedule), against
    the plain per-graph path on the same GPU (each graph built and counted
    alone); every per-graph count checked against the plain path's. Returns
    the figures ("summary" holds the few that the default bench line carries)."""
    import xxtric_b200 as xt
    spec = xt.batch_spec(BATCH_GRAPHS, SEED)
    eoff, d_src, d_dst = ctx.gen_batch(spec)
    voff = np.concatenate([[0], np.cumsum(spec["n"])]).astype(np.int64)
    ng = BATCH_GRAPHS
    t0 = time.perf_counter()
    bg = ctx.graph_from_batch(voff, eoff, d_src, d_dst, device=True)
    build_s = time.perf_counter() - t0
    tune = bg.autotune(reps=2)
    bg.capture()
    info = bg.info()
    d_total = torch.zeros(1, dtype=torch.int64, device="cuda")
    d_per = torch.zeros(ng, dtype=torch.int64, device="cuda")
    for _ in range(warmup):
        bg.count_groups_async(d_total, d_per)
    torch.cuda.synchronize()
    l0 = ctx.launches
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        bg.count_groups_async(d_total, d_per)
    b.record(stream)
    torch.cuda.synchronize()
    launches = ctx.launches - l0
    t_batch = a.elapsed_time(b) / 1e3
    per = d_per.cpu().numpy()
    total = int(d_total.item())
    bg.free()
    # end to end, batched: host edge lists -> device -> one build -> one count -> per-graph counts
    ts = torch.as_tensor(d_src, device="cuda")
    td = torch.as_tensor(d_dst, device="cuda")
    h_src = torch.empty(len(ts), dtype=torch.int32, pin_memory=True)
    h_dst = torch.empty(len(td), dtype=torch.int32, pin_memory=True)
    h_src.copy_(ts)
    h_dst.copy_(td)
    hs, hd = h_src.numpy(), h_dst.numpy()
    g2 = ctx.graph_from_batch(voff, eoff, hs, hd)
    g2.count_groups()
    g2.free()
    torch.cuda.synchronize()
    ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ea.record(stream)
    for _ in range(e2e_steps):
        g2 = ctx.graph_from_batch(voff, eoff, hs, hd)
        _, per_e2e = g2.count_groups()
        g2.free()
    eb.record(stream)
    torch.cuda.synchronize()
    t_e2e = ea.elapsed_time(eb) / 1e3 / e2e_steps
    if not (per_e2e == per).all():
        raise RuntimeError("end-to-end batch counts differ from the device-resident ones")
    # plain per-graph path: each graph built and counted on its own
    plain_count_s = 0.0
    plain_ok = True
    torch.cuda.synchronize()
    p0 = time.perf_counter()
    for g in range(ng):
        e0, e1 = int(eoff[g]), int(eoff[g + 1])
        pg = ctx.graph_from_device_edges(int(spec["n"][g]), e1 - e0, ts[e0:e1], td[e0:e1])
        ca, cb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ca.record(stream)
        pg.count_async(d_total)
        cb.record(stream)
        cb.synchronize()
        plain_count_s += ca.elapsed_time(cb) / 1e3
        plain_ok &= int(d_total.item()) == int(per[g])
        pg.free()
    torch.cuda.synchronize()
    plain_e2e_s = time.perf_counter() - p0
    d_src.free()
    d_dst.free()
    del ts, td, h_src, h_dst
    torch.cuda.empty_cache()
    graphs_per_s = ng * steps / t_batch
    out = {
        "graphs": ng, "vertices": int(voff[-1]), "edges_generated": int(eoff[-1]), "oriented_edges": info["n_edges"],
        "triangles": total, "t_batch": t_batch, "steps": steps, "launches": launches,
        "graphs_per_s": graphs_per_s, "oriented_edges_per_s": info["n_edges"] * steps / t_batch,
        "e2e_graphs_per_s": ng / t_e2e, "e2e_ms": 1e3 * t_e2e,
        "h2d_bytes_per_step": 8 * int(eoff[-1]) + 16 * (ng + 1), "d2h_bytes_per_step": 8 * (ng + 1),
        "plain_count_graphs_per_s": ng / plain_count_s, "plain_e2e_graphs_per_s": ng / plain_e2e_s,
        "plain_count_s": plain_count_s, "plain_e2e_s": plain_e2e_s,
        "per_graph_counts_equal_plain": bool(plain_ok), "build_s": build_s, "autotune": tune.get("best", tune),
    }
    out["summary"] = {
        "workload": BATCH_WORKLOAD, "graphs_per_s": round(graphs_per_s, 1),
        "plain_graphs_per_s": round(ng / plain_count_s, 1), "speedup_vs_plain": round(graphs_per_s * plain_count_s / ng, 3),
        "e2e_graphs_per_s": round(ng / t_e2e, 1), "plain_e2e_graphs_per_s": round(ng / plain_e2e_s, 1),
        "e2e_speedup_vs_plain": round(plain_e2e_s / t_e2e, 3),
        "per_graph_counts_equal_plain": bool(plain_ok), "triangles": total, "ms_per_batch_count": 1e3 * t_batch / steps,
        "autotune_best": tune.get("best", tune),
        "note": "count: device time of one captured launch over all graphs vs the sum of per-graph count times; "
                "e2e: host edge lists in, per-graph counts out, vs building and counting each graph alone",
    }
    return out


def run_batch(args) -> None:
    """The batching form's own bench line (graphs/s)."""
    import torch

    import xxtric_b200 as xt
    from xxtric_b200 import replicas

    rank, world, local = replicas.init(backend="nccl")
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    ctx = xt.Context(local)
    ctx.set_stream(stream.cuda_stream)
    replicas.barrier()
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if sampler:
        sampler.start()
    m = measure_batch(ctx, stream, torch, args.steps, args.warmup, args.e2e_steps)
    clocks = sampler.stop() if sampler else None
    value, _, t_max = replicas.aggregate(m["graphs"] * args.steps, m["t_batch"])
    replicas.finish()
    if rank != 0:
        return
    ng = m["graphs"]
    line = {
        "metric": "graphs/s (batched count, 4096 graphs)", "value": value, "unit": "graphs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "graphs": ng, "vertices": m["vertices"],
                   "edges_generated": m["edges_generated"], "oriented_edges": m["oriented_edges"], "seed": SEED,
                   "l2": "inputs larger than L2, no flush", "launch": "one persistent kernel, captured CUDA graph"},
        "triangles": m["triangles"],
        "oriented_edges_per_s": m["oriented_edges"] * args.steps * world / t_max,
        "e2e": {"value": m["e2e_graphs_per_s"], "unit": "graphs/s", "ms_per_step": m["e2e_ms"],
                "h2d_bytes_per_step": m["h2d_bytes_per_step"], "d2h_bytes_per_step": m["d2h_bytes_per_step"]},
        "plain": {"count_graphs_per_s": m["plain_count_graphs_per_s"], "e2e_graphs_per_s": m["plain_e2e_graphs_per_s"],
                  "count_s": m["plain_count_s"], "e2e_s": m["plain_e2e_s"],
                  "note": "each graph built and counted alone (device edge lists), same GPU"},
        "speedup_vs_plain": {"count": m["graphs_per_s"] / m["plain_count_graphs_per_s"],
                             "e2e": m["e2e_graphs_per_s"] / m["plain_e2e_graphs_per_s"]},
        "per_graph_counts_equal_plain": m["per_graph_counts_equal_plain"], "build_s": m["build_s"],
        "autotune": m["autotune"], "gpu_launches": m["launches"], "clocks": clocks,
    }
    print(json.dumps(line))


SERVE_WORKLOAD = ("count queries on R-MAT graphs (a=.57 b=.19 c=.19 d=.05, edge factor 16, 10% noise, ids "
                  "permuted), scale uniform in {10..20} (log-uniform vertex count), Poisson arrivals; host edge "
                  "lists (int32) copied in per query; degree-oriented")
SERVE_RATES = (10, 30, 100, 300, 1000, 3000, 10000)
SERVE_POOL = 48
# the default bench line: one rate below saturation, one above
SERVE_RATES_DEFAULT = (100, 3000)


def _pct(xs, q):
    return float(np.percentile(np.asarray(xs) * 1e3, q)) if len(xs) else None


def measure_serve(ctx, local: int, torch, rates, max_queries: int = 600) -> dict:
    """Serving form: Poisson arrival streams at the given rates, served with
    admission by memory budget and continuous batching (xt_serve_*), against
    the plain per-query path (build + count per query, one at a time) under
    the same arrivals. Every served and plain count is checked against the
    query's solo count. Returns the sweep ("summary": the default line's)."""
    import xxtric_b200 as xt
    rng = np.random.default_rng(SEED + 5)
    pool = []  # (nv, pinned src, pinned dst)
    for i in range(SERVE_POOL):
        scale = int(rng.integers(10, 21))
        ne = EDGE_FACTOR << scale
        ds = torch.empty(ne, dtype=torch.int32, device="cuda")
        dd = torch.empty_like(ds)
        ctx.gen_rmat(scale, ne, 1000 + i, ds, dd)
        hs = torch.empty(ne, dtype=torch.int32, pin_memory=True)
        hd = torch.empty(ne, dtype=torch.int32, pin_memory=True)
        hs.copy_(ds)
        hd.copy_(dd)
        pool.append((1 << scale, hs.numpy(), hd.numpy(), scale))
    del ds, dd
    torch.cuda.synchronize()

    def plain_one(i):
        nv, hs, hd, _ = pool[i]
        g = ctx.graph_from_edges(nv, hs, hd)
        t = g.count()
        g.free()
        return t

    solo = [plain_one(i) for i in range(SERVE_POOL)]  # also warms the plain path
    srv = xt.Server(local, budget_bytes=150 << 30, slots=3)
    for i in range(SERVE_POOL):  # warm the server's slots and pool allocator
        srv.wait(srv.submit(*pool[i][:3]))
    st0 = srv.stats()
    sweep = []
    exact = True
    l_plain0 = ctx.launches
    for lam in rates:
        n = int(min(max_queries, max(30, 3 * lam)))
        arr = np.cumsum(rng.exponential(1.0 / lam, n))
        arr -= arr[0]
        which = rng.integers(0, SERVE_POOL, n)
        # served: submit on schedule, results timed by the server (submit -> result)
        t0 = time.perf_counter()
        sub = []
        for k in range(n):
            d = t0 + arr[k] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            ts = time.perf_counter()
            sub.append((srv.submit(*pool[which[k]][:3]), ts))
        lat, done = [], []
        for k, (tk, ts) in enumerate(sub):
            c, l = srv.wait(tk)
            exact &= c == solo[which[k]]
            lat.append(l)
            done.append(ts + l)
        served_s = max(done) - t0
        bl = srv.batches()[-n:]
        bl = [b for b in bl if b["take"] >= bl[-1]["take"] - served_s - 1.0]
        # plain: one query at a time in arrival order, each waiting for the previous
        t0 = time.perf_counter()
        plat = []
        for k in range(n):
            d = t0 + arr[k] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            exact &= plain_one(which[k]) == solo[which[k]]
            plat.append(time.perf_counter() - (t0 + arr[k]))
        plain_s = time.perf_counter() - t0
        edges = int(sum(len(pool[w][1]) for w in which))
        sweep.append({"rate_per_s": lam, "queries": n, "edge_rows": edges,
                      "served": {"p50_ms": _pct(lat, 50), "p99_ms": _pct(lat, 99), "graphs_per_s": n / served_s,
                                 "batches": len(bl), "graphs_per_batch": float(np.mean([b["graphs"] for b in bl])),
                                 "build_ms_mean": 1e3 * float(np.mean([b["built"] - b["take"] for b in bl])),
                                 "count_ms_mean": 1e3 * float(np.mean([b["done"] - b["built"] for b in bl])),
                                 "batch_ms_max": 1e3 * float(max(b["done"] - b["take"] for b in bl))},
                      "plain": {"p50_ms": _pct(plat, 50), "p99_ms": _pct(plat, 99), "graphs_per_s": n / plain_s}})
    st = srv.stats()
    srv.close()
    out = {"pool": pool, "sweep": sweep, "exact": bool(exact), "stats": st, "stats0": st0,
           "plain_launches": ctx.launches - l_plain0}
    out["summary"] = {
        "workload": SERVE_WORKLOAD, "budget_bytes": st["budget_bytes"], "slots": 3,
        "rates": [{"rate_per_s": r["rate_per_s"], "queries": r["queries"],
                   "served_p50_ms": round(r["served"]["p50_ms"], 2), "served_p99_ms": round(r["served"]["p99_ms"], 2),
                   "served_graphs_per_s": round(r["served"]["graphs_per_s"], 1),
                   "plain_p50_ms": round(r["plain"]["p50_ms"], 2), "plain_p99_ms": round(r["plain"]["p99_ms"], 2),
                   "plain_graphs_per_s": round(r["plain"]["graphs_per_s"], 1),
                   "graphs_per_batch": round(r["served"]["graphs_per_batch"], 2)} for r in sweep],
        "counts_equal_solo": bool(exact),
        "note": "served: xt_serve_* with admission by device-memory budget and continuous batching; plain: "
                "build + count per query, one at a time, same arrivals; latency = submit to result",
    }
    return out


def run_serve(args) -> None:
    """The serving form's own bench line: the full rate sweep."""
    import torch

    import xxtric_b200 as xt
    from xxtric_b200 import replicas

    rank, world, local = replicas.init(backend="nccl")
    torch.cuda.set_device(local)
    ctx = xt.Context(local)
    m = measure_serve(ctx, local, torch, SERVE_RATES)
    sweep, st, st0, pool = m["sweep"], m["stats"], m["stats0"], m["pool"]
    top = sweep[-1]
    line = {
        "metric": "graphs/s (served count queries, Poisson arrivals)", "value": top["served"]["graphs_per_s"],
        "unit": "graphs/s", "n_gpus": world, "steps": len(SERVE_RATES), "warmup": 1,
        "ms_per_step": 1e3 / top["served"]["graphs_per_s"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": SERVE_WORKLOAD, "pool_graphs": SERVE_POOL,
                   "pool_scales": [p[3] for p in pool], "rates_per_s": list(SERVE_RATES),
                   "budget_bytes": st["budget_bytes"], "slots": 3, "seed": SEED,
                   "l2": "inputs larger than L2 for the large queries; each query copied in from host memory"},
        "sweep": sweep,
        "e2e": {"value": top["served"]["graphs_per_s"], "unit": "graphs/s",
                "h2d_bytes_per_step": 8 * top["edge_rows"], "d2h_bytes_per_step": 8 * top["queries"],
                "note": "a step is one rate's stream; the served path is end to end by construction"},
        "speedup_vs_plain_at_top_rate": top["served"]["graphs_per_s"] / top["plain"]["graphs_per_s"],
        "counts_equal_solo": m["exact"],
        "server": {k: st[k] - st0.get(k, 0) if k in ("submitted", "completed", "batches", "launches") else st[k]
                   for k in ("submitted", "completed", "failed", "rejected", "batches", "max_batch", "budget_peak",
                             "device_peak", "launches")},
        "gpu_launches": st["launches"] - st0["launches"],
        "plain_launches": m["plain_launches"],
    }
    ctx.close()
    replicas.finish()
    if rank == 0:
        print(json.dumps(line))
    if not m["exact"]:
        raise SystemExit("served counts differ from the solo counts")


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--impl", choices=["xtric", "reference"], default="xtric")
    ap.add_argument("--workload", choices=["rmat24", "chunglu", "rgg", "batch", "serve"], default="rmat24",
                    help="rmat24: the headline single-graph count (R-MAT scale 24); chunglu: the heavy-skew "
                         "Chung-Lu graph; rgg: the reference's small random geometric graph; batch: the batching "
                         "form; serve: the serving form (Poisson arrival sweep)")
    ap.add_argument("--scale", type=int, default=SCALE,
                    help="R-MAT scale of the single-graph workload (24 is the headline; smaller scales are the "
                         "small cases that profiler captures run on)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="leave the batching and serving summaries out of the default line")
    ap.add_argument("--mode", choices=["global", "per-vertex", "per-edge"], default="global",
                    help="the count the timed step runs: the global count (the headline), or with per-vertex or "
                         "per-edge counts into device memory")
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: count one graph on all GPUs together (each rank a shard of the schedule, then an "
                         "NCCL all-reduce) instead of independent replicas")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end leg (profiler captures of the count kernel)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)  # timing rule: at least 3 untimed warm-up steps
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_xtric(args)


if __name__ == "__main__":
    main()
