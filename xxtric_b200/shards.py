"""Edge-sharded count of one graph over several GPUs (one process per GPU).

The reference's multi-GPU engine (TriangleCounting::count,
xxtric-gpu-vmm-mpi.hpp:89-129) has every GPU count its part of the graph and
then sums the parts with MPI_Reduce on rank 0. Here every rank holds the
whole graph in its own GPU's memory (built from the same input; an R-MAT
scale-24 graph takes about 6 GB of the 180 GB) and counts one shard of the
count's schedule: the tasks of every tier whose index is the rank modulo the
world size (xt_count_shard_async / xt_count_edges_shard_async). Every
triangle belongs to exactly one task, so the parts sum to the whole count;
one all-reduce over NCCL (an in-place sum of int64 words on the device)
gives every rank the global count and, when asked, the per-vertex counts or
per-edge supports. Ranks run no kernel that waits on another rank: the only
exchange is the collective after the count.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def world(group=None) -> tuple[int, int]:
    """(rank, world size) of the group, (0, 1) without a process group."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def reduce_parts(parts: torch.Tensor, group=None) -> torch.Tensor:
    """Sums every rank's int64 parts in place (all ranks get the sum) and
    returns the tensor. int64 throughout: counts are exact past 2^53."""
    if parts.dtype != torch.int64:
        raise TypeError("shard parts are int64 counts")
    if world(group)[1] > 1:
        dist.all_reduce(parts, op=dist.ReduceOp.SUM, group=group)
    return parts


def count_sharded(graph, per_vertex: bool = False, group=None, out: torch.Tensor | None = None):
    """Global count (and per-vertex counts in the graph's input numbering when
    per_vertex) of `graph`, a DeviceGraph every rank built from the same
    input, with this rank's GPU counting its shard of the schedule.

    The library's context must run on torch's current stream (Context.set_stream)
    so the collective is ordered after the shard's count. Returns (count,
    per-vertex tensor on the device or None); `out`, if given, is an int64
    device tensor of 1 (+ nv) words reused across calls."""
    rank, nranks = world(group)
    nv = graph.nv
    n = 1 + (nv if per_vertex else 0)
    d = out if out is not None else torch.empty(n, dtype=torch.int64, device="cuda")
    if d.numel() < n or d.dtype != torch.int64:
        raise ValueError(f"out must hold {n} int64 words")
    graph.count_shard_async(rank, nranks, d[:1], d[1:n] if per_vertex else None)
    reduce_parts(d[:n], group)
    return int(d[0].item()), (d[1:n] if per_vertex else None)


def count_edges_sharded(graph, group=None, out: torch.Tensor | None = None):
    """Global count and per-edge supports (order of DeviceGraph.csr()) of
    `graph`, sharded like count_sharded. Returns (count, supports on the device)."""
    rank, nranks = world(group)
    ne = int(graph.info()["n_edges"])
    n = 1 + ne
    d = out if out is not None else torch.empty(n, dtype=torch.int64, device="cuda")
    if d.numel() < n or d.dtype != torch.int64:
        raise ValueError(f"out must hold {n} int64 words")
    graph.count_edges_shard_async(rank, nranks, d[:1], d[1:n])
    reduce_parts(d[:n], group)
    return int(d[0].item()), d[1:n]
