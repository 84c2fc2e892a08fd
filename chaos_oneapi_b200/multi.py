"""Sharding one sweep over the ranks of a process group (one process per GPU).

Every parameter point is independent, so a grid splits into contiguous
blocks, one per rank, with no exchange during integration; the spectra are
gathered once at the end.  Unlike the reference, which gives every GPU
`nodes / num_GPUs` points and drops the remainder (tasklyapunov.cpp:19), the
remainder is spread over the first ranks.
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def shard_bounds(P: int, world: int, rank: int) -> tuple[int, int]:
    """[start, end) of rank's contiguous block; sizes differ by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    base, extra = divmod(P, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def gpu_compute(sweep):
    """compute(params, inits) -> (spectrum, status) on this rank's GPU."""
    def compute(params, inits):
        return sweep.run_host(np.ascontiguousarray(params), np.ascontiguousarray(inits))
    return compute


def run_sharded(params: np.ndarray, inits: np.ndarray, k: int,
                compute: Callable[[np.ndarray, np.ndarray], tuple], group=None):
    """Runs this rank's block through `compute` and all-gathers the spectra
    (P x k, float64) and statuses (P, int32) in point order on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    P = params.shape[0]
    s, e = shard_bounds(P, world, rank)
    spec = np.full((e - s, k), np.nan)
    status = np.zeros(e - s, dtype=np.int32)
    if e > s:
        spec, status = compute(params[s:e], inits[s:e])
    # all_gather needs equal shapes: pad to the largest block
    n_max = shard_bounds(P, world, 0)[1]
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    buf = torch.full((n_max, k + 1), float("nan"), dtype=torch.float64, device=dev)
    if e > s:
        buf[:e - s, :k] = torch.from_numpy(np.asarray(spec, dtype=np.float64))
        buf[:e - s, k] = torch.from_numpy(np.asarray(status, dtype=np.float64))
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out_spec = np.empty((P, k))
    out_status = np.empty(P, dtype=np.int32)
    for r, part in enumerate(parts):
        rs, re_ = shard_bounds(P, world, r)
        a = part[:re_ - rs].cpu().numpy()
        out_spec[rs:re_] = a[:, :k]
        out_status[rs:re_] = a[:, k].astype(np.int32)
    return out_spec, out_status
