"""Multi-GPU batches: the uneven batch split over ranks (one process per GPU) with no exchange on the data path.

Independent generalized problems shard naturally (the reference runs its throughput sweeps as independent processes,
Sources/EigenBench/main.swift:464-497).  Every rank computes the same partition from the sizes alone
(xtb_batch_partition: longest first on the library's cost model of n), solves its own problems with the batch call on
its GPU, and keeps its results on the host; nothing crosses between GPUs.  Collecting the results on one rank, when a
caller wants that, is a host-side gather after the solves (``gather_to_rank0``), outside the hot path.
"""
from __future__ import annotations

import numpy as np

import xtbeig


def partition(sizes, parts: int) -> np.ndarray:
    """part_of[i] in 0..parts-1 for every problem size in `sizes` (the C ABI's xtb_batch_partition)."""
    ns = np.ascontiguousarray(np.asarray(sizes, dtype=np.int32))
    out = np.zeros(max(len(ns), 1), np.int32)
    rc = xtbeig.lib().xtb_batch_partition(int(len(ns)), xtbeig._p(ns), int(parts), xtbeig._p(out))
    if rc != 0:
        raise ValueError(f"xtb_batch_partition returned {rc}")
    return out[: len(ns)]


def my_problems(sizes, rank: int, world: int) -> list:
    """Indices of the problems this rank solves, in batch order."""
    part = partition(sizes, world)
    return [i for i in range(len(sizes)) if part[i] == rank]


def solve_batch_sharded(hs, ss, rank: int, world: int):
    """Solve this rank's share of a batch of host problems (lists H_i, S_i) on the current GPU.  Returns
    (indices, w, C, U, info) for the rank's problems only."""
    sizes = [np.asarray(h).shape[0] for h in hs]
    idx = my_problems(sizes, rank, world)
    if not idx:
        return idx, [], [], [], np.zeros(0, np.int32)
    w, c, u, info, ret = xtbeig.dsygvd_batched([hs[i] for i in idx], [ss[i] for i in idx])
    if ret < -1:
        raise RuntimeError(f"xtb_dsygvd_batched returned {ret}: {xtbeig.last_error()}")
    return idx, w, c, u, info


def gather_to_rank0(local, rank: int, world: int):
    """Host-side gather of per-rank Python objects to rank 0 through torch.distributed (any backend); returns the
    list of every rank's object on rank 0 and None elsewhere."""
    import torch.distributed as dist

    if world == 1:
        return [local]
    out = [None] * world if rank == 0 else None
    dist.gather_object(local, out, dst=0)
    return out
