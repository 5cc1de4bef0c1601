"""Batch sharding over ranks, on CPU with the gloo backend (world sizes 2 and 3; no GPU).

The uneven batch (256 sizes uniform in [124, 1788], seed 3) is split by xtb_batch_partition.  Every rank computes the
partition from the sizes alone; the test gathers each rank's share to rank 0 over gloo and checks that every problem
is assigned exactly once, that all ranks computed the same partition, and that the cost model's load is balanced
(largest share within 2 % of the mean, the longest-first bound for this draw).  Invalid arguments return the documented
codes.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import inputs

import shard
import xtbeig


def _cost(n):
    return 5.0 * n + 1.3e-6 * float(n) ** 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, sizes, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mine = shard.my_problems(sizes, rank, world)
        part = shard.partition(sizes, world)
        got = shard.gather_to_rank0((rank, mine, part.tolist()), rank, world)
        if rank == 0:
            np.save(os.path.join(out_dir, "gathered.npy"), np.array(got, dtype=object), allow_pickle=True)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_batch_partition_over_gloo_ranks(tmp_path, world):
    sizes = inputs.batch_sizes(256, seed=3)
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, sizes, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(os.path.join(tmp_path, "gathered.npy"), allow_pickle=True)
    assert len(got) == world
    parts = [g[2] for g in got]
    assert all(p == parts[0] for p in parts), "every rank must compute the same partition"
    seen = sorted(i for g in got for i in g[1])
    assert seen == list(range(len(sizes))), "every problem exactly once"
    loads = [sum(_cost(sizes[i]) for i in g[1]) for g in got]
    assert max(loads) <= 1.02 * (sum(loads) / world)


def test_batch_partition_arguments():
    lib = xtbeig.lib()
    ns = np.array([10, 5, 300], np.int32)
    out = np.zeros(3, np.int32)
    assert lib.xtb_batch_partition(3, xtbeig._p(ns), 0, xtbeig._p(out)) == -3
    assert lib.xtb_batch_partition(-1, xtbeig._p(ns), 2, xtbeig._p(out)) == -1
    assert lib.xtb_batch_partition(3, None, 2, xtbeig._p(out)) == -2
    bad = np.array([10, -5, 300], np.int32)
    assert lib.xtb_batch_partition(3, xtbeig._p(bad), 2, xtbeig._p(out)) == -2
    assert lib.xtb_batch_partition(0, None, 2, None) == 0
    # one part: everything in part 0; more parts than problems: each problem alone, largest first
    assert list(shard.partition([10, 5, 300], 1)) == [0, 0, 0]
    p = shard.partition([10, 5, 300], 5)
    assert len(set(p.tolist())) == 3 and p[2] == 0
