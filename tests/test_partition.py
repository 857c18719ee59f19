"""Host logic of the multi-GPU batched workload (CPU): the size-balanced
partition of independent boxes over ranks, and the whole-job reduction
(particles summed, time maxed) run by two gloo ranks."""

import os
import socket

import numpy as np
import pytest


def test_partition_covers_every_box_once_and_balances(pkg):
    from importlib import import_module

    part = import_module("lsmps3d_b200.partition")
    sizes = [c for c in (pkg.cases.uniform01(7, 64) * 192_000 + 8_000).astype(int)]
    for world in (1, 2, 3, 4, 8):
        parts = part.partition_boxes(sizes, world)
        assert len(parts) == world
        flat = sorted(b for p in parts for b in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[b] for b in p) for p in parts]
        bound = max(sum(sizes) / world, max(sizes))
        assert max(loads) <= 4.0 / 3.0 * bound
    assert part.partition_boxes([], 2) == [[], []]
    with pytest.raises(ValueError):
        part.partition_boxes([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, sizes, out_dir):
    import sys

    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import __graft_entry__ as e

    e.load_package()
    from importlib import import_module

    part = import_module("lsmps3d_b200.partition")
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = part.partition_boxes(sizes, world)[rank]
    particles = sum(sizes[b] for b in mine)
    ms = 10.0 + rank  # a stand-in for the rank's measured time
    total, slowest = part.reduce_rank_results(world, particles, ms)
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(f"{','.join(map(str, mine))};{particles};{total};{slowest}\n")
    dist.destroy_process_group()


def test_two_gloo_ranks_split_boxes_and_reduce(pkg, tmp_path):
    import torch.multiprocessing as mp

    sizes = [int(c.n_fluid) for c in pkg.cases.batched_boxes(count=12, n_min=2_000, n_max=20_000)]
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), sizes, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    rows = [open(tmp_path / f"rank{r}.txt").read().strip().split(";") for r in range(world)]
    boxes = sorted(int(b) for r in rows for b in r[0].split(",") if b)
    assert boxes == list(range(len(sizes)))
    assert all(int(r[2]) == sum(sizes) for r in rows)
    assert all(float(r[3]) == 10.0 + world - 1 for r in rows)
    assert abs(int(rows[0][1]) - int(rows[1][1])) <= max(sizes)
