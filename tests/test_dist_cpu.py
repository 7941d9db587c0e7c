"""The multi-replica path of bench.py on the CPU: two `gloo` ranks.

A single solve does not shard ("replicas only"): N ranks run N independent
solves and the bench reports the units of all ranks over the slowest rank's
time, with no data-path collective.  These tests run that reduction and the
batched workload's seed partition on two CPU processes.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        # rank r: (r + 1) * 100 ms for (r + 1) * 1e9 units
        value, max_ms = bench.replica_value(100.0 * (rank + 1), 1e9 * (rank + 1), world)
        seeds = bench.batch_seeds(rank, 4)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{value!r} {max_ms!r} {' '.join(map(str, seeds))}\n")
    finally:
        dist.destroy_process_group()


def test_replica_value_two_gloo_ranks(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    seen = set()
    for rank in range(world):
        value, max_ms, *seeds = open(tmp_path / f"rank{rank}.txt").read().split()
        # all ranks agree: (1e9 + 2e9) units over the slowest rank's 200 ms
        assert float(max_ms) == 200.0
        assert abs(float(value) - 3e9 / 0.2 / 1e9) < 1e-9
        s = set(map(int, seeds))
        assert not (s & seen)
        seen |= s
    assert seen == set(range(8))


def test_replica_value_single_rank():
    pytest.importorskip("torch")
    sys.path.insert(0, ROOT)
    import bench
    value, max_ms = bench.replica_value(500.0, 2e12, 1)
    assert max_ms == 500.0 and abs(value - 4000.0) < 1e-9
