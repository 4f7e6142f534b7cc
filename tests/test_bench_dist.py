"""The multi-process plumbing of bench.py on CPU: two gloo ranks take the max of their
timings and aggregate the whole-job rate exactly as the GPU ranks do over NCCL."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    r, local, w = bench.dist_env()
    dist = bench.dist_init(w, "gloo")
    bench.barrier(dist, "cpu")
    mx = bench.reduce_max(1.5 + r, dist, "cpu")
    rate = bench.aggregate_rate(4096 * 4096, 100, w, mx)
    out[rank] = (r, local, w, mx, rate)
    dist.destroy_process_group()


def test_two_rank_max_and_aggregate():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(worker, args=(world, free_port(), out), nprocs=world, join=True, start_method="spawn")
    assert sorted(out.keys()) == [0, 1]
    for rank in range(world):
        r, local, w, mx, rate = out[rank]
        assert (r, local, w) == (rank, rank, world)
        assert mx == 2.5  # the slower rank's time
        assert rate == pytest.approx(world * 4096 * 4096 * 100 / 2.5 / 1e9)


def test_single_process_defaults():
    import bench
    os.environ.pop("WORLD_SIZE", None)
    assert bench.dist_init(1, "gloo") is None
    assert bench.reduce_max(3.25, None, "cpu") == 3.25
