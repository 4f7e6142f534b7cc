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


def test_shard_members_partitions_by_cell_count():
    import bench
    import fg2_b200
    sizes = bench.batch_sizes()
    biggest = max(a * b for a, b in sizes)
    for world in (1, 2, 3, 4, 8):
        shards = fg2_b200.shard_members(sizes, world)
        assert len(shards) == world
        assert sorted(k for s in shards for k in s) == list(range(len(sizes)))
        loads = [sum(sizes[k][0] * sizes[k][1] for k in s) for s in shards]
        assert max(loads) - min(loads) <= biggest
        assert shards == fg2_b200.shard_members(sizes, world)  # deterministic
    assert fg2_b200.shard_members([(64, 64)], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        fg2_b200.shard_members(sizes, 0)


def shard_worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    import fg2_b200
    r, _, w = bench.dist_env()
    dist = bench.dist_init(w, "gloo")
    mine = fg2_b200.shard_members(bench.batch_sizes(), w)[r]
    everyone = [None] * w
    dist.all_gather_object(everyone, mine)
    cells = sum(a * b for a, b in (bench.batch_sizes()[k] for k in mine))
    mx = bench.reduce_max(cells, dist, "cpu")  # the slowest rank is the one with the most cells
    out[rank] = (everyone, cells, mx)
    dist.destroy_process_group()


def test_two_ranks_own_disjoint_member_shards():
    """Each gloo rank takes its share of the 512-member batch as the bench's batch leg does at
    N > 1; together the shards are the whole batch, each member on exactly one rank."""
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(shard_worker, args=(world, free_port(), out), nprocs=world, join=True, start_method="spawn")
    import bench
    total = sum(a * b for a, b in bench.batch_sizes())
    shards0, c0, mx = out[0]
    shards1, c1, _ = out[1]
    assert shards0 == shards1
    assert sorted(shards0[0] + shards0[1]) == list(range(len(bench.batch_sizes())))
    assert c0 + c1 == total and mx == max(c0, c1)
