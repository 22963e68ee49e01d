"""Sharding of batched problems over ranks (host logic) and the result gather over a world of two
gloo ranks on the CPU: every instance is solved on exactly one rank, loads are balanced, and the
merged results come back in instance order on every rank."""
import os

import numpy as np
import pytest

from specann_b200 import sharding


def sizes_c3(count=64, seed=7):
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(np.log(2 ** 10), np.log(2 ** 17), count)).astype(int)
    return [(int(x), int(20 * x)) for x in n]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shards_partition_and_balance(world):
    sizes = sizes_c3()
    shards = sharding.shard_instances(sizes, world)
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(len(sizes)))
    costs = [sum(sharding.instance_cost(*sizes[i]) for i in s) for s in shards]
    biggest = max(sharding.instance_cost(*s) for s in sizes)
    assert max(costs) - min(costs) <= biggest + 1e-6


def test_merge_rejects_duplicates():
    with pytest.raises(ValueError):
        sharding.merge_results([{0: [1]}, {0: [2]}])


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sizes = sizes_c3(10)
    mine = sharding.shard_instances(sizes, world)[rank]
    # stand-in per-problem results (the GPU solve is not part of this CPU test)
    local = {i: [{"instance": i, "seed": s, "energy": -float(i * 10 + s)} for s in (1, 2)] for i in mine}
    gathered = [None] * world
    dist.all_gather_object(gathered, local)
    merged = sharding.merge_results(gathered)
    np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([r["energy"] for r in merged]))
    dist.barrier()
    dist.destroy_process_group()


def test_gather_over_two_gloo_ranks(tmp_path):
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    expect = np.array([-float(i * 10 + s) for i in range(10) for s in (1, 2)])
    for r in range(2):
        assert np.array_equal(np.load(tmp_path / f"r{r}.npy"), expect)
