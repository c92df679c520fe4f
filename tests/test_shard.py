"""Case sharding of the batched form over ranks: the assignment, and the
end-of-run reductions run as two gloo ranks on CPU (no GPU)."""
import os
import socket

import numpy as np
import pytest

from minifs_b200 import shard


def _cells_of_batched_workload(ncase=64, seed=2024):
    import bench
    return [6 * c["n"] ** 3 for c in bench.batched_workload(ncase, seed)["cases"]]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_assignment_complete_disjoint_balanced(world):
    cells = _cells_of_batched_workload()
    owner = shard.assign_cases(cells, world)
    assert len(owner) == len(cells) and set(owner) <= set(range(world))
    parts = [shard.rank_cases(cells, world, r) for r in range(world)]
    assert sorted(k for p in parts for k in p) == list(range(len(cells)))
    loads = [sum(cells[k] for k in p) for p in parts]
    assert max(loads) - sum(cells) / world < max(cells)
    assert shard.assign_cases(cells, world) == owner  # deterministic


def test_assignment_edge_cases():
    assert shard.assign_cases([], 4) == []
    assert shard.assign_cases([5, 5, 5], 1) == [0, 0, 0]
    assert shard.assign_cases([1, 9, 3], 3) == [2, 0, 1]
    with pytest.raises(ValueError):
        shard.assign_cases([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    cells = _cells_of_batched_workload()
    mine = shard.rank_cases(cells, world, rank)
    local = sum(cells[k] for k in mine)
    total = shard.reduce_sum(local, dist)
    fake_ms = 10.0 + rank  # the slower rank decides the job time
    ms = shard.reduce_max(fake_ms, dist)
    np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([local, total, ms, len(mine)]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    cells = _cells_of_batched_workload()
    r = [np.load(tmp_path / f"r{k}.npy") for k in range(world)]
    assert r[0][1] == r[1][1] == sum(cells)
    assert r[0][0] + r[1][0] == sum(cells)
    assert r[0][2] == r[1][2] == 11.0
    assert r[0][3] + r[1][3] == len(cells)
