"""One batch of instances split across ranks (pdhcg_b200/shard.py), on the
CPU: the nonzero-balanced partition covers every instance exactly once and
keeps the bins within one instance's weight of each other; with two gloo
ranks, each rank solves only its bin and rank 0 gets every result back in
the batch's order.  The solver is a stand-in (no GPU); the batched kernel
itself is tested on the GPU in test_gpu_batch.py."""
import os
import socket

import numpy as np
import pytest

from pdhcg_b200 import instances, shard


def _check_bins(weights, bins):
    flat = sorted(i for b in bins for i in b)
    assert flat == list(range(len(weights)))  # every instance exactly once
    for b in bins:
        assert b == sorted(b)
    loads = [sum(weights[i] for i in b) for b in bins]
    assert max(loads) - min(loads) <= max(weights) + 1e-9


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_partition_covers_once_and_balances(parts):
    w = instances.mpc_nnz  # the batched workload's weights
    weights = [w(int(t)) for t in instances.mpc_horizons(4, 4096)]
    bins = shard.partition(weights, parts)
    assert len(bins) == parts
    _check_bins(weights, bins)
    assert shard.partition(weights, parts) == bins  # a pure function of the weights


def test_partition_edge_cases():
    assert shard.partition([], 3) == [[], [], []]
    assert shard.partition([5.0], 4) == [[0], [], [], []]
    bins = shard.partition([1.0] * 7, 2)
    _check_bins([1.0] * 7, bins)
    with pytest.raises(ValueError):
        shard.partition([1.0], 0)


def _fake_solver(problems, params):
    return [{"status": "OPTIMAL", "tag": p["tag"], "solved_by": os.environ["RANK"]} for p in problems]


def _worker(rank, world, port, weights, out_path):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        built = []

        def build(idx):
            built.extend(idx)
            return [{"tag": 1000 + i} for i in idx]

        res = shard.solve_batch_sharded(weights, build, {}, solver=_fake_solver, rank=rank, world=world)
        # this rank built exactly its own bin
        assert built == shard.partition(weights, world)[rank]
        if rank == 0:
            np.save(out_path, np.array([[r["tag"], int(r["solved_by"])] for r in res]))
        else:
            assert res is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_solve_world2_gloo(tmp_path):
    import torch.multiprocessing as mp
    weights = [instances.mpc_nnz(int(t)) for t in instances.mpc_horizons(4, 257)]
    out = str(tmp_path / "res.npy")
    mp.start_processes(_worker, args=(2, _free_port(), weights, out), nprocs=2, join=True, start_method="spawn")
    res = np.load(out)
    assert res[:, 0].tolist() == [1000 + i for i in range(len(weights))]  # the batch's order
    bins = shard.partition(weights, 2)
    for r in (0, 1):
        assert sorted(np.nonzero(res[:, 1] == r)[0].tolist()) == bins[r]  # solved where the partition put it
