"""CPU: the multi-GPU split of the batched workload (longest-processing-time
partition, computed identically on every rank) and the one host gather of
results after the run, with two gloo ranks.  No GPU: the instances' results
are stand-ins built from their index."""
import os
import socket

import numpy as np
import pytest

import llg
import shard


def test_lpt_partition_is_balanced_and_deterministic(llg_lib):
    rng = np.random.default_rng(5)
    costs = rng.uniform(1.0, 100.0, 64)
    for parts in (1, 2, 3, 4, 8):
        part, load = shard.partition_lpt(costs, parts)
        assert part.min() >= 0 and part.max() < parts
        assert np.allclose([costs[part == r].sum() for r in range(parts)], load)
        lower = max(costs.sum() / parts, costs.max())          # bound on the optimal makespan
        assert load.max() <= (4.0 / 3.0) * lower + 1e-9
        again, _ = shard.partition_lpt(costs, parts)
        assert np.array_equal(part, again)
    # textbook instance: 2 parts, costs 3 3 2 2 2 -> LPT makespan 7 (optimum 6)
    part, load = shard.partition_lpt([3, 3, 2, 2, 2], 2)
    assert list(load) == [7.0, 5.0] and list(part) == [0, 1, 0, 1, 0]
    with pytest.raises(llg.LLGError):
        shard.partition_lpt([1.0, -1.0], 2)


def test_config4_split_covers_every_instance_once(llg_lib):
    insts = llg.config4_instances(64, 12345)
    seen = []
    for r in range(4):
        seen += shard.my_instances(insts, 4, r)
    assert sorted(seen) == list(range(64))
    costs = [shard.instance_cost(x["params"]) for x in insts]
    _, load = shard.partition_lpt(costs, 4)
    assert load.max() / load.mean() < 1.05


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    import datetime
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "gpu-micromagnetics-irregular_b200"))
    import torch.distributed as dist
    import llg as _llg
    import shard as _shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        insts = _llg.config4_instances(64, 12345)
        mine = _shard.my_instances(insts, world, rank)
        # stand-in results: a final "state" and counters derived from the index
        local = {i: {"rank": rank, "nst": 100 + i, "m": np.full(3, float(i))} for i in mine}
        merged = _shard.gather_results(local, world, rank)
        if rank == 0:
            np.save(out_path, np.array([[k, v["rank"], v["nst"], v["m"][0]] for k, v in merged.items()]))
        else:
            assert merged is None
    finally:
        dist.destroy_process_group()


def test_two_rank_split_and_gather_over_gloo(llg_lib, tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "merged.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    rows = np.load(out)
    assert rows.shape == (64, 4)
    assert list(rows[:, 0].astype(int)) == list(range(64))          # every instance once, in order
    insts = llg.config4_instances(64, 12345)
    part, _ = shard.partition_lpt([shard.instance_cost(x["params"]) for x in insts], 2)
    assert np.array_equal(rows[:, 1].astype(int), part)             # gathered from the rank that owns it
    assert np.array_equal(rows[:, 2], 100 + np.arange(64)) and np.array_equal(rows[:, 3], np.arange(64))
