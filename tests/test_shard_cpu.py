"""Multi-rank path of the batched workload, on CPU: the cost partition of
independent problems across ranks and the gather of their results, run as two
gloo ranks. The per-rank stepping is the CPU oracle here (no GPU); on GPUs each
rank steps its share as one `Batch`, with the same partition and gather."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fdtd_b200 import problem as P
from fdtd_b200.shard import gather_results, imbalance, partition_by_cost, problem_cost, shard_for_rank


def test_partition_covers_every_problem_once():
    rng = np.random.default_rng(3)
    for world in range(1, 9):
        costs = rng.uniform(1.0, 100.0, size=37)
        shares = partition_by_cost(costs, world)
        flat = sorted(q for s in shares for q in s)
        assert flat == list(range(37))
        assert shares == partition_by_cost(list(costs), world)  # deterministic
        # longest-processing-time bound: max load <= 4/3 optimum (+ one job)
        assert imbalance(costs, shares) <= 4.0 / 3.0 + costs.max() / (costs.sum() / world)


def test_partition_of_the_batched_workload_is_balanced():
    probs = P.config3(128, steps=3000)
    costs = [problem_cost(p) for p in probs]
    for world in (2, 4, 8):
        shares = partition_by_cost(costs, world)
        assert imbalance(costs, shares) < 1.05
        assert [shard_for_rank(probs, r, world) for r in range(world)] == shares


def test_partition_rejects_bad_arguments():
    with pytest.raises(ValueError):
        partition_by_cost([1.0], 0)
    with pytest.raises(ValueError):
        shard_for_rank([], 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _small_batch():
    return P.config3(5, steps=24, seed=11, nmin=30, nmax=48, npml=4, nrect=2)


def _rank_main(rank, world, port, out_path):
    import sys
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    import pyoracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        probs = _small_batch()
        mine = shard_for_rank(probs, rank, world)
        local = {q: pyoracle.run_oracle(probs[q]).get("Hz") for q in mine}
        merged = gather_results(local)
        if rank == 0:
            np.savez(out_path, **{str(q): v for q, v in merged.items()})
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_step_their_shares_and_gather(oracle, tmp_path):
    out = str(tmp_path / "gathered.npz")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    probs = _small_batch()
    assert sorted(int(k) for k in got.files) == list(range(len(probs)))
    for q, p in enumerate(probs):
        ref = oracle.run_oracle(p).get("Hz")
        assert np.array_equal(got[str(q)], ref)
