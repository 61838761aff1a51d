"""Host logic of the batched workload and of the multi-rank runs (CPU only).

The worlds of a batch are independent (one bake stage each,
bake/globe/erosion/run.py); ranks share them out with no collective on the
data path and reduce only their work and time at the end.  The multi-rank
test runs that logic as two ``gloo`` ranks on the CPU.
"""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "procedural-generation_b200"))

from pgerosion import batch  # noqa: E402
from pgerosion.params import max_steps_of  # noqa: E402


def test_batch_worlds_follow_the_workload():
    a = batch.batch_worlds(64, seed=3)
    b = batch.batch_worlds(64, seed=3)
    assert [w.N for w in a] == [w.N for w in b]
    assert [w.params.erosion.friction for w in a] == [w.params.erosion.friction for w in b]
    assert len(a) == 64
    assert set(w.N for w in a) <= set(batch.BATCH_SIZES)
    assert len(set(w.N for w in a)) >= 4  # the sizes really vary
    base = batch.ErosionParams()
    for w in a:
        ep = w.params.erosion
        assert w.n_particles == 6 * w.N * w.N // 8
        assert max_steps_of(ep, w.N) == 2 * w.N
        for name in ("friction", "erodibility", "deposition_rate", "evap_rate"):
            r = getattr(ep, name) / getattr(base, name)
            assert 1 - batch.BATCH_JITTER - 1e-12 <= r <= 1 + batch.BATCH_JITTER + 1e-12
        assert abs(w.params.world.cell_size_m * w.N - 9773.0 * 1024) < 1e-6
    assert [w.N for w in batch.batch_worlds(64, seed=4)] != [w.N for w in a]


@pytest.mark.parametrize("world_size", [1, 2, 3, 8])
def test_assign_is_complete_disjoint_and_balanced(world_size):
    costs = [w.cost for w in batch.batch_worlds(64, seed=0)]
    parts = batch.assign(costs, world_size)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    # longest-first greedy: no rank exceeds another by more than the largest world
    assert max(loads) - min(loads) <= max(costs) + 1e-9
    assert parts == batch.assign(costs, world_size)  # every rank computes the same split


def test_assign_more_ranks_than_worlds():
    parts = batch.assign([5.0, 1.0], 4)
    assert parts == [[0], [1], [], []]


def _rank_main(rank, world_size, init_file, out_dir):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"file://{init_file}", rank=rank, world_size=world_size)
    try:
        costs = [w.cost for w in batch.batch_worlds(16, seed=1)]
        mine = batch.my_worlds(costs, rank, world_size)
        everyone = [None] * world_size
        dist.all_gather_object(everyone, mine)
        flat = sorted(i for p in everyone for i in p)
        assert flat == list(range(len(costs))), flat
        # the job's work is the sum over ranks, its time the slowest rank's
        sums, maxes = batch.reduce_totals(dist, [len(mine), sum(costs[i] for i in mine)], [10.0 + rank, -rank])
        assert sums[0] == len(costs)
        assert abs(sums[1] - sum(costs)) < 1e-6 * sum(costs)
        assert maxes == [10.0 + world_size - 1, 0.0]
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array(mine, dtype=np.int64))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_worlds_and_reduce(tmp_path):
    import torch.multiprocessing as mp

    init_file = tmp_path / "pg_init"
    mp.spawn(_rank_main, args=(2, str(init_file), str(tmp_path)), nprocs=2, join=True)
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    assert len(set(r0) & set(r1)) == 0
    assert len(r0) + len(r1) == 16


def test_reduce_totals_single_rank():
    sums, maxes = batch.reduce_totals(None, [1, 2.5], [3.0])
    assert sums == [1.0, 2.5] and maxes == [3.0]


def test_thread_quota_shares_the_ledger_threads_by_cost():
    costs = [w.cost for w in batch.batch_worlds(64, seed=0)]
    q = batch.thread_quota(costs)
    assert all(v % 256 == 0 and 256 <= v <= batch.LEDGER_THREADS for v in q)
    # in proportion to cost, every world at least one block; the total about the GPU's resident threads
    big, small = max(range(64), key=lambda i: costs[i]), min(range(64), key=lambda i: costs[i])
    assert q[big] > q[small] == 256
    assert batch.LEDGER_THREADS <= sum(q) <= batch.LEDGER_THREADS + 64 * 256
