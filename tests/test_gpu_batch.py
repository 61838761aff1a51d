"""Worlds stepped together on one GPU equal their own single-world runs.

A batch is independent erosion stages (bake/globe/erosion/run.py, one world
each); running them concurrently, one CUDA stream per world, must not change
any world's result.  The exact (ordered) apply is deterministic, so the
comparison is bit for bit.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "procedural-generation_b200"))

pytestmark = pytest.mark.gpu

FIELDS = ("height", "sediment", "discharge", "momentum", "pending")


def _worlds():
    from pgerosion import batch

    return batch.batch_worlds(4, seed=7, iterations=2, sizes=(24, 32, 40))


def test_concurrent_worlds_equal_their_single_runs(cuda):
    import torch

    from pgerosion import batch
    from pgerosion import maps as gm

    ws = _worlds()
    counts = [min(w.n_particles, 1500) for w in ws]
    together = batch.build_states(ws)
    runner = batch.Runner(together, [w.params for w in ws])
    stats = runner.step(2, n_particles=counts)
    assert all(len(s) == 2 for s in stats)
    alone = batch.build_states(ws)
    for i, (st, w) in enumerate(zip(alone, ws)):
        for it in range(2):
            s = gm.step(st, w.params, it, n_particles=counts[i])
            assert s["droplet_steps"] == stats[i][it]["droplet_steps"]
    torch.cuda.synchronize()
    for a, b in zip(together, alone):
        assert a.iteration == b.iteration == 2
        for f in FIELDS:
            assert torch.equal(getattr(a, f), getattr(b, f)), f


def test_fewer_streams_than_worlds(cuda):
    import torch

    from pgerosion import batch

    ws = _worlds()
    counts = [min(w.n_particles, 800) for w in ws]
    a = batch.build_states(ws)
    b = batch.build_states(ws)
    batch.Runner(a, [w.params for w in ws], streams=2).step(1, n_particles=counts)
    batch.Runner(b, [w.params for w in ws], streams=4).step(1, n_particles=counts)
    for x, y in zip(a, b):
        for f in FIELDS:
            assert torch.equal(getattr(x, f), getattr(y, f)), f


def test_packed_lanes_are_exact(cuda):
    """Several droplets per warp in the trace and in the apply (the footprint
    settings for worlds sharing the GPU) give the same result bit for bit."""
    import torch

    from pgerosion import batch
    from pgerosion import maps as gm

    ws = batch.batch_worlds(1, seed=11, iterations=2, sizes=(48,))
    a = batch.build_states(ws)[0]
    b = batch.build_states(ws)[0]
    n = 3000
    for it in range(2):
        sa = gm.step(a, ws[0].params, it, n_particles=n)
        sb = gm.step(b, ws[0].params, it, n_particles=n, trace_lanes=32, apply_lanes=4)
        assert sa["droplet_steps"] == sb["droplet_steps"]
    torch.cuda.synchronize()
    for f in FIELDS:
        assert torch.equal(getattr(a, f), getattr(b, f)), f


def test_wave_apply_worlds_with_thread_shares_equal_their_single_runs(cuda):
    """The wave apply's worlds stepped together, each with a share of the
    ledger threads (``max_threads``: smaller own-change tables, a smaller
    persistent launch), equal the same worlds stepped alone with every
    thread: the int64 sums do not depend on which thread took a droplet."""
    import torch

    from pgerosion import _lib, batch
    from pgerosion import maps as gm

    ws = _worlds()
    counts = [min(w.n_particles, 1500) for w in ws]
    kw = {"apply": _lib.APPLY_WAVE, "wave": 4000}
    together = batch.build_states(ws)
    for st, q in zip(together, batch.thread_quota([w.cost for w in ws], total=1024)):
        st.max_threads = q
    batch.Runner(together, [w.params for w in ws], **kw).step(2, n_particles=counts)
    alone = batch.build_states(ws)
    for i, (st, w) in enumerate(zip(alone, ws)):
        for it in range(2):
            gm.step(st, w.params, it, n_particles=counts[i], **kw)
    torch.cuda.synchronize()
    assert all(st._ws_threads <= 1024 for st in together)
    for a, b in zip(together, alone):
        for f in FIELDS:
            assert torch.equal(getattr(a, f), getattr(b, f)), f
