"""Many independent worlds: the batched workload of worlds of different
sizes and rates, eroded together.

The reference bakes one world per process: the erosion stage
(bake/globe/erosion/run.py) steps one ``ErosionState`` through
``maps.step`` (bake/globe/erosion/maps.py:1516-1617).  A batch of worlds is
that stage run for each world; nothing couples them.  Here:

* on one GPU, every world steps on its own CUDA stream, driven from its own
  host thread, so the latency-bound waves of many worlds overlap on the
  SMs (one world's exact pass occupies a small part of the GPU);
* across GPUs (one process per GPU), the worlds are shared out between the
  ranks by estimated cost, with no collective on the data path; only the
  per-world statistics and the timing are reduced at the end.

Each world's results are those of its own single-world run, bit for bit:
the exact (ordered) apply is deterministic and the worlds share no state.
"""
from __future__ import annotations

import dataclasses
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from .params import ErosionParams, WorldGroup, WorldParams, plain_knobs

#: world sizes of the batched workload, drawn per world by seed
BATCH_SIZES = (64, 96, 128, 192, 256, 384, 512)
#: the rates jittered per world (friction, erodibility, deposition, evaporation), +- this fraction
BATCH_JITTER = 0.30


@dataclasses.dataclass
class BatchWorld:
    """One world of a batch: its parameters and droplets per iteration."""

    params: WorldParams
    n_particles: int

    @property
    def N(self) -> int:
        return int(self.params.world.N_c)

    @property
    def cost(self) -> float:
        """Relative cost of one iteration: droplets x their lifetime bound."""
        return float(self.n_particles) * float(2 * self.N)


def batch_worlds(n_worlds: int = 64, seed: int = 0, iterations: int = 50, sizes=BATCH_SIZES,
                 jitter: float = BATCH_JITTER) -> list[BatchWorld]:
    """The batched workload: ``n_worlds`` Earth-like worlds, each with N_c
    drawn from ``sizes`` and friction, erodibility, deposition rate and
    evaporation rate scaled by U(1 - jitter, 1 + jitter), all from
    ``seed``; 6 N^2 / 8 droplets per iteration; max_steps = the reference's
    default 2 N (``erosion.max_steps = 0``); the same planet at every
    resolution (cell size 9773 m x 1024 / N)."""
    rng = np.random.default_rng([seed, 64])
    base = ErosionParams()
    out = []
    for i in range(n_worlds):
        N = int(sizes[int(rng.integers(len(sizes)))])
        f = 1.0 + jitter * (2.0 * rng.random(4) - 1.0)
        ep = ErosionParams(iterations=iterations, max_steps=0, uplift_mode="replay",
                           friction=base.friction * f[0], erodibility=base.erodibility * f[1],
                           deposition_rate=base.deposition_rate * f[2], evap_rate=base.evap_rate * f[3], **plain_knobs())
        wp = WorldParams(world=WorldGroup(seed=seed * 1000 + i, N_c=N, cell_size_m=9773.0 * 1024.0 / N, land_fraction=0.29,
                                          halo=2), erosion=ep)
        out.append(BatchWorld(wp, 6 * N * N // 8))
    return out


def assign(costs, world_size: int) -> list[list[int]]:
    """Share worlds out between ``world_size`` ranks: longest first, each to
    the least-loaded rank (ties to the lowest rank).  Deterministic, so
    every rank computes the same assignment without communicating."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world_size
    out: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(costs[i])
    return [sorted(x) for x in out]


#: resident droplet threads of the wave apply's ledger kernel on a B200: one block of 256 a multiprocessor
LEDGER_THREADS = 148 * 256


def thread_quota(costs, total: int = LEDGER_THREADS) -> list[int]:
    """Each world's share of the wave apply's resident ledger threads, in
    proportion to its cost, rounded up to whole blocks of 256 (at least
    one): the per-thread own-change tables of many worlds at once then fit
    in HBM (``ErosionState.max_threads``)."""
    tot = float(sum(costs)) or 1.0
    return [int(min(total, max(256, -(-int(total * float(c) / tot) // 256) * 256))) for c in costs]


def my_worlds(costs, rank: int, world_size: int) -> list[int]:
    """The worlds rank ``rank`` erodes."""
    return assign(costs, world_size)[rank]


def reduce_totals(dist, sums, maxes, device="cpu"):
    """Across ranks: element-wise sums of ``sums`` and maxima of ``maxes``
    (the job's work and its slowest rank's time).  ``dist`` None: one rank."""
    import torch

    s = torch.tensor([float(x) for x in sums], dtype=torch.float64, device=device)
    m = torch.tensor([float(x) for x in maxes], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(s)
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
    return [float(x) for x in s.cpu()], [float(x) for x in m.cpu()]


class Runner:
    """Step many worlds concurrently on one GPU: world ``i`` runs on its own
    CUDA stream from its own host thread (the library call of a droplet pass
    releases the interpreter while its waves are launched).

    The costliest worlds (droplets x lifetime bound, ``costs``) get the
    highest stream priority: they set the batch's makespan, and the small
    worlds fill the SMs around them.  The CUDA runtime multiplexes streams
    onto ``CUDA_DEVICE_MAX_CONNECTIONS`` hardware queues (8 by default);
    set it to 32 before CUDA starts for up to 32 truly independent queues.

    Each world's trace runs 32 droplets per warp (``trace_lanes``): alone, a
    wave's trace is fastest spread thin, but many worlds at once are limited
    by the registers their resident warps hold (measured on the 64-world
    batch: 234 M droplet-steps/s at 32 per warp against 191 M spread thin).
    The apply keeps one droplet per warp: packing several made the batch
    slower (lanes of one warp that wait on different hand-offs take turns)."""

    def __init__(self, states, params, streams: int | None = None, costs=None, trace_lanes: int = 32, **step_kw):
        import torch

        if len(states) != len(params):
            raise ValueError("one params per state")
        self.states = list(states)
        self.params = list(params)
        n = len(self.states) if streams is None else max(1, min(int(streams), len(self.states)))
        if costs is None:
            costs = [float(s.N) ** 3 for s in self.states]
        lo, hi = torch.cuda.Stream.priority_range()  # (lowest, highest): higher priority = smaller number
        top = max(costs) if len(costs) else 1.0
        self.streams = []
        for i in range(n):
            pr = hi if costs[i] >= 0.5 * top else lo
            self.streams.append(torch.cuda.Stream(device=self.states[i].height.device, priority=pr))
        self.step_kw = dict(step_kw)
        if len(self.states) > 1:
            self.step_kw.setdefault("trace_lanes", int(trace_lanes))
        # one long-lived pool: a world's host passes (the lake balance keeps its scratch per thread) run on
        # threads that stay, so later refreshes reuse their pages
        self._pool = ThreadPoolExecutor(max_workers=len(self.streams))

    def close(self) -> None:
        """Stop the runner's host threads (their per-thread scratch goes with them)."""
        self._pool.shutdown(wait=True)

    def _run(self, i: int, iterations: int, first: int | None, kw: dict, spawns) -> list[dict]:
        import torch

        from . import maps as gm

        st, p = self.states[i], self.params[i]
        out = []
        with torch.cuda.stream(self.streams[i % len(self.streams)]):
            for k in range(iterations):
                it = st.iteration if first is None else first + k
                extra = {}
                if spawns is not None:
                    extra["predrawn"] = spawns(i, it)
                out.append(gm.step(st, p, it, **kw, **extra))
            torch.cuda.current_stream().synchronize()
        return out

    def step(self, iterations: int = 1, first: int | None = None, n_particles=None, spawns=None) -> list[list[dict]]:
        """``iterations`` plain iterations of every world; returns each
        world's per-iteration statistics.  ``n_particles``: one count per
        world (None: the worlds' defaults).  ``spawns(i, iteration)``: the
        world's pre-drawn spawn uniforms (``maps.draw_spawns`` output moved
        to the device), or None to draw them on the host each iteration."""
        import torch

        torch.cuda.synchronize()
        kws = []
        for i in range(len(self.states)):
            kw = dict(self.step_kw)
            if n_particles is not None:
                kw["n_particles"] = int(n_particles[i])
            kws.append(kw)
        # the costliest worlds first, so their threads start their passes first
        order = sorted(range(len(self.states)), key=lambda i: -self.states[i].N)
        futs = {i: self._pool.submit(self._run, i, iterations, first, kws[i], spawns) for i in order}
        res = [futs[i].result() for i in range(len(self.states))]
        torch.cuda.synchronize()
        return res


def build_states(batch: list[BatchWorld], device="cuda"):
    """ErosionStates of a batch (Earth-like synthetic stage inputs), with the
    uplift replay started as the stage does."""
    from . import maps as gm
    from .synth import earth_world

    states = []
    for bw in batch:
        w = bw.params.world
        world = earth_world(seed=int(w.seed), N=int(w.N_c), cell_size_m=float(w.cell_size_m), land_fraction=float(w.land_fraction))
        st = gm.ErosionState.from_world(world, device=device)
        gm.start_replay(st, bw.params)
        states.append(st)
    return states
