"""Benchmark: droplet-steps/s of the erosion stage on the Earth-default world.

Workload (one "step" = one full plain erosion iteration): cube-sphere
N_c = 1024, halo 2, 6 x 1028 x 1028 float32 fBm + ridge bedrock (-8000..+6000 m,
29 % land), latitude-banded rain 0.1..3.0, uplift replay 0..2 mm/iteration,
1,572,864 droplets per iteration (+ re-injected stockpiles), max lifetime 96
steps.  A droplet-step is one change-list entry of volume >= 0 (one step
that reaches the mass-transfer section).  Data: seeded synthetic world.

Arms
  default          the CUDA library (libpgerosion.so) through pgerosion.maps
  --impl reference the reference algorithm's CPU restatement (the oracle, a
                   port of the numba code; numba itself is not installed
                   where the bench runs), timed on all host cores

Multi-GPU: ``torchrun --nproc-per-node N bench.py --gpus N``: every rank
erodes its own world (seed = rank), no collective on the data path (weak
scaling); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for p in (ROOT, ROOT / "procedural-generation_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

#: algorithmic bytes of one droplet-step on the plain path: gathered 2x2
#: surface (16 B), 2x2 momentum a/b and discharge (48 B), inverse metric and
#: metric (24 B), base / evap / hardness / sediment (16 B), mask (1 B);
#: scattered int64 terrain change, discharge and two momentum tracks (32 B)
BYTES_PER_STEP = 137
#: the brush measurement (radius 3, BASELINE's c1 / c2 brush): the same gathers (105 B), the
#: int64 terrain change scattered over the footprint (45 cells within distance < 4: 360 B) and the
#: discharge and two momentum tracks on the step's own cell (24 B)
BRUSH_RADIUS = 3
BRUSH_CELLS = 45
BRUSH_BYTES_PER_STEP = 105 + 8 * BRUSH_CELLS + 24
#: the planet level's brush (radius 2): 25 cells within distance < 3
PLANET_BRUSH_CELLS = 25


def run_batched(args, rank, world_size, dist, dev):
    """The batched workload: 64 Earth-like worlds, N_c drawn from 64..512, rates jittered +-30 %,
    6 N^2 / 8 droplets and max_steps 2 N each, shared out between the ranks.  Timed per rank with
    CUDA events (max over ranks): one iteration with the worlds stepped one by one on one stream,
    then iterations with every world on its own stream at once (pgerosion.batch.Runner)."""
    import torch

    from pgerosion import batch
    from pgerosion import maps as gm

    worlds = batch.batch_worlds(args.batch_worlds, seed=0)
    mine = batch.my_worlds([w.cost for w in worlds], rank, world_size)
    sub = [worlds[i] for i in mine]
    counts = [w.n_particles for w in sub]
    k = max(1, args.batch_steps)
    states = batch.build_states(sub, device=dev)
    # every world's spawn uniforms for the timed iterations, drawn up front and resident in HBM
    pre = {}
    for i, w in enumerate(sub):
        for it in range(1, 2 + k):
            rng, u, off = gm.draw_spawns(w.params, "erosion", (it,), counts[i])
            pre[(i, it)] = (rng, torch.as_tensor(u, device=dev), torch.as_tensor(off, device=dev))
    from pgerosion import _lib

    wave_kw = {} if args.batch_apply == "ordered" else {"apply": _lib.APPLY_WAVE, "wave": max(counts) * 2 if counts else 1}
    wave = args.batch_apply == "wave"
    # the wave apply's own-change tables: every world at once holds a share of the GPU's resident ledger threads
    # (by cost), so that 64 worlds' tables fit; one by one, each world gets all of them (below)
    quota = batch.thread_quota([w.cost for w in sub]) if wave else [0] * len(sub)
    for st, q in zip(states, quota):
        st.max_threads = q
    runner = batch.Runner(states, [w.params for w in sub], costs=[w.cost for w in sub], trace_lanes=args.batch_trace_lanes,
                          streams=args.batch_streams or None, **wave_kw) if sub else None
    if runner:
        runner.step(1, n_particles=counts)  # warm-up: workspaces, first pass of every world
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev[0].record()
    one, worst = 0, 0.0
    ms_alone = 0.0
    for i, (st, w) in enumerate(zip(states, sub)):
        if wave:  # alone, a world's pass takes every resident ledger thread: its full tables, made before timing
            st.max_threads = 0
            st.reserve(counts[i] + st.F * st.N * st.N, gm.list_steps_of(w.params.erosion, st.N), 1, wave_tables=True)
            torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        one += gm.step(st, w.params, st.iteration, n_particles=counts[i], predrawn=pre[(i, st.iteration)], **wave_kw)["droplet_steps"]
        e1.record()
        e1.synchronize()
        worst = max(worst, e0.elapsed_time(e1))
        ms_alone += e0.elapsed_time(e1)
        if wave:  # back to the world's share, made again now (outside the timed passes)
            st.max_threads = quota[i]
            st.reserve(counts[i] + st.F * st.N * st.N, gm.list_steps_of(w.params.erosion, st.N), 1, wave_tables=True)
    ev[1].record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev[2].record()
    res = runner.step(k, n_particles=counts, spawns=lambda i, it: pre[(i, it)]) if runner else []
    ev[3].record()
    torch.cuda.synchronize()
    if runner:
        runner.close()
    together = sum(s["droplet_steps"] for r in res for s in r)
    # one by one: the sum of the worlds' own passes, each timed on the device (the host's turns between them, and
    # with the wave apply the workspaces made between them, are not counted)
    (one_all, tog_all), (ms_one, ms_tog, worst) = batch.reduce_totals(
        dist, [one, together], [ms_alone, ev[2].elapsed_time(ev[3]), worst], device=dev)
    sizes = sorted(w.N for w in worlds)
    v_one, v_tog = one_all / (ms_one * 1e-3), tog_all / (ms_tog * 1e-3)
    del runner, states
    torch.cuda.empty_cache()
    return {"workload": f"{len(worlds)} worlds, N_c {sizes[0]}..{sizes[-1]} (mean N_c^2 {np.mean(np.square(sizes)):.0f}), "
                        f"6 N^2/8 droplets, max_steps 2N, rates +-30 %, {args.batch_apply} apply",
            "one_by_one": {"value": v_one, "unit": "droplet-steps/s", "ms_per_step": ms_one},
            "concurrent": {"value": v_tog, "unit": "droplet-steps/s", "ms_per_step": ms_tog / k, "steps": k},
            "speedup": v_tog / v_one,
            "slowest_world_ms_per_step": worst}


def run_adjoint(args, dev):
    """The calibration workload: N_c = 256 Earth-like world, 2^17 droplets per
    iteration, 50 iterations, a checkpoint every 5; loss = mean squared
    height difference over land to a target made by the same run with the
    four rates jittered +-30 % (another seed); gradients with respect to a
    per-cell erodibility field (1 +- 0.2) and the four rates.  Times the
    forward (the run) and the adjoint (backward: recompute from the
    checkpoints with the passes taped, then the reverse) with CUDA events, for
    the default truncated gradient and for the exact one along the recorded
    paths."""
    import torch

    from pgerosion import adjoint as adj

    N, P, iters = args.adjoint_n, args.adjoint_droplets, args.adjoint_iterations
    params = adj.calibration_params(seed=0, N=N, iterations=iters)
    st = adj.calibration_state(params, device=dev)
    calib = adj.Calibration(st, params, iters, P, checkpoint_every=adj.CALIB_CHECKPOINT)
    target = calib.run(None, adj.rates_of(adj.calibration_params(seed=0, N=N, iterations=iters, jitter=0.3, jitter_seed=1)).tolist())
    land = torch.zeros_like(target, dtype=torch.bool)
    land[st.interior] = target[st.interior] > 0.0
    out = {"workload": f"calibration: N_c={N}, {P} droplets/iteration, {iters} "
                       f"iterations, checkpoint every {adj.CALIB_CHECKPOINT}, wave apply (one wave per iteration), loss = "
                       "mean squared land height difference (m^2) to a target from rates +-30 %",
           "metric": "adjoint/forward time ratio", "higher_is_better": False, "modes": {}}
    for name, cp, ct in (("truncated", False, False), ("exact_on_paths", True, True)):
        calib.carry_path, calib.carry_terrain = cp, ct
        fw, bw = [], []
        for rep in range(1 + max(1, args.adjoint_reps)):
            erod = adj.erodibility_init(st, seed=0).requires_grad_(True)
            rates = adj.rates_of(params).to(dev).requires_grad_(True)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            torch.cuda.synchronize()
            ev[0].record()
            loss = adj.land_loss(adj.erode(erod, rates, calib), target, land, st.height_unit_m)
            ev[1].record()
            loss.backward()
            ev[2].record()
            torch.cuda.synchronize()
            if rep > 0:  # the first repetition allocates the tapes
                fw.append(ev[0].elapsed_time(ev[1]))
                bw.append(ev[1].elapsed_time(ev[2]))
        g = rates.grad.detach().cpu().tolist()
        fin = bool(np.all(np.isfinite(g))) and bool(torch.isfinite(erod.grad).all())
        out["modes"][name] = {"carry_path": cp, "carry_terrain": ct, "forward_ms": float(np.median(fw)),
                              "adjoint_ms": float(np.median(bw)), "ratio": float(np.median(bw) / np.median(fw)),
                              "loss_m2": float(loss.detach()), "finite": fin,
                              "rate_gradient": g if fin else None,
                              "field_gradient_l1": float(erod.grad.double().abs().sum()) if fin else None}
    if args.calibrate_steps > 0:
        # gradient descent from the start (rates of the base parameters, field 1 +- 0.2) toward the target
        # made with the rates +-30 %: the loss at every step, and where the rates went
        calib.carry_path, calib.carry_terrain = False, False
        t0 = time.perf_counter()
        bl = lambda z: adj.block_loss(z, target, land, st.height_unit_m, N, st.H, block=8)
        cal = adj.calibrate(calib, target, land, adj.erodibility_init(st, seed=0), adj.rates_of(params), steps=args.calibrate_steps,
                            method="line", loss_fn=bl)
        torch.cuda.synchronize()
        tgt = adj.rates_of(adj.calibration_params(seed=0, N=N, iterations=iters, jitter=0.3, jitter_seed=1)).tolist()
        dist = lambda r: float(np.linalg.norm(np.log(np.asarray(r)) - np.log(np.asarray(tgt))))
        r0 = adj.rates_of(params).tolist()
        out["calibration"] = {"method": "line search along the normalised truncated gradient (log rates)",
                              "loss": "8x8-block land loss (m^2)", "steps": args.calibrate_steps, "loss_m2": cal["loss"],
                              "eta": cal["eta"], "forwards": cal["forwards"], "adjoints": cal["adjoints"],
                              "rates": cal["rates"][-1] if cal["rates"] else r0, "start_rates": r0, "target_rates": tgt,
                              "log_rate_distance_to_target": [dist(r0)] + [dist(r) for r in cal["rates"]],
                              "wall_s": time.perf_counter() - t0}
    out["value"] = out["modes"]["truncated"]["ratio"]
    out["droplet_steps_per_iteration"] = float(np.mean([s_.get("droplet_steps", 0) for s_ in calib.stats]))
    del calib, st
    torch.cuda.empty_cache()
    return out


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_world(seed: int, N: int | None = None):
    from pgerosion import synth

    params, P = synth.config_params("earth", seed=seed)
    if N is not None and N != params.world.N_c:
        params.world.N_c = N
        P = 6 * N * N // 4
    w = synth.earth_world(seed=seed, N=params.world.N_c)
    return params, P, w


def cpu_baseline(params, P, world, seconds=20.0):
    """The oracle (CPU restatement of the reference) on all host cores: full
    iterations of the same workload until ``seconds`` have passed."""
    from oracle import oracle as orc

    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    st = orc.OracleState.from_world(world, params)
    orc.start_replay(st, params)
    steps, t_all, n_it = 0, 0.0, 0
    while t_all < seconds and n_it < 50:
        t0 = time.perf_counter()
        s = orc.step(st, params, n_it, n_particles=P)
        t_all += time.perf_counter() - t0
        steps += s["droplet_steps"]
        n_it += 1
    return {"value": steps / t_all, "unit": "droplet-steps/s", "cores": threads, "kind": "port",
            "sample": f"{n_it} full iteration(s) of the same N_c={params.world.N_c} world, {t_all:.1f} s"}


def launches_per_iteration(nw: int, pending: bool, creep: bool, ordered: bool) -> int:
    """Kernels of this library one plain iteration launches (library kernels
    -- CUB scan / sort / select -- not counted)."""
    # weights, counts, quantised weights, CDF, the total's pairwise sum (plan, leaves, fold), search; the stockpiles
    spawn = 8 + (1 if pending else 0)
    if ordered:   # pack x2, terrain; per wave: trace, keys, flags, ranks, ordered apply, gather, finish; error report, mode, fold+EMA
        droplets = 3 + 7 * nw + 3
    else:         # pack x2; waves and the refreshes between them; mode, fold+EMA
        droplets = 2 + nw + (nw - 1) + 2
    thermal = 4 * (2 if creep else 1)
    uplift = 4    # the mean's pairwise sum (plan, leaves, fold), the add
    datum = 1 + 8 * 2 + 1
    halo = 4
    return spawn + droplets + thermal + uplift + datum + halo


def _side_leg(st, params, P, kw, it0, nsteps, dev, dist, bytes_per_step):
    """A secondary measurement on the evolved world: 3 untimed iterations with
    ``kw``, then ``nsteps`` timed ones (CUDA events around the whole steps and
    around each droplet pass); returns its result and the next iteration key."""
    import torch

    from pgerosion import maps as gm

    for k in range(3):
        rng, u, off = gm.draw_spawns(params, "erosion", (it0 + k,), P)
        gm.step(st, params, it0 + k, predrawn=(rng, torch.as_tensor(u, device=dev), torch.as_tensor(off, device=dev)), **kw)
    pre = []
    for k in range(nsteps):
        rng, u, off = gm.draw_spawns(params, "erosion", (it0 + 3 + k,), P)
        pre.append((rng, torch.as_tensor(u, device=dev), torch.as_tensor(off, device=dev)))
    ta = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e2 = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    e2[0].record()
    steps = 0
    for k in range(nsteps):
        s2 = gm.step(st, params, it0 + 3 + k, predrawn=pre[k], events=ta[k], **kw)
        steps += s2["droplet_steps"]
    e2[1].record()
    torch.cuda.synchronize()
    t2 = torch.tensor([steps, e2[0].elapsed_time(e2[1])], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(t2[:1])
        dist.all_reduce(t2[1:], op=dist.ReduceOp.MAX)
    avg = float(np.mean([a.elapsed_time(b) for a, b in ta]))
    ach = steps / max(nsteps, 1) * bytes_per_step / (avg * 1e-3) / 1e9
    peak, _ = _peaks()
    res = {"value": float(t2[0]) / (float(t2[1]) * 1e-3), "unit": "droplet-steps/s", "steps": nsteps,
           "ms_per_step": float(t2[1]) / nsteps,
           "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "ms_per_launch": avg}}
    return res, it0 + 3 + nsteps


def run_b200(args, rank, world_size, dist):
    import torch

    from pgerosion import _lib
    from pgerosion import maps as gm
    from pgerosion.batch import reduce_totals

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    params, P, world = make_world(seed=rank, N=args.n)
    st = gm.ErosionState.from_world(world)
    gm.start_replay(st, params)
    prec = _lib.PREC_F64 if args.precision == "f64" else _lib.PREC_F32
    wave = None if args.wave == 0 else args.wave
    apply = _lib.APPLY_ORDERED if args.apply == "ordered" else _lib.APPLY_WAVE
    kw = dict(n_particles=P, wave=wave, precision=prec, blocks_per_sm=args.blocks_per_sm, apply=apply, apply_lanes=args.apply_lanes)
    n_total = args.warmup + args.steps

    # value: spawn uniforms of every iteration drawn up front and resident in HBM
    pre = []
    for it in range(n_total):
        rng, u, off = gm.draw_spawns(params, "erosion", (it,), P)
        pre.append((rng, torch.as_tensor(u, device=dev), torch.as_tensor(off, device=dev)))
    for it in range(args.warmup):
        gm.step(st, params, it, predrawn=pre[it], **kw)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    # the droplet pass (pge_trace_apply) timed on its own stream with events
    ta = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    steps_done = 0
    n_waves = 0
    pend_any = False
    with ClockSampler(dev.index) as clk:
        torch.cuda.synchronize()
        ev[0].record()
        for k in range(args.steps):
            it = args.warmup + k
            st_k = gm.step(st, params, it, predrawn=pre[it], events=ta[k], **kw)
            steps_done += st_k["droplet_steps"]
            n_waves += -(-st_k["particles"] // st_k["chunk"])
            pend_any |= st_k["released"] > 0
        ev[1].record()
        torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1])
    ta_ms = [a.elapsed_time(b) for a, b in ta]
    # e2e: the public API with host buffers: spawns drawn on the host and
    # copied from pinned memory every step, stats read back every step
    h2d = d2h = 0
    e2e_steps = 0
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    # the public API's host feeder: each iteration's spawn uniforms drawn on the host (one iteration
    # ahead, into pinned memory) and copied to the device inside the step
    feeder = gm.SpawnFeeder(params, P, device=dev)
    feeder.prefetch((n_total,))
    e0 = time.perf_counter()
    ee = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ee[0].record()
    for k in range(args.steps):
        it = n_total + k
        rng, u_d, off_d, nbytes = feeder.get((it,))
        s = gm.step(st, params, it, predrawn=(rng, u_d, off_d), **kw)
        h2d += nbytes + 8 * _n_pending(s)
        d2h += (_lib.STATS_WORDS + 4 + 4) * 8
        e2e_steps += s["droplet_steps"]
    ee[1].record()
    torch.cuda.synchronize()
    e2e_ms = ee[0].elapsed_time(ee[1])
    feeder.close()
    (steps_all, e2e_all), (ms_max, e2e_ms_max) = reduce_totals(dist, [steps_done, e2e_steps], [ms, e2e_ms], device=dev)
    alt = brush = f32 = None
    it_next = n_total + args.steps
    if apply == _lib.APPLY_ORDERED and not args.no_alt:
        # the order-free wave apply on the same world (one wave per iteration): faster, not the
        # reference's serial apply
        kw_alt = dict(kw, apply=_lib.APPLY_WAVE, wave=max(P + P // 8, 1))
        alt, it_next = _side_leg(st, params, P, kw_alt, it_next, args.alt_steps, dev, dist, BYTES_PER_STEP)
        alt["apply"] = "wave (order-free, int64 fixed point; not the reference's serial apply)"
        if not args.no_brush:
            # the same with the erode / deposit brush of radius 3 (BASELINE's c2 brush; no reference counterpart)
            import dataclasses

            pb = dataclasses.replace(params, erosion=dataclasses.replace(params.erosion, brush_radius=BRUSH_RADIUS))
            brush, it_next = _side_leg(st, pb, P, kw_alt, it_next, args.alt_steps, dev, dist, BRUSH_BYTES_PER_STEP)
            brush["apply"] = f"wave apply with the erode / deposit brush, radius {BRUSH_RADIUS} ({BRUSH_CELLS} cells)"
            brush["bytes_per_step"] = BRUSH_BYTES_PER_STEP
        if not args.no_f32 and prec == _lib.PREC_F64:
            # the exact pass with the trace in float32 (the ledger and the apply stay float64): what float64
            # arithmetic costs the trace; its paths are not the reference's (tests: >= 90 % identical)
            kw32 = dict(kw, precision=_lib.PREC_F32)
            f32, it_next = _side_leg(st, params, P, kw32, it_next, min(args.alt_steps, 3), dev, dist, BYTES_PER_STEP)
            f32["trace"] = "float32 trace, float64 ordered apply (reference chunk waves)"
    batched = None
    if not args.no_batch:
        batched = run_batched(args, rank, world_size, dist, dev)
    if rank != 0:
        return None
    # the routing surface of the evolved N_c = 1024 terrain (erosion.flood_every's refresh), CUDA-event timed
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    sweeps = st.refresh_route(float(params.erosion.route_eps) / st.height_unit_m)
    e1.record()
    e1.synchronize()
    surf = st.height + st.sediment
    route_flood = {"what": "epsilon-filled routing surface (pge_route_flood + linear halo exchange) of the evolved world",
                   "ms": e0.elapsed_time(e1), "sweeps": sweeps, "filled_cells": int((st.route > surf).sum().item())}
    # the planet's lake refresh of the same terrain (erosion.lake_balance: the sea mask on the device, then the
    # host pass -- surface and sea off the device, flood, D8, evaporation balance, flags and levels back), wall clock
    # around synchronised calls: the host pass is not a kernel
    base0 = st.base.clone()
    st.refresh_base(0.02)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lk = st.refresh_lakes(6.0, 0.5 / st.height_unit_m, 0.02, 3.0)
    torch.cuda.synchronize()
    lake_balance = {"what": "planet lake refresh (refresh_lakes: D2H of surface and sea, the host flood + D8 + "
                            "evaporation balance of pge_lake_balance, H2D of flags and closed levels), lake_evap 6, land_evap 3",
                    "ms": (time.perf_counter() - t0) * 1e3, "host_threads": torch.get_num_threads(), **lk}
    st.route = st.lake_flag = st.sea_mask = st.base_at = None
    st.base = base0
    adjoint = None
    if not args.no_adjoint:
        adjoint = run_adjoint(args, dev)
    peak, peak_kind = _peaks()
    per_launch_steps = steps_done / max(args.steps, 1)
    avg_ta = float(np.mean(ta_ms))
    achieved = per_launch_steps * BYTES_PER_STEP / (avg_ta * 1e-3) / 1e9
    # DRAM bytes per droplet pass, from ncu (dram__bytes_read.sum + dram__bytes_write.sum) over the waves of an
    # exact pass of the N_c = 256 world: with the caches kept from kernel to kernel, as the live pass runs, 40 B
    # a droplet-step (scaled by the pass's droplet-steps); with ncu's flush before every kernel, 33.7 MB a wave
    # (the per-wave workspace is fixed, so that one scales with the waves)
    exact = apply == _lib.APPLY_ORDERED
    traffic = TRAFFIC_PER_STEP * per_launch_steps if exact else None
    traffic_cold = TRAFFIC_PER_WAVE_COLD * n_waves / max(args.steps, 1) if exact else None
    out = {
        "metric": "droplet-steps/s", "value": steps_all / (ms_max * 1e-3), "unit": "droplet-steps/s", "n_gpus": world_size,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == _lib.PREC_F64 else "f32",
        "data": "synthetic (seeded fBm + ridge Earth-default world per rank)",
        "config": {"workload": f"plain erosion iteration, cube-sphere N_c={params.world.N_c}, H=2, {P} droplets/iteration, "
                               f"max_steps 96, uplift replay", "N_c": params.world.N_c, "droplets_per_iteration": P,
                   "wave": "reference chunk" if wave is None else wave, "apply": args.apply,
                   "l2": "inputs larger than L2 (state > 1 GB)",
                   "parallelism": f"replicas x{world_size}"},
        "e2e": {"value": e2e_all / (e2e_ms_max * 1e-3), "unit": "droplet-steps/s", "h2d_bytes_per_step": h2d // max(args.steps, 1),
                "d2h_bytes_per_step": d2h // max(args.steps, 1)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_cold": traffic_cold, "peak_kind": peak_kind,
                     "kernel": "droplet pass (pge_trace_apply: trace waves, ordered apply or wave refreshes, pack, fold)",
                     "ms_per_launch": avg_ta, "bytes_per_step": BYTES_PER_STEP},
        "gpu_launches": launches_per_iteration(max(n_waves // max(args.steps, 1), 1), pend_any, params.erosion.creep_rate > 0,
                                               apply == _lib.APPLY_ORDERED) * args.steps,
        "clocks": clk.summary(),
    }
    if alt is not None:
        out["alt_wave_apply"] = alt
    if brush is not None:
        out["brush"] = brush
    if f32 is not None:
        out["f32_trace"] = f32
    if batched is not None:
        out["batched_worlds"] = batched
    if adjoint is not None:
        out["adjoint"] = adjoint
    out["route_flood"] = route_flood
    out["lake_balance"] = lake_balance
    if world_size == 1 and not args.no_cpu:
        w_host = world
        out["cpu_baseline"] = cpu_baseline(params, P, w_host, seconds=args.cpu_seconds)
    return out


def run_planet(args, dev):
    """Config c5: the planet-wide N_c = 8192 level on one GPU (pgerosion.planet): 2^24 droplets an
    iteration, max_steps 128, the wave apply with the brush of radius 2, heights to pinned host memory
    every 20 iterations.  Prints its own JSON line."""
    import torch

    from pgerosion import _lib
    from pgerosion import maps as gm
    from pgerosion import planet

    N = args.n or planet.PLANET_N
    params = planet.planet_params(N=N)
    P = planet.PLANET_DROPLETS if N == planet.PLANET_N else max(1, (6 * N * N) // 24)
    t0 = time.time()
    st = planet.planet_state(N=N, device=dev)
    build_s = time.time() - t0
    kw = dict(n_particles=P, apply=_lib.APPLY_WAVE, wave=P + P // 8)
    timeline = planet.Timeline(st, every=20)
    # the rain draws of the next iteration made on the host while the device runs this one (the public API's feeder)
    feeder = gm.SpawnFeeder(params, P, device=dev)
    feeder.prefetch((0,))
    total = args.warmup + args.steps if args.planet_iterations <= 0 else args.planet_iterations
    for it in range(args.warmup if args.planet_iterations <= 0 else 0):
        gm.step(st, params, it, predrawn=feeder.get((it,))[:3], **kw)
        timeline.maybe(it)
    torch.cuda.synchronize()
    first = args.warmup if args.planet_iterations <= 0 else 0
    ta = []
    steps = 0
    with ClockSampler(dev.index) as clk:
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        w0 = time.perf_counter()
        ev[0].record()
        for it in range(first, total):
            e = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            s = gm.step(st, params, it, events=e, predrawn=feeder.get((it,))[:3], **kw)
            timeline.maybe(it + 1)
            steps += s["droplet_steps"]
            ta.append(e)
        ev[1].record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - w0
    timeline.wait()
    feeder.close()
    ms = ev[0].elapsed_time(ev[1])
    n = total - first
    avg = float(np.mean([a.elapsed_time(b) for a, b in ta]))
    bytes_step = 105 + 8 * PLANET_BRUSH_CELLS + 24
    ach = steps / n * bytes_step / (avg * 1e-3) / 1e9
    peak, peak_kind = _peaks()
    a = st.to_numpy() if N <= 2048 else None
    out = {"metric": "droplet-steps/s", "value": steps / (ms * 1e-3), "unit": "droplet-steps/s", "n_gpus": 1, "steps": n,
           "warmup": first, "ms_per_step": ms / n, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded N_c=1024 fBm + ridge base, bicubic to N_c=8192, + 3 detail octaves; built on the device)",
           "config": {"workload": f"planet level: cube-sphere N_c={N}, H=2, {P} droplets/iteration, max_steps 128, wave apply, "
                                  f"brush radius 2, timeline every 20 iterations", "N_c": N, "droplets_per_iteration": P},
           "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind,
                        "kernel": "droplet pass (pge_trace_apply, one wave)", "ms_per_launch": avg, "bytes_per_step": bytes_step},
           "stage": {"iterations": n, "wall_s": wall, "build_s": build_s, "timeline_frames": [f for f, _ in timeline.frames],
                     "device_gb_peak": torch.cuda.max_memory_allocated(dev) / 1e9},
           "clocks": clk.summary()}
    if a is not None:
        out["stage"]["land_fraction"] = float(np.mean((a["height"] + a["sediment"])[st.interior] >= 0))
    return out


def _n_pending(stats) -> int:
    """Stockpile droplets of an iteration (their directions are host-drawn and copied)."""
    return int(stats.get("n_pending", 0))


def run_reference(args, rank):
    if rank != 0:
        return None
    params, P, world = make_world(seed=0, N=args.n)
    from oracle import oracle as orc

    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    st = orc.OracleState.from_world(world, params)
    orc.start_replay(st, params)
    for it in range(args.warmup):
        orc.step(st, params, it, n_particles=P)
    steps = 0
    t0 = time.perf_counter()
    for k in range(args.steps):
        s = orc.step(st, params, args.warmup + k, n_particles=P)
        steps += s["droplet_steps"]
    dt = time.perf_counter() - t0
    v = steps / dt
    return {"metric": "droplet-steps/s", "value": v, "unit": "droplet-steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded fBm + ridge Earth-default world)", "impl": "reference",
            "config": {"workload": f"plain erosion iteration, cube-sphere N_c={params.world.N_c}, H=2, {P} droplets/iteration, "
                                   f"max_steps 96, uplift replay", "N_c": params.world.N_c, "droplets_per_iteration": P},
            "cpu_baseline": {"value": v, "unit": "droplet-steps/s", "cores": threads, "kind": "port",
                             "sample": f"{args.steps} full iterations after {args.warmup} warm-up"},
            "e2e": {"value": v, "unit": "droplet-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    # the batched measurement runs up to 64 streams at once: let the runtime give them 32 hardware
    # queues instead of 8 (a property of this process's CUDA context, set before CUDA starts)
    os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--wave", type=int, default=-1, help="droplets per wave; 0 = the reference's chunk; -1 = default")
    ap.add_argument("--precision", default="f64", choices=("f64", "f32"))
    ap.add_argument("--blocks-per-sm", type=int, default=0, help="droplet kernel: 2 selects the two-blocks-per-SM variant")
    ap.add_argument("--apply", default="ordered", choices=("ordered", "wave"),
                    help="ordered: the reference's serial apply (default); wave: per-droplet ledgers against wave-start terrain")
    ap.add_argument("--n", "--nc", dest="n", type=int, default=None,
                    help="override N_c (tests; under torchrun use --nc, which torchrun's own options do not abbreviate)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-alt", action="store_true", help="skip the secondary wave-apply measurement")
    ap.add_argument("--alt-steps", type=int, default=5)
    ap.add_argument("--no-brush", action="store_true", help="skip the brush (radius 3) measurement")
    ap.add_argument("--no-f32", action="store_true", help="skip the float32-trace measurement")
    ap.add_argument("--apply-lanes", type=int, default=0, help="ordered apply: droplets per warp (0 = 1)")
    ap.add_argument("--config", default="c2", choices=("c2", "c5"),
                    help="c2: the Earth-default N_c=1024 line (default); c5: the N_c=8192 planet level on one GPU")
    ap.add_argument("--planet-iterations", type=int, default=0, help="c5: run this many iterations as the timed stage")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-worlds measurement")
    ap.add_argument("--batch-worlds", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=2)
    ap.add_argument("--batch-apply", default="ordered", choices=("ordered", "wave"), help="the batched worlds' apply")
    ap.add_argument("--batch-trace-lanes", type=int, default=32, help="the batched worlds' trace: droplets per warp")
    ap.add_argument("--batch-streams", type=int, default=0, help="the batched worlds' streams (0: one a world)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the calibration (adjoint) measurement")
    ap.add_argument("--adjoint-reps", type=int, default=2)
    ap.add_argument("--adjoint-only", action="store_true", help="run the calibration (adjoint) measurement alone")
    ap.add_argument("--adjoint-n", type=int, default=256, help="calibration world N_c (the workload: 256)")
    ap.add_argument("--adjoint-droplets", type=int, default=1 << 17, help="calibration droplets per iteration (the workload: 2^17)")
    ap.add_argument("--adjoint-iterations", type=int, default=50, help="calibration iterations (the workload: 50)")
    ap.add_argument("--calibrate-steps", type=int, default=0, help="calibration: run this many line-search gradient steps as well")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.wave == -1:
        args.wave = DEFAULT_WAVE
    rank = int(os.environ.get("RANK", 0))
    world_size = int(os.environ.get("WORLD_SIZE", 1))
    dist = None
    if args.impl == "reference":
        out = run_reference(args, rank)
    elif args.config == "c5":
        import torch

        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
        torch.cuda.set_device(dev)
        out = run_planet(args, dev) if rank == 0 else None
    elif args.adjoint_only:
        import torch

        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
        torch.cuda.set_device(dev)
        out = {"adjoint": run_adjoint(args, dev)} if rank == 0 else None
    else:
        if world_size > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        out = run_b200(args, rank, world_size, dist)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


#: droplets per wave of the default run (0 = the reference's chunk of 2048)
DEFAULT_WAVE = 0
#: DRAM bytes of the exact pass (trace, sort, ranks, apply, finish) per droplet-step, caches kept between
#: kernels, and per wave with the caches flushed before every kernel; both from ncu captures of the N_c = 256 pass
TRAFFIC_PER_STEP = 40.0
TRAFFIC_PER_WAVE_COLD = 33.7e6

if __name__ == "__main__":
    main()
