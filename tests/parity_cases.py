"""Parity cases shared by the tests and the smoke check (test infrastructure).

Each case is built from a committed golden fixture (tests/golden/, written
by gen_golden.py from the reference itself) and carries an ``oracle``
callable that recomputes the reference result with the C oracle.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "procedural-generation_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

from pgerosion.geometry import get_grid  # noqa: E402
from pgerosion.params import ErosionParams, WorldGroup, WorldParams  # noqa: E402

GOLDEN = ROOT / "tests" / "golden"


def erosion_params(js: str) -> ErosionParams:
    d = json.loads(js)
    return ErosionParams(**{k: v for k, v in d.items() if k in ErosionParams.__dataclass_fields__})


def isolated_case(path=GOLDEN / "trace_isolated.npz") -> dict:
    """Droplets with pairwise-disjoint paths on an N=48 six-face world."""
    t = np.load(path)
    N, H = int(t["N"]), int(t["H"])
    cs = float(t["cell_size_m"])
    grid = get_grid(N, H, cs)
    ep = erosion_params(str(t["params"]))
    case = {k: t[k] for k in t.files if k not in ("params",)}
    case.update(grid=grid, params=ep, N=N, H=H, cell_size_m=cs, volume0=float(t["volume0"]), conc_scale=float(t["conc_scale"]),
                cap=int(t["cap"]))

    def oracle():
        from oracle import oracle as orc

        F, NE = 6, N + 2 * H
        st = orc.OracleState(height=t["height"].copy(), sediment=t["sediment"].copy(), discharge=t["discharge"].copy(),
                             momentum=t["momentum"].copy(), hardness=t["hardness"], precip=np.ones((F, NE, NE), np.float32),
                             evap=t["evap"], uplift=np.zeros((F, NE, NE)), mask=t["mask"],
                             metric=np.ascontiguousarray(np.broadcast_to(grid.metric_face, (F, NE, NE, 3))),
                             metric_inv=np.ascontiguousarray(np.broadcast_to(grid.metric_inv_face, (F, NE, NE, 3))),
                             N=N, H=H, spherical=True, height_unit_m=cs, grid=grid, base=t["base"].copy())
        st.pack()
        tp = orc.trace_params(st, ep, case["volume0"], case["conc_scale"])
        cl = orc.trace(st, tp, t["sp_face"], t["sp_x"], t["sp_y"], t["sp_sed"], t["sp_dir"], case["volume0"])
        out = orc.apply(st, orc.apply_params(st, ep, ep.iter_deposit / cs), cl, case["cap"])
        names = ("cl_cell", "cl_delta", "cl_vol", "cl_mom", "cl_count", "cl_lo", "cl_hi", "sp_death")
        r = dict(zip(names, cl))
        r.update(acc=st.acc, pending=st.pending, disch_track=st.disch_track, mom_track=st.mom_track, apply_out=np.array(out, float))
        return r

    case["oracle"] = oracle
    return case


def window_case(path=GOLDEN / "window_trace.npz") -> dict:
    """One face of the N=48 world as a window (spherical=False, F = 1; mask:
    active basin, frozen margin, outside ring; deposit_on_exit) with droplets
    that share cells, and the reference's change lists and serial apply
    (``roots_trace.npz``: the same with a roots field)."""
    t = np.load(path)
    N, H = int(t["N"]), int(t["H"])
    cs = float(t["cell_size_m"])
    ep = erosion_params(str(t["params"]))
    case = {k: t[k] for k in t.files if k not in ("params",)}
    case.update(params=ep, N=N, H=H, cell_size_m=cs, volume0=float(t["volume0"]), conc_scale=float(t["conc_scale"]),
                cap=int(t["cap"]))

    def oracle():
        from oracle import oracle as orc

        NE = N + 2 * H
        st = orc.OracleState(height=t["height"].copy(), sediment=t["sediment"].copy(), discharge=t["discharge"].copy(),
                             momentum=t["momentum"].copy(), hardness=t["hardness"], precip=np.ones((1, NE, NE), np.float32),
                             evap=t["evap"], uplift=np.zeros((1, NE, NE)), mask=t["mask"], metric=t["metric"],
                             metric_inv=t["metric_inv"], N=N, H=H, spherical=False, height_unit_m=cs, base=t["base"].copy(),
                             deposit_on_exit=bool(t["deposit_on_exit"]))
        if "roots" in t.files:
            st.roots = np.ascontiguousarray(t["roots"], np.float32)
        if "lake_id" in t.files:  # the lake parks' window: route, lakes with room, their ids and rooms
            st.route = t["route"].copy()
            st.lake_flag = t["lake_flag"].copy()
            st.lake_load = np.zeros_like(st.height)
            st.lake_id = np.ascontiguousarray(t["lake_id"], np.int32)
            st.lake_room = t["lake_room"].copy()
        st.pack()
        tp = orc.trace_params(st, ep, case["volume0"], case["conc_scale"])
        if "lake_id" in t.files:
            tp.lake_park = 1.0
        cl = orc.trace(st, tp, t["sp_face"], t["sp_x"], t["sp_y"], t["sp_sed"], t["sp_dir"], case["volume0"])
        out = orc.apply(st, orc.apply_params(st, ep, ep.iter_deposit / cs), cl, case["cap"])
        names = ("cl_cell", "cl_delta", "cl_vol", "cl_mom", "cl_count", "cl_lo", "cl_hi", "sp_death")
        r = dict(zip(names, cl))
        r.update(acc=st.acc, pending=st.pending, disch_track=st.disch_track, mom_track=st.mom_track, apply_out=np.array(out, float))
        if "lake_id" in t.files:
            r.update(lake_load=st.lake_load, room_after=st.lake_room)
        return r

    case["oracle"] = oracle
    return case


def lake_case(path=GOLDEN / "lake_trace.npz") -> dict:
    """The window of window_case with the routing surface and the lakes of
    the reference's refresh_lakes_window packed, droplets spawned on the
    lakes too, and the reference's change lists and serial apply."""
    t = np.load(path)
    N, H = int(t["N"]), int(t["H"])
    cs = float(t["cell_size_m"])
    ep = erosion_params(str(t["params"]))
    case = {k: t[k] for k in t.files if k not in ("params",)}
    case.update(params=ep, N=N, H=H, cell_size_m=cs, volume0=float(t["volume0"]), conc_scale=float(t["conc_scale"]),
                cap=int(t["cap"]), eps=float(t["eps"]), min_depth=float(t["min_depth"]))

    def oracle_state():
        from oracle import oracle as orc

        NE = N + 2 * H
        return orc.OracleState(height=t["height"].copy(), sediment=t["sediment"].copy(), discharge=t["discharge"].copy(),
                               momentum=t["momentum"].copy(), hardness=t["hardness"], precip=np.ones((1, NE, NE), np.float32),
                               evap=t["evap"], uplift=np.zeros((1, NE, NE)), mask=t["mask"], metric=t["metric"],
                               metric_inv=t["metric_inv"], N=N, H=H, spherical=False, height_unit_m=cs, base=t["base"].copy(),
                               deposit_on_exit=bool(t["deposit_on_exit"]))

    def oracle():
        from oracle import oracle as orc

        st = oracle_state()
        orc.refresh_route(st, case["eps"])
        lakes = orc.refresh_lakes_window(st, case["min_depth"])
        st.pack()
        tp = orc.trace_params(st, ep, case["volume0"], case["conc_scale"])
        cl = orc.trace(st, tp, t["sp_face"], t["sp_x"], t["sp_y"], t["sp_sed"], t["sp_dir"], case["volume0"])
        out = orc.apply(st, orc.apply_params(st, ep, ep.iter_deposit / cs), cl, case["cap"])
        names = ("cl_cell", "cl_delta", "cl_vol", "cl_mom", "cl_count", "cl_lo", "cl_hi", "sp_death")
        r = dict(zip(names, cl))
        r.update(acc=st.acc, pending=st.pending, disch_track=st.disch_track, mom_track=st.mom_track, apply_out=np.array(out, float),
                 route=st.route, lake_flag=st.lake_flag, rflag_after=st.samp[..., orc.S_RFLAG].copy(), lakes=lakes)
        return r

    case["oracle"] = oracle
    case["oracle_state"] = oracle_state
    return case


def step_case(path=GOLDEN / "step_tiny.npz") -> dict:
    """A six-face N=32 world and the reference's state after a few steps."""
    from pgerosion.synth import World

    t = np.load(path)
    N, H, cs = int(t["N"]), int(t["H"]), float(t["cell_size_m"])
    ep = erosion_params(str(t["params"]))
    params = WorldParams(world=WorldGroup(seed=int(t["seed"]), N_c=N, cell_size_m=cs, land_fraction=float(t["land_fraction"]),
                                          halo=H), erosion=ep)
    world = World(get_grid(N, H, cs), t["bedrock"], t["hardness"], t["precip"], t["evap"], t["uplift"], float(t["land_fraction"]))
    return {"t": t, "params": params, "world": world, "iterations": int(t["iterations"]), "n_particles": int(t["n_particles"]),
            "stats": json.loads(str(t["stats"]))}


def changelist_rows(res: dict, cap: int):
    """Per-droplet (cells, deltas, vols, moms) lists of a change list."""
    cnt = res["cl_count"]
    rows = []
    for p in range(cnt.size):
        sl = slice(p * cap, p * cap + int(cnt[p]))
        rows.append((res["cl_cell"][sl], res["cl_delta"][sl], res["cl_vol"][sl], np.asarray(res["cl_mom"]).reshape(-1, 2)[sl]))
    return rows


def hypsometry(height, sediment, interior, unit, pct=(1, 5, 10, 25, 50, 75, 90, 95, 99)):
    """Cell-count percentiles (metres) of the interior surface."""
    s = (np.asarray(height) + np.asarray(sediment))[interior] * unit
    return np.percentile(s, pct)


def window_world(kind: str, N: int = 48, H: int = 2, cell: float = 50.0, seed: int = 0, writeoff: float | None = None):
    """Single-face windows (spherical=False, deposit_on_exit) for the
    reference's conservation tests (bake/tests/test_erosion.py:191-289):
    ``closed`` -- a bowl above sea level, nothing can leave as ocean deposit;
    ``tilt`` -- a plane tilted into the sea, an open coast; ``shelf`` -- land
    sloping to a seafloor one ``dep_floor_m`` below the waterline, walled off
    at the far edge, so every load that reaches the sea is surplus.
    Returns the window arrays (cell units) and WorldParams."""
    from pgerosion.params import ErosionParams, WorldGroup, WorldParams, plain_knobs

    NE = N + 2 * H
    g = get_grid(N, H, cell)
    i, j = np.meshgrid(np.arange(NE), np.arange(NE), indexing="ij")
    u = (i - H + 0.5) / N
    v = (j - H + 0.5) / N
    rough = 2.0 * np.random.default_rng(seed).standard_normal((NE, NE))
    if kind == "closed":
        bed = 60.0 + 400.0 * ((u - 0.5) ** 2 + (v - 0.5) ** 2) + rough
    elif kind == "tilt":
        bed = 80.0 * (0.55 - u) + 8.0 * np.sin(6.0 * v) + rough
    elif kind == "shelf":
        bed = np.where(u < 0.6, 60.0 * (0.6 - u) + 1.0 + np.abs(rough), -0.9)
        bed = np.where(u >= 0.9, 300.0, bed)
    else:
        raise KeyError(kind)
    mask = np.zeros((1, NE, NE), np.uint8)
    mask[0, H:H + N, H:H + N] = 1
    ep = ErosionParams(iterations=40, max_steps=64, friction=0.05, erodibility=0.3, deposition_rate=0.3, evap_rate=0.01,
                       uplift_mode="stack", particles_per_cell=1.0, **plain_knobs())
    if writeoff is not None:
        ep.offshore_writeoff = float(writeoff)
    p = WorldParams(world=WorldGroup(seed=seed, N_c=N, cell_size_m=cell, land_fraction=0.5, halo=H), erosion=ep)
    arr = dict(height=(bed / cell)[None].astype(np.float64), mask=mask, metric=np.ascontiguousarray(g.metric_face[None]),
               metric_inv=np.ascontiguousarray(g.metric_inv_face[None]), N=N, H=H, cell=cell)
    return arr, p


def gpu_window(arr):
    """A device ErosionState of ``window_world``'s arrays."""
    import torch

    from pgerosion import maps as gm

    dev = torch.device("cuda")
    sh = arr["height"].shape
    f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64), device=dev)
    f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device=dev)
    return gm.ErosionState(height=f64(arr["height"]), sediment=f64(np.zeros(sh)), discharge=f64(np.zeros(sh)),
                           momentum=f64(np.zeros(sh + (2,))), hardness=f32(np.full(sh, 0.5)), precip=f32(np.ones(sh)),
                           evap=f32(np.ones(sh)), uplift=f64(np.zeros(sh)),
                           mask=torch.as_tensor(arr["mask"], device=dev), metric=f32(arr["metric"][0]),
                           metric_inv=f32(arr["metric_inv"][0]), N=arr["N"], H=arr["H"], spherical=False,
                           height_unit_m=arr["cell"], deposit_on_exit=True)

