"""Overflowing lakes on the device against the reference (needs a B200).

The kernel side of the lakes (particle.py:186-190, 626-636, 751-763, 952-956,
1010-1012) and the window lake refresh (maps.py:629-673), checked against the
fixtures the reference made (tests/golden/lake_trace.npz: a window with its
lakes, one trace + serial apply; tests/golden/step_lake.npz: sphere steps
with lake flags set by the caller) and against the oracle, which equals both
bit for bit.

Tolerances: the routing flood and the lake flags are integer / comparison
work and must be identical.  The traces are float64 with the reference's
operation order; a trajectory can still end a few ulp apart (libm) and flip
a branch downstream, so at least 99 % of the droplets must keep identical
cell paths and deaths, with deltas / volumes / momenta within 1e-5 relative;
a pass's fields follow the routed pass's bound (at most 0.5 % of values off
1e-5 relative, the worst within 5 % of the field's scale, >= 99 % of heights
bit-identical); steps follow the hypsometry bound of the plain steps.
"""
import ctypes
import json

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from pgerosion import _lib
from pgerosion import maps as gm
from tests.parity_cases import GOLDEN, changelist_rows, hypsometry, lake_case, step_case
from tests.test_gpu_parity import HYPS_TOL_MANY

pytestmark = pytest.mark.gpu


def _gpu_window(case):
    dev = torch.device("cuda")
    f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64), device=dev)
    f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device=dev)
    NE = case["N"] + 2 * case["H"]
    return gm.ErosionState(height=f64(case["height"]), sediment=f64(case["sediment"]), discharge=f64(case["discharge"]),
                           momentum=f64(case["momentum"]), hardness=f32(case["hardness"]), precip=f32(np.ones((1, NE, NE))),
                           evap=f32(case["evap"]), uplift=f64(np.zeros((1, NE, NE))),
                           mask=torch.as_tensor(np.ascontiguousarray(case["mask"], np.uint8), device=dev),
                           metric=f32(case["metric"][0]), metric_inv=f32(case["metric_inv"][0]), N=case["N"], H=case["H"],
                           spherical=False, height_unit_m=case["cell_size_m"], base=f64(case["base"]),
                           deposit_on_exit=bool(case["deposit_on_exit"]))


def _lake_window(case):
    g = _gpu_window(case)
    g.refresh_route(case["eps"])
    info = g.refresh_lakes_window(case["min_depth"])
    return g, info


def test_window_route_and_lake_flags_equal_the_reference(cuda):
    case = lake_case()
    g, info = _lake_window(case)
    assert g.route.cpu().numpy().tobytes() == case["route"].tobytes()
    assert np.array_equal(g.lake_flag.cpu().numpy(), case["lake_flag"])
    assert info["lake_cells"] == int((case["lake_flag"] > 0).sum()) > 10
    # without a route there are no lakes
    g2 = _gpu_window(case)
    assert g2.refresh_lakes_window(case["min_depth"]) == {"lake_cells": 0}
    assert int(g2.lake_flag.sum()) == 0


def test_window_lake_change_lists_match_reference(cuda):
    """The reference's change lists with the lakes packed: crossing entries
    (no exchange on a lake), the shore trap, no pit count on the water."""
    case = lake_case()
    g, _ = _lake_window(case)
    res = gm.trace_changelist(g, case["params"], case["sp_face"], case["sp_x"], case["sp_y"], case["sp_sed"], case["sp_dir"],
                              case["volume0"], case["conc_scale"], precision=_lib.PREC_F64)
    cap = case["cap"]
    lake = case["lake_flag"].reshape(-1) > 0
    same = 0
    crossing = 0
    rows = list(zip(changelist_rows(res, cap), changelist_rows(case, cap)))
    for p, (a, b) in enumerate(rows):
        if res["sp_death"][p] != case["sp_death"][p] or not np.array_equal(a[0], b[0]):
            continue
        crossing += int((lake[a[0]] & (a[1] == 0.0)).sum())
        if np.allclose(a[1], b[1], rtol=1e-5, atol=1e-12) and np.allclose(a[2], b[2], rtol=1e-5, atol=0) and \
                np.allclose(a[3], b[3], rtol=1e-5, atol=1e-7):
            same += 1
    assert same >= 0.99 * len(rows), (same, len(rows))
    assert crossing > 1000


def _oracle_window(case):
    o = case["oracle_state"]()
    orc.refresh_route(o, case["eps"])
    orc.refresh_lakes_window(o, case["min_depth"])
    return o


def _oracle_chunked_pass(o, ep, f, x, y, sed, dirs, v0):
    P = len(f)
    chunk = orc.chunk_size(ep, P)
    o.pack()
    o.acc[...] = 0.0
    tp = orc.trace_params(o, ep, v0, chunk / (v0 * P))
    ap = orc.apply_params(o, ep, ep.iter_deposit / o.height_unit_m)
    cap = orc.change_list_cap(tp.max_steps)
    clamped = 0
    for c0 in range(0, P, chunk):
        sl = slice(c0, c0 + chunk)
        cl = orc.trace(o, tp, f[sl], x[sl], y[sl], sed[sl], dirs[sl], v0)
        clamped += orc.apply(o, ap, cl, cap)[0]
    lib = orc.lib()
    lib.orc_fold(ctypes.c_int64(o.height.size), orc._p(o.height), orc._p(o.sediment), orc._p(o.acc), orc._p(o.mask))
    lib.orc_ema(ctypes.c_int64(o.height.size), orc._p(o.discharge), orc._p(o.momentum), orc._p(o.disch_track), orc._p(o.mom_track),
                orc._p(o.mask), ctypes.c_double(float(ep.ema)))
    return clamped


def _close_fields(a, o, keys=("height", "sediment", "discharge", "momentum", "pending")):
    for k in keys:
        want = getattr(o, k)
        off = ~np.isclose(a[k], want, rtol=1e-5, atol=1e-8)
        worst = np.abs(a[k] - want).max()
        assert off.mean() <= 5e-3 and worst <= 0.05 * max(np.abs(want).max(), 1e-12), (k, int(off.sum()), worst)
    assert np.mean(a["height"] == o.height) > 0.99


def test_window_lake_ordered_pass_matches_oracle(cuda):
    """The lake window's droplets through the ordered apply in the
    reference's chunks against the oracle's chunked serial pass; no lake bed
    is eroded (its floor is the water level, above the bed)."""
    case = lake_case()
    ep = case["params"]
    g, _ = _lake_window(case)
    s0 = (g.height + g.sediment).cpu().numpy()
    f, x, y, sed, dirs, v0 = case["sp_face"], case["sp_x"], case["sp_y"], case["sp_sed"], case["sp_dir"], case["volume0"]
    s = gm.apply_spawns(g, ep, f, x, y, sed, dirs, v0)
    o = _oracle_window(case)
    clamped = _oracle_chunked_pass(o, ep, f, x, y, sed, dirs, v0)
    a = g.to_numpy()
    _close_fields(a, o)
    assert abs(s["clamped"] - clamped) <= 1e-3 * clamped, (s["clamped"], clamped)
    lake = case["lake_flag"] > 0
    s1 = a["height"] + a["sediment"]
    assert (s1[lake] >= s0[lake] - 1e-12).all()
    assert (s1[lake] > s0[lake]).any()  # the shore trap and crossing droplets' loads do reach lake cells


def test_window_lake_wave_pass_keeps_lake_beds_and_mass(cuda):
    """The order-free wave apply with the lakes packed: lake beds are not
    eroded, and the pass balances (change of height + sediment + pending =
    minus what left the window)."""
    case = lake_case()
    ep = case["params"]
    g, _ = _lake_window(case)
    s0 = (g.height + g.sediment).cpu().numpy()
    m0 = g.total_mass()
    f, x, y, sed, dirs, v0 = case["sp_face"], case["sp_x"], case["sp_y"], case["sp_sed"], case["sp_dir"], case["volume0"]
    s = gm.apply_spawns(g, ep, f, x, y, sed, dirs, v0, apply=_lib.APPLY_WAVE)
    a = g.to_numpy()
    lake = case["lake_flag"] > 0
    s1 = a["height"] + a["sediment"]
    assert (s1[lake] >= s0[lake] - 1e-12).all()
    assert s["entries"] > 0
    # the loaded spawns bring their loads in from outside the window's mass
    brought = float(np.sum(sed))
    out = s["lost_offshore"] - s["deficit_out"]  # a deficit left at a list's end is mass the pass creates
    assert abs(s["eroded"] + brought - (s["deposited"] + s["to_pending"] + out)) <= 1e-6 * max(s["eroded"], 1.0), s
    assert abs((g.total_mass() - m0) - brought + out) <= 1e-6 * max(s["eroded"], 1.0), (m0, g.total_mass(), s)


def test_lake_steps_follow_the_reference(cuda):
    """Sphere steps with the reference fixture's lake flags (1 and 2, halos
    from the nearest interior cell) and the routing flood every 2
    iterations: the hypsometry within the chaotic bound of the plain steps,
    and the flags read (a pass without them ends elsewhere)."""
    c = step_case(GOLDEN / "step_lake.npz")
    t = c["t"]
    g = gm.ErosionState.from_world(c["world"])
    gm.start_replay(g, c["params"])
    g.lake_flag = torch.as_tensor(t["lake_flag"], device="cuda")
    for it in range(c["iterations"]):
        gm.step(g, c["params"], it, n_particles=c["n_particles"])
    a = g.to_numpy()
    inter = g.interior
    hg = hypsometry(a["height"], a["sediment"], inter, 50.0)
    hr = hypsometry(t["height"], t["sediment"], inter, 50.0)
    assert np.abs(hg - hr).max() <= HYPS_TOL_MANY, (hg, hr)
    # the same first iteration without lake flags is a different pass
    g1 = gm.ErosionState.from_world(c["world"])
    gm.start_replay(g1, c["params"])
    g1.lake_flag = torch.as_tensor(t["lake_flag"], device="cuda")
    g2 = gm.ErosionState.from_world(c["world"])
    gm.start_replay(g2, c["params"])
    gm.step(g1, c["params"], 0, n_particles=c["n_particles"])
    gm.step(g2, c["params"], 0, n_particles=c["n_particles"])
    assert not np.array_equal(g1.to_numpy()["height"], g2.to_numpy()["height"])


def _balance_world():
    from pgerosion.params import WorldGroup, WorldParams
    from pgerosion.synth import World
    from pgerosion.geometry import get_grid
    from tests.parity_cases import erosion_params
    import json

    fx = np.load(GOLDEN / "lake_balance.npz")
    N, H, cs = int(fx["N"]), int(fx["H"]), float(fx["cell_size_m"])
    ep = erosion_params(str(fx["params"]))
    params = WorldParams(world=WorldGroup(seed=int(fx["seed"]), N_c=N, cell_size_m=cs, land_fraction=float(fx["land_fraction"]),
                                          halo=H), erosion=ep)
    world = World(get_grid(N, H, cs), fx["bedrock"], fx["hardness"], fx["precip"], fx["evap"], fx["uplift"],
                  float(fx["land_fraction"]))
    return fx, params, world, json.loads(str(fx["stats"]))


@pytest.mark.parametrize("tag,land_evap", [("budyko", 3.0), ("plain", 0.0)])
def test_planet_lake_refresh_equals_the_reference(cuda, tag, land_evap):
    """ErosionState.refresh_lakes on the device state (surface and sea mask
    copied off the device, the host balance, flags and closed levels copied
    back with halos from the nearest interior cell): the reference's flags
    and base level, halos included, bit for bit."""
    fx, params, world, _ = _balance_world()
    g = gm.ErosionState.from_world(world)
    g.height.copy_(torch.as_tensor(fx["u_height"]))
    g.sediment.copy_(torch.as_tensor(fx["u_sediment"]))
    mf = float(fx["ocean_min_fraction"])
    g.refresh_base(mf)
    assert np.array_equal(g.sea_mask.cpu().numpy(), fx["u_sea"].reshape(g.sea_mask.shape))
    assert g.base.cpu().numpy().tobytes() == np.ascontiguousarray(fx["u_base"]).tobytes()
    g.refresh_route(float(params.erosion.route_eps) / g.height_unit_m)
    info = g.refresh_lakes(float(fx["lake_evap"]), float(fx["min_depth"]), mf, land_evap)
    want = json.loads(str(fx[f"{tag}_info"]))
    assert {k: info[k] for k in info} == {k: want[k] for k in info}
    assert np.array_equal(g.lake_flag.cpu().numpy(), fx[f"{tag}_flag"])
    assert g.base.cpu().numpy().tobytes() == np.ascontiguousarray(fx[f"{tag}_base"]).tobytes()


def test_planet_lake_steps_follow_the_reference(cuda):
    """maps.step with erosion.lake_balance (lake_fill off), the sea mask and
    the routing flood every 2 iterations: the lakes refreshed on the same
    iterations as the reference's, the hypsometry within the chaotic bound of
    the plain steps, and the mass balance of one more pass with the lakes."""
    from tests.test_gpu_parity import _mass_balance

    fx, params, world, stats = _balance_world()
    g = gm.ErosionState.from_world(world)
    gm.start_replay(g, params)
    got = []
    for it in range(int(fx["iterations"])):
        s = gm.step(g, params, it, n_particles=int(fx["n_particles"]))
        assert ("lakes" in s) == ("lakes" in stats[it]), it
        got.append(s.get("lakes"))
    want = [st.get("lakes") for st in stats]
    # the first refresh sees the same surface as the reference's: the same lakes
    assert got[0] == want[0], (got, want)
    assert all(x is None or x["depressions"] > 0 for x in got), (got, want)
    a = g.to_numpy()
    inter = g.interior
    hg = hypsometry(a["height"], a["sediment"], inter, 50.0)
    hr = hypsometry(fx["height"], fx["sediment"], inter, 50.0)
    assert np.abs(hg - hr).max() <= HYPS_TOL_MANY, (hg, hr)
    m0 = g.total_mass()
    s = gm.run_iteration(g, params, int(fx["iterations"]), n_particles=int(fx["n_particles"]))
    _mass_balance(s, m0, g.total_mass())


def test_basin_fill_equals_the_reference(cuda):
    """maps.fill_basins on the device state from the reference's start (the open
    ocean on the device, the host flood and graded plain of pge_basin_fill,
    the sediment added and the halos exchanged on the device): the
    reference's interior sediment bit for bit, its halos within 1e-12 (the
    halo gather sums in another order), and its statistics."""
    from pgerosion.params import WorldGroup, WorldParams
    from pgerosion.synth import World
    from pgerosion.geometry import get_grid
    from tests.parity_cases import erosion_params

    fx = np.load(GOLDEN / "basin_fill.npz")
    N, H, cs = int(fx["N"]), int(fx["H"]), float(fx["cell_size_m"])
    ep = erosion_params(str(fx["params"]))
    params = WorldParams(world=WorldGroup(seed=int(fx["seed"]), N_c=N, cell_size_m=cs, land_fraction=float(fx["land_fraction"]),
                                          halo=H), erosion=ep)
    world = World(get_grid(N, H, cs), fx["bedrock"], fx["hardness"], fx["precip"], fx["evap"], fx["uplift"],
                  float(fx["land_fraction"]))
    g = gm.ErosionState.from_world(world)
    gm.start_replay(g, params)
    # the reference's start (its replay's datum hold may differ in the last bits: the fill is compared on one surface)
    g.height.copy_(torch.as_tensor(fx["h_start"]))
    g.sediment.copy_(torch.as_tensor(fx["s_start"]))
    info = gm.fill_basins(g, params)
    want = json.loads(str(fx["info"]))
    assert info == want, (info, want)
    a = g.to_numpy()
    inter = g.interior
    assert a["sediment"][inter].tobytes() == np.ascontiguousarray(fx["sediment"][inter]).tobytes()
    np.testing.assert_allclose(a["sediment"], fx["sediment"], rtol=0, atol=1e-12)
    # off, or on a window: nothing
    ep0 = type(ep)(**{**{k: getattr(ep, k) for k in ep.__dataclass_fields__}, "basin_fill_grade": 0.0})
    assert gm.fill_basins(g, WorldParams(world=params.world, erosion=ep0)) is None


@pytest.mark.parametrize("tag", ["a", "b"])
def test_window_lake_balance_on_the_state_equals_the_reference(cuda, tag):
    """ErosionState.refresh_lakes_window with window_lake_evap > 0 on the
    device window state (the routing flood on the device, the balance on the
    host, flags and the lowered route back): the reference's flags, route
    and counts, bit for bit."""
    fx = np.load(GOLDEN / "window_lake_balance.npz")
    N, H = int(fx["N"]), int(fx["H"])
    NE = N + 2 * H
    dev = torch.device("cuda")
    f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64), device=dev)
    f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device=dev)
    from pgerosion.geometry import get_grid

    grid = get_grid(N, H, float(fx["cell_size_m"]))
    g = gm.ErosionState(height=f64(fx["height"]), sediment=f64(fx["sediment"]), discharge=f64(np.zeros((1, NE, NE))),
                        momentum=f64(np.zeros((1, NE, NE, 2))), hardness=f32(np.full((1, NE, NE), 0.5)), precip=f32(fx["precip"]),
                        evap=f32(fx["evap"]), uplift=f64(np.zeros((1, NE, NE))),
                        mask=torch.as_tensor(np.ascontiguousarray(fx["mask"], np.uint8), device=dev),
                        metric=f32(grid.metric_face), metric_inv=f32(grid.metric_inv_face), N=N, H=H, spherical=False,
                        height_unit_m=float(fx["cell_size_m"]), deposit_on_exit=True)
    g.route = f64(fx[f"{tag}_route0"])
    info = g.refresh_lakes_window(float(fx["min_depth"]), float(fx[f"{tag}_lake_evap"]))
    want = json.loads(str(fx[f"{tag}_info"]))
    assert info == want, (info, want)
    assert np.array_equal(g.lake_flag.cpu().numpy(), fx[f"{tag}_flag"])
    assert g.route.cpu().numpy().tobytes() == np.ascontiguousarray(fx[f"{tag}_route"]).tobytes()
