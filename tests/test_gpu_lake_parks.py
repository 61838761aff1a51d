"""The lake parks (erosion.lake_fill) on the device against the reference (needs a B200).

* tests/golden/lake_parks.npz (made by the reference's trace_particles with
  lake_park on and one serial apply_changes, on a window whose lakes are all
  flagged as having room, with small rooms so that the countdown refuses
  loads): the change lists with their park entries (volume -3 on the lake
  cell entered), then one exact pass of the same droplets -- the rooms
  counted down in droplet order, the loads the lakes took, the refused rest
  joining each droplet's stockpile -- against the reference's accumulators.
* tests/golden/lake_fill_steps.npz (the reference's maps.step with
  lake_balance and lake_fill on the six-face N=32 world): steps with the
  parks and the host settle at every refresh; the first refresh is the
  reference's, the hypsometry within the chaotic bound of the plain steps,
  and one more pass balances its mass with the parked loads counted.

Tolerances: the change lists as the other window traces (>= 99 % of droplets
with identical cell paths and deaths, values within 1e-5 relative); the park
countdown and the loads the lakes take are float64 sums in the serial order,
identical where the traces are.
"""
import numpy as np
import pytest
import torch

from pgerosion import _lib
from pgerosion import maps as gm
from tests.parity_cases import GOLDEN, changelist_rows, hypsometry, window_case
from tests.test_gpu_lakes import _gpu_window
from tests.test_gpu_parity import HYPS_TOL_MANY, _mass_balance

pytestmark = pytest.mark.gpu


def _park_window(case):
    g = _gpu_window(case)
    dev = g.height.device
    g.route = torch.as_tensor(np.ascontiguousarray(case["route"], np.float64), device=dev)
    g.lake_flag = torch.as_tensor(np.ascontiguousarray(case["lake_flag"], np.uint8), device=dev)
    g.lake_id = torch.as_tensor(np.ascontiguousarray(case["lake_id"], np.int32), device=dev)
    g.lake_room = torch.as_tensor(np.ascontiguousarray(case["lake_room"], np.float64), device=dev)
    g.lake_load = torch.zeros_like(g.height)
    return g


def test_lake_park_change_lists_match_reference(cuda):
    case = window_case(GOLDEN / "lake_parks.npz")
    g = _park_window(case)
    res = gm.trace_changelist(g, case["params"], case["sp_face"], case["sp_x"], case["sp_y"], case["sp_sed"], case["sp_dir"],
                              case["volume0"], case["conc_scale"], precision=_lib.PREC_F64, parks=True)
    cap = case["cap"]
    rows = list(zip(changelist_rows(res, cap), changelist_rows(case, cap)))
    same, parks = 0, 0
    for p, (a, b) in enumerate(rows):
        if res["sp_death"][p] != case["sp_death"][p] or not np.array_equal(a[0], b[0]) or not np.array_equal(a[2] == -3.0, b[2] == -3.0):
            continue
        parks += int((a[2] == -3.0).sum())
        if np.allclose(a[1], b[1], rtol=1e-5, atol=1e-12) and np.allclose(a[2], b[2], rtol=1e-5, atol=0) and \
                np.allclose(a[3], b[3], rtol=1e-5, atol=1e-7):
            same += 1
    want_parks = int((case["cl_vol"] == -3.0).sum())
    print(f"{same} of {len(rows)} droplets identical; park entries {parks} of the reference's {want_parks}")
    assert same >= 0.99 * len(rows), (same, len(rows))
    assert parks >= 0.98 * want_parks and want_parks > 50
    # the hook records the lists only: nothing applied
    assert np.abs(res["acc"]).max() == 0.0


def test_lake_park_ordered_pass_matches_reference(cuda):
    """One exact pass of the fixture's droplets as one wave (the reference's
    single trace and serial apply): the rooms run out (every lake at 0, as
    the reference's), the loads each lake cell took, the stockpiles (the
    refused rest included) and the terrain change equal the reference's."""
    case = window_case(GOLDEN / "lake_parks.npz")
    ep = case["params"]
    g = _park_window(case)
    s0 = (g.height + g.sediment).cpu().numpy()
    P = len(case["sp_face"])
    s = gm.apply_spawns(g, ep, case["sp_face"], case["sp_x"], case["sp_y"], case["sp_sed"], case["sp_dir"], case["volume0"],
                        wave=P, parks=True, conc_scale=case["conc_scale"])
    load = g.lake_load.cpu().numpy()
    room = g.lake_room.cpu().numpy()
    a = g.to_numpy()
    want_load = case["lake_load"]
    same_load = float(np.mean(load[want_load > 0] == want_load[want_load > 0]))
    print(f"park cells {int((want_load > 0).sum())}, bit-identical loads {same_load:.4%}; parked {load.sum():.6f} vs "
          f"{want_load.sum():.6f}; clamped {s['clamped']} vs {int(case['apply_out'][0])}")
    assert np.array_equal(room, case["room_after"]) and (room == 0.0).all()
    np.testing.assert_allclose(load, want_load, rtol=1e-6, atol=1e-12)
    assert same_load >= 0.95
    np.testing.assert_allclose(a["pending"], case["pending"], rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose((a["height"] + a["sediment"]) - s0, case["acc"], rtol=1e-5, atol=1e-9)
    assert abs(s["to_pending"] - case["apply_out"][1]) <= 1e-6 * max(case["apply_out"][1], 1e-12)


def _fill_world():
    import json

    from pgerosion.geometry import get_grid
    from pgerosion.params import WorldGroup, WorldParams
    from pgerosion.synth import World
    from tests.parity_cases import erosion_params

    fx = np.load(GOLDEN / "lake_fill_steps.npz")
    N, H, cs = int(fx["N"]), int(fx["H"]), float(fx["cell_size_m"])
    params = WorldParams(world=WorldGroup(seed=int(fx["seed"]), N_c=N, cell_size_m=cs, land_fraction=float(fx["land_fraction"]),
                                          halo=H), erosion=erosion_params(str(fx["params"])))
    world = World(get_grid(N, H, cs), fx["bedrock"], fx["hardness"], fx["precip"], fx["evap"], fx["uplift"],
                  float(fx["land_fraction"]))
    return fx, params, world, json.loads(str(fx["stats"]))


def test_lake_fill_steps_follow_the_reference(cuda):
    fx, params, world, stats = _fill_world()
    assert gm.lake_fill_args(gm.ErosionState.from_world(world), params) is not None
    g = gm.ErosionState.from_world(world)
    gm.start_replay(g, params)
    got, parked = [], 0.0
    for it in range(int(fx["iterations"])):
        s = gm.step(g, params, it, n_particles=int(fx["n_particles"]))
        assert ("lakes" in s) == ("lakes" in stats[it]), it
        got.append(s.get("lakes"))
        parked += s.get("parked", 0.0)
    want = [st.get("lakes") for st in stats]
    print("lakes", got, "\nreference", want, "\nparked by the passes", parked)
    # the first refresh sees the reference's surface: the same lakes, nothing parked yet
    assert {k: got[0][k] for k in ("lake_cells", "lake_cells_closed", "depressions", "overflowing", "closed", "dry")} == \
        {k: want[0][k] for k in ("lake_cells", "lake_cells_closed", "depressions", "overflowing", "closed", "dry")}
    assert got[0]["load_lakes"] == want[0]["load_lakes"] and got[0]["load_parked"] == 0.0
    assert parked > 0.0 and any(x is not None and x["load_laid"] > 0.0 for x in got[1:])
    a = g.to_numpy()
    inter = g.interior
    hg = hypsometry(a["height"], a["sediment"], inter, 50.0)
    hr = hypsometry(fx["height"], fx["sediment"], inter, 50.0)
    assert np.abs(hg - hr).max() <= HYPS_TOL_MANY, (hg, hr)
    m0 = g.total_mass()
    s = gm.run_iteration(g, params, int(fx["iterations"]), n_particles=int(fx["n_particles"]))
    _mass_balance(s, m0, g.total_mass())


def test_lake_parks_need_the_exact_apply(cuda):
    fx, params, world, _ = _fill_world()
    g = gm.ErosionState.from_world(world)
    gm.start_replay(g, params)
    gm.step(g, params, 0, n_particles=1024)  # the lakes of the first refresh
    with pytest.raises(_lib.PgeError, match="ordered apply only"):
        gm.run_iteration(g, params, 1, n_particles=1024, apply=_lib.APPLY_WAVE)
