"""The CPU oracle against the reference's own outputs (golden fixtures
written by tests/golden/gen_golden.py from the bake's numba code)."""
import hashlib
import json

import numpy as np
import pytest

from oracle import oracle as orc
from tests.parity_cases import GOLDEN, changelist_rows, isolated_case, lake_case, step_case, window_case


def test_cubesphere_vectors_bit_exact():
    g = np.load(GOLDEN / "cubesphere_vectors.npz")
    assert np.array_equal(orc.to_sphere(g["face"], g["u"], g["v"]), g["xyz"])
    f2, u2, v2 = orc.from_sphere(g["xyz"])
    assert np.array_equal(f2, g["face2"]) and np.array_equal(u2, g["u2"]) and np.array_equal(v2, g["v2"])
    tf, tu, tv, ta, tb = orc.transfer_velocity(g["t_face"], g["t_u"], g["t_v"], g["t_a"], g["t_b"])
    assert np.array_equal(tf, g["t_face2"])
    assert np.array_equal(np.stack([tu, tv, ta, tb], 1), g["t_out"])


def test_reference_vector_file_if_present():
    """The bake's own checked-in vector file (tests/data/cubesphere_vectors.bin),
    read when the environment variable PGE_BAKE_DIR names a bake checkout."""
    import os
    import struct
    from pathlib import Path

    bake = os.environ.get("PGE_BAKE_DIR")
    if not bake:
        pytest.skip("PGE_BAKE_DIR not set (a bake checkout with tests/data/cubesphere_vectors.bin)")
    path = Path(bake) / "tests" / "data" / "cubesphere_vectors.bin"
    if not path.exists():
        pytest.skip(f"{path} not found")
    rec_t = np.dtype([("face", "<i4"), ("u", "<f8"), ("v", "<f8"), ("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("face2", "<i4"),
                      ("u2", "<f8"), ("v2", "<f8")])
    with open(path, "rb") as fh:
        assert fh.read(4) == b"CSV2"
        (K,) = struct.unpack("<i", fh.read(4))
        rec = np.frombuffer(fh.read(), dtype=rec_t)
    assert rec.shape[0] == K
    xyz = orc.to_sphere(rec["face"], rec["u"], rec["v"])
    assert np.array_equal(xyz, np.stack([rec["x"], rec["y"], rec["z"]], 1))
    f2, u2, v2 = orc.from_sphere(xyz)
    assert np.array_equal(f2, rec["face2"]) and np.array_equal(u2, rec["u2"]) and np.array_equal(v2, rec["v2"])


def test_trace_and_apply_match_reference_bit_exact():
    case = isolated_case()
    res = case["oracle"]()
    cap = case["cap"]
    for k in ("cl_count", "cl_lo", "cl_hi", "sp_death"):
        assert np.array_equal(res[k], case[k]), k
    for a, b in zip(changelist_rows(res, cap), changelist_rows(case, cap)):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    for k in ("acc", "pending", "disch_track", "mom_track"):
        assert np.array_equal(res[k], case[k]), k
    assert np.array_equal(res["apply_out"], case["apply_out"])


def test_window_trace_and_serial_apply_match_reference_bit_exact():
    """Window mode (spherical=False, F = 1, outside / frozen / active masks,
    deposit_on_exit) with droplets sharing cells: the oracle's trace and
    serial apply equal the reference's bit for bit."""
    case = window_case()
    res = case["oracle"]()
    cap = case["cap"]
    for k in ("cl_count", "cl_lo", "cl_hi", "sp_death"):
        assert np.array_equal(res[k], case[k]), k
    assert (case["sp_death"] == orc.DEATH_NAMES.index("exit")).sum() > 10  # droplets do leave the window
    for a, b in zip(changelist_rows(res, cap), changelist_rows(case, cap)):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    for k in ("acc", "pending", "disch_track", "mom_track"):
        assert np.array_equal(res[k], case[k]), k
    assert np.array_equal(res["apply_out"], case["apply_out"])


def test_full_steps_match_reference_bit_exact():
    c = step_case()
    t = c["t"]
    st = orc.OracleState.from_world(c["world"], c["params"])
    orc.start_replay(st, c["params"])
    assert np.array_equal(st.height, t["h_start"])
    for it in range(c["iterations"]):
        s = orc.step(st, c["params"], it, n_particles=c["n_particles"])
        r = c["stats"][it]
        for k in ("particles", "entries", "clamped", "deaths"):
            assert s[k] == r[k], (it, k)
        assert s["datum_shift"] == r["datum_shift"]
        assert s["lost_offshore"] == r["lost_offshore"]
    for k in ("height", "sediment", "discharge", "momentum", "pending"):
        assert np.array_equal(getattr(st, k), t[k]), k


def test_oracle_conserves_mass_in_a_particle_pass():
    """Delta (h + s + pending) over the active interior = deficit_out - lost_offshore (a deficit left at a
    list's end is erosion the droplet carried but the terrain could not give, particle.py:964-966, 1043)."""
    c = step_case()
    st = orc.OracleState.from_world(c["world"], c["params"])
    for it in range(3):
        m0 = st.total_mass()
        s = orc.run_iteration(st, c["params"], it, n_particles=2048)
        m1 = st.total_mass()
        assert abs((m1 - m0) + s["lost_offshore"] - s["deficit_out"]) <= 1e-9 * max(abs(m0), 1.0), it
        orc.thermal_erosion(st, c["params"])
        orc.apply_uplift(st)
        orc.hold_datum(st, st.land_target)
        st.exchange_halos()


def test_isostasy_steps_match_reference_bit_exact():
    """Four reference steps with isostasy on (0.8, every 2 iterations): the
    oracle's step bound, its isostasy statistics and the final state are
    the reference's, bit for bit."""
    c = step_case(GOLDEN / "isostasy_tiny.npz")
    t = c["t"]
    st = orc.OracleState.from_world(c["world"], c["params"])
    orc.start_replay(st, c["params"])
    assert orc.smoothing_kappa(st) == float(t["kappa"])
    for it in range(c["iterations"]):
        s = orc.step(st, c["params"], it, n_particles=c["n_particles"])
        r = c["stats"][it]
        assert s["entries"] == r["entries"] and s["clamped"] == r["clamped"], it
        assert ("isostasy" in s) == ("isostasy" in r), it
        if "isostasy" in r:
            for k, v in r["isostasy"].items():
                assert s["isostasy"][k] == v, (it, k)
        assert s["datum_shift"] == r["datum_shift"], it
    for k in ("height", "sediment", "discharge", "momentum", "pending"):
        assert np.array_equal(getattr(st, k), t[k]), k


def test_route_flood_matches_reference_bit_exact():
    """The oracle's heap flood against the reference's (route.py:31-125),
    on the sphere (with a basin that has its own base level) and on a window."""
    fx = np.load(GOLDEN / "route_flood.npz")
    surf = fx["height"] + fx["sediment"]
    got = orc.priority_flood_eps(surf, fx["mask"], fx["owner"], int(fx["H"]), int(fx["N"]), float(fx["eps"]), fx["base"])
    assert got.tobytes() == fx["route"].tobytes()
    wsurf = fx["w_height"] + fx["w_sediment"]
    got = orc.priority_flood_eps(wsurf, fx["w_mask"], fx["w_owner"], int(fx["H"]), int(fx["N"]), float(fx["eps"]), np.zeros_like(wsurf))
    assert got.tobytes() == fx["w_route"].tobytes()


def test_routed_steps_match_reference_bit_exact():
    """Full steps with the routing surface on (erosion.flood_every = 2: the
    flood refreshed before iterations 0, 2 and 4, particles steering on it,
    maps.py:1553-1554 and particle.py:453-460, 556-559)."""
    c = step_case(GOLDEN / "step_route.npz")
    t = c["t"]
    st = orc.OracleState.from_world(c["world"], c["params"])
    orc.start_replay(st, c["params"])
    assert np.array_equal(st.height, t["h_start"])
    for it in range(c["iterations"]):
        s = orc.step(st, c["params"], it, n_particles=c["n_particles"])
        r = c["stats"][it]
        for k in ("particles", "entries", "clamped", "deaths"):
            assert s[k] == r[k], (it, k)
        assert s["datum_shift"] == r["datum_shift"]
    for k in ("height", "sediment", "discharge", "momentum", "pending"):
        assert np.array_equal(getattr(st, k), t[k]), k
    # the route's interior bit for bit; its halos come from the linear halo gather, summed in another order (1 ulp)
    inter = (slice(None), slice(st.H, st.H + st.N), slice(st.H, st.H + st.N))
    assert np.array_equal(st.route[inter], t["route"][inter])
    np.testing.assert_allclose(st.route, t["route"], rtol=0, atol=1e-12)


def test_sea_mask_matches_reference_bit_exact():
    """The oracle's sea mask (maps.py:360-420, hydro/run.py:64-83) on the
    reference fixture's world, and full steps with the sea mask and the
    routing flood on (sea_mask_every = flood_every = 2)."""
    c = step_case(GOLDEN / "step_sea.npz")
    t = c["t"]
    st = orc.OracleState.from_world(c["world"], c["params"])
    st.height[...] = t["b_height"]
    st.sediment[...] = t["b_sediment"]
    info = orc.refresh_base(st, float(t["ocean_min_fraction"]))
    assert info == json.loads(str(t["b_info"]))
    assert info["closed_basins"] > 0
    assert np.array_equal(st.base, t["b_base"])
    st = orc.OracleState.from_world(c["world"], c["params"])
    orc.refresh_base(st, float(t["ocean_min_fraction"]))
    orc.start_replay(st, c["params"])
    assert np.array_equal(st.height, t["h_start"])
    for it in range(c["iterations"]):
        s = orc.step(st, c["params"], it, n_particles=c["n_particles"])
        r = c["stats"][it]
        for k in ("particles", "entries", "clamped", "deaths", "datum_shift"):
            assert s[k] == r[k], (it, k)
        assert s.get("sea") == r.get("sea"), it
    for k in ("height", "sediment", "discharge", "momentum", "pending", "base"):
        assert np.array_equal(getattr(st, k), t[k]), k


def test_glacial_steps_match_reference_bit_exact():
    """Steps with the glacial pass on (erosion/glacial.py: every 2 iterations
    on a world frozen poleward of 50 degrees): its statistics and the state."""
    c = step_case(GOLDEN / "step_glacial.npz")
    t = c["t"]
    st = orc.OracleState.from_world(c["world"], c["params"])
    orc.start_replay(st, c["params"])
    assert np.array_equal(st.height, t["h_start"])
    n_carves = 0
    for it in range(c["iterations"]):
        s = orc.step(st, c["params"], it, n_particles=c["n_particles"])
        r = c["stats"][it]
        for k in ("particles", "entries", "clamped", "deaths", "datum_shift"):
            assert s[k] == r[k], (it, k)
        assert s.get("glacial") == r.get("glacial"), it
        n_carves += "glacial" in s
    assert n_carves == 2
    inter = st.interior
    for k in ("height", "sediment", "discharge", "momentum"):
        assert np.array_equal(getattr(st, k), t[k]), k
    assert np.array_equal(st.pending[inter], t["pending"][inter])


def test_window_lakes_trace_and_apply_match_reference_bit_exact():
    """Lakes on a window (erosion.window_lakes, maps.py:629-673): the
    oracle's routing flood and lake flags equal the reference's, and with
    them packed (flag 2 on a lake) the trace and serial apply equal the
    reference's bit for bit: no exchange while crossing a lake, the load
    dropped at the shore, no pit count on the water, the bed never eroded
    below the water level, lake flags kept by the apply."""
    case = lake_case()
    res = case["oracle"]()
    assert res["route"].tobytes() == case["route"].tobytes()
    assert np.array_equal(res["lake_flag"], case["lake_flag"])
    assert res["lakes"]["lake_cells"] > 10
    cap = case["cap"]
    for k in ("cl_count", "cl_lo", "cl_hi", "sp_death"):
        assert np.array_equal(res[k], case[k]), k
    rows_ref = changelist_rows(case, cap)
    for a, b in zip(changelist_rows(res, cap), rows_ref):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    # the lake branches are exercised: entries with no exchange on lake cells
    lake = case["lake_flag"].reshape(-1) > 0
    crossing = sum(int(((lake[c]) & (d == 0.0)).sum()) for c, d, _, _ in rows_ref)
    assert crossing > 1000
    for k in ("acc", "pending", "disch_track", "mom_track", "rflag_after"):
        assert np.array_equal(res[k], case[k]), k
    assert np.array_equal(res["apply_out"], case["apply_out"])


def test_lake_flag_changes_the_pass():
    """Planting mistakes in the oracle shows the fixture can tell: without
    the lake flags, or with another shore trap, the change lists differ."""
    case = lake_case()
    from oracle import oracle as orc

    def run(flags, trap):
        st = case["oracle_state"]()
        orc.refresh_route(st, case["eps"])
        st.lake_flag = flags
        st.pack()
        ep = case["params"]
        ep_t = type(ep)(**{**{k: getattr(ep, k) for k in ep.__dataclass_fields__}, "lake_trap": trap})
        tp = orc.trace_params(st, ep_t, case["volume0"], case["conc_scale"])
        return orc.trace(st, tp, case["sp_face"], case["sp_x"], case["sp_y"], case["sp_sed"], case["sp_dir"], case["volume0"])

    ep = case["params"]
    base = run(case["lake_flag"], float(ep.lake_trap))
    assert np.array_equal(base[1], case["cl_delta"])
    assert not np.array_equal(run(None, float(ep.lake_trap))[1], case["cl_delta"])
    assert not np.array_equal(run(case["lake_flag"], 0.5)[1], case["cl_delta"])


def test_lake_steps_match_reference_bit_exact():
    """Full steps on the sphere with caller-set lake flags (1 and 2, halos
    from the nearest interior cell) and the routing flood every 2
    iterations: the oracle's state equals the reference's bit for bit."""
    c = step_case(GOLDEN / "step_lake.npz")
    t = c["t"]
    st = orc.OracleState.from_world(c["world"], c["params"])
    orc.start_replay(st, c["params"])
    assert np.array_equal(st.height, t["h_start"])
    st.lake_flag = t["lake_flag"].copy()
    for it in range(c["iterations"]):
        s = orc.step(st, c["params"], it, n_particles=c["n_particles"])
        r = c["stats"][it]
        for k in ("particles", "entries", "clamped", "deaths"):
            assert s[k] == r[k], (it, k)
        assert s["datum_shift"] == r["datum_shift"]
    for k in ("height", "sediment", "discharge", "momentum", "pending"):
        assert np.array_equal(getattr(st, k), t[k]), k
    inter = (slice(None), slice(st.H, st.H + st.N), slice(st.H, st.H + st.N))
    assert np.array_equal(st.route[inter], t["route"][inter])


def test_roots_trace_and_serial_apply_match_reference_bit_exact():
    """Roots (erosion.vegetation: the exchange on land scaled by 1 - roots,
    particle.py:615-618) on the window: the oracle's trace and serial apply
    equal the reference's bit for bit, and the roots change the pass."""
    case = window_case(GOLDEN / "roots_trace.npz")
    res = case["oracle"]()
    cap = case["cap"]
    for k in ("cl_count", "cl_lo", "cl_hi", "sp_death"):
        assert np.array_equal(res[k], case[k]), k
    for a, b in zip(changelist_rows(res, cap), changelist_rows(case, cap)):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    for k in ("acc", "pending", "disch_track", "mom_track"):
        assert np.array_equal(res[k], case[k]), k
    assert np.array_equal(res["apply_out"], case["apply_out"])
    bare = window_case(GOLDEN / "window_trace.npz")
    assert not np.array_equal(case["cl_delta"][:1000], bare["cl_delta"][:1000])


def _window_steps_state(t, ep):
    NE = int(t["N"]) + 2 * int(t["H"])
    st = orc.OracleState(height=t["start_height"].copy(), sediment=t["start_sediment"].copy(),
                         discharge=t["start_discharge"].copy(), momentum=t["start_momentum"].copy(), hardness=t["hardness"],
                         precip=t["precip"], evap=t["evap"], uplift=np.zeros((1, NE, NE)), mask=t["mask"], metric=t["metric"],
                         metric_inv=t["metric_inv"], N=int(t["N"]), H=int(t["H"]), spherical=False,
                         height_unit_m=float(t["cell_size_m"]), base=t["base"].copy(), deposit_on_exit=True)
    st.inflow_volume = float(t["inflow_volume"])
    return st


def test_window_steps_with_inflow_match_reference_bit_exact():
    """Full steps on a window (maps.step, spherical=False: masks, deposit on
    exit, no halo exchange or datum hold) with the cell-count discharge
    scales on and part of the spawn weight declared as inflow across the
    window's edge (maps.py:913-917): the oracle's state equals the
    reference's bit for bit, and the inflow changes the run."""
    from tests.parity_cases import erosion_params

    from pgerosion.params import WorldGroup, WorldParams

    t = np.load(GOLDEN / "window_steps.npz")
    ep = erosion_params(str(t["params"]))
    params = WorldParams(world=WorldGroup(seed=int(t["seed"]), N_c=int(t["N"]), cell_size_m=float(t["cell_size_m"]),
                                          land_fraction=float(t["land_fraction"]), halo=int(t["H"])), erosion=ep)
    st = _window_steps_state(t, ep)
    stats = json.loads(str(t["stats"]))
    for it in range(int(t["iterations"])):
        s = orc.step(st, params, it, n_particles=int(t["n_particles"]))
        for k in ("particles", "entries", "clamped", "deaths"):
            assert s[k] == stats[it][k], (it, k)
    for k in ("height", "sediment", "discharge", "momentum", "pending"):
        assert np.array_equal(getattr(st, k), t[k]), k
    st2 = _window_steps_state(t, ep)
    st2.inflow_volume = 0.0
    orc.step(st2, params, 0, n_particles=int(t["n_particles"]))
    st1 = _window_steps_state(t, ep)
    orc.step(st1, params, 0, n_particles=int(t["n_particles"]))
    assert not (np.array_equal(st1.sediment, st2.sediment) and np.array_equal(st1.discharge, st2.discharge))


def test_bank_cut_trace_and_serial_apply_match_reference_bit_exact():
    """The bank cut on the outside of bends (erosion.lateral_rate,
    particle.py:699-738: an entry of volume -2 after the step's own, applied
    under the erosion caps, no discharge, the path unchanged) on the window:
    the oracle's trace and serial apply equal the reference's bit for bit."""
    case = window_case(GOLDEN / "lateral_trace.npz")
    res = case["oracle"]()
    cap = case["cap"]
    assert cap == orc.change_list_cap(int(case["max_steps"]), True)
    for k in ("cl_count", "cl_lo", "cl_hi", "sp_death"):
        assert np.array_equal(res[k], case[k]), k
    for a, b in zip(changelist_rows(res, cap), changelist_rows(case, cap)):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    assert int(sum((r[2] == -2.0).sum() for r in changelist_rows(case, cap))) > 1000
    for k in ("acc", "pending", "disch_track", "mom_track"):
        assert np.array_equal(res[k], case[k]), k
    assert np.array_equal(res["apply_out"], case["apply_out"])


def test_bank_cut_steps_match_reference_bit_exact():
    """Full steps on the sphere with lateral_rate = 0.5: the oracle's state
    equals the reference's bit for bit."""
    c = step_case(GOLDEN / "step_lateral.npz")
    t = c["t"]
    st = orc.OracleState.from_world(c["world"], c["params"])
    orc.start_replay(st, c["params"])
    assert np.array_equal(st.height, t["h_start"])
    for it in range(c["iterations"]):
        s = orc.step(st, c["params"], it, n_particles=c["n_particles"])
        r = c["stats"][it]
        for k in ("particles", "entries", "clamped", "deaths"):
            assert s[k] == r[k], (it, k)
        assert s["datum_shift"] == r["datum_shift"]
    for k in ("height", "sediment", "discharge", "momentum", "pending"):
        assert np.array_equal(getattr(st, k), t[k]), k


def test_planet_lake_refresh_and_steps_match_reference_bit_exact():
    """The oracle's restatement of the planet's lake refresh (maps.py:422-479
    with lake_fill off: the hydro flood, D8, the evaporation balance) on the
    reference fixture's surface, for both balance branches, and full steps
    with lake_balance, the sea mask and the routing flood every 2
    iterations: flags, base level and state equal the reference's bit for
    bit."""
    import json as _json

    from pgerosion.params import WorldGroup, WorldParams
    from tests.parity_cases import erosion_params

    fx = np.load(GOLDEN / "lake_balance.npz")
    N, H, cs = int(fx["N"]), int(fx["H"]), float(fx["cell_size_m"])
    ep = erosion_params(str(fx["params"]))
    params = WorldParams(world=WorldGroup(seed=int(fx["seed"]), N_c=N, cell_size_m=cs, land_fraction=float(fx["land_fraction"]),
                                          halo=H), erosion=ep)
    from pgerosion.synth import World
    from pgerosion.geometry import get_grid

    world = World(get_grid(N, H, cs), fx["bedrock"], fx["hardness"], fx["precip"], fx["evap"], fx["uplift"],
                  float(fx["land_fraction"]))
    for tag, le in (("budyko", 3.0), ("plain", 0.0)):
        st = orc.OracleState.from_world(world, params)
        st.height[...] = fx["u_height"]
        st.sediment[...] = fx["u_sediment"]
        orc.refresh_base(st, float(fx["ocean_min_fraction"]))
        assert np.array_equal(st.sea.reshape(-1), fx["u_sea"].reshape(-1))
        info = orc.refresh_lakes(st, float(fx["lake_evap"]), float(fx["min_depth"]), float(fx["ocean_min_fraction"]), le)
        want = _json.loads(str(fx[f"{tag}_info"]))
        assert info == {k: want[k] for k in info}, (info, want)
        assert np.array_equal(st.lake_flag, fx[f"{tag}_flag"])
        assert st.base.tobytes() == np.ascontiguousarray(fx[f"{tag}_base"]).tobytes()
    st = orc.OracleState.from_world(world, params)
    orc.start_replay(st, params)
    assert np.array_equal(st.height, fx["h_start"])
    stats = _json.loads(str(fx["stats"]))
    for it in range(int(fx["iterations"])):
        s = orc.step(st, params, it, n_particles=int(fx["n_particles"]))
        for k in ("particles", "entries", "clamped", "deaths"):
            assert s[k] == stats[it][k], (it, k)
        if "lakes" in stats[it]:
            assert s["lakes"] == {k: stats[it]["lakes"][k] for k in s["lakes"]}, it
    for k in ("height", "sediment", "discharge", "momentum", "pending", "base", "lake_flag"):
        assert np.array_equal(getattr(st, k), fx[k]), k


def test_basin_fill_matches_reference_bit_exact():
    """The oracle's fill_basins (maps.py:1278-1326) on the reference's fresh
    world after start_replay: the reference's sediment bit for bit."""
    import json as _json

    from pgerosion.geometry import get_grid
    from pgerosion.params import WorldGroup, WorldParams
    from pgerosion.synth import World
    from tests.parity_cases import erosion_params

    fx = np.load(GOLDEN / "basin_fill.npz")
    N, H, cs = int(fx["N"]), int(fx["H"]), float(fx["cell_size_m"])
    params = WorldParams(world=WorldGroup(seed=int(fx["seed"]), N_c=N, cell_size_m=cs, land_fraction=float(fx["land_fraction"]),
                                          halo=H), erosion=erosion_params(str(fx["params"])))
    world = World(get_grid(N, H, cs), fx["bedrock"], fx["hardness"], fx["precip"], fx["evap"], fx["uplift"],
                  float(fx["land_fraction"]))
    st = orc.OracleState.from_world(world, params)
    orc.start_replay(st, params)
    assert np.array_equal(st.height, fx["h_start"]) and np.array_equal(st.sediment, fx["s_start"])
    info = orc.fill_basins(st, params)
    assert info["basin_cells"] == _json.loads(str(fx["info"]))["basin_cells"]
    assert np.array_equal(st.sediment, fx["sediment"])


@pytest.mark.parametrize("tag", ["a", "b"])
def test_window_lake_balance_matches_reference_bit_exact(tag):
    """The oracle's restatement of a window's lake balance (maps.py:675-736,
    window_lake_evap > 0) on the reference fixture's window and route: the
    flags, the lowered route and the counts, bit for bit."""
    fx = np.load(GOLDEN / "window_lake_balance.npz")
    N, H = int(fx["N"]), int(fx["H"])
    NE = N + 2 * H
    from pgerosion.geometry import get_grid

    grid = get_grid(N, H, float(fx["cell_size_m"]))
    st = orc.OracleState(height=fx["height"].copy(), sediment=fx["sediment"].copy(), discharge=np.zeros((1, NE, NE)),
                         momentum=np.zeros((1, NE, NE, 2)), hardness=np.full((1, NE, NE), 0.5, np.float32), precip=fx["precip"],
                         evap=fx["evap"], uplift=np.zeros((1, NE, NE)), mask=fx["mask"],
                         metric=np.ascontiguousarray(grid.metric_face[None]), metric_inv=np.ascontiguousarray(grid.metric_inv_face[None]),
                         N=N, H=H, spherical=False, height_unit_m=float(fx["cell_size_m"]), deposit_on_exit=True)
    st.route = fx[f"{tag}_route0"].copy()
    info = orc.refresh_lakes_window(st, float(fx["min_depth"]), float(fx[f"{tag}_lake_evap"]))
    assert info == json.loads(str(fx[f"{tag}_info"]))
    assert np.array_equal(st.lake_flag, fx[f"{tag}_flag"])
    assert st.route.tobytes() == np.ascontiguousarray(fx[f"{tag}_route"]).tobytes()


def test_lake_parks_trace_and_serial_apply_match_reference_bit_exact():
    """Lake parks (erosion.lake_fill; particle.py:626-636, 672-696 in the
    trace, 912-933 and 1019 in the apply) on the lake window with every lake
    flagged as having room and small rooms: the park entries (volume -3 on
    the lake cell entered), the serial room countdown, the parked loads and
    the refused rest added to the particle's surplus equal the reference's
    bit for bit."""
    case = window_case(GOLDEN / "lake_parks.npz")
    res = case["oracle"]()
    cap = case["cap"]
    for k in ("cl_count", "cl_lo", "cl_hi", "sp_death"):
        assert np.array_equal(res[k], case[k]), k
    for a, b in zip(changelist_rows(res, cap), changelist_rows(case, cap)):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    assert int((case["cl_vol"] == -3.0).sum()) > 50
    for k in ("acc", "pending", "disch_track", "mom_track", "lake_load", "room_after"):
        assert np.array_equal(res[k], case[k]), k
    assert np.array_equal(res["apply_out"], case["apply_out"])
    assert float(case["lake_load"].sum()) > 0.0 and (case["room_after"] == 0.0).all()  # rooms ran out: loads refused


def test_lake_fill_steps_match_reference_bit_exact():
    """Full steps with the bake's default lakes (lake_balance and lake_fill:
    park entries, the serial room countdown, the loads laid over the lake
    floors and the rooms given at each refresh, maps.py:490-628), the sea
    mask and the routing flood every 2 iterations: the oracle's state, lake
    loads, ids, rooms and flags equal the reference's bit for bit."""
    import json as _json

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
    st = orc.OracleState.from_world(world, params)
    orc.start_replay(st, params)
    assert np.array_equal(st.height, fx["h_start"])
    stats = _json.loads(str(fx["stats"]))
    for it in range(int(fx["iterations"])):
        s = orc.step(st, params, it, n_particles=int(fx["n_particles"]))
        for k in ("particles", "entries", "clamped", "deaths"):
            assert s[k] == stats[it][k], (it, k)
        if "lakes" in stats[it]:
            assert s["lakes"] == stats[it]["lakes"], it
    for k in ("height", "sediment", "discharge", "momentum", "pending", "base", "lake_flag", "lake_load", "lake_id", "lake_room"):
        assert np.array_equal(getattr(st, k), fx[k]), k


def test_brush_restatement_conserves_and_spreads():
    """oracle.brush_spread (the library's brush, no reference counterpart): a unit
    change in the middle of a face spreads over the footprint in proportion to
    the weights; next to a face edge the weights renormalise over the interior;
    the total is kept."""
    N, H, r = 16, 2, 3
    NE = N + 2 * H
    acc = np.zeros((6, NE, NE))
    acc[2, 10, 10] = 1.0
    acc[4, H, H + 5] = -2.0  # on the interior's first row: the footprint is cut by the edge
    out = orc.brush_spread(acc, np.ones(acc.shape, np.uint8), N, H, r)
    assert abs(out.sum() - acc.sum()) < 1e-12
    q = orc.brush_weights(r)
    assert q[r, r] == 1024 * (r + 1) and q[0, 0] == 0  # corners beyond r + 1
    np.testing.assert_allclose(out[2, 10 - r:10 + r + 1, 10 - r:10 + r + 1], q / q.sum(), rtol=1e-14)
    assert np.all(out[4, :H] == 0.0) and np.all(out[4, :, :H] == 0.0)  # nothing on the halo
    assert abs(out[4].sum() + 2.0) < 1e-12
