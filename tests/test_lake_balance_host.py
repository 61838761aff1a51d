"""The planet's lake balance (``pge_lake_balance``: ErosionState.refresh_lakes,
globe/erosion/maps.py:422-479, with erosion.lake_fill off) against the
reference's own refresh on the same surface (tests/golden/lake_balance.npz,
made by tests/golden/gen_golden.py).

``pge_lake_balance`` is the library's host code (the reference's sequence
follows the flood's serial pop order), so it runs here without a GPU; the
arrays it takes are what ``ErosionState.refresh_lakes`` copies off the
device.  Flags, closed levels and the water surface are comparison and
float32 work on the reference's own operation order: identical."""
import ctypes
import json

import numpy as np
import pytest

from pgerosion import _lib
from pgerosion.geometry import get_grid
from pgerosion.isostasy import sqrt_det_metric
from tests.parity_cases import GOLDEN


def _inputs():
    fx = np.load(GOLDEN / "lake_balance.npz")
    N, H, cs = int(fx["N"]), int(fx["H"]), float(fx["cell_size_m"])
    grid = get_grid(N, H, cs)
    inter = (slice(None), slice(H, H + N), slice(H, H + N))
    c = lambda a, t: np.ascontiguousarray(np.asarray(a)[inter], dtype=t)
    surf = c(fx["u_height"] + fx["u_sediment"], np.float32)
    sq = sqrt_det_metric(grid)[H:H + N, H:H + N]
    area = np.ascontiguousarray(np.broadcast_to((sq.astype(np.float64) * cs ** 2).astype(np.float32), (6, N, N)))
    return dict(fx=fx, grid=grid, N=N, H=H, cs=cs, inter=inter, surf=surf, ocean=np.ascontiguousarray(fx["u_sea"], np.uint8),
                precip=c(fx["precip"], np.float32), pet=c(fx["evap"], np.float32), area=area,
                owner=np.ascontiguousarray(grid.owner, np.int32), metric=np.ascontiguousarray(grid.metric_face, np.float32))


def _balance(d, land_evap):
    N = d["N"]
    g = _lib.PgeGrid(F=6, N=N, H=d["H"], spherical=1, metric_shared=1, max_steps=1, max_droplets=1, max_wave=1)
    flag = np.empty((6, N, N), np.uint8)
    water = np.empty((6, N, N), np.float32)
    level = np.empty((6, N, N), np.float32)
    info = _lib.PgeLakeInfo()
    _lib.check(_lib.load().pge_lake_balance(ctypes.byref(g), d["owner"].ctypes.data, d["metric"].ctypes.data, d["area"].ctypes.data,
                                            d["cs"], d["surf"].ctypes.data, d["ocean"].ctypes.data, d["precip"].ctypes.data,
                                            d["pet"].ctypes.data, float(d["fx"]["lake_evap"]), float(land_evap),
                                            float(d["fx"]["min_depth"]), flag.ctypes.data, water.ctypes.data, level.ctypes.data,
                                            ctypes.byref(info)), "pge_lake_balance")
    return flag, water, level, info


@pytest.mark.parametrize("tag,land_evap", [("budyko", 3.0), ("plain", 0.0)])
def test_lake_balance_equals_the_reference(tag, land_evap):
    d = _inputs()
    fx, inter = d["fx"], d["inter"]
    flag, water, level, info = _balance(d, land_evap)
    want = json.loads(str(fx[f"{tag}_info"]))
    got = {k: int(getattr(info, k)) for k in ("lake_cells", "lake_cells_closed", "depressions", "overflowing", "closed", "dry")}
    assert got == {k: want[k] for k in got}, (got, want)
    assert np.array_equal(flag, fx[f"{tag}_flag"][inter])
    assert water.tobytes() == np.ascontiguousarray(fx[f"{tag}_water"], np.float32).tobytes()
    # the closed lakes' levels are the base level there, the rest of the base is untouched
    base = np.array(fx["u_base"][inter])
    closed = ~np.isnan(level)
    base[closed] = level[closed]
    assert base.tobytes() == np.ascontiguousarray(fx[f"{tag}_base"][inter]).tobytes()
    assert got["lake_cells"] > 0 and got["closed"] > 0 and got["overflowing"] > 0


def test_lake_balance_without_evaporation_is_the_spill_fill():
    """lake_evap = land_evap = 0: every depression stands at its spill
    point, overflowing, and no lake is closed."""
    d = _inputs()
    d["fx"] = dict(d["fx"])
    d["fx"]["lake_evap"] = np.float64(0.0)
    flag, water, level, info = _balance(d, 0.0)
    assert info.lake_cells_closed == 0 and np.isnan(level).all()
    assert (water >= d["surf"]).all()
    assert int(flag.sum()) == int(info.lake_cells) > 0


def test_lake_balance_rejects_a_window():
    N = 8
    g = _lib.PgeGrid(F=1, N=N, H=2, spherical=0, metric_shared=1, max_steps=1, max_droplets=1, max_wave=1)
    a = np.zeros((1, N, N), np.float32)
    r = _lib.load().pge_lake_balance(ctypes.byref(g), a.ctypes.data, a.ctypes.data, a.ctypes.data, 1.0, a.ctypes.data, a.ctypes.data,
                                     a.ctypes.data, a.ctypes.data, 1.0, 0.0, 0.0, a.ctypes.data, None, None, None)
    assert r == _lib.PGE_E_UNSUPPORTED


def test_basin_fill_equals_the_reference():
    """``pge_basin_fill`` (fill_basins, maps.py:1278-1326, on the host) on the
    reference fixture's fresh world after start_replay, with the open ocean
    of the oracle's sea mask (pinned to the reference): the sediment the
    reference lays, bit for bit, and its basin count."""
    from oracle import oracle as orc

    fx = np.load(GOLDEN / "basin_fill.npz")
    N, H, cs = int(fx["N"]), int(fx["H"]), float(fx["cell_size_m"])
    grid = get_grid(N, H, cs)
    inter = (slice(None), slice(H, H + N), slice(H, H + N))
    surf = np.ascontiguousarray((fx["h_start"] + fx["s_start"])[inter], np.float32)
    below, labels, keep = orc.below_sea_components(surf, grid, 0.02)[:3]
    ocean = np.ascontiguousarray((below & keep[np.maximum(labels, 0)]).reshape(surf.shape), np.uint8)
    ep = json.loads(str(fx["params"]))
    step = float(ep["basin_fill_grade"]) * (cs / 1000.0) / cs
    add = np.empty((6, N, N))
    basin = np.empty((6, N, N), np.uint8)
    nb = ctypes.c_int64(0)
    g = _lib.PgeGrid(F=6, N=N, H=H, spherical=1, metric_shared=1, max_steps=1, max_droplets=1, max_wave=1)
    owner = np.ascontiguousarray(grid.owner, np.int32)
    _lib.check(_lib.load().pge_basin_fill(ctypes.byref(g), owner.ctypes.data, surf.ctypes.data, ocean.ctypes.data, step,
                                          float(ep["basin_fill_min_m"]) / cs, add.ctypes.data, basin.ctypes.data,
                                          ctypes.byref(nb)), "pge_basin_fill")
    info = json.loads(str(fx["info"]))
    assert int(nb.value) == info["basin_cells"] > 0
    sed = np.array(fx["s_start"])
    sed[inter] += add
    assert sed[inter].tobytes() == np.ascontiguousarray(fx["sediment"][inter]).tobytes()


@pytest.mark.parametrize("tag", ["a", "b"])
def test_window_lake_balance_equals_the_reference(tag):
    """``pge_window_lake_balance`` (ErosionState._balance_window_lakes,
    maps.py:675-736, on the host) on the reference fixture's window after
    its routing flood: the reference's lake flags, lowered routing surface
    and counts, bit for bit, at two evaporation rates (overflowing and closed
    lakes)."""
    fx = np.load(GOLDEN / "window_lake_balance.npz")
    N, H = int(fx["N"]), int(fx["H"])
    NE = N + 2 * H
    surf = np.ascontiguousarray((fx["height"] + fx["sediment"])[0], np.float32)
    active = np.ascontiguousarray(fx["mask"][0] == 1, np.uint8)
    precip = np.ascontiguousarray(fx["precip"][0], np.float32)
    evap = np.ascontiguousarray(fx["evap"][0], np.float32)
    route = np.ascontiguousarray(fx[f"{tag}_route0"][0], np.float64).copy()
    lake = np.empty((NE, NE), np.uint8)
    counts = np.zeros(5, np.int64)
    g = _lib.PgeGrid(F=1, N=N, H=H, spherical=0, metric_shared=1, max_steps=1, max_droplets=1, max_wave=1)
    _lib.check(_lib.load().pge_window_lake_balance(ctypes.byref(g), surf.ctypes.data, active.ctypes.data, precip.ctypes.data,
                                                   evap.ctypes.data, float(fx[f"{tag}_lake_evap"]), float(fx["min_depth"]),
                                                   route.ctypes.data, lake.ctypes.data, counts.ctypes.data),
               "pge_window_lake_balance")
    info = json.loads(str(fx[f"{tag}_info"]))
    assert {"depressions": int(counts[0]), "overflowing": int(counts[1]), "closed": int(counts[2]), "dry": int(counts[3])} == \
        {k: info[k] for k in ("depressions", "overflowing", "closed", "dry")}
    flag = np.zeros((NE, NE), np.uint8)
    flag[H:H + N, H:H + N] = lake[H:H + N, H:H + N]
    assert np.array_equal(flag, fx[f"{tag}_flag"][0])
    assert int(flag.sum()) == info["lake_cells"]
    assert route.tobytes() == np.ascontiguousarray(fx[f"{tag}_route"][0]).tobytes()
    assert info["closed"] > 0


def _oracle_lakes(surf, ocean, precip, pet, grid, lake_evap, land_evap, min_depth):
    """The oracle's restatement of the planet lake refresh (pinned to the
    reference above) on raw interior arrays: flags, water, closed levels."""
    from oracle import oracle as orc

    N, H = grid.N, grid.H
    nbr = orc._cell_neighbors(grid)
    s32 = surf.reshape(-1)
    oc = ocean.reshape(-1).astype(bool)
    filled, parent, order, pop_seq = orc.hydro_flood(s32, oc, nbr, N)
    down = orc.flow_down(filled, oc, parent, nbr, grid.metric_face, N, H)
    topo = pop_seq[::-1]
    topo = topo[~oc[topo]]
    water, bal = orc.balance_lakes(s32, filled, oc, order, down, topo, precip, pet, orc.interior_cell_area(grid), grid.cell_size_m,
                                   nbr, lake_evap, land_evap)
    lake = ((water - s32) > np.float32(min_depth)) & ~oc
    closed = lake & (water < filled - np.float32(1e-4))
    return (lake & ~closed).astype(np.uint8), water, closed, bal


@pytest.mark.parametrize("case", ["noise", "no_ocean", "plateau", "all_ocean_but_one"])
@pytest.mark.parametrize("land_evap", [0.0, 3.0])
def test_lake_balance_equals_the_oracle_on_edge_cases(case, land_evap):
    """Seeded small worlds the fixtures do not cover -- rough noise with a
    sea, no ocean at all (an error, as in the reference), a flat plateau with
    pits (flats drain to their flood parent), a world that is ocean but for
    one cell -- checked against the oracle's restatement of the reference."""
    N, H, cs = 12, 2, 1000.0
    grid = get_grid(N, H, cs)
    rng = np.random.default_rng(hash((case, land_evap)) % 2**32)
    if case == "noise":
        surf = rng.normal(0.5, 1.0, (6, N, N)).astype(np.float32)
    elif case == "no_ocean":
        surf = (2.0 + rng.random((6, N, N))).astype(np.float32)
    elif case == "plateau":
        surf = np.full((6, N, N), 3.0, np.float32)
        surf[:, 3:5, 3:5] = 2.0
        surf[0, :2, :] = -1.0
    else:
        surf = np.full((6, N, N), -5.0, np.float32)
        surf[2, 6, 6] = 1.0
    ocean = np.zeros((6, N, N), np.uint8)
    if case != "no_ocean":
        from oracle import oracle as orc

        below, labels, keep = orc.below_sea_components(surf, grid, 0.02)[:3]
        if labels is not None:
            ocean = np.ascontiguousarray((below & keep[np.maximum(labels, 0)]).reshape(surf.shape), np.uint8)
    precip = (0.2 + rng.random((6, N, N))).astype(np.float32)
    pet = rng.random((6, N, N)).astype(np.float32)
    sq = sqrt_det_metric(grid)[H:H + N, H:H + N]
    area = np.ascontiguousarray(np.broadcast_to((sq.astype(np.float64) * cs ** 2).astype(np.float32), (6, N, N)))
    d = dict(fx={"lake_evap": np.float64(2.0), "min_depth": np.float64(1e-3)}, N=N, H=H, cs=cs, surf=np.ascontiguousarray(surf),
             ocean=ocean, precip=precip, pet=pet, area=area, owner=np.ascontiguousarray(grid.owner, np.int32),
             metric=np.ascontiguousarray(grid.metric_face, np.float32))
    if case == "no_ocean":
        # the flood drains the lowest cell, but D8 holds it to be land with nowhere to go: the reference's
        # flow_directions raises (hydro/routing.py:86-89), and so do the oracle and the library
        with pytest.raises(RuntimeError):
            _oracle_lakes(surf, ocean, precip, pet, grid, 2.0, land_evap, 1e-3)
        with pytest.raises(_lib.PgeError, match="no flow direction"):
            _balance(d, land_evap)
        return
    flag, water, level, info = _balance(d, land_evap)
    want_flag, want_water, closed, bal = _oracle_lakes(surf, ocean, precip, pet, grid, 2.0, land_evap, 1e-3)
    assert np.array_equal(flag.reshape(-1), want_flag)
    assert water.reshape(-1).tobytes() == want_water.tobytes()
    assert np.array_equal(~np.isnan(level.reshape(-1)), closed)
    assert {k: int(getattr(info, k)) for k in bal} == bal


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_basin_fill_equals_the_oracle_on_noise_worlds(seed):
    """``pge_basin_fill`` against the oracle's restatement (pinned to the
    reference above) on seeded rough worlds with a sea and many closed
    basins, at a steep grade so the plain's slope shows."""
    from oracle import oracle as orc

    N, H, cs = 12, 2, 1000.0
    grid = get_grid(N, H, cs)
    rng = np.random.default_rng(seed)
    surf = rng.normal(0.3, 1.0, (6, N, N)).astype(np.float32)
    below, labels, keep = orc.below_sea_components(surf, grid, 0.02)[:3]
    ocean = np.ascontiguousarray((below & keep[np.maximum(labels, 0)]).reshape(surf.shape), np.uint8)
    step, depth = 0.05, 0.01
    add = np.empty((6, N, N))
    basin = np.empty((6, N, N), np.uint8)
    nb = ctypes.c_int64(0)
    g = _lib.PgeGrid(F=6, N=N, H=H, spherical=1, metric_shared=1, max_steps=1, max_droplets=1, max_wave=1)
    owner = np.ascontiguousarray(grid.owner, np.int32)
    _lib.check(_lib.load().pge_basin_fill(ctypes.byref(g), owner.ctypes.data, surf.ctypes.data, ocean.ctypes.data, step, depth,
                                          add.ctypes.data, basin.ctypes.data, ctypes.byref(nb)), "pge_basin_fill")
    s32 = surf.reshape(-1)
    oc = ocean.reshape(-1).astype(bool)
    filled, parent, order, pop_seq = orc.hydro_flood(s32, oc, orc._cell_neighbors(grid), N)
    gr = s32.astype(np.float64)
    for c in pop_seq:
        q = parent[c]
        if q >= 0 and gr[q] + step > gr[c]:
            gr[c] = gr[q] + step
    want_basin = ((filled - s32) > np.float32(depth)) & ~oc
    want = np.where(want_basin, np.maximum(gr - s32, 0.0), 0.0)
    assert np.array_equal(basin.reshape(-1).astype(bool), want_basin) and want_basin.any()
    assert add.reshape(-1).tobytes() == want.tobytes()
    assert int(nb.value) == int(want_basin.sum())


def test_lake_fill_refresh_equals_the_oracle(monkeypatch):
    """``pge_lake_balance_fill`` (the lake refresh with erosion.lake_fill:
    the parked loads laid over the lake floors, the lakes numbered and given
    their room, maps.py:422-479, 490-628) against the oracle's refresh, which
    reproduces the reference's steps on tests/golden/lake_fill_steps.npz bit
    for bit: at every refresh of those steps, on the same state, the flags,
    the sediment laid, the stockpiles, the lake numbers and rooms, the
    isostatic load and the closed lakes' levels are identical."""
    import json as _json

    from oracle import oracle as orc
    from pgerosion.params import WorldGroup, WorldParams
    from pgerosion.synth import World
    from tests.parity_cases import erosion_params

    fx = np.load(GOLDEN / "lake_fill_steps.npz")
    N, H, cs = int(fx["N"]), int(fx["H"]), float(fx["cell_size_m"])
    params = WorldParams(world=WorldGroup(seed=int(fx["seed"]), N_c=N, cell_size_m=cs, land_fraction=float(fx["land_fraction"]),
                                          halo=H), erosion=erosion_params(str(fx["params"])))
    grid = get_grid(N, H, cs)
    world = World(grid, fx["bedrock"], fx["hardness"], fx["precip"], fx["evap"], fx["uplift"], float(fx["land_fraction"]))
    st = orc.OracleState.from_world(world, params)
    orc.start_replay(st, params)
    inter = (slice(None), slice(H, H + N), slice(H, H + N))
    sq = sqrt_det_metric(grid)[H:H + N, H:H + N]
    area = np.ascontiguousarray(np.broadcast_to((sq.astype(np.float64) * cs ** 2).astype(np.float32), (6, N, N)))
    owner = np.ascontiguousarray(grid.owner, np.int32)
    metric = np.ascontiguousarray(grid.metric_face, np.float32)
    centres = np.ascontiguousarray(grid.centers()[:, H:H + N, H:H + N], np.float64)
    g = _lib.PgeGrid(F=6, N=N, H=H, spherical=1, metric_shared=1, max_steps=1, max_droplets=1, max_wave=1)
    original = orc.refresh_lakes
    seen = []

    def checked(state, lake_evap, min_depth, min_fraction, land_evap=0.0, fill=None):
        if fill is None:
            return original(state, lake_evap, min_depth, min_fraction, land_evap, fill)
        c = lambda a, t: np.ascontiguousarray(np.asarray(a)[inter], dtype=t)
        surf = c(state.height + state.sediment, np.float32)
        sea = getattr(state, "sea", None)
        if sea is None:
            below, labels, keep = orc.below_sea_components(surf, grid, float(min_fraction))
            sea = np.zeros(surf.shape, bool) if labels is None else (below & keep[np.maximum(labels, 0)]).reshape(surf.shape)
        ocean = np.ascontiguousarray(np.asarray(sea, bool).reshape(surf.shape), np.uint8)
        pet = getattr(state, "lake_pet", None)
        pet = c(state.evap if pet is None else pet, np.float32)
        if state.lake_load is None:
            load, ids = np.zeros((6, N, N)), np.full((6, N, N), -1, np.int32)
        else:
            load, ids = c(state.lake_load, np.float64), c(state.lake_id, np.int32)
        sed0, pend0 = c(state.sediment, np.float64), c(state.pending, np.float64)
        iso0 = None if getattr(state, "iso_acc", None) is None else c(state.iso_acc, np.float64)
        lay, padd, room = np.zeros((6, N, N)), np.zeros((6, N, N)), np.zeros(6 * N * N)
        flag = np.empty((6, N, N), np.uint8)
        water = np.empty((6, N, N), np.float32)
        level = np.empty((6, N, N), np.float32)
        evap = c(state.evap, np.float32)
        height = c(state.height, np.float64)
        precip = c(state.precip, np.float32)  # every array handed over is held by a name until the call returns
        fl = _lib.PgeLakeFill(grade=fill[0], ice_evap=fill[1], rise=fill[2], evap=evap.ctypes.data, centres=centres.ctypes.data,
                              height=height.ctypes.data, sediment=sed0.ctypes.data, lake_load=load.ctypes.data,
                              lake_id=ids.ctypes.data, lay=lay.ctypes.data, pending=padd.ctypes.data, lake_room=room.ctypes.data,
                              lake_room_cap=room.size)
        info = _lib.PgeLakeInfo()
        _lib.check(_lib.load().pge_lake_balance_fill(ctypes.byref(g), owner.ctypes.data, metric.ctypes.data, area.ctypes.data, cs,
                                                     surf.ctypes.data, ocean.ctypes.data, precip.ctypes.data,
                                                     pet.ctypes.data, float(lake_evap), float(land_evap), float(min_depth),
                                                     flag.ctypes.data, water.ctypes.data, level.ctypes.data, ctypes.byref(fl),
                                                     ctypes.byref(info)), "pge_lake_balance_fill")
        base0 = c(state.base, np.float64)
        out = original(state, lake_evap, min_depth, min_fraction, land_evap, fill)
        assert np.array_equal(flag, np.asarray(state.lake_flag)[inter])
        assert (sed0 + lay).tobytes() == c(state.sediment, np.float64).tobytes()
        assert (pend0 + padd).tobytes() == c(state.pending, np.float64).tobytes()
        assert np.array_equal(ids, c(state.lake_id, np.int32))
        assert room[:max(int(fl.lakes), 1)].tobytes() == np.ascontiguousarray(state.lake_room, np.float64).tobytes()
        if iso0 is not None:
            assert (iso0 + fill[3] * lay).tobytes() == c(state.iso_acc, np.float64).tobytes()
        closed = ~np.isnan(level)
        base0[closed] = level[closed]
        assert base0.tobytes() == c(state.base, np.float64).tobytes()
        assert int(info.lake_cells) == out["lake_cells"] and int(info.lake_cells_closed) == out["lake_cells_closed"]
        assert int(fl.lakes) == out["load_lakes"]
        for k in ("parked", "laid", "stray", "room"):
            assert abs(getattr(fl, k) - out[f"load_{k}"]) <= 1e-12 * max(abs(out[f"load_{k}"]), 1.0), k
        seen.append((int(fl.lakes), float(fl.parked), float(fl.laid)))
        return out

    monkeypatch.setattr(orc, "refresh_lakes", checked)
    for it in range(int(fx["iterations"])):
        orc.step(st, params, it, n_particles=int(fx["n_particles"]))
    print("refreshes (lakes taking load, parked, laid):", seen)
    assert len(seen) >= 3 and any(p > 0.0 for _, p, _ in seen) and any(n > 0 for n, _, _ in seen)
    for k in ("height", "sediment", "lake_load", "lake_id", "lake_room"):
        assert np.array_equal(getattr(st, k), fx[k]), k
