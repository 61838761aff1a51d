"""Host logic: parameters, random streams, workloads."""
import numpy as np
import pytest

from pgerosion import params as pp
from pgerosion import synth


def test_rng_streams_follow_the_reference_key():
    p = pp.WorldParams(world=pp.WorldGroup(seed=7))
    a = p.rng("erosion", 3).random(4)
    b = np.random.default_rng([(7 + 3000) & ((1 << 64) - 1), 1, 3]).random(4)
    assert np.array_equal(a, b)
    assert not np.array_equal(p.rng("erosion").random(2), p.rng("erosion", 0).random(2))
    with pytest.raises(KeyError):
        p.rng("nope")


def test_chunk_and_steps():
    ep = pp.ErosionParams()
    assert pp.chunk_size(ep, 1_572_864) == 2048
    assert pp.chunk_size(ep, 4096) == 256
    assert pp.max_steps_of(ep, 128) == 256
    assert pp.max_steps_of(pp.ErosionParams(max_steps=96), 1024) == 96


def test_plain_path_guard():
    pp.check_plain(pp.ErosionParams(**pp.plain_knobs()))
    with pytest.raises(ValueError):
        pp.check_plain(pp.ErosionParams())  # the ice sheet
    # the bake's lakes with their parks run (the exact apply)
    pp.check_plain(pp.ErosionParams(**{**pp.plain_knobs(), "lake_balance": True, "lake_fill": True, "flood_every": 10}))


def test_small_world_inputs():
    w = synth.plain_small_world(0)
    H, N = w.grid.H, w.grid.N
    inter = w.bedrock[:, H:H + N, H:H + N]
    assert abs(float((inter >= 0).mean()) - 0.30) < 1e-3
    assert inter.min() >= -4000.0 - 1e-3 and inter.max() <= 3000.0 + 1e-3
    assert w.bedrock.dtype == np.float32 and w.precip.min() == 1.0
    p, P = synth.config_params("small")
    assert P == 65536 and p.erosion.max_steps == 64 and p.world.N_c == 128


def test_stage_land_target_and_volcano_field_without_gpu(tmp_path):
    """The stage driver's host logic (run.py:229-261, maps.py:1413-1430):
    the held land fraction is world.land_fraction, or in shelf mode the
    bedrock's own share of cells at or above 0; the active volcanic cones
    are read from the store only when it has them."""
    import dataclasses

    from pgerosion import stage
    from pgerosion.geometry import get_grid
    from pgerosion.params import TectonicsGroup, WorldGroup, WorldParams

    p = WorldParams(world=WorldGroup(N_c=8, halo=2, land_fraction=0.3))
    bed = np.array([-1.0, 0.0, 2.0, 3.0])
    assert stage.datum_land_fraction(p, bed) == 0.3
    ps = dataclasses.replace(p, tectonics=TectonicsGroup(shelf_fraction=0.1))
    assert stage.datum_land_fraction(ps, bed) == 0.75
    store = stage.LocalStore(tmp_path)
    grid = get_grid(8, 2, 50.0)
    assert stage.active_volcanoes(store, grid) is None
    cone = np.zeros((6, grid.NE, grid.NE), np.float32)
    cone[1, 4, 5] = 1200.0
    store.save_field(stage.VOLCANO_FIELD, cone, grid.H)
    got = stage.active_volcanoes(store, grid)
    assert got is not None and float(got[1, 4, 5]) == 1200.0
