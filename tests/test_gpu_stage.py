"""The GPU stage driver end to end: outputs, checkpoints, and a resumed run
that lands on the continuous run's outputs byte for byte
(bake/tests/test_erosion.py:456-493 adapted)."""
import numpy as np
import pytest

from pgerosion import stage, synth
from pgerosion.params import ErosionParams, WorldGroup, WorldParams, plain_knobs

pytestmark = pytest.mark.gpu


def _world_store(tmp_path):
    w = synth.earth_world(seed=4, N=32, H=2, cell_size_m=50.0, land_fraction=0.3)
    st = stage.LocalStore(tmp_path)
    for name in ("bedrock", "hardness", "precip", "evap", "uplift"):
        st.save_field(name, getattr(w, name), w.grid.H)
    p = WorldParams(world=WorldGroup(seed=4, N_c=32, cell_size_m=50.0, land_fraction=0.3, halo=2),
                    erosion=ErosionParams(**{**plain_knobs(), "iterations": 6, "checkpoint_every": 3, "max_steps": 48,
                                             "friction": 0.05, "erodibility": 0.3, "deposition_rate": 0.3, "evap_rate": 0.01,
                                             "uplift_mode": "replay", "particles_per_cell": 0.5}))
    return st, p


def test_stage_run_checkpoints_and_resume(cuda, tmp_path):
    st, p = _world_store(tmp_path)
    info = stage.run(st, p, log=lambda m: None)
    assert info["iterations"] == 6 and info["backend"] == "b200"
    out = {n: np.stack([np.load(st.coarse / f"{n}.f{k}.npy") for k in range(6)]) for n in stage.OUTPUTS}
    assert out["height"].dtype == np.float32 and out["momentum"].shape[-1] == 2
    assert (st.checkpoint_dir / "erosion_iter0003.npz").exists() and (st.checkpoint_dir / "erosion_iter0006.json").exists()
    with np.load(st.checkpoint_dir / "erosion_iter0006.npz") as z:
        assert set(z.files) >= {"height", "sediment", "discharge", "momentum", "pending", "lake_load"}
        assert z["height"].dtype == np.float64
    # drop the last checkpoint: the stage resumes from iteration 3 and lands on the same outputs
    for suf in (".npz", ".json"):
        (st.checkpoint_dir / f"erosion_iter0006{suf}").unlink()
    msgs = []
    stage.run(st, p, log=msgs.append)
    assert any("resumed" in m and "iteration 3" in m for m in msgs), msgs
    for n in stage.OUTPUTS:
        again = np.stack([np.load(st.coarse / f"{n}.f{k}.npy") for k in range(6)])
        assert again.tobytes() == out[n].tobytes(), n


def test_background_checkpoints_equal_synchronous_ones(cuda, tmp_path):
    """Checkpoints written while the iterations go on hold the same arrays
    as the synchronous writer's, and the final outputs are the same."""
    a_dir, b_dir = tmp_path / "a", tmp_path / "b"
    sa, p = _world_store(a_dir)
    sb, _ = _world_store(b_dir)
    stage.run(sa, p, log=lambda m: None, async_checkpoints=True)
    stage.run(sb, p, log=lambda m: None, async_checkpoints=False)
    for it in (3, 6):
        with np.load(sa.checkpoint_dir / f"erosion_iter{it:04d}.npz") as za, np.load(sb.checkpoint_dir / f"erosion_iter{it:04d}.npz") as zb:
            assert set(za.files) == set(zb.files)
            for k in za.files:
                assert za[k].tobytes() == zb[k].tobytes(), (it, k)
    for n in stage.OUTPUTS:
        for k in range(6):
            assert np.load(sa.coarse / f"{n}.f{k}.npy").tobytes() == np.load(sb.coarse / f"{n}.f{k}.npy").tobytes()


def test_isostasy_state_is_checkpointed_and_resumed(cuda, tmp_path):
    """With isostasy on, the rebound not yet applied (iso_acc) is part of the
    checkpoint (run.py:100-139) and a resumed run lands on the continuous
    run's outputs."""
    import dataclasses

    st, p = _world_store(tmp_path)
    p = dataclasses.replace(p, erosion=dataclasses.replace(p.erosion, isostasy=0.8, isostasy_every=4))
    stage.run(st, p, log=lambda m: None)
    with np.load(st.checkpoint_dir / "erosion_iter0003.npz") as z:
        assert "iso_acc" in z.files and np.abs(z["iso_acc"]).max() > 0.0
    out = {n: np.stack([np.load(st.coarse / f"{n}.f{k}.npy") for k in range(6)]) for n in stage.OUTPUTS}
    for suf in (".npz", ".json"):
        (st.checkpoint_dir / f"erosion_iter0006{suf}").unlink()
    stage.run(st, p, log=lambda m: None)
    for n in stage.OUTPUTS:
        again = np.stack([np.load(st.coarse / f"{n}.f{k}.npy") for k in range(6)])
        assert again.tobytes() == out[n].tobytes(), n


def test_host_refreshes_are_checkpointed_and_resumed(cuda, tmp_path):
    """With the routing flood, the sea mask, the planet's lake balance and the
    glacial pass on (every 2 iterations, ice poleward of 50 degrees) and the
    basin fill at the start, the route, the base level, the lake flags and the
    sticky ice are part of the checkpoint (run.py:104-128, 200-223) and a
    resumed run lands on the continuous run's outputs byte for byte."""
    import dataclasses

    w = synth.earth_world(seed=4, N=32, H=2, cell_size_m=50.0, land_fraction=0.3)
    w.evap[...] = np.where(np.abs(w.grid.latitude()) > np.radians(50.0), 0.0, 1.0).astype(np.float32)
    st = stage.LocalStore(tmp_path)
    for name in ("bedrock", "hardness", "precip", "evap", "uplift"):
        st.save_field(name, getattr(w, name), w.grid.H)
    _, p = _world_store(tmp_path / "unused")
    p = dataclasses.replace(p, erosion=dataclasses.replace(p.erosion, flood_every=2, sea_mask_every=2, glacial_every=2,
                                                           glacial_from=0.0, lake_balance=True, lake_fill=False,
                                                           basin_fill_grade=0.1))
    stage.run(st, p, log=lambda m: None)
    with np.load(st.checkpoint_dir / "erosion_iter0003.npz") as z:
        assert {"route", "base", "ice_prev", "lake_flag", "lake_id", "lake_room"} <= set(z.files)
        assert z["ice_prev"].dtype == np.uint8 and z["ice_prev"].any()
    out = {n: np.stack([np.load(st.coarse / f"{n}.f{k}.npy") for k in range(6)]) for n in stage.OUTPUTS}
    for suf in (".npz", ".json"):
        (st.checkpoint_dir / f"erosion_iter0006{suf}").unlink()
    stage.run(st, p, log=lambda m: None)
    for n in stage.OUTPUTS:
        again = np.stack([np.load(st.coarse / f"{n}.f{k}.npy") for k in range(6)])
        assert again.tobytes() == out[n].tobytes(), n


def test_active_volcanoes_are_taken_off_and_put_back(cuda, tmp_path):
    """A store with active volcanic cones (volcano_active, run.py:229-311):
    the stage erodes the ground under them and puts them back on top at its
    end, so its outputs are those of the same run on the bedrock without the
    cones, with the cones added to the height (float32 metres); the other
    outputs are untouched."""
    import dataclasses

    sa, p = _world_store(tmp_path / "a")
    p = dataclasses.replace(p, erosion=dataclasses.replace(p.erosion, checkpoint_every=0, resume=False))
    from pgerosion.geometry import get_grid

    grid = get_grid(32, 2, 50.0)
    bed = stage._field(sa, "bedrock", grid)
    cone = np.zeros_like(bed)
    cone[2, 10:13, 14:17] = 900.0
    cone[4, 20, 8] = 2500.0
    sa.save_field(stage.VOLCANO_FIELD, cone, grid.H)
    info = stage.run(sa, p, log=lambda m: None)
    assert info["volcano_cells"] == 10 and info["volcano_max_m"] == 2500.0
    sb, _ = _world_store(tmp_path / "b")
    sb.save_field("bedrock", (bed - cone).astype(np.float32), grid.H)
    stage.run(sb, p, log=lambda m: None)
    out = lambda s_, n: np.stack([np.load(s_.coarse / f"{n}.f{k}.npy") for k in range(6)])
    H, N = grid.H, grid.N
    ha, hb = out(sa, "height"), out(sb, "height")
    np.testing.assert_allclose(ha, hb + cone[:, H:H + N, H:H + N], rtol=0, atol=1e-3)
    for n in ("sediment", "discharge", "momentum"):
        assert out(sa, n).tobytes() == out(sb, n).tobytes(), n


def test_lake_parks_are_checkpointed_and_resumed(cuda, tmp_path):
    """The bake's default lakes (lake_balance with lake_fill: loads parked in
    the lakes, laid over their floors at each refresh and at the end): the
    parked loads, the lakes' numbers and rooms are part of the checkpoint
    (run.py:104-128, 200-224) and a resumed run lands on the continuous run's
    outputs byte for byte."""
    import dataclasses

    w = synth.earth_world(seed=11, N=32, H=2, cell_size_m=50.0, land_fraction=0.45)
    st = stage.LocalStore(tmp_path)
    for name in ("bedrock", "hardness", "precip", "evap", "uplift"):
        st.save_field(name, getattr(w, name), w.grid.H)
    _, p = _world_store(tmp_path / "unused")
    p = dataclasses.replace(p, erosion=dataclasses.replace(p.erosion, flood_every=2, sea_mask_every=2, lake_balance=True,
                                                           lake_fill=True, basin_fill_grade=0.1))
    info = stage.run(st, p, log=lambda m: None)
    assert info.get("lakes_end") is not None
    with np.load(st.checkpoint_dir / "erosion_iter0003.npz") as z:
        assert {"lake_load", "lake_id", "lake_room", "lake_flag"} <= set(z.files)
        assert (z["lake_id"] >= 0).any() and z["lake_room"].size >= 1
    out = {n: np.stack([np.load(st.coarse / f"{n}.f{k}.npy") for k in range(6)]) for n in stage.OUTPUTS}
    for suf in (".npz", ".json"):
        (st.checkpoint_dir / f"erosion_iter0006{suf}").unlink()
    stage.run(st, p, log=lambda m: None)
    for n in stage.OUTPUTS:
        again = np.stack([np.load(st.coarse / f"{n}.f{k}.npy") for k in range(6)])
        assert again.tobytes() == out[n].tobytes(), n
