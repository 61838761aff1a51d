"""Stage driver host logic: checkpoint hash, prune, find, and the store layout
(bake/globe/erosion/run.py:68-225 semantics).  No GPU."""
import dataclasses
import json

import numpy as np

from pgerosion import stage
from pgerosion.geometry import Grid
from pgerosion.params import ErosionParams, WorldGroup, WorldParams, plain_knobs


def _params(**kw):
    return WorldParams(world=WorldGroup(seed=1, N_c=16, cell_size_m=50.0, land_fraction=0.3, halo=2),
                       erosion=ErosionParams(**{**plain_knobs(), **kw}))


def test_hash_normalises_run_control_knobs():
    a = _params(uplift_mode="stack", iterations=10)
    b = _params(uplift_mode="stack", iterations=20, checkpoint_every=3, resume=False)
    assert stage.ckpt_hash(a, 0) == stage.ckpt_hash(b, 0)
    # in replay mode the start depends on the iteration count: it stays in the hash
    assert stage.ckpt_hash(_params(uplift_mode="replay", iterations=10), 0) != stage.ckpt_hash(_params(uplift_mode="replay", iterations=20), 0)
    assert stage.ckpt_hash(a, 0) != stage.ckpt_hash(_params(uplift_mode="stack", friction=0.1), 0)
    assert stage.ckpt_hash(a, 0) != stage.ckpt_hash(a, 1)  # the apply mode is part of the identity


def test_hash_covers_upstream_groups_and_outputs(tmp_path):
    """A re-baked tectonics or climate output (same parameters, new manifest
    hash) and a changed tectonics group both refuse the old checkpoint, as
    run.py:68-97's hash does."""
    st = stage.LocalStore(tmp_path)
    d = st.checkpoint_dir
    d.mkdir(parents=True)
    p = _params(uplift_mode="stack")

    def manifest(tect, clim):
        (tmp_path / "manifest.json").write_text(json.dumps(
            {"stages": {"tectonics": {"done": True, "hash": tect}, "climate": {"done": True, "hash": clim}}}))

    manifest("t1", "c1")
    h = stage.ckpt_hash(p, 0, st)
    assert h != stage.ckpt_hash(p, 0)  # the upstream output hashes are part of it
    _fake_ckpt(d, 4, h)
    assert stage.find_checkpoint(st, p, 0)[1]["iteration"] == 4
    manifest("t2", "c1")  # tectonics re-baked with the same parameters
    assert stage.find_checkpoint(st, p, 0) is None
    manifest("t1", "c2")  # climate re-baked
    assert stage.find_checkpoint(st, p, 0) is None
    manifest("t1", "c1")
    assert stage.find_checkpoint(st, p, 0)[1]["iteration"] == 4
    q = dataclasses.replace(p, tectonics=dataclasses.replace(p.tectonics, shelf_fraction=0.25))
    assert stage.find_checkpoint(st, q, 0) is None  # a changed tectonics group


def _fake_ckpt(d, it, h):
    p = d / f"erosion_iter{it:04d}.npz"
    np.savez(p, height=np.zeros(1))
    p.with_suffix(".json").write_text(json.dumps({"iteration": it, "params_hash": h}))


def test_prune_and_find(tmp_path):
    st = stage.LocalStore(tmp_path)
    d = st.checkpoint_dir
    d.mkdir(parents=True)
    p = _params(uplift_mode="stack")
    h = stage.ckpt_hash(p, 0, st)
    for it in (3, 6, 9):
        _fake_ckpt(d, it, h)
    _fake_ckpt(d, 1, "other")
    stage.prune_checkpoints(d, h, keep=2)
    kept = sorted(q.name for q in d.glob("erosion_iter*.npz"))
    assert kept == ["erosion_iter0001.npz", "erosion_iter0006.npz", "erosion_iter0009.npz"]
    assert stage.find_checkpoint(st, p, 0)[1]["iteration"] == 9
    assert stage.find_checkpoint(st, p, 0, max_iteration=8)[1]["iteration"] == 6
    # a truncated .json (a crash between the npz and the json) falls back to the previous one
    (d / "erosion_iter0009.json").write_text('{"iteration": 9, "par')
    assert stage.find_checkpoint(st, p, 0)[1]["iteration"] == 6
    assert stage.find_checkpoint(st, _params(uplift_mode="stack", friction=0.2), 0) is None


def test_local_store_round_trip(tmp_path):
    g = Grid(16, 2, 50.0)
    c = g.centers()
    f = (c[..., 0] * 100.0 + c[..., 2] ** 2).astype(np.float32)
    st = stage.LocalStore(tmp_path)
    st.save_field("bedrock", f, g.H)
    back = st.load_field("bedrock", g)
    H, N = g.H, g.N
    assert np.array_equal(back[:, H:H + N, H:H + N], f[:, H:H + N, H:H + N])
    assert np.abs(back - f).max() < 0.5  # halos refilled by the cubic exchange
