"""Parity at the benchmarked workloads (needs a B200).

* Gate 1 on the N_c = 128 small world and the N_c = 1024 Earth-default world:
  isolated droplets traced by the float64 kernel against the reference's own
  change lists and accumulators (tests/golden/trace_isolated_{c1,n1024}.npz,
  made by trace_particles / apply_changes): cells and death causes identical,
  deltas / volumes / momenta within 1e-5 relative, the accumulators within
  1e-5 relative.
* Device spawns (pge_spawn_rain) against the oracle's spawn_particles (the
  reference's maps.py:809-833, pinned by the step fixtures): the same
  (face, x, y) for every droplet and the same total weight, bit for bit, on
  both worlds and on a rain field of float32 values from 1e-6 to 3 whose
  cumulative sum the integer scan cannot hold exactly (there the totals stay
  bit-identical -- numpy's pairwise order -- and the cells may differ only
  where a uniform falls within rounding of a cell boundary).
* One ordered (exact) pass at both workloads with the oracle's spawns on the
  same terrain: every field within 1e-5 relative, and the share of
  bit-identical heights printed and held above 99 %.  The remaining cells
  come from face crossings where the C library's tan / atan are off by one
  ulp (tests/test_crmath.py): the kernel's are correctly rounded.
"""
import ctypes
import hashlib
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from pgerosion import _lib
from pgerosion import maps as gm
from pgerosion import synth
from tests.parity_cases import erosion_params

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).parent / "golden"

_WORLDS = {}


def _world(name):
    """The fresh world of a workload (the noise on the GPU: the same float64 operations as on the host)."""
    if name not in _WORLDS:
        if name == "c1":
            _WORLDS[name] = (synth.plain_small_world(0),) + synth.config_params("small")
        else:
            _WORLDS[name] = (synth.earth_world(seed=0, N=1024),) + synth.config_params("earth")
    return _WORLDS[name]


@pytest.mark.parametrize("name", ["c1", "n1024"])
def test_isolated_droplets_on_benchmarked_worlds_match_reference(cuda, name):
    t = np.load(GOLD / f"trace_isolated_{name}.npz")
    world = _world(name)[0]
    assert hashlib.sha256(np.ascontiguousarray(world.bedrock).tobytes()).hexdigest() == str(t["bedrock_sha"]), \
        "the rebuilt world differs from the one the reference traced"
    ep = erosion_params(str(t["params"]))
    st = gm.ErosionState.from_world(world)
    res = gm.trace_changelist(st, ep, t["sp_face"], t["sp_x"], t["sp_y"], t["sp_sed"], t["sp_dir"], float(t["volume0"]),
                              float(t["conc_scale"]), precision=_lib.PREC_F64)
    cap = int(res["cap"])
    cnt = t["cl_count"]
    assert np.array_equal(res["cl_count"], cnt), "entry counts differ"
    assert np.array_equal(res["sp_death"], t["sp_death"]), "death causes differ"
    sel = np.concatenate([np.arange(q * cap, q * cap + cnt[q]) for q in range(cnt.size)])
    assert np.array_equal(res["cl_cell"][sel], t["cl_cell"]), "cell paths differ"
    d_ours, d_ref = res["cl_delta"][sel], t["cl_delta"]
    np.testing.assert_allclose(d_ours, d_ref, rtol=1e-5, atol=1e-12)
    np.testing.assert_allclose(res["cl_vol"][sel], t["cl_vol"], rtol=1e-5, atol=0)
    np.testing.assert_allclose(res["cl_mom"][sel], t["cl_mom"], rtol=1e-5, atol=1e-7)
    exact = np.mean(d_ours == d_ref)
    print(f"{name}: {cnt.size} isolated droplets, {sel.size} entries; deltas bit-identical in {exact:.4%}")
    touched = t["touched"]
    for k, ref in (("acc", t["acc"]), ("pending", t["pending"]), ("disch_track", t["disch_track"])):
        ours = res[k].reshape(-1)
        np.testing.assert_allclose(ours[touched], ref, rtol=1e-5, atol=1e-11, err_msg=k)
        rest = np.ones(ours.size, bool)
        rest[touched] = False
        assert np.abs(ours[rest]).max() <= 1e-11, f"{k} changed cells the reference left alone"
    np.testing.assert_allclose(res["mom_track"].reshape(-1, 2)[touched], t["mom_track"], rtol=1e-5, atol=1e-8)


def _wide_rain_world():
    w = synth.plain_small_world(0)
    rng = np.random.default_rng(5)
    w.precip[...] = (10.0 ** rng.uniform(-6.0, np.log10(3.0), w.precip.shape)).astype(np.float32)
    return w


@pytest.mark.parametrize("name", ["c1", "n1024", "wide_rain"])
def test_device_spawns_match_reference_draws(cuda, name):
    if name == "wide_rain":
        world, (params, P) = _wide_rain_world(), synth.config_params("small")
    else:
        world, params, P = _world(name)
    o = orc.OracleState.from_world(world, params)
    f, x, y, v0 = orc.spawn_particles(o, P, params.rng("erosion", 3))
    g = gm.ErosionState.from_world(world)
    r2 = params.rng("erosion", 3)
    u = r2.random(P)
    off = r2.random((P, 2))
    d = gm.spawn_rain(g, u, off)
    assert d["total"] / P == v0, "volume0 differs from w.sum() / P"
    same = (d["face"] == f) & (d["x"] == x) & (d["y"] == y)
    print(f"{name}: {P} spawns, identical {same.mean():.6%}; volume0 {v0!r}")
    if name == "wide_rain":
        assert same.mean() > 1.0 - 1e-4
    else:
        assert same.all(), np.flatnonzero(~same)[:10]


def _ordered_pass(world, params, P):
    """One exact pass on the device and the oracle's chunked serial pass on the same spawns and terrain."""
    o = orc.OracleState.from_world(world, params)
    replay = str(params.erosion.uplift_mode) == "replay"
    if replay:
        orc.start_replay(o, params)
    f, x, y, v0 = orc.spawn_particles(o, P, params.rng("erosion", 0))
    g = gm.ErosionState.from_world(world)
    if replay:
        # the replayed start: the interior lowered by the run's uplift less its mean (numpy's pairwise
        # order on both sides) is bit-identical; the halos come from the cubic exchange, whose 16-term sums
        # numpy's einsum orders its own way (within 1e-12); then both passes start from the same terrain
        gm.start_replay(g, params)
        gh = g.height.cpu().numpy()
        inter = g.interior
        assert np.array_equal(gh[inter], o.height[inter]), "replayed interior differs"
        np.testing.assert_allclose(gh, o.height, rtol=1e-12, atol=1e-12)
        g.height.copy_(torch.as_tensor(o.height))
    z = np.zeros(len(f))
    s = gm.apply_spawns(g, params, f, x, y, z, z, v0)
    ep = params.erosion
    chunk = orc.chunk_size(ep, P)
    o.pack()
    o.acc[...] = 0.0
    tp = orc.trace_params(o, ep, v0, chunk / (v0 * P))
    ap = orc.apply_params(o, ep, ep.iter_deposit / o.height_unit_m)
    cap = orc.change_list_cap(tp.max_steps)
    clamped = 0
    for c0 in range(0, P, chunk):
        cl = orc.trace(o, tp, f[c0:c0 + chunk], x[c0:c0 + chunk], y[c0:c0 + chunk], z[c0:c0 + chunk], z[c0:c0 + chunk], v0)
        clamped += orc.apply(o, ap, cl, cap)[0]
    lib = orc.lib()
    lib.orc_fold(ctypes.c_int64(o.height.size), orc._p(o.height), orc._p(o.sediment), orc._p(o.acc), orc._p(o.mask))
    lib.orc_ema(ctypes.c_int64(o.height.size), orc._p(o.discharge), orc._p(o.momentum), orc._p(o.disch_track), orc._p(o.mom_track),
                orc._p(o.mask), ctypes.c_double(float(ep.ema)))
    a = g.to_numpy()
    worst = {}
    for k in ("height", "sediment", "discharge", "momentum", "pending"):
        ref = getattr(o, k)
        worst[k] = float(np.abs(a[k] - ref).max() / max(np.abs(ref).max(), 1e-300))
        np.testing.assert_allclose(a[k], ref, rtol=1e-5, atol=1e-8, err_msg=k)
    return float(np.mean(a["height"] == o.height)), float(np.mean(a["sediment"] == o.sediment)), worst, s["clamped"], clamped


@pytest.mark.parametrize("name", ["c1", "n1024"])
def test_ordered_pass_at_benchmarked_worlds_matches_oracle(cuda, name):
    world, params, P = _world(name)
    same, same_s, worst, cl_gpu, cl_orc = _ordered_pass(world, params, P)
    print(f"{name}: one exact pass of {P} droplets: heights bit-identical in {same:.4%}, sediment in {same_s:.4%}; "
          f"largest difference / largest value {worst}; clamped entries {cl_gpu} vs {cl_orc}")
    assert same > 0.99 and same_s > 0.99
    assert abs(cl_gpu - cl_orc) <= 1e-3 * max(cl_orc, 1)
