"""Edge cases of the droplet pass on the device (needs a B200), against the
oracle where it has an answer.

* A world under the sea everywhere: no cell can spawn (the reference's
  ``spawn_weights`` are all zero, maps.py:793-807), the pass spawns nothing
  and changes nothing, and the step goes on (map passes, datum hold).
* A pass over no spawns at all (``apply_spawns`` with empty arrays), in both
  apply modes: the state is untouched.
* Waves of one droplet (the serial apply reduced to its definition): the
  exact apply and the order-free wave apply agree bit for bit, since no two
  droplets ever share a wave.
* Zero rain on land: spawns only where the rain is positive; a world with no
  rain at all spawns nothing.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as orc
from pgerosion import _lib
from pgerosion import maps as gm
from pgerosion import synth

pytestmark = pytest.mark.gpu

FIELDS = ("height", "sediment", "discharge", "momentum", "pending")


def _small(N=32, seed=3):
    w = synth.plain_small_world(seed, N=N)
    params, _ = synth.config_params("small")
    return w, params


def test_world_under_the_sea_spawns_nothing(cuda):
    w, params = _small()
    w.bedrock[...] = np.minimum(w.bedrock, -10.0)
    o = orc.OracleState.from_world(w, params)
    so = orc.run_iteration(o, params, 0, n_particles=2000)
    g = gm.ErosionState.from_world(w)
    before = g.to_numpy()
    s = gm.run_iteration(g, params, 0, n_particles=2000)
    assert s["particles"] == 0 and so["particles"] == 0
    after = g.to_numpy()
    for k in FIELDS:
        assert np.array_equal(before[k], after[k]), k
    st = gm.step(g, params, 1, n_particles=2000)  # the map passes run on regardless
    assert st["particles"] == 0


@pytest.mark.parametrize("apply", [_lib.APPLY_ORDERED, _lib.APPLY_WAVE])
def test_pass_over_no_spawns_changes_nothing(cuda, apply):
    w, params = _small()
    g = gm.ErosionState.from_world(w)
    before = g.to_numpy()
    z = np.zeros(0)
    s = gm.apply_spawns(g, params, np.zeros(0, np.int32), z, z, z, z, 1.0, apply=apply)
    assert s["droplets"] == 0 and s["entries"] == 0 and s["eroded"] == 0.0
    after = g.to_numpy()
    for k in ("height", "sediment", "pending"):
        assert np.array_equal(before[k], after[k]), k


def test_one_droplet_waves_agree_between_apply_modes(cuda):
    w, params = _small()
    o = orc.OracleState.from_world(w, params)
    f, x, y, v0 = orc.spawn_particles(o, 600, params.rng("erosion", 0))
    z = np.zeros(len(f))
    outs = []
    for apply in (_lib.APPLY_ORDERED, _lib.APPLY_WAVE):
        g = gm.ErosionState.from_world(w)
        gm.apply_spawns(g, params, f, x, y, z, z, v0, wave=1, apply=apply)
        outs.append(g.to_numpy())
    # the wave apply sums int64 fixed point (2^-40), the exact apply float64: with one droplet a wave both
    # are the serial apply, apart from the fixed point's rounding (which can turn a later droplet's step)
    for k in ("height", "sediment"):
        close = np.abs(outs[0][k] - outs[1][k]) <= 1e-9
        print(k, "cells within 1e-9:", close.mean())
        assert close.mean() > 0.99, k


def test_rain_only_where_it_falls(cuda):
    w, params = _small()
    H, N = w.grid.H, w.grid.N
    w.precip[...] = 0.0
    w.precip[1, H:H + N // 2, H:H + N // 2] = 1.0
    g = gm.ErosionState.from_world(w)
    rng = params.rng("erosion", 0)
    d = gm.spawn_rain(g, rng.random(1000), rng.random((1000, 2)))
    assert (d["face"] == 1).all()
    assert (d["x"] < N // 2 + 1e-9).all() and (d["y"] < N // 2 + 1e-9).all()
    w.precip[...] = 0.0
    g2 = gm.ErosionState.from_world(w)
    assert gm.run_iteration(g2, params, 0, n_particles=1000)["particles"] == 0
