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
        pp.check_plain(pp.ErosionParams())


def test_small_world_inputs():
    w = synth.plain_small_world(0)
    H, N = w.grid.H, w.grid.N
    inter = w.bedrock[:, H:H + N, H:H + N]
    assert abs(float((inter >= 0).mean()) - 0.30) < 1e-3
    assert inter.min() >= -4000.0 - 1e-3 and inter.max() <= 3000.0 + 1e-3
    assert w.bedrock.dtype == np.float32 and w.precip.min() == 1.0
    p, P = synth.config_params("small")
    assert P == 65536 and p.erosion.max_steps == 64 and p.world.N_c == 128
