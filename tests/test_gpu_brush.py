"""The erode / deposit brush (PgeParams.brush_radius; no reference counterpart).

The reference writes one cell a step (bake/globe/erosion/particle.py:662-671);
the brush spreads each applied erosion or deposition of the wave apply over
the active cells of its face within distance < r + 1, weights r + 1 -
distance, in int64 fixed point (shares truncated, the rest on the entry's own
cell).  Its oracle is the reference's own result composed with the brush
restated in numpy (oracle.brush_spread):

* isolated droplets of the N_c = 128 small world (the reference's change
  lists and serial apply, tests/golden/trace_isolated_c1.npz): the device's
  spread net change equals brush_spread of the reference's net change within
  1e-5 relative (the gate-1 tolerance), and sums to it;
* a full pass with r = 3 balances mass as the one-cell pass does, and repeats
  bit for bit.
"""
import dataclasses
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as orc
from pgerosion import _lib
from pgerosion import maps as gm
from pgerosion import synth
from tests.parity_cases import erosion_params
from tests.test_gpu_parity import _mass_balance

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).parent / "golden"


@pytest.mark.parametrize("r", [1, 3])
def test_brush_on_isolated_droplets_matches_reference_then_brush(cuda, r):
    t = np.load(GOLD / "trace_isolated_c1.npz")
    world = synth.plain_small_world(0)
    ep = dataclasses.replace(erosion_params(str(t["params"])), brush_radius=r)
    st = gm.ErosionState.from_world(world)
    res = gm.trace_changelist(st, ep, t["sp_face"], t["sp_x"], t["sp_y"], t["sp_sed"], t["sp_dir"], float(t["volume0"]),
                              float(t["conc_scale"]), precision=_lib.PREC_F64)
    ref = np.zeros(st.height.numel())
    ref[t["touched"]] = t["acc"]
    ref = ref.reshape(tuple(st.height.shape))
    want = orc.brush_spread(ref, np.ones(ref.shape, np.uint8), st.N, st.H, r, spherical=True)
    got = res["acc"]
    scale = np.abs(want).max()
    err = np.abs(got - want).max() / scale
    spread = np.count_nonzero(got) / max(np.count_nonzero(ref), 1)
    print(f"r={r}: {np.count_nonzero(ref)} cells changed without the brush, {np.count_nonzero(got)} with it "
          f"({spread:.1f}x); largest difference {err:.2e} of the largest change")
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-11 + 1e-9 * scale)
    assert abs(got.sum() - ref.sum()) <= 1e-9 * np.abs(ref).sum()  # conserving
    assert spread > 1.5


def test_brush_pass_balances_and_repeats(cuda):
    params, P = synth.config_params("small")
    params = dataclasses.replace(params, erosion=dataclasses.replace(params.erosion, brush_radius=3))
    w = synth.plain_small_world(0)
    outs = []
    for _ in range(2):
        g = gm.ErosionState.from_world(w)
        for it in range(2):
            m0 = g.total_mass()
            s = gm.run_iteration(g, params, it, n_particles=P, apply=_lib.APPLY_WAVE, wave=P)
            _mass_balance(s, m0, g.total_mass())
        outs.append(g.to_numpy())
    for k in outs[0]:
        assert outs[0][k].tobytes() == outs[1][k].tobytes(), k


def test_brush_needs_the_wave_apply(cuda):
    params, P = synth.config_params("small")
    params = dataclasses.replace(params, erosion=dataclasses.replace(params.erosion, brush_radius=2))
    g = gm.ErosionState.from_world(synth.plain_small_world(0))
    with pytest.raises(_lib.PgeError, match="brush"):
        gm.run_iteration(g, params, 0, n_particles=1024)
