"""The sea mask (ErosionState.refresh_base, globe/erosion/maps.py:360-420 with
globe/hydro/run.py:64-83) on the device against the reference's: the base
level bit for bit and the statistics equal on the fixture the reference made
(tests/golden/step_sea.npz), and steps with the sea mask and the routing flood
on following the reference's own run."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "procedural-generation_b200"))

pytestmark = pytest.mark.gpu


def test_sea_base_equals_the_reference(cuda):
    import torch

    from pgerosion import maps as gm
    from tests.parity_cases import GOLDEN, step_case

    c = step_case(GOLDEN / "step_sea.npz")
    t = c["t"]
    g = gm.ErosionState.from_world(c["world"])
    g.height.copy_(torch.as_tensor(t["b_height"]))
    g.sediment.copy_(torch.as_tensor(t["b_sediment"]))
    info = g.refresh_base(float(t["ocean_min_fraction"]))
    assert info == json.loads(str(t["b_info"]))
    assert info["closed_basins"] > 0
    assert g.base.cpu().numpy().tobytes() == t["b_base"].tobytes()
    assert g.base_at == 0


def test_sea_masked_routed_steps_follow_the_reference(cuda):
    """sea_mask_every = flood_every = 2: each refresh's statistics as the
    reference's (counts exactly, the deepest floor to 1e-12: the replayed
    start differs from the reference's in the last bit), and the hypsometry
    within the chaotic bound of the reference's run."""
    from pgerosion import maps as gm
    from tests.parity_cases import GOLDEN, hypsometry, step_case
    from tests.test_gpu_parity import HYPS_TOL_MANY

    c = step_case(GOLDEN / "step_sea.npz")
    t = c["t"]
    g = gm.ErosionState.from_world(c["world"])
    g.refresh_base(float(t["ocean_min_fraction"]))
    gm.start_replay(g, c["params"])
    for it in range(c["iterations"]):
        s = gm.step(g, c["params"], it, n_particles=c["n_particles"])
        r = c["stats"][it]
        assert ("sea" in s) == ("sea" in r), it
        if it == 0:
            for k in ("closed_cells", "closed_basins", "sea_cells"):
                assert s["sea"][k] == r["sea"][k], (it, k)
            assert abs(s["sea"]["deepest_basin_floor"] - r["sea"]["deepest_basin_floor"]) <= 1e-12 * abs(r["sea"]["deepest_basin_floor"])
    a = g.to_numpy()
    hg = hypsometry(a["height"], a["sediment"], g.interior, 50.0)
    hr = hypsometry(t["height"], t["sediment"], g.interior, 50.0)
    assert np.abs(hg - hr).max() <= HYPS_TOL_MANY, (hg, hr)
