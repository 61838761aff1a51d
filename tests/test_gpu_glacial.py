"""The glacial pass (erosion/glacial.py:162-257, the ice line of the
evaporation field) on the device against the oracle, which is pinned bit for
bit to the reference (tests/test_oracle.py), and steps with it on against the
reference's own run (tests/golden/step_glacial.npz).

Tolerances: the interior state and the pass's sums to 1e-12 relative (the
carved total and the margin weights are float64 sums whose order differs from
numpy's; the moraine is the carved total spread by the weights); cell counts
exactly."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "procedural-generation_b200"))

pytestmark = pytest.mark.gpu


def _pair():
    import torch

    from oracle import oracle as orc
    from pgerosion import maps as gm
    from tests.parity_cases import GOLDEN, step_case

    c = step_case(GOLDEN / "step_glacial.npz")
    t = c["t"]
    g = gm.ErosionState.from_world(c["world"])
    o = orc.OracleState.from_world(c["world"], c["params"])
    for k in ("height", "sediment", "discharge", "momentum", "pending"):
        getattr(g, k).copy_(torch.as_tensor(t[k]))
        getattr(o, k)[...] = t[k]
    return c, g, o


def test_glacial_pass_matches_oracle(cuda):
    from oracle import oracle as orc
    from pgerosion import maps as gm

    c, g, o = _pair()
    inter = g.interior
    for rep in range(2):  # the second pass reads the first's ice (erosion.glacial_sticky)
        sg = gm.glacial_carve(g, c["params"])
        so = orc.glacial_carve(o, c["params"])
        assert sg["ice_cells"] == so["ice_cells"] > 0 and sg["moraine_cells"] == so["moraine_cells"] > 0, rep
        for k in ("carved", "max_carve", "outwash"):
            assert abs(sg[k] - so[k]) <= 1e-12 * abs(so[k]), (rep, k, sg[k], so[k])
        a = g.to_numpy()
        for k in ("height", "sediment", "pending"):
            np.testing.assert_allclose(a[k][inter], getattr(o, k)[inter], rtol=1e-12, atol=1e-14, err_msg=f"{rep} {k}")
        assert np.array_equal(g.ice_prev.cpu().numpy().astype(bool), o.ice_prev)


def test_glacial_steps_follow_the_reference(cuda):
    """glacial_every = 2: the passes run when the reference's do, their ice
    and moraine within 2 % of the reference's cells (the states they carve
    drift apart in the last bits, as every run of this erosion does), and the
    hypsometry within the chaotic bound of the reference's run."""
    from pgerosion import maps as gm
    from tests.parity_cases import GOLDEN, hypsometry, step_case
    from tests.test_gpu_parity import HYPS_TOL_MANY

    c = step_case(GOLDEN / "step_glacial.npz")
    t = c["t"]
    g = gm.ErosionState.from_world(c["world"])
    gm.start_replay(g, c["params"])
    for it in range(c["iterations"]):
        s = gm.step(g, c["params"], it, n_particles=c["n_particles"])
        r = c["stats"][it]
        assert ("glacial" in s) == ("glacial" in r), it
        if "glacial" in s:
            for k in ("ice_cells", "moraine_cells"):
                assert abs(s["glacial"][k] - r["glacial"][k]) <= 0.02 * r["glacial"][k], (it, k, s["glacial"], r["glacial"])
            assert s["glacial"]["carved"] > 0.0
    a = g.to_numpy()
    hg = hypsometry(a["height"], a["sediment"], g.interior, 50.0)
    hr = hypsometry(t["height"], t["sediment"], g.interior, 50.0)
    assert np.abs(hg - hr).max() <= HYPS_TOL_MANY, (hg, hr)
