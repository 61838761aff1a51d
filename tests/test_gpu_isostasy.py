"""Isostasy on the device (maps.py:1331-1410) against the oracle, which is
pinned bit for bit to the reference (tests/test_oracle.py).

Tolerances: one smoothing step is bit-identical (the same float64
operations per cell and the same float32 rounding of the operator); the
step bound and a whole pass are within 1e-11 relative -- the power
iteration's norms, the halo gathers' sums and the mean are reductions whose
order differs from numpy's.
"""
import dataclasses

import numpy as np
import pytest
import torch

from oracle import oracle as orc
from pgerosion import isostasy as giso
from pgerosion import maps as gm
from tests.parity_cases import GOLDEN, step_case

pytestmark = pytest.mark.gpu


def _case():
    c = step_case(GOLDEN / "isostasy_tiny.npz")
    g = gm.ErosionState.from_world(c["world"])
    o = orc.OracleState.from_world(c["world"], c["params"])
    return c, g, o


def test_one_smoothing_step_is_bit_identical(cuda):
    from pgerosion.geometry import exchange_halos as xh

    c, g, o = _case()
    rng = np.random.default_rng(3)
    f = rng.standard_normal(o.height.shape)
    xh(o.grid, f, linear=True)
    kappa, cell = 0.083, float(o.height_unit_m)
    want = f + kappa * orc.laplacian(o, f).astype(np.float64) * (cell * cell)
    src = torch.as_tensor(f, device="cuda")
    dst = torch.empty_like(src)
    giso._step(g, src, dst, kappa, keep=True)
    assert dst.cpu().numpy().tobytes() == want.tobytes()
    # the bare operator in cell units (the step bound's power iteration)
    giso._step(g, src, dst, 1.0, keep=False)
    assert dst.cpu().numpy().tobytes() == (orc.laplacian(o, f).astype(np.float64) * (cell * cell)).tobytes()


def test_step_bound_matches_oracle(cuda):
    c, g, o = _case()
    kg = giso.smoothing_kappa(g)
    ko = orc.smoothing_kappa(o)
    assert abs(kg - ko) <= 1e-11 * ko
    assert abs(ko - float(c["t"]["kappa"])) == 0.0


def test_isostasy_pass_matches_oracle(cuda):
    c, g, o = _case()
    rng = np.random.default_rng(8)
    load = rng.normal(0.0, 0.5, o.height.shape)
    o.iso_acc = load.copy()
    g.iso_acc = torch.as_tensor(load.copy(), device="cuda")
    g.height.copy_(torch.as_tensor(o.height))
    so = orc.apply_isostasy(o, c["params"])
    sg = giso.apply_isostasy(g, c["params"])
    assert sg["diffusion_steps"] == so["diffusion_steps"] > 0
    for k in ("sigma_cells", "kappa", "load_abs_cells", "rebound_max", "rebound_min"):
        assert abs(sg[k] - so[k]) <= 1e-11 * max(abs(so[k]), 1e-300), k
    h = g.height.cpu().numpy()
    np.testing.assert_allclose(h, o.height, rtol=1e-11, atol=1e-11)
    assert float(g.iso_acc.abs().max()) == 0.0


def test_steps_schedule_isostasy_like_the_reference(cuda):
    """maps.step with isostasy on: the load is the particles' and the mass
    wasting's surface change, applied every isostasy_every iterations with
    the reference's step count; the plain passes are unchanged."""
    c, g, o = _case()
    gm.start_replay(g, c["params"])
    ref = c["stats"]
    for it in range(c["iterations"]):
        s = gm.step(g, c["params"], it, n_particles=c["n_particles"])
        assert ("isostasy" in s) == ("isostasy" in ref[it]), it
        if "isostasy" in s:
            assert s["isostasy"]["diffusion_steps"] == ref[it]["isostasy"]["diffusion_steps"]
            assert abs(s["isostasy"]["kappa"] - ref[it]["isostasy"]["kappa"]) <= 1e-11 * ref[it]["isostasy"]["kappa"]
            assert float(g.iso_acc.abs().max()) == 0.0
        else:
            assert float(g.iso_acc.abs().max()) > 0.0
    # without isostasy the same run ends elsewhere: the rebound is applied
    p2 = dataclasses.replace(c["params"], erosion=dataclasses.replace(c["params"].erosion, isostasy=0.0))
    g2 = gm.ErosionState.from_world(c["world"])
    gm.start_replay(g2, p2)
    for it in range(c["iterations"]):
        gm.step(g2, p2, it, n_particles=c["n_particles"])
    assert float((g.height - g2.height).abs().max()) > 1e-3
