"""The bank cut on the outside of bends (erosion.lateral_rate,
particle.py:699-738) on the device, against the reference's fixtures
(tests/golden/lateral_trace.npz: a window trace + serial apply;
tests/golden/step_lateral.npz: sphere steps), which the oracle equals bit for
bit.  Tolerances as for the plain path: change lists of >= 99 % of the
droplets identical in cells and deaths with values within 1e-5 relative; a
pass within the routed pass's bound of the oracle's; steps within the
hypsometry bound."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as orc
from pgerosion import _lib
from pgerosion import maps as gm
from tests.parity_cases import GOLDEN, changelist_rows, hypsometry, step_case, window_case
from tests.test_gpu_parity import HYPS_TOL_MANY, _gpu_window_state

pytestmark = pytest.mark.gpu


def test_window_bank_cut_change_lists_match_reference(cuda):
    case = window_case(GOLDEN / "lateral_trace.npz")
    assert float(case["params"].lateral_rate) > 0.0
    st = _gpu_window_state(case)
    res = gm.trace_changelist(st, case["params"], case["sp_face"], case["sp_x"], case["sp_y"], case["sp_sed"], case["sp_dir"],
                              case["volume0"], case["conc_scale"], precision=_lib.PREC_F64)
    cap = case["cap"]
    rows = list(zip(changelist_rows(res, cap), changelist_rows(case, cap)))
    same = banks = 0
    for p, (a, b) in enumerate(rows):
        if res["sp_death"][p] != case["sp_death"][p] or not np.array_equal(a[0], b[0]) or not np.array_equal(a[2] == -2.0, b[2] == -2.0):
            continue
        banks += int((a[2] == -2.0).sum())
        if np.allclose(a[1], b[1], rtol=1e-5, atol=1e-12) and np.allclose(a[2], b[2], rtol=1e-5, atol=0) and \
                np.allclose(a[3], b[3], rtol=1e-5, atol=1e-7):
            same += 1
    assert same >= 0.99 * len(rows), (same, len(rows))
    assert banks > 1000


def test_window_bank_cut_ordered_pass_matches_oracle(cuda):
    case = window_case(GOLDEN / "lateral_trace.npz")
    ep = case["params"]
    g = _gpu_window_state(case)
    f, x, y, sed, dirs, v0 = case["sp_face"], case["sp_x"], case["sp_y"], case["sp_sed"], case["sp_dir"], case["volume0"]
    P = len(f)
    s = gm.apply_spawns(g, ep, f, x, y, sed, dirs, v0)
    o = orc.OracleState(height=case["height"].copy(), sediment=case["sediment"].copy(), discharge=case["discharge"].copy(),
                        momentum=case["momentum"].copy(), hardness=case["hardness"], precip=np.ones_like(case["hardness"]),
                        evap=case["evap"], uplift=np.zeros_like(case["height"]), mask=case["mask"], metric=case["metric"],
                        metric_inv=case["metric_inv"], N=case["N"], H=case["H"], spherical=False,
                        height_unit_m=case["cell_size_m"], base=case["base"].copy(), deposit_on_exit=bool(case["deposit_on_exit"]))
    chunk = orc.chunk_size(ep, P)
    o.pack()
    o.acc[...] = 0.0
    tp = orc.trace_params(o, ep, v0, chunk / (v0 * P))
    ap = orc.apply_params(o, ep, ep.iter_deposit / o.height_unit_m)
    cap = orc.change_list_cap(tp.max_steps, True)
    clamped = 0
    for c0 in range(0, P, chunk):
        sl = slice(c0, c0 + chunk)
        cl = orc.trace(o, tp, f[sl], x[sl], y[sl], sed[sl], dirs[sl], v0)
        clamped += orc.apply(o, ap, cl, cap)[0]
    lib = orc.lib()
    lib.orc_fold(ctypes.c_int64(o.height.size), orc._p(o.height), orc._p(o.sediment), orc._p(o.acc), orc._p(o.mask))
    lib.orc_ema(ctypes.c_int64(o.height.size), orc._p(o.discharge), orc._p(o.momentum), orc._p(o.disch_track), orc._p(o.mom_track),
                orc._p(o.mask), ctypes.c_double(float(ep.ema)))
    a = g.to_numpy()
    for k in ("height", "sediment", "discharge", "momentum", "pending"):
        want = getattr(o, k)
        off = ~np.isclose(a[k], want, rtol=1e-5, atol=1e-8)
        worst = np.abs(a[k] - want).max()
        assert off.mean() <= 5e-3 and worst <= 0.05 * max(np.abs(want).max(), 1e-12), (k, int(off.sum()), worst)
    assert np.mean(a["height"] == o.height) > 0.99
    assert abs(s["clamped"] - clamped) <= 1e-3 * clamped, (s["clamped"], clamped)


@pytest.mark.parametrize("apply", [_lib.APPLY_ORDERED, _lib.APPLY_WAVE])
def test_bank_cut_steps_follow_the_reference(cuda, apply):
    """Sphere steps with lateral_rate = 0.5 (ordered apply: the reference's
    semantics, the hypsometry within the chaotic bound; wave apply: the
    order-free ledger with the same bank entries), and the mass balance of
    one more pass over every cell.  On the sphere every cell is active, halo
    cells included, so a bank one cell across the flow can be a halo cell:
    the reference cuts it there and its next halo exchange overwrites the
    cut, so the balance holds over all cells of the pass, not over the
    interior (the oracle, bit-identical to the reference, shows the same)."""
    c = step_case(GOLDEN / "step_lateral.npz")
    t = c["t"]
    g = gm.ErosionState.from_world(c["world"])
    gm.start_replay(g, c["params"])
    for it in range(c["iterations"]):
        gm.step(g, c["params"], it, n_particles=c["n_particles"], apply=apply)
    a = g.to_numpy()
    inter = g.interior
    if apply == _lib.APPLY_ORDERED:
        # the wave apply is order-free (every droplet of a wave cuts against the wave's start terrain), not the
        # reference's serial model, so only the ordered apply is held to the reference's hypsometry
        hg = hypsometry(a["height"], a["sediment"], inter, 50.0)
        hr = hypsometry(t["height"], t["sediment"], inter, 50.0)
        assert np.abs(hg - hr).max() <= HYPS_TOL_MANY, (hg, hr)
    full = lambda: float((g.height + g.sediment + g.pending).sum().item())
    m0 = full()
    s = gm.run_iteration(g, c["params"], c["iterations"], n_particles=c["n_particles"], apply=apply)
    out = s["lost_offshore"] - s["deficit_out"]  # a deficit left at a list's end is mass the pass creates
    assert abs((full() - m0) + out) <= 1e-6 * max(s["eroded"], 1e-12), (m0, full(), s)
