"""The reference's conservation and stockpile tests on windows
(bake/tests/test_erosion.py:191-289), adapted to the device path: the same
invariants on single-face windows (spherical=False, deposit_on_exit) built by
``parity_cases.window_world`` (a closed bowl, a tilted coast, a walled
shelf).  Every statistic the device returns is summed in int64 fixed point
(2^-40 cell units), so the exactness bounds of the reference (1e-9 of the
values) hold with room to spare."""
import numpy as np
import pytest

from pgerosion import maps as gm
from tests.parity_cases import gpu_window, window_world

pytestmark = pytest.mark.gpu


def _sea_pending(st):
    s = (st.height + st.sediment)
    return float(st.pending[s < 0].sum())


def test_conservation_closed_window(cuda):
    arr, p = window_world("closed")
    st = gpu_window(arr)
    assert float((st.height + st.sediment)[st.interior].min()) > 0  # no ocean: nothing can leave as ocean deposit
    m0 = st.total_mass()
    clamped = 0
    for it in range(20):
        s = gm.step(st, p, it)
        assert s["particles"] > 0
        clamped += s["clamped"]
    m1 = st.total_mass()
    assert abs(m1 - m0) <= 1e-6 * abs(m0), (m0, m1)
    assert clamped > 0  # the live caps were exercised, and mass still balances
    assert float(st.sediment[st.interior].max()) > 0
    assert float(st.sediment.min()) >= 0 and float(st.pending.min()) >= 0


def test_offshore_loss_is_accounted(cuda):
    """Open coast: what leaves the surface is exactly lost_offshore; every
    sea-death surplus splits 1 - w : w between its cell's stockpile and the
    write-off (up to the dust the kernel writes off outright, as the
    reference's shelf test allows); the old rule (w = 1) deletes more and
    parks nothing."""
    out = {}
    for label, wo in (("park", None), ("delete", 1.0)):
        arr, p = window_world("tilt", writeoff=wo)
        w = p.erosion.offshore_writeoff
        st = gpu_window(arr)
        m0 = st.total_mass()
        lost = parked = 0.0
        for it in range(25):
            s = gm.step(st, p, it)
            lost += s["lost_offshore"]
            assert s["deficit_out"] <= 1e-12 * abs(m0)
            sea_pending = _sea_pending(st)
            parked += sea_pending
            # the kept share is (1 - w) / w of the write-off, less the dust written off outright (a
            # kept share under 1e-4 cell units) and less what later deposits lifted above the sea
            gap = (1.0 - w) / w * s["lost_offshore"] - sea_pending
            assert -1e-8 * (sea_pending + s["lost_offshore"]) <= gap <= 1e-2 * (1.0 - w) / w * s["lost_offshore"] + 1e-8, (label, it, gap)
        m1 = st.total_mass()
        assert abs((m1 + lost) - m0) <= 1e-6 * abs(m0), (label, m0, m1, lost)
        assert s["deaths"]["ocean"] > 0
        out[label] = (lost, parked)
    assert out["delete"][0] > 0.0 and out["delete"][1] == 0.0
    assert out["park"][1] > 0.0 and out["park"][0] < out["delete"][0], out


def test_seafloor_stockpile_is_bounded(cuda):
    """A shelf nothing can be placed on: the stockpile that comes back decays
    (each re-injection writes w of it off), a geometric series, where parking
    everything would grow linearly."""
    arr, p = window_world("shelf")
    w = p.erosion.offshore_writeoff
    st = gpu_window(arr)
    sea0 = (st.height + st.sediment) < 0
    assert bool(sea0[st.interior].any())
    m0 = st.total_mass()
    n = 40
    lost_k = np.zeros(n)
    pend_k = np.zeros(n)
    for it in range(n):
        s = gm.step(st, p, it)
        assert s["lost_offshore"] > 0.0, it
        lost_k[it] = s["lost_offshore"]
        pend_k[it] = _sea_pending(st)
        gap = (1.0 - w) / w * lost_k[it] - pend_k[it]
        assert -1e-8 * (pend_k[it] + lost_k[it]) <= gap <= 1e-2 * (1.0 - w) / w * lost_k[it] + 1e-8, (it, gap)
    assert bool(((st.height + st.sediment)[sea0] < 0.0).all())  # sea never turned into land
    m1 = st.total_mass()
    assert abs((m1 + lost_k.sum()) - m0) <= 1e-6 * abs(m0), (m0, m1, lost_k.sum())
    fresh = lost_k / w - np.concatenate([[0.0], pend_k[:-1]])
    assert fresh.max() > 0.0
    assert pend_k.max() <= (1.0 - w) / w * fresh.max() * (1.0 + 1e-8)
    assert pend_k[-1] < 0.25 * np.sum((1.0 - w) * fresh), (pend_k[-1], np.sum((1.0 - w) * fresh))
    assert pend_k[3 * n // 4:].max() < 2.0 * pend_k[n // 4: n // 2].max(), pend_k


def test_window_steps_with_inflow_follow_the_reference(cuda):
    """maps.step on a window with the cell-count discharge scales and part of
    the spawn weight declared as inflow across its edge (maps.py:913-917;
    the reference's own steps in tests/golden/window_steps.npz, which the
    oracle equals bit for bit): the hypsometry of the active interior within
    the chaotic bound of the plain steps after three iterations."""
    import json

    import torch

    from pgerosion.params import WorldGroup, WorldParams
    from tests.parity_cases import GOLDEN, erosion_params
    from tests.test_gpu_parity import HYPS_TOL_MANY

    t = np.load(GOLDEN / "window_steps.npz")
    ep = erosion_params(str(t["params"]))
    params = WorldParams(world=WorldGroup(seed=int(t["seed"]), N_c=int(t["N"]), cell_size_m=float(t["cell_size_m"]),
                                          land_fraction=float(t["land_fraction"]), halo=int(t["H"])), erosion=ep)
    dev = torch.device("cuda")
    f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64), device=dev)
    f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device=dev)
    NE = int(t["N"]) + 2 * int(t["H"])
    st = gm.ErosionState(height=f64(t["start_height"]), sediment=f64(t["start_sediment"]), discharge=f64(t["start_discharge"]),
                         momentum=f64(t["start_momentum"]), hardness=f32(t["hardness"]), precip=f32(t["precip"]),
                         evap=f32(t["evap"]), uplift=f64(np.zeros((1, NE, NE))),
                         mask=torch.as_tensor(np.ascontiguousarray(t["mask"], np.uint8), device=dev), metric=f32(t["metric"][0]),
                         metric_inv=f32(t["metric_inv"][0]), N=int(t["N"]), H=int(t["H"]), spherical=False,
                         height_unit_m=float(t["cell_size_m"]), base=f64(t["base"]), deposit_on_exit=True,
                         inflow_volume=float(t["inflow_volume"]))
    stats = json.loads(str(t["stats"]))
    for it in range(int(t["iterations"])):
        s = gm.step(st, params, it, n_particles=int(t["n_particles"]))
        if it == 0:  # later iterations re-inject stockpiles the run itself made
            assert s["particles"] == stats[it]["particles"]
    a = st.to_numpy()
    act = np.asarray(t["mask"]) == 1
    hg = np.percentile((a["height"] + a["sediment"])[act] * float(t["cell_size_m"]), [1, 5, 10, 25, 50, 75, 90, 95, 99])
    hr = np.percentile((t["height"] + t["sediment"])[act] * float(t["cell_size_m"]), [1, 5, 10, 25, 50, 75, 90, 95, 99])
    assert np.abs(hg - hr).max() <= HYPS_TOL_MANY, (hg, hr)
