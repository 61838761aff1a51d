"""The routing surface (ErosionState.refresh_route, globe/erosion/maps.py:351-358
and globe/erosion/route.py:31-125) on the device against the reference's own
flood: bit for bit on the fixture made by the reference (tests/golden/route_flood.npz),
on the sphere and on a window."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "procedural-generation_b200"))

pytestmark = pytest.mark.gpu


def _flood(fx, prefix, spherical):
    import ctypes

    import torch

    from pgerosion import _lib
    from pgerosion.maps import _ptr, _stream

    h = torch.as_tensor(fx[prefix + "height"], device="cuda")
    s = torch.as_tensor(fx[prefix + "sediment"], device="cuda")
    base = torch.as_tensor(fx["base"] if spherical else np.zeros_like(fx[prefix + "height"]), device="cuda")
    mask = torch.as_tensor(fx[prefix + "mask"], device="cuda")
    owner = torch.as_tensor(fx[prefix + "owner"].astype(np.int32), device="cuda")
    F, NE = h.shape[0], h.shape[1]
    N, H = int(fx["N"]), int(fx["H"])
    g = _lib.PgeGrid(F=F, N=N, H=H, spherical=int(spherical), metric_shared=1, max_steps=8, max_droplets=16, max_wave=16)
    L = _lib.load()
    ws = torch.empty(int(L.pge_workspace_bytes(ctypes.byref(g))), dtype=torch.uint8, device="cuda")
    st = _lib.PgeState(height=_ptr(h), sediment=_ptr(s), base=_ptr(base), mask=_ptr(mask))
    route = torch.empty_like(h)
    n = ctypes.c_int64(0)
    _lib.check(L.pge_route_flood(ctypes.byref(g), ctypes.byref(st), _ptr(owner), float(fx["eps"]), _ptr(route), 1 << 20,
                                 ctypes.byref(n), _ptr(ws), ws.numel(), _stream()), "pge_route_flood")
    torch.cuda.synchronize()
    return route.cpu().numpy(), int(n.value)


def test_route_flood_equals_the_reference_on_the_sphere(cuda):
    fx = np.load(ROOT / "tests" / "golden" / "route_flood.npz")
    got, sweeps = _flood(fx, "", True)
    H, N = int(fx["H"]), int(fx["N"])
    inter = (slice(None), slice(H, H + N), slice(H, H + N))
    assert sweeps > 0
    assert got[inter].tobytes() == fx["route"][inter].tobytes()
    assert (got > fx["height"] + fx["sediment"]).sum() > 0


def test_route_flood_equals_the_reference_on_a_window(cuda):
    fx = np.load(ROOT / "tests" / "golden" / "route_flood.npz")
    got, _ = _flood(fx, "w_", False)
    assert got.tobytes() == fx["w_route"].tobytes()


def test_refresh_route_on_a_state(cuda):
    """The state method: interior bit-identical to the oracle's flood, halos
    from the linear exchange, and the datum hold shifts the route with the
    terrain."""
    import torch

    from oracle import oracle as orc
    from pgerosion import maps as gm
    from pgerosion.synth import plain_small_world

    st = gm.ErosionState.from_world(plain_small_world(seed=4, N=24))
    eps = 1e-3
    st.refresh_route(eps)
    surf = (st.height + st.sediment).cpu().numpy()
    own = st.grid.owner
    want = orc.priority_flood_eps(surf, np.ones(surf.shape, np.uint8), own, st.H, st.N, eps, st.base.cpu().numpy())
    got = st.route.cpu().numpy()
    inter = st.interior
    assert got[inter].tobytes() == want[inter].tobytes()
    r0 = st.route.clone()
    q = gm.hold_datum(st, 0.5)
    assert q != 0.0
    torch.testing.assert_close(st.route, r0 - q, rtol=0, atol=0)


def test_routed_ordered_pass_matches_oracle(cuda):
    """One exact (ordered) pass with particles steering on the routing
    surface (particle.py:453-460, 556-559; the route flags following the live
    surface, particle.py:1010-1012) against the oracle's chunked serial pass
    on the same spawns, start terrain and route -- to the tolerance of the
    plain pass's parity test -- and the route changes the pass."""
    import torch

    from oracle import oracle as orc
    from pgerosion import maps as gm
    from tests.parity_cases import GOLDEN, step_case

    c = step_case(GOLDEN / "step_route.npz")
    ep = c["params"].erosion
    o = orc.OracleState.from_world(c["world"], c["params"])
    orc.start_replay(o, c["params"])
    eps = float(ep.route_eps) / o.height_unit_m
    orc.refresh_route(o, eps)
    f, x, y, v0 = orc.spawn_particles(o, c["n_particles"], c["params"].rng("erosion", 0))
    P = len(f)
    z = np.zeros(P)
    g = gm.ErosionState.from_world(c["world"])
    g.height.copy_(torch.as_tensor(o.height))
    g.route = torch.as_tensor(o.route.copy(), device="cuda")
    s = gm.apply_spawns(g, c["params"], f, x, y, z, z, v0)
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
    import ctypes

    lib = orc.lib()
    lib.orc_fold(ctypes.c_int64(o.height.size), orc._p(o.height), orc._p(o.sediment), orc._p(o.acc), orc._p(o.mask))
    lib.orc_ema(ctypes.c_int64(o.height.size), orc._p(o.discharge), orc._p(o.momentum), orc._p(o.disch_track), orc._p(o.mom_track),
                orc._p(o.mask), ctypes.c_double(float(ep.ema)))
    a = g.to_numpy()
    # a few trajectories differ in their last bits (libm: the face transfer, the discharge power), which
    # can flip a branch downstream and move the cells (and the tracks summed along) the rest of their
    # path; every other value within the plain pass's tolerance
    for k in ("height", "sediment", "discharge", "momentum", "pending"):
        want = getattr(o, k)
        off = ~np.isclose(a[k], want, rtol=1e-5, atol=1e-8)
        worst = np.abs(a[k] - want).max()
        assert off.mean() <= 5e-3 and worst <= 0.05 * max(np.abs(want).max(), 1e-12), (k, int(off.sum()), worst)
    assert np.mean(a["height"] == o.height) > 0.99
    assert abs(s["clamped"] - clamped) <= 1e-3 * clamped, (s["clamped"], clamped)
    # without the route the same pass ends elsewhere
    g2 = gm.ErosionState.from_world(c["world"])
    o2 = orc.OracleState.from_world(c["world"], c["params"])
    orc.start_replay(o2, c["params"])
    g2.height.copy_(torch.as_tensor(o2.height))
    gm.apply_spawns(g2, c["params"], f, x, y, z, z, v0)
    assert not np.array_equal(g2.to_numpy()["height"], a["height"])


def test_routed_steps_follow_the_reference(cuda):
    """maps.step with erosion.flood_every = 2 (the flood refreshed before
    iterations 0, 2 and 4): the hypsometry within the chaotic bound of the
    reference's own routed run, the routing surface of the final terrain
    bit-identical to the oracle's flood of it, and the mass balance of a
    routed pass."""
    from oracle import oracle as orc
    from pgerosion import maps as gm
    from tests.parity_cases import GOLDEN, hypsometry, step_case
    from tests.test_gpu_parity import HYPS_TOL_MANY, _mass_balance

    c = step_case(GOLDEN / "step_route.npz")
    t = c["t"]
    ep = c["params"].erosion
    g = gm.ErosionState.from_world(c["world"])
    gm.start_replay(g, c["params"])
    inter = g.interior
    for it in range(c["iterations"]):
        refresh = it % int(ep.flood_every) == 0
        s = gm.step(g, c["params"], it, n_particles=c["n_particles"])
        if refresh:
            assert s["seconds_route"] > 0.0
        assert g.route is not None
    a = g.to_numpy()
    hg = hypsometry(a["height"], a["sediment"], inter, 50.0)
    hr = hypsometry(t["height"], t["sediment"], inter, 50.0)
    assert np.abs(hg - hr).max() <= HYPS_TOL_MANY, (hg, hr)
    # the route of the final terrain against the oracle's flood of it
    g.refresh_route(float(ep.route_eps) / g.height_unit_m)
    surf = a["height"] + a["sediment"]
    want = orc.priority_flood_eps(surf, np.ones(surf.shape, np.uint8), g.grid.owner, g.H, g.N, float(ep.route_eps) / g.height_unit_m,
                                  g.base.cpu().numpy())
    assert g.route.cpu().numpy()[inter].tobytes() == want[inter].tobytes()
    # mass balance of one more routed pass
    m0 = g.total_mass()
    s = gm.run_iteration(g, c["params"], c["iterations"], n_particles=c["n_particles"])
    _mass_balance(s, m0, g.total_mass())
