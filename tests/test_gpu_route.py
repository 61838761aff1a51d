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
