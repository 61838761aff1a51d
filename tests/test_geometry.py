"""Host geometry tables against the reference's Grid (golden fixture)."""
import hashlib
import json

import numpy as np

from pgerosion.geometry import Grid
from tests.parity_cases import GOLDEN


def test_halo_tables_match_reference():
    g = np.load(GOLDEN / "halo_N8_H2.npz")
    grid = Grid(8, 2, 50.0)
    hm = grid.halo
    for k in ("dst", "src", "nearest"):
        assert np.array_equal(getattr(hm, k), g[k]), k
    for k in ("w", "w_lin", "rot"):
        assert np.array_equal(getattr(hm, k), g[k]), k
    assert np.array_equal(grid.owner, g["owner"])
    assert np.array_equal(grid.metric_face, g["metric"])
    assert np.array_equal(grid.metric_inv_face, g["metric_inv"])


def test_halo_table_digests_match_reference():
    dig = json.loads(str(np.load(GOLDEN / "halo_N8_H2.npz")["digests"]))
    for N, H, c in ((16, 2, 50.0), (32, 4, 9773.0)):
        grid = Grid(N, H, c)
        hm = grid.halo
        for k in ("dst", "src", "w", "w_lin", "rot", "nearest"):
            assert hashlib.sha256(np.ascontiguousarray(getattr(hm, k)).tobytes()).hexdigest() == dig[f"{N}_{H}_{k}"], (N, k)
        assert hashlib.sha256(np.ascontiguousarray(grid.owner).tobytes()).hexdigest() == dig[f"{N}_{H}_owner"]
        assert hashlib.sha256(np.ascontiguousarray(grid.metric_face).tobytes()).hexdigest() == dig[f"{N}_{H}_metric"]


def test_halo_exchange_reproduces_smooth_field():
    from pgerosion.geometry import exchange_halos

    grid = Grid(32, 2, 50.0)
    c = grid.centers()
    f = c[..., 0] * 0.3 + c[..., 2] ** 2
    g = f.copy()
    g[:, :2] = 0
    g[:, -2:] = 0
    g[:, :, :2] = 0
    g[:, :, -2:] = 0
    exchange_halos(grid, g)
    assert np.abs(g - f).max() < 1e-4
