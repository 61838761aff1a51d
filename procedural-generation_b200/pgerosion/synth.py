"""Seeded synthetic worlds for the erosion benchmarks and tests.

No real planet or dataset is used: every input field is generated here from
a seed, with the shapes, ranges and land fractions of the workloads the
stage is measured on (cube-sphere N_c = 128 / 1024 / 8192 worlds, a batch of
uneven worlds, a calibration world).

The bedrock is value-noise fBm evaluated on the unit sphere (a 3-D lattice
per octave, smoothstep-trilinear interpolation -- the same family of noise
as the bake's ``globe/stubs.py:fbm_at``, seamless across cube edges because
it lives in space), optionally plus ridged octaves ``1 - |2n - 1|``, then
mapped rank-preservingly onto ``[lo, 0)`` below and ``[0, hi]`` above the
land-fraction quantile.  Fields are computed on interior cells and their
halos filled with the grid's cubic halo exchange, as the bake's
``FaceField.load`` does for stage inputs.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .geometry import Grid, exchange_halos, get_grid


def _device():
    try:
        import torch

        return torch.device("cuda") if torch.cuda.is_available() else None
    except ImportError:  # pragma: no cover
        return None


def value_noise(p, rng: np.random.Generator, freq: float):
    """One octave of lattice value noise in [0, 1] at unit vectors ``p``
    (numpy array, or a float64 torch tensor on any device)."""
    n = int(np.ceil(freq)) + 2
    lattice = rng.random((n + 1, n + 1, n + 1))
    if not isinstance(p, np.ndarray):
        import torch

        lat = torch.as_tensor(lattice, device=p.device).reshape(-1)
        q = (p + 1.0) * 0.5 * freq
        i0 = torch.floor(q).to(torch.int64)
        t = q - i0
        t = t * t * (3.0 - 2.0 * t)
        i0 = i0.clamp(0, n - 1)
        out = torch.zeros(p.shape[:-1], dtype=p.dtype, device=p.device)
        for dx in (0, 1):
            wx = t[..., 0] if dx else 1.0 - t[..., 0]
            for dy in (0, 1):
                wy = t[..., 1] if dy else 1.0 - t[..., 1]
                for dz in (0, 1):
                    wz = t[..., 2] if dz else 1.0 - t[..., 2]
                    idx = ((i0[..., 0] + dx) * (n + 1) + (i0[..., 1] + dy)) * (n + 1) + (i0[..., 2] + dz)
                    out += wx * wy * wz * lat[idx]
        return out
    q = (p + 1.0) * 0.5 * freq
    i0 = np.floor(q).astype(np.int64)
    t = q - i0
    t = t * t * (3.0 - 2.0 * t)
    i0 = np.clip(i0, 0, n - 1)
    out = np.zeros(p.shape[:-1])
    for dx in (0, 1):
        wx = t[..., 0] if dx else 1.0 - t[..., 0]
        for dy in (0, 1):
            wy = t[..., 1] if dy else 1.0 - t[..., 1]
            for dz in (0, 1):
                wz = t[..., 2] if dz else 1.0 - t[..., 2]
                out += wx * wy * wz * lattice[i0[..., 0] + dx, i0[..., 1] + dy, i0[..., 2] + dz]
    return out


def fbm(p, rng: np.random.Generator, octaves: int = 6, base_freq: float = 2.0, ridged: bool = False):
    """Fractal sum of ``octaves`` octaves in [-1, 1] (ridged: in [0, 1])."""
    out = 0.0
    amp, total = 1.0, 0.0
    for o in range(octaves):
        n = value_noise(p, rng, base_freq * 2 ** o)
        out = out + amp * ((1.0 - abs(2.0 * n - 1.0)) if ridged else (2.0 * n - 1.0))
        total += amp
        amp *= 0.5
    return out / total


def _host(a) -> np.ndarray:
    return a if isinstance(a, np.ndarray) else a.detach().cpu().numpy()


def rank_map(v: np.ndarray, land_fraction: float, lo: float, hi: float) -> np.ndarray:
    """Monotone piecewise-linear map putting the ``1 - land_fraction`` quantile
    at 0, the minimum at ``lo`` and the maximum at ``hi``."""
    q = float(np.quantile(v, 1.0 - land_fraction))
    vmin, vmax = float(v.min()), float(v.max())
    return np.where(v < q, lo * (q - v) / max(q - vmin, 1e-30), hi * (v - q) / max(vmax - q, 1e-30))


def interior_points(grid: Grid, device=None):
    """(6, N, N, 3) unit vectors of the interior cell centres (a torch
    tensor on ``device`` when one is given)."""
    i = np.arange(grid.N) + grid.H
    EI, EJ = np.meshgrid(i, i, indexing="ij")
    p = np.stack([grid.centers_of(f, EI, EJ) for f in range(6)])
    if device is None:
        return p
    import torch

    return torch.as_tensor(p, device=device)


def _extend(grid: Grid, interior: np.ndarray, dtype) -> np.ndarray:
    H, N = grid.H, grid.N
    out = np.zeros((6, grid.NE, grid.NE), dtype=np.float64)
    out[:, H:H + N, H:H + N] = interior
    exchange_halos(grid, out)
    return out.astype(dtype)


@dataclass
class World:
    """Stage inputs of one synthetic world (extended (6, NE, NE) arrays, metres)."""

    grid: Grid
    bedrock: np.ndarray  # float32 m
    hardness: np.ndarray  # float32 [0, 1]
    precip: np.ndarray  # float32 spawn weight
    evap: np.ndarray  # float32 multiplier
    uplift: np.ndarray  # float32 m / iteration
    land_fraction: float


def plain_small_world(seed: int = 0, N: int = 128, H: int = 2, cell_size_m: float = 50.0, land_fraction: float = 0.30) -> World:
    """N_c = 128 world: 6-octave fBm bedrock mapped to -4000..+3000 m with 30 %
    of cells above 0, uniform rain 1.0, no uplift, hardness 0.5 +- 0.25 fBm,
    evaporation multiplier 1."""
    grid = get_grid(N, H, cell_size_m)
    rng = np.random.default_rng([seed, 128])
    p = interior_points(grid)
    bed = rank_map(fbm(p, rng, 6), land_fraction, -4000.0, 3000.0)
    hard = np.clip(0.5 + 0.25 * fbm(p, rng, 4), 0.0, 1.0)
    ones = np.ones((6, grid.NE, grid.NE), np.float32)
    return World(grid, _extend(grid, bed, np.float32), _extend(grid, hard, np.float32), ones.copy(), ones.copy(),
                 np.zeros((6, grid.NE, grid.NE), np.float32), land_fraction)


def earth_world(seed: int = 0, N: int = 1024, H: int = 2, cell_size_m: float = 9773.0, land_fraction: float = 0.29,
                device="auto") -> World:
    """Earth-default world: fBm (6 octaves) plus ridged noise (4 octaves)
    mapped to -8000..+6000 m with 29 % land; latitude-banded rain 0.1..3.0
    modulated by fBm; uplift 0..2 mm per iteration from fBm; hardness
    0.5 +- 0.25 fBm; evaporation multiplier 1.  The noise is evaluated on
    the GPU when one is present (``device="auto"``), in the same float64
    operations as on the host."""
    grid = get_grid(N, H, cell_size_m)
    rng = np.random.default_rng([seed, 1024])
    dev = _device() if device == "auto" else device
    p = interior_points(grid, dev)
    base = _host(fbm(p, rng, 6) + 0.6 * fbm(p, rng, 4, base_freq=4.0, ridged=True))
    bed = rank_map(base, land_fraction, -8000.0, 6000.0)
    ph = _host(p)
    lat = np.arcsin(np.clip(ph[..., 2], -1.0, 1.0))
    band = np.exp(-(lat / 0.25) ** 2) + 0.6 * np.exp(-((np.abs(lat) - 1.0) / 0.2) ** 2)
    band = band / band.max()
    rain = np.clip(0.1 + 2.9 * band * (0.6 + 0.8 * (0.5 + 0.5 * _host(fbm(p, rng, 4)))), 0.1, 3.0)
    upl = 0.002 * np.clip(0.5 + 0.5 * _host(fbm(p, rng, 4)), 0.0, 1.0)
    hard = np.clip(0.5 + 0.25 * _host(fbm(p, rng, 4)), 0.0, 1.0)
    ones = np.ones((6, grid.NE, grid.NE), np.float32)
    return World(grid, _extend(grid, bed, np.float32), _extend(grid, hard, np.float32),
                 np.clip(_extend(grid, rain, np.float32), 0.1, 3.0), ones, _extend(grid, upl, np.float32), land_fraction)


def config_params(name: str, seed: int = 0):
    """WorldParams and droplet count of a named workload.

    ``small``: N_c = 128, 65,536 droplets, max_steps 64, friction 0.05,
    erodibility 0.3, deposition 0.3, evaporation 0.01, 20 iterations.
    ``earth``: N_c = 1024, 6 N^2 / 4 droplets, max_steps 96, uplift replay,
    400 iterations.  Both run the plain path (every host-refreshed process
    off) with halo 2."""
    from .params import ErosionParams, WorldGroup, WorldParams, plain_knobs

    if name == "small":
        ep = ErosionParams(iterations=20, max_steps=64, friction=0.05, erodibility=0.3, deposition_rate=0.3,
                           evap_rate=0.01, uplift_mode="stack", **plain_knobs())
        return WorldParams(world=WorldGroup(seed=seed, N_c=128, cell_size_m=50.0, land_fraction=0.30, halo=2), erosion=ep), 65536
    if name == "earth":
        ep = ErosionParams(iterations=400, max_steps=96, uplift_mode="replay", **plain_knobs())
        return WorldParams(world=WorldGroup(seed=seed, N_c=1024, cell_size_m=9773.0, land_fraction=0.29, halo=2), erosion=ep), 6 * 1024 * 1024 // 4
    raise KeyError(name)
