"""The planet-wide 1.2 km level: one N_c = 8192 cube-sphere world on one GPU.

The reference reaches this resolution only by tiling the planet into zoom
windows (bake/globe/zoom/planet.py:65, docs/zoom-windows.md:815-820: 3.0 h of
tile time per 80 iterations on 20 cores); its global state cannot be built at
this size on the host (the Grid's float64 (6, NE, NE, 3) tables,
cubesphere.py:464-502).  Here the whole sphere is one state in HBM: the
geometry is one face-shared metric table and the halo tables, and the fields
are built on the device face by face, never as host arrays.

Workload: bedrock from a seeded N_c = 1024 fBm + ridge base upsampled
bicubically to N_c = 8192 per face, plus 3 octaves of detail noise, rank
mapped to -8000..+6000 m with ~29 % land (the land quantile taken from a
16 M-cell sample); latitude-banded rain 0.1..3.0 as the Earth-default world;
hardness 0.5 +- 0.25 fBm; no uplift.  2^24 droplets per iteration, max_steps
128, the wave apply with the erode / deposit brush of radius 2.

Device memory at N_c = 8192 (403 M extended cells): state ~32 GB (seven
float64 fields, momentum two; three float32 fields), the library workspace
~93 GB (packed samples, accumulators, spawn CDF, thermal scratch, the
ordered apply's per-cell words) and ~18 GB of spawn buffers sized for the
worst case of a stockpile on every cell: ~143 GB of the B200's 183 GB.
"""
from __future__ import annotations

import numpy as np
import torch

from . import maps as gm
from .geometry import get_grid
from .params import ErosionParams, WorldGroup, WorldParams, plain_knobs
from .synth import fbm

#: the 1.2 km level's cell: the Earth-default 9773 m cell at N_c = 1024 divided by 8
PLANET_CELL_M = 9773.0 * 1024 / 8192
PLANET_N = 8192
PLANET_DROPLETS = 1 << 24


def planet_params(seed: int = 0, N: int = PLANET_N, iterations: int = 200, brush_radius: int = 2):
    """The level's knobs: the plain path, max_steps 128, the brush of radius 2."""
    ep = ErosionParams(iterations=iterations, max_steps=128, uplift_mode="stack", brush_radius=brush_radius, **plain_knobs())
    cell = 9773.0 * 1024 / N
    return WorldParams(world=WorldGroup(seed=seed, N_c=N, cell_size_m=cell, land_fraction=0.29, halo=2), erosion=ep)


def _face_points(grid, f, device):
    """(N, N, 3) unit vectors of face f's interior cell centres, float64 on the device."""
    H, N = grid.H, grid.N
    i = np.arange(N) + H
    EI, EJ = np.meshgrid(i, i, indexing="ij")
    return torch.as_tensor(grid.centers_of(f, EI, EJ), device=device)


def _halo_fill(state, field64):
    """Fill the halo rows of a (6, NE, NE) float64 device field from its interior (the cubic tables)."""
    import ctypes

    from . import _lib
    from ._lib import PgeHalo

    dst, src, w, rot = state.halo_tables()
    h = PgeHalo(K=int(dst.shape[0]), dst=gm._ptr(dst), src=gm._ptr(src), w=gm._ptr(w), rot=gm._ptr(rot))
    _lib.check(_lib.load().pge_halo_gather(ctypes.byref(h), gm._ptr(field64), 0, gm._stream()), "pge_halo_gather")


def planet_state(seed: int = 0, N: int = PLANET_N, H: int = 2, device="cuda", base_n: int = 1024, land_fraction: float = 0.29):
    """The level's ErosionState, built on the device (see the module docstring)."""
    dev = torch.device(device)
    grid = get_grid(N, H, 9773.0 * 1024 / N)
    base_grid = get_grid(base_n, H, 9773.0)
    NE = grid.NE
    # one generator state per field, restored for every face (and row block) so that all of them draw
    # the same noise lattices
    base_state = np.random.default_rng([seed, N, 0]).bit_generator.state
    field_state = np.random.default_rng([seed, N, 1]).bit_generator.state
    rough = torch.empty((6, N, N), dtype=torch.float32, device=dev)
    for f in range(6):
        g = np.random.default_rng()
        g.bit_generator.state = base_state
        p = _face_points(base_grid, f, dev)
        coarse = fbm(p, g, 6) + 0.6 * fbm(p, g, 4, base_freq=4.0, ridged=True)
        up = torch.nn.functional.interpolate(coarse[None, None].float(), size=(N, N), mode="bicubic", align_corners=False)[0, 0]
        # 3 octaves of detail at the fine cells (the generator continues where the base left it: the same
        # lattices on every face)
        pf = _face_points(grid, f, dev)
        rough[f] = up + (0.5 ** 6) * fbm(pf, g, 3, base_freq=2.0 * 2 ** 6).float()
        del p, pf, coarse, up
    # rank map to -8000..+6000 m with land_fraction above 0 (the quantile from a 16 M-cell sample)
    flat = rough.reshape(-1)
    gen = torch.Generator(device=dev).manual_seed(seed)
    sample, _ = torch.sort(flat[torch.randint(0, flat.numel(), (1 << 24,), device=dev, generator=gen)])
    q = float(sample[int((1.0 - land_fraction) * (sample.numel() - 1))])
    vmin, vmax = float(flat.min()), float(flat.max())
    unit = grid.cell_size_m
    height = torch.zeros((6, NE, NE), dtype=torch.float64, device=dev)
    inter = height[:, H:H + N, H:H + N]
    for f in range(6):
        v = rough[f].double()
        inter[f] = torch.where(v < q, -8000.0 * (q - v) / max(q - vmin, 1e-30), 6000.0 * (v - q) / max(vmax - q, 1e-30)) / unit
    del rough, flat, sample
    # rain and hardness at the fine cells
    rain64 = torch.zeros((6, NE, NE), dtype=torch.float64, device=dev)
    hard64 = torch.zeros((6, NE, NE), dtype=torch.float64, device=dev)
    for f in range(6):
        g = np.random.default_rng()
        g.bit_generator.state = field_state
        pf = _face_points(grid, f, dev)
        lat = torch.asin(torch.clamp(pf[..., 2], -1.0, 1.0))
        band = torch.exp(-(lat / 0.25) ** 2) + 0.6 * torch.exp(-((lat.abs() - 1.0) / 0.2) ** 2)
        band = band / (1.0 + 0.6 * float(np.exp(-25.0)))  # the band's largest value (at the equator)
        rain64[f, H:H + N, H:H + N] = torch.clamp(0.1 + 2.9 * band * (0.6 + 0.8 * (0.5 + 0.5 * fbm(pf, g, 4))), 0.1, 3.0)
        hard64[f, H:H + N, H:H + N] = torch.clamp(0.5 + 0.25 * fbm(pf, g, 4), 0.0, 1.0)
        del pf, lat, band
    z = lambda: torch.zeros((6, NE, NE), dtype=torch.float64, device=dev)
    st = gm.ErosionState(height=height, sediment=z(), discharge=z(), momentum=torch.zeros((6, NE, NE, 2), dtype=torch.float64, device=dev),
                         hardness=torch.zeros((6, NE, NE), dtype=torch.float32, device=dev),
                         precip=torch.zeros((6, NE, NE), dtype=torch.float32, device=dev),
                         evap=torch.ones((6, NE, NE), dtype=torch.float32, device=dev), uplift=z(), mask=None,
                         metric=torch.as_tensor(np.ascontiguousarray(grid.metric_face), device=dev),
                         metric_inv=torch.as_tensor(np.ascontiguousarray(grid.metric_inv_face), device=dev), N=N, H=H,
                         spherical=True, height_unit_m=unit, grid=grid, land_target=land_fraction)
    st.exchange_halos()
    _halo_fill(st, rain64)
    _halo_fill(st, hard64)
    st.precip.copy_(torch.clamp(rain64, 0.1, 3.0).float())
    st.hardness.copy_(torch.clamp(hard64, 0.0, 1.0).float())
    del rain64, hard64
    torch.cuda.synchronize(dev)
    return st


class Timeline:
    """Heights (float32 metres of height + sediment, the interior faces) copied
    to pinned host memory every ``every`` iterations on a side stream, ordered
    after the iteration that made them; the copies overlap the next
    iterations.  ``frames`` holds (iteration, pinned tensor) pairs."""

    def __init__(self, state, every: int = 20, keep: int = 10):
        self.every, self.keep = int(every), int(keep)
        self.frames: list = []
        self._stream = torch.cuda.Stream()
        self._snap = None
        self._state = state

    def maybe(self, iteration: int) -> None:
        if self.every <= 0 or iteration % self.every != 0:
            return
        st = self._state
        H, N = st.H, st.N
        if self._snap is None:
            self._snap = torch.empty((6, N, N), dtype=torch.float32, device=st.height.device)
        # the snapshot on the iteration stream (after the side stream's previous copy out of it), the copy
        # to the host on the side stream
        torch.cuda.current_stream().wait_stream(self._stream)
        self._snap.copy_((st.height[:, H:H + N, H:H + N] + st.sediment[:, H:H + N, H:H + N]) * st.height_unit_m)
        host = torch.empty((6, N, N), dtype=torch.float32, pin_memory=True)
        ready = torch.cuda.Event()
        ready.record()
        with torch.cuda.stream(self._stream):
            self._stream.wait_event(ready)
            host.copy_(self._snap, non_blocking=True)
        self.frames.append((iteration, host))
        if len(self.frames) > self.keep:
            self.frames.pop(0)

    def wait(self) -> None:
        self._stream.synchronize()
