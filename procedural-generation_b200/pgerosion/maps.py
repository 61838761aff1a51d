"""GPU erosion state and the per-iteration driver (the drop-in for the bake's
``globe.erosion.maps`` plain path).

Same names and argument meaning as the reference module
(bake/globe/erosion/maps.py):

* :class:`ErosionState` -- ``maps.ErosionState`` (maps.py:56-191), its arrays
  held as CUDA tensors: float64 height / sediment / discharge / momentum /
  pending / base / uplift, float32 hardness / precip / evap, uint8 mask, and
  the face-shared float32 metric tables.
* :func:`run_iteration` -- maps.py:839-1047: spawns drawn on the host by
  ``params.rng(rng_stage, *key)`` in the reference's order (rain uniforms,
  rain offsets, then the stockpiles' directions), inverse CDF, stockpile
  re-injection and the droplet pass on the device (``pge_spawn_rain``,
  ``pge_collect_pending``, ``pge_trace_apply``).  Returns the reference's
  stats dict.
* :func:`thermal_erosion`, :func:`apply_uplift`, :func:`start_replay`,
  :func:`hold_datum`, :func:`step` -- maps.py:1050-1213, 1446-1617, plain path.

Waves.  The reference freezes the terrain for a chunk of particles and
applies their changes serially; here a wave of ``wave`` droplets is traced on
frozen terrain and each droplet applies its own ledger (see
``csrc/pge_droplets.cuh``).  ``wave=None`` uses the reference's own chunk
size (``erosion.chunk`` / 16 chunks minimum); a larger wave keeps more of
the GPU busy, and the trace-time concurrency divisor ``conc_scale`` follows
the wave size as the reference's follows its chunk.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import PgeGrid, PgeHalo, PgeParams, PgeSpawns, PgeState, PgeStats, check
from .params import cell_units, check_plain, chunk_size, erosion_group, max_steps_of

MASK_OUTSIDE, MASK_ACTIVE, MASK_FROZEN = 0, 1, 2


def _ptr(t: torch.Tensor | None):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


@dataclass
class ErosionState:
    """GPU-resident erosion state (see the module docstring)."""

    height: torch.Tensor
    sediment: torch.Tensor
    discharge: torch.Tensor
    momentum: torch.Tensor
    hardness: torch.Tensor
    precip: torch.Tensor
    evap: torch.Tensor
    uplift: torch.Tensor
    mask: torch.Tensor | None
    metric: torch.Tensor  # (NE, NE, 3) float32, shared by every face
    metric_inv: torch.Tensor
    N: int
    H: int
    spherical: bool
    height_unit_m: float
    grid: object = None
    pending: torch.Tensor = None
    base: torch.Tensor = None
    iteration: int = 0
    land_target: float | None = None
    deposit_on_exit: bool = False
    #: window mode: the part of the spawn weight that is water flowing in across the window's edge, not rain on it
    #: (zoom tiles); excluded from the rain per cell the cell-count discharge scales use
    inflow_volume: float = 0.0
    max_droplets: int = 0
    max_steps: int = 0
    max_wave: int = 0
    wave_tables: bool = False
    #: the wave apply's resident droplet threads with own-change tables (0: the GPU's maximum); set lower
    #: (then call reserve) for a world that shares the GPU with others, to keep its workspace small
    max_threads: int = 0
    _ws_threads: int = field(default=-1, repr=False)
    _ws: torch.Tensor = field(default=None, repr=False)
    _halo: tuple = field(default=None, repr=False)
    _erode_cap: torch.Tensor = field(default=None, repr=False)
    iso_acc: torch.Tensor = field(default=None, repr=False)
    #: per-cell multiplier of erosion.erodibility (float32, (F, NE, NE)) or None: the calibrated field of the
    #: adjoint (pgerosion.adjoint); the wave apply only
    erodibility: torch.Tensor = field(default=None, repr=False)
    #: the epsilon-filled routing surface (float64, (F, NE, NE), cell units) or None (refresh_route)
    route: torch.Tensor = field(default=None, repr=False)
    #: overflowing lakes (uint8, (F, NE, NE): 1 a lake, 2 a lake with room for its rivers' load; maps.py:87) or None:
    #: set by the caller (the hydro stage's balance) or by refresh_lakes_window; read with the routing surface only
    lake_flag: torch.Tensor = field(default=None, repr=False)
    #: the share of a droplet's exchange with the bed the plants hold back (float32 (F, NE, NE) in [0, 1],
    #: erosion.vegetation) or None: bare ground
    roots: torch.Tensor = field(default=None, repr=False)
    #: the potential evaporation the planet's lake balance runs on (float32, (F, NE, NE)) in place of evap, or None
    lake_pet: torch.Tensor = field(default=None, repr=False)
    #: the lake parks (erosion.lake_fill, maps.py:105-107): float64 load per cell that droplets parked in a lake with
    #: room since the last refresh, the int32 lake of lake_room each cell belongs to (-1 none), and float64 room per
    #: lake; None until the first pass with parks
    lake_load: torch.Tensor = field(default=None, repr=False)
    lake_id: torch.Tensor = field(default=None, repr=False)
    lake_room: torch.Tensor = field(default=None, repr=False)
    #: the open sea of the last sea-mask refresh (bool, (F, N, N)), the lake balance's drains; None before the first
    sea_mask: torch.Tensor = field(default=None, repr=False)
    #: iteration of the last sea-mask refresh (refresh_base), None before the first
    base_at: int = None
    #: the last glacial pass's ice (uint8, (F, NE, NE)) for erosion.glacial_sticky, None before the first
    ice_prev: torch.Tensor = field(default=None, repr=False)
    _owner: torch.Tensor = field(default=None, repr=False)
    _sea: tuple = field(default=None, repr=False)
    _spawn: dict = field(default=None, repr=False)
    _lake_inputs: tuple = field(default=None, repr=False)
    _centres: np.ndarray = field(default=None, repr=False)

    def __post_init__(self):
        dev = self.height.device
        if dev.type != "cuda":
            raise RuntimeError("ErosionState lives on a CUDA device (the b200 backend has no CPU path)")
        if self.pending is None:
            self.pending = torch.zeros_like(self.height)
        if self.base is None:
            self.base = torch.zeros_like(self.height)

    # -- constructors ----------------------------------------------------------
    @classmethod
    def from_arrays(cls, grid, height, sediment, discharge, momentum, hardness, precip, evap, uplift, mask=None,
                    height_unit_m=None, pending=None, base=None, device="cuda", land_target=None) -> "ErosionState":
        """From (6, NE, NE[, 2]) numpy arrays already in cell units."""
        d = torch.device(device)
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=d)
        f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=d)
        m = None if mask is None or np.all(np.asarray(mask) == MASK_ACTIVE) else torch.as_tensor(np.ascontiguousarray(mask, np.uint8), device=d)
        return cls(height=f64(height), sediment=f64(sediment), discharge=f64(discharge), momentum=f64(momentum),
                   hardness=f32(hardness), precip=f32(precip), evap=f32(evap), uplift=f64(uplift), mask=m,
                   metric=f32(grid.metric_face), metric_inv=f32(grid.metric_inv_face), N=grid.N, H=grid.H, spherical=True,
                   height_unit_m=float(grid.cell_size_m if height_unit_m is None else height_unit_m), grid=grid,
                   pending=None if pending is None else f64(pending), base=None if base is None else f64(base),
                   land_target=land_target)

    @classmethod
    def from_grid(cls, grid, bedrock_m, hardness, precip, evap, uplift_m, eparams=None, mask=None, device="cuda") -> "ErosionState":
        """Global six-face state from extended arrays in metres, as the
        reference's ``ErosionState.from_grid`` (maps.py:152-191) builds it."""
        unit = float(grid.cell_size_m)
        arr = lambda x: np.asarray(getattr(x, "data", x))
        F, NE = 6, grid.NE
        return cls.from_arrays(grid, arr(bedrock_m).astype(np.float64) / unit, np.zeros((F, NE, NE)), np.zeros((F, NE, NE)),
                               np.zeros((F, NE, NE, 2)), arr(hardness), arr(precip), arr(evap),
                               arr(uplift_m).astype(np.float64) / unit, mask=mask, height_unit_m=unit, device=device)

    @classmethod
    def from_world(cls, world, device="cuda") -> "ErosionState":
        st = cls.from_grid(world.grid, world.bedrock, world.hardness, world.precip, world.evap, world.uplift, device=device)
        st.land_target = float(world.land_fraction)
        return st

    # -- views ------------------------------------------------------------------
    @property
    def F(self) -> int:
        return self.height.shape[0]

    @property
    def NE(self) -> int:
        return self.height.shape[1]

    @property
    def interior(self):
        H, N = self.H, self.N
        return (slice(None), slice(H, H + N), slice(H, H + N))

    def surface(self) -> torch.Tensor:
        return self.height + self.sediment

    def total_mass(self) -> float:
        """Sum of height + sediment + pending (+ lake_load, the loads parked in
        lakes) over the active interior (cell units), as maps.py:323-326."""
        t = self.height + self.sediment + self.pending
        if self.lake_load is not None:
            t = t + self.lake_load
        t = t[self.interior]
        if self.mask is not None:
            t = t[self.mask[self.interior] == MASK_ACTIVE]
        return float(t.sum().item())

    def to_numpy(self) -> dict:
        return {k: getattr(self, k).detach().cpu().numpy() for k in ("height", "sediment", "discharge", "momentum", "pending", "base")}

    # -- library plumbing ---------------------------------------------------------
    def pge_grid(self) -> PgeGrid:
        return PgeGrid(F=self.F, N=self.N, H=self.H, spherical=int(bool(self.spherical)),
                       deposit_on_exit=int(bool(self.deposit_on_exit)), metric_shared=1, max_steps=int(self.max_steps),
                       wave_tables=int(self.wave_tables), max_droplets=int(self.max_droplets), max_wave=int(self.max_wave),
                       max_threads=int(self.max_threads))

    def pge_state(self, parks: bool = False) -> PgeState:
        """The C view of the state; with ``parks`` the lake parks' arrays
        (:meth:`ensure_lake_parks` first), else none (parks off)."""
        ps = PgeState(height=_ptr(self.height), sediment=_ptr(self.sediment), discharge=_ptr(self.discharge),
                      momentum=_ptr(self.momentum), pending=_ptr(self.pending), base=_ptr(self.base), uplift=_ptr(self.uplift),
                      hardness=_ptr(self.hardness), precip=_ptr(self.precip), evap=_ptr(self.evap), mask=_ptr(self.mask),
                      metric=_ptr(self.metric), metric_inv=_ptr(self.metric_inv), erodibility=_ptr(self.erodibility),
                      route=_ptr(self.route), lake_flag=_ptr(self.lake_flag), roots=_ptr(self.roots))
        if parks:
            ps.lake_load, ps.lake_id, ps.lake_room = _ptr(self.lake_load), _ptr(self.lake_id), _ptr(self.lake_room)
            ps.lakes = int(self.lake_room.numel())
        return ps

    def ensure_lake_parks(self) -> None:
        """The lake parks' arrays at their initial values (maps.py:128-133):
        no load parked, no lake numbered, one zero room."""
        dev = self.height.device
        if self.lake_load is None:
            self.lake_load = torch.zeros_like(self.height)
        if self.lake_id is None:
            self.lake_id = torch.full(self.height.shape, -1, dtype=torch.int32, device=dev)
        if self.lake_room is None:
            self.lake_room = torch.zeros(1, dtype=torch.float64, device=dev)

    def reserve(self, max_droplets: int, max_steps: int, max_wave: int = 1, wave_tables: bool = False) -> None:
        """Size the library workspace and spawn buffers for up to
        ``max_droplets`` spawns of ``max_steps`` steps and ordered-apply
        waves of up to ``max_wave`` droplets (grows, never shrinks)."""
        if (max_droplets <= self.max_droplets and max_steps <= self.max_steps and max_wave <= self.max_wave
                and (self.wave_tables or not wave_tables) and self._ws is not None and self._ws_threads == self.max_threads):
            return
        self._ws_threads = int(self.max_threads)
        self._ws = None  # the old workspace goes before the new one is made
        self.wave_tables = bool(self.wave_tables or wave_tables)
        self.max_droplets = max(int(max_droplets), self.max_droplets)
        self.max_steps = max(int(max_steps), self.max_steps)
        self.max_wave = max(int(max_wave), self.max_wave, 1)
        L = _lib.load()
        g = self.pge_grid()
        nbytes = int(L.pge_workspace_bytes(ctypes.byref(g)))
        if nbytes == 0:
            raise _lib.PgeError("pge_workspace_bytes rejected the grid: " + _lib.last_error())
        self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.height.device)
        n = self.max_droplets
        d = self.height.device
        self._spawn = {
            "face": torch.empty(n, dtype=torch.int32, device=d),
            "x": torch.empty(n, dtype=torch.float64, device=d),
            "y": torch.empty(n, dtype=torch.float64, device=d),
            "sed": torch.empty(n, dtype=torch.float64, device=d),
            "dir": torch.empty(n, dtype=torch.float64, device=d),
            "scal": torch.zeros(4, dtype=torch.float64, device=d),  # spawn total weight, datum shift
            "cnt": torch.zeros(4, dtype=torch.int64, device=d),  # spawnable cells, stockpiles
            "stats": torch.zeros(_lib.STATS_WORDS, dtype=torch.int64, device=d),
            "host_scal": torch.zeros(4, dtype=torch.float64).pin_memory(),
            "host_cnt": torch.zeros(4, dtype=torch.int64).pin_memory(),
            "host_stats": torch.zeros(_lib.STATS_WORDS, dtype=torch.int64).pin_memory(),
        }

    @property
    def workspace(self) -> torch.Tensor:
        return self._ws

    def halo_tables(self, linear: bool = False):
        """The grid's halo tables on the device (dst, src, weights, rotations):
        cubic weights by default, the monotone linear ones with ``linear``."""
        if self._halo is None:
            hm = self.grid.halo
            d = self.height.device
            self._halo = (torch.as_tensor(hm.dst.astype(np.int32), device=d), torch.as_tensor(hm.src.astype(np.int32), device=d),
                          torch.as_tensor(hm.w, device=d), torch.as_tensor(np.ascontiguousarray(hm.rot), device=d),
                          torch.as_tensor(np.ascontiguousarray(hm.w_lin), device=d))
        dst, src, w, rot, wl = self._halo
        return dst, src, (wl if linear else w), rot

    def exchange_field(self, field: torch.Tensor, vector: bool = False, linear: bool = False) -> None:
        """Fill the halos of one (F, NE, NE[, 2]) float64 field from its interior
        (FaceField.exchange_halos, field.py:104-125)."""
        if not self.spherical:
            return
        dst, src, w, rot = self.halo_tables(linear)
        h = PgeHalo(K=int(dst.shape[0]), dst=_ptr(dst), src=_ptr(src), w=_ptr(w), rot=_ptr(rot))
        check(_lib.load().pge_halo_gather(ctypes.byref(h), _ptr(field), 1 if vector else 0, _stream()), "pge_halo_gather")

    def exchange_halos(self) -> None:
        """Refresh the halos of height, sediment, discharge and the rotated
        momentum (maps.py:329-340)."""
        if not self.spherical:
            return
        dst, src, w, rot = self.halo_tables()
        h = PgeHalo(K=int(dst.shape[0]), dst=_ptr(dst), src=_ptr(src), w=_ptr(w), rot=_ptr(rot))
        L = _lib.load()
        st = _stream()
        for t in (self.height, self.sediment, self.discharge):
            check(L.pge_halo_gather(ctypes.byref(h), _ptr(t), 0, st), "pge_halo_gather")
        check(L.pge_halo_gather(ctypes.byref(h), _ptr(self.momentum), 1, st), "pge_halo_gather")

    def owner_table(self) -> torch.Tensor:
        """int32 flat index of the interior cell owning every extended cell
        (cubesphere.py:664-674; the identity for a window), on the device."""
        if self._owner is None:
            F, NE = self.F, self.N + 2 * self.H
            own = self.grid.owner if self.spherical else np.arange(F * NE * NE).reshape(F, NE, NE)
            self._owner = torch.as_tensor(np.ascontiguousarray(own, dtype=np.int32), device=self.height.device)
        return self._owner

    def refresh_route(self, eps: float, max_sweeps: int = 1 << 22) -> int:
        """Recompute the routing surface from the current terrain
        (maps.py:351-358: route.priority_flood_eps, then the linear halo
        exchange); returns the relaxation sweeps run."""
        _ensure_workspace(self)
        if self.route is None or self.route.shape != self.height.shape:
            self.route = torch.empty_like(self.height)
        n = ctypes.c_int64(0)
        check(_lib.load().pge_route_flood(ctypes.byref(self.pge_grid()), ctypes.byref(self.pge_state()), _ptr(self.owner_table()),
                                          float(eps), _ptr(self.route), int(max_sweeps), ctypes.byref(n), _ptr(self.workspace),
                                          self.workspace.numel(), _stream()), "pge_route_flood")
        self.exchange_field(self.route, linear=True)
        return int(n.value)

    def refresh_lakes_window(self, min_depth: float, lake_evap: float = 0.0) -> dict:
        """The lakes of a window (maps.py:629-736, erosion.window_lakes): every
        depression the routing surface fills more than ``min_depth`` (cell
        units) deep is an overflowing lake, flagged on the interior's active
        cells; particles cross it without touching the bed, drop their load at
        its shore and are not counted as climbing inside it.  With
        ``lake_evap > 0`` (erosion.window_lake_evap) each depression settles
        where the rain reaching it meets its evaporation instead
        (``pge_window_lake_balance``, a host pass over the flat flood), and the
        routing surface is lowered to the water on its lake cells.  Must run
        after :meth:`refresh_route`."""
        if self.lake_flag is None or self.lake_flag.shape != self.height.shape:
            self.lake_flag = torch.zeros(self.height.shape, dtype=torch.uint8, device=self.height.device)
        if self.route is None:
            self.lake_flag.zero_()
            return {"lake_cells": 0}
        if float(lake_evap) > 0.0:
            if self.spherical or self.F != 1:
                raise ValueError("the evaporation balance of window lakes runs on a window (F = 1)")
            host = lambda t: np.ascontiguousarray(t.detach().cpu().numpy())
            surf = host((self.height + self.sediment)[0].float())
            active = host(self.mask[0] == MASK_ACTIVE) if self.mask is not None else np.ones(surf.shape, bool)
            active = np.ascontiguousarray(active, np.uint8)
            precip = host(self.precip[0])
            evap = host(self.evap[0])
            route = host(self.route[0]).copy()
            lake = np.empty(surf.shape, np.uint8)
            counts = np.zeros(5, np.int64)
            check(_lib.load().pge_window_lake_balance(ctypes.byref(self.pge_grid()), surf.ctypes.data, active.ctypes.data,
                                                      precip.ctypes.data, evap.ctypes.data, float(lake_evap), float(min_depth),
                                                      route.ctypes.data, lake.ctypes.data, counts.ctypes.data),
                  "pge_window_lake_balance")
            dev = self.height.device
            self.route[0] = torch.as_tensor(route, device=dev)
            H, N = self.H, self.N
            self.lake_flag.zero_()
            self.lake_flag[0, H:H + N, H:H + N] = torch.as_tensor(lake[H:H + N, H:H + N], device=dev)
            return {"lake_cells": int(lake[H:H + N, H:H + N].sum()), "depressions": int(counts[0]), "overflowing": int(counts[1]),
                    "closed": int(counts[2]), "dry": int(counts[3])}
        n = torch.zeros(1, dtype=torch.int64, device=self.height.device)
        check(_lib.load().pge_window_lakes(ctypes.byref(self.pge_grid()), ctypes.byref(self.pge_state()), float(min_depth),
                                           _ptr(self.lake_flag), _ptr(n), _stream()), "pge_window_lakes")
        return {"lake_cells": int(n.item())}

    def refresh_base(self, min_fraction: float = 0.02, max_sweeps: int = 1 << 22) -> dict:
        """Recompute the base level (maps.py:360-420): 0 on the open ocean
        and on land, a closed below-sea basin's deepest surface on its cells
        (hydro/run.py:64-83: a below-sea body is open ocean when it covers
        ``min_fraction`` of the globe, and the largest always is); halos
        copied from their nearest interior source.  Returns the reference's
        statistics."""
        info = {"closed_cells": 0, "closed_basins": 0, "sea_cells": 0, "deepest_basin_floor": 0.0}
        if not self.spherical:
            self.base = torch.zeros_like(self.height)
            self.base_at = self.iteration
            return info
        base, labels = self._sea_base(min_fraction, max_sweeps)
        b = base[self.interior]
        below = labels >= 0
        closed = below & (b < 0.0)
        self.sea_mask = below & ~closed
        info["sea_cells"] = int(self.sea_mask.sum().item())
        info["closed_cells"] = int(closed.sum().item())
        if info["closed_cells"]:
            info["closed_basins"] = int(torch.unique(labels[closed]).numel())
            info["deepest_basin_floor"] = float(b[closed].min().item())
        self.base = base
        self.base_at = self.iteration
        return info

    def _sea_tables(self):
        """(interior cell areas float32 (F, N, N), their float64 sum, halo dst, halo nearest) on the device."""
        if self._sea is None:
            from .isostasy import sqrt_det_metric

            dev = self.height.device
            H, N = self.H, self.N
            sq = sqrt_det_metric(self.grid)[H:H + N, H:H + N]
            area = np.ascontiguousarray(np.broadcast_to((sq.astype(np.float64) * float(self.grid.cell_size_m) ** 2)
                                                        .astype(np.float32), (self.F, N, N)))
            hm = self.grid.halo
            self._sea = (torch.as_tensor(area, device=dev), float(area.reshape(-1).astype(np.float64).sum()),
                         torch.as_tensor(hm.dst.astype(np.int64), device=dev), torch.as_tensor(hm.nearest.astype(np.int64), device=dev))
        return self._sea

    def _sea_base(self, min_fraction: float, max_sweeps: int = 1 << 22):
        """pge_sea_base of the current surface: (base (F, NE, NE) with its halos copied from their nearest
        interior cells, component labels (F, N, N))."""
        _ensure_workspace(self)
        area, total, dst, nearest = self._sea_tables()
        base = torch.empty_like(self.height)
        labels = torch.empty((self.F, self.N, self.N), dtype=torch.int32, device=self.height.device)
        n = ctypes.c_int64(0)
        check(_lib.load().pge_sea_base(ctypes.byref(self.pge_grid()), ctypes.byref(self.pge_state()), _ptr(self.owner_table()),
                                       _ptr(area), float(min_fraction) * total, _ptr(base), _ptr(labels), int(max_sweeps),
                                       ctypes.byref(n), _ptr(self.workspace), self.workspace.numel(), _stream()), "pge_sea_base")
        flat = base.view(-1)
        flat[dst] = flat[nearest]  # the halo is an exact copy of the cell it mirrors (a jump at a basin rim)
        return base, labels

    def refresh_lakes(self, lake_evap: float, min_depth: float, min_fraction: float = 0.02, land_evap: float = 0.0,
                      fill: tuple | None = None) -> dict:
        """The planet's lakes (maps.py:422-479, erosion.lake_balance): the
        hydro stage's flood, D8 routing and evaporation balance on the
        eroding surface (``pge_lake_balance``, a host pass: its every step
        follows the flood's serial pop order).  Overflowing lakes deeper than
        ``min_depth`` (cell units) are flagged (``lake_flag``); a lake drawn
        below its rim is a closed sea, its level written into ``base``.  The
        drains are the sea of the last :meth:`refresh_base`, else the open
        ocean of the current surface; the balance runs on ``lake_pet`` when
        set, else ``evap``.  Must run after :meth:`refresh_base` and
        :meth:`refresh_route`.  With ``fill`` (:func:`lake_fill_args`,
        erosion.lake_fill) the lakes first take the loads parked on them
        (``pge_lake_balance_fill``, maps.py:490-628): laid over their floors
        as sediment (and isostatic load), the lakes with room numbered in
        ``lake_id`` / ``lake_room`` and flagged 2."""
        if not self.spherical:
            raise ValueError("refresh_lakes is the planet's lake balance; a window's lakes come from refresh_lakes_window")
        inter = self.interior
        if self.sea_mask is not None:
            sea = self.sea_mask
        else:
            sb, labels = self._sea_base(min_fraction)
            sea = (labels >= 0) & (sb[inter] == 0.0)
        area, _, dst, nearest = self._sea_tables()
        pet = self.lake_pet if self.lake_pet is not None else self.evap
        host = lambda t: np.ascontiguousarray(t.detach().cpu().numpy())
        # every array handed to the host pass is held by a name until it returns
        surf = host((self.height + self.sediment)[inter].float())
        ocean = host(sea.to(torch.uint8))
        precip = host(self.precip[inter])
        pet_h = host(pet[inter].float())
        if self._lake_inputs is None:
            self._lake_inputs = (host(self.owner_table()), host(self.metric), host(area))
        owner, metric, area_h = self._lake_inputs
        F, N = self.F, self.N
        flag = np.empty((F, N, N), np.uint8)
        level = np.empty((F, N, N), np.float32)
        info = _lib.PgeLakeInfo()
        dev = self.height.device
        settled = {}
        if fill is None:
            check(_lib.load().pge_lake_balance(ctypes.byref(self.pge_grid()), owner.ctypes.data, metric.ctypes.data,
                                               area_h.ctypes.data, float(self.grid.cell_size_m), surf.ctypes.data,
                                               ocean.ctypes.data, precip.ctypes.data, pet_h.ctypes.data, float(lake_evap),
                                               float(land_evap), float(min_depth), flag.ctypes.data, None, level.ctypes.data,
                                               ctypes.byref(info)), "pge_lake_balance")
        else:
            grade, ice_evap, rise, load_share = (float(v) for v in fill)
            self.ensure_lake_parks()
            evap_h = host(self.evap[inter])
            height_h, sed_h = host(self.height[inter]), host(self.sediment[inter])
            load_h, id_h = host(self.lake_load[inter]), host(self.lake_id[inter])
            H = self.H
            if self._centres is None:
                self._centres = np.ascontiguousarray(self.grid.centers()[:, H:H + N, H:H + N], dtype=np.float64)
            lay = np.zeros((F, N, N))
            pend_add = np.zeros((F, N, N))
            room = np.zeros(F * N * N)  # at most one lake a cell
            fl = _lib.PgeLakeFill(grade=grade, ice_evap=ice_evap, rise=rise, evap=evap_h.ctypes.data,
                                  centres=self._centres.ctypes.data, height=height_h.ctypes.data, sediment=sed_h.ctypes.data,
                                  lake_load=load_h.ctypes.data, lake_id=id_h.ctypes.data, lay=lay.ctypes.data,
                                  pending=pend_add.ctypes.data, lake_room=room.ctypes.data, lake_room_cap=room.size)
            check(_lib.load().pge_lake_balance_fill(ctypes.byref(self.pge_grid()), owner.ctypes.data, metric.ctypes.data,
                                                    area_h.ctypes.data, float(self.grid.cell_size_m), surf.ctypes.data,
                                                    ocean.ctypes.data, precip.ctypes.data, pet_h.ctypes.data, float(lake_evap),
                                                    float(land_evap), float(min_depth), flag.ctypes.data, None,
                                                    level.ctypes.data, ctypes.byref(fl), ctypes.byref(info)),
                  "pge_lake_balance_fill")
            lay_d = torch.as_tensor(lay, device=dev)
            sed_i = self.sediment[inter]  # views: the laid sediment and stockpiles land in the state itself
            sed_i += lay_d
            if self.iso_acc is not None:
                iso_i = self.iso_acc[inter]
                iso_i += load_share * lay_d
            pend_i = self.pending[inter]
            pend_i += torch.as_tensor(pend_add, device=dev)
            self.lake_load.zero_()
            self.lake_id.fill_(-1)
            self.lake_id[inter] = torch.as_tensor(id_h, device=dev)
            self.lake_room = torch.as_tensor(room[:max(int(fl.lakes), 1)].copy(), device=dev)
            settled = {"parked": fl.parked, "laid": fl.laid, "stray": fl.stray, "room": fl.room, "lakes": int(fl.lakes)}
        lf = torch.zeros(self.height.shape, dtype=torch.uint8, device=dev)
        lf[inter] = torch.as_tensor(flag, device=dev)
        closed = ~np.isnan(level)
        if closed.any():
            b = self.base[inter]  # a view: the closed lakes' levels land in the base itself
            cl = torch.as_tensor(closed, device=dev)
            b[cl] = torch.as_tensor(level, device=dev)[cl].double()
        for t in (lf, self.base):  # exact copies of the cells they mirror (maps.py:476-479)
            flat = t.view(-1)
            flat[dst] = flat[nearest]
        self.lake_flag = lf
        return {"lake_cells": int(info.lake_cells), "lake_cells_closed": int(info.lake_cells_closed),
                "depressions": int(info.depressions), "overflowing": int(info.overflowing), "closed": int(info.closed),
                "dry": int(info.dry), **{f"load_{k}": v for k, v in settled.items()}}

    def n_active_interior(self) -> int:
        if self.mask is None:
            return self.F * self.N * self.N
        return int((self.mask[self.interior] == MASK_ACTIVE).sum().item())


# --------------------------------------------------------------------------
# one iteration
# --------------------------------------------------------------------------
def list_steps_of(ep, N) -> int:
    """Steps' worth of change-list room a droplet needs: two entries a step
    with the bank cut (erosion.lateral_rate, particle.py:259-272)."""
    m = max_steps_of(ep, N)
    return 2 * m if float(getattr(ep, "lateral_rate", 0.0)) > 0.0 else m


def default_wave(ep, n_particles: int) -> int:
    """The reference's chunk size: the wave that reproduces its terrain freezes."""
    return chunk_size(ep, n_particles)


def make_params(state: ErosionState, ep, volume0: float, P: int, wave: int, precision: int, mom_scale=1.0, disc_sat=None,
                iter_deposit=None, threads_per_block=0, blocks_per_sm=0, apply=_lib.APPLY_ORDERED, trace_lanes=0,
                apply_lanes=0) -> PgeParams:
    """The kernel's parameters in cell units.  ``erosion.brush_radius`` (no
    counterpart in the reference; 0 when the group has no such knob) spreads
    the wave apply's changes over a brush (PgeParams.brush_radius)."""
    u = state.height_unit_m
    return PgeParams(
        dt=float(ep.dt), density=float(ep.density), friction=float(ep.friction), deposition_rate=float(ep.deposition_rate),
        evap_rate=float(ep.evap_rate), k_mom=float(ep.k_mom), mom_scale=float(mom_scale), k_disc=float(ep.k_disc),
        disc_saturation=float(ep.disc_saturation if disc_sat is None else disc_sat), disc_exponent=float(ep.disc_exponent),
        slope_gain=float(ep.slope_gain), slope_sat=float(ep.slope_saturation), erodibility=float(ep.erodibility),
        cover_depth=cell_units(ep, "cover_depth", u), min_volume=float(ep.min_volume_frac) * float(volume0),
        max_erode=cell_units(ep, "max_erode", u), conc_scale=float(wave / (volume0 * P)) if P > 0 and volume0 > 0.0 else 0.0, ocean_rate=float(ep.ocean_deposition_rate),
        fan_room=cell_units(ep, "fan_room", u), dep_floor=cell_units(ep, "dep_floor_m", u), iter_erode=cell_units(ep, "iter_erode", u),
        iter_deposit=float(cell_units(ep, "iter_deposit", u) if iter_deposit is None else iter_deposit),
        fan_slope=float(ep.fan_slope), offshore_writeoff=float(ep.offshore_writeoff), ema=float(ep.ema),
        lake_trap=float(getattr(ep, "lake_trap", 0.9)), lateral_rate=float(getattr(ep, "lateral_rate", 0.0)),
        max_steps=max_steps_of(ep, state.N), pit_steps=int(ep.pit_steps), ocean_steps=int(ep.ocean_steps), wave=int(wave),
        precision=int(precision), apply=int(apply), use_erode_cap=0, threads_per_block=int(threads_per_block),
        blocks_per_sm=int(blocks_per_sm), trace_lanes=int(trace_lanes), apply_lanes=int(apply_lanes),
        brush_radius=int(getattr(ep, "brush_radius", 0)))


def draw_spawns(params, rng_stage: str, key, P: int):
    """The rain draws of one iteration in the reference's order: ``P``
    uniforms, then ``(P, 2)`` offsets; the generator is returned for the
    stockpile directions that follow."""
    rng = params.rng(rng_stage, *key)
    u = rng.random(P)
    off = rng.random((P, 2))
    return rng, u, off


def spawn_rain(state: ErosionState, u, off) -> dict:
    """The rain spawns of ``u`` (P uniforms, unsorted) and ``off`` ((P, 2)
    offsets) on the device (``pge_spawn_rain``: maps.spawn_particles,
    maps.py:809-833): ``face``, ``x``, ``y`` (host arrays), the total spawn
    weight (``w.sum()``, so ``volume0 = total / P``) and the count of
    spawnable cells."""
    P = int(np.asarray(u).shape[0])
    state.reserve(P, 1, 1)
    L = _lib.load()
    dev = state.height.device
    u_d = torch.as_tensor(u, dtype=torch.float64, device=dev)
    off_d = torch.as_tensor(off, dtype=torch.float64, device=dev).contiguous()
    face = torch.zeros(P, dtype=torch.int32, device=dev)
    xs, ys, sed, dirs = (torch.zeros(P, dtype=torch.float64, device=dev) for _ in range(4))
    scal = torch.zeros(1, dtype=torch.float64, device=dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    spawns = PgeSpawns(face=_ptr(face), x=_ptr(xs), y=_ptr(ys), sed=_ptr(sed), dir=_ptr(dirs), count=P, volume0=0.0)
    check(L.pge_spawn_rain(ctypes.byref(state.pge_grid()), ctypes.byref(state.pge_state()), _ptr(u_d), _ptr(off_d), P,
                           ctypes.byref(spawns), _ptr(scal), _ptr(cnt), _ptr(state.workspace), state.workspace.numel(), _stream()),
          "pge_spawn_rain")
    torch.cuda.synchronize()
    return {"face": face.cpu().numpy(), "x": xs.cpu().numpy(), "y": ys.cpu().numpy(), "total": float(scal.item()),
            "n_spawnable": int(cnt.item())}


class SpawnFeeder:
    """The host-drawn spawn uniforms of successive iterations, ready before
    they are needed: while the device runs iteration ``k``, a background
    thread draws iteration ``k + 1``'s ``P`` uniforms and ``(P, 2)`` offsets
    (``draw_spawns``, the reference's order) into pinned host memory; ``get``
    copies them to the device on the current stream and returns what
    ``run_iteration(predrawn=...)`` takes.  Two pinned buffers alternate; a
    buffer is refilled only after its last copy to the device has finished."""

    def __init__(self, params, P: int, rng_stage: str = "erosion", device="cuda"):
        from concurrent.futures import ThreadPoolExecutor

        self.params, self.P, self.stage = params, int(P), rng_stage
        self._pin = [(torch.empty(self.P, dtype=torch.float64).pin_memory(),
                      torch.empty((self.P, 2), dtype=torch.float64).pin_memory()) for _ in range(2)]
        self._copied = [None, None]
        d = torch.device(device)
        self._dev = [(torch.empty(self.P, dtype=torch.float64, device=d), torch.empty((self.P, 2), dtype=torch.float64, device=d))
                     for _ in range(2)]
        self._ex = ThreadPoolExecutor(max_workers=1)
        self._fut = {}
        self._slot = 0

    @staticmethod
    def _key(key):
        return tuple(key) if isinstance(key, (tuple, list)) else (int(key),)

    def _draw(self, key, slot):
        ev = self._copied[slot]
        if ev is not None:
            ev.synchronize()  # the buffer's previous copy to the device is done
        u, off = self._pin[slot]
        rng = self.params.rng(self.stage, *key)
        rng.random(out=u.numpy())
        rng.random(out=off.numpy())
        return rng

    def prefetch(self, key) -> None:
        key = self._key(key)
        if key not in self._fut:
            self._fut[key] = (self._ex.submit(self._draw, key, self._slot), self._slot)
            self._slot ^= 1

    def get(self, key):
        """``(rng, u, off)`` of iteration ``key`` with ``u`` and ``off`` on the
        device; starts drawing the next iteration.  Returns the bytes copied
        to the device as a fourth item."""
        key = self._key(key)
        self.prefetch(key)
        fut, slot = self._fut.pop(key)
        rng = fut.result()
        u_p, off_p = self._pin[slot]
        u_d, off_d = self._dev[slot]
        u_d.copy_(u_p, non_blocking=True)
        off_d.copy_(off_p, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        self._copied[slot] = ev
        self.prefetch(key[:-1] + (key[-1] + 1,))
        return rng, u_d, off_d, u_p.numel() * 8 + off_p.numel() * 8

    def close(self) -> None:
        self._ex.shutdown(wait=True)


def run_iteration(state: ErosionState, params, iteration_key, n_particles: int | None = None,
                  particles_per_cell: float | None = None, rng_stage: str = "erosion", log=None, wave: int | None = None,
                  precision: int = _lib.PREC_F64, predrawn=None, threads_per_block: int = 0, blocks_per_sm: int = 0,
                  events=None, apply: int = _lib.APPLY_ORDERED, trace_lanes: int = 0, apply_lanes: int = 0,
                  tape=None, parks: bool | None = None) -> dict:
    """One particle pass (maps.py:839-1047) on the device; see the module
    docstring.  ``parks``: the lake parks (erosion.lake_fill; default: on
    where :func:`lake_fill_args` is, as the reference's pass has them,
    maps.py:996).  ``predrawn`` may carry ``draw_spawns``' result for this
    iteration (drawn ahead, host or device arrays); ``events`` a pair of
    CUDA events recorded around the droplet pass (``pge_trace_apply``).
    ``tape``: a callable ``(n_droplets, max_steps, waves, cells) -> PgeTape``
    -- the pass then runs as the float64 wave apply, recorded for the
    adjoint (``pge_trace_apply_tape``); the spawns, parameters and tape are
    returned under ``stats["adjoint"]``."""
    ep = erosion_group(params)
    check_plain(ep)
    key = iteration_key if isinstance(iteration_key, (tuple, list)) else (int(iteration_key),)
    t0 = time.time()
    if n_particles is None:
        ppc = ep.particles_per_cell if particles_per_cell is None else particles_per_cell
        n_particles = max(1, int(round(ppc * state.n_active_interior())))
    P = int(n_particles)
    max_steps = max_steps_of(ep, state.N)
    # stockpiles re-injected: at most one per interior cell; the reference's chunk is at most erosion.chunk
    state.reserve(P + state.F * state.N * state.N, list_steps_of(ep, state.N),
                  (int(ep.chunk) if wave is None else int(wave)) if apply == _lib.APPLY_ORDERED else 1,
                  wave_tables=apply == _lib.APPLY_WAVE)
    rng, u, off = predrawn if predrawn is not None else draw_spawns(params, rng_stage, key, P)
    L = _lib.load()
    g = state.pge_grid()
    if parks is None:  # no lakes yet (no route or flags): nothing can be parked
        parks = lake_fill_args(state, params) is not None and state.route is not None and state.lake_flag is not None
    if parks:
        state.ensure_lake_parks()
        parked0 = state.lake_load.sum()
    s = state.pge_state(parks)
    sp = state._spawn
    ws = state.workspace
    st = _stream()
    dev = state.height.device
    u_d = torch.as_tensor(u, device=dev)
    off_d = torch.as_tensor(off, device=dev)
    spawns = PgeSpawns(face=_ptr(sp["face"]), x=_ptr(sp["x"]), y=_ptr(sp["y"]), sed=_ptr(sp["sed"]), dir=_ptr(sp["dir"]),
                       count=P, volume0=0.0)
    scal, cnt = sp["scal"], sp["cnt"]
    nsp_ptr = ctypes.c_void_p(cnt.data_ptr())
    npend_ptr = ctypes.c_void_p(cnt.data_ptr() + 8)
    check(L.pge_spawn_rain(ctypes.byref(g), ctypes.byref(s), _ptr(u_d), _ptr(off_d), P, ctypes.byref(spawns), _ptr(scal),
                           nsp_ptr, _ptr(ws), ws.numel(), st), "pge_spawn_rain")
    check(L.pge_count_pending(ctypes.byref(g), ctypes.byref(s), npend_ptr, _ptr(ws), ws.numel(), st), "pge_count_pending")
    hs, hc = sp["host_scal"], sp["host_cnt"]
    hs.copy_(scal, non_blocking=True)
    hc.copy_(cnt, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    total = float(hs[0])
    n_spawnable, n_pend = int(hc[0]), int(hc[1])
    stats = {"particles": 0, "entries": 0, "steps_mean": 0.0}
    if n_spawnable == 0 or not (total > 0.0):
        return stats
    volume0 = total / P
    stats_d = sp["stats"]
    stats_d.zero_()
    if n_pend:
        dirs = torch.as_tensor(rng.random(n_pend) * (2.0 * np.pi), device=dev)
        sp["dir"][P:P + n_pend].copy_(dirs)
        check(L.pge_collect_pending(ctypes.byref(g), ctypes.byref(s), ctypes.byref(spawns), P, _ptr(stats_d), _ptr(ws), ws.numel(),
                                    st), "pge_collect_pending")
    Ptot = P + n_pend
    spawns.count = Ptot
    spawns.volume0 = volume0
    disc_sat = float(ep.disc_saturation)
    mom_scale = 1.0
    if float(ep.disc_saturation_cells) > 0.0 or float(ep.momentum_saturation_cells) > 0.0:
        # the window's inflow across its edge is not rain on it (maps.py:913-917)
        rain_total = volume0 * P
        rain_per_cell = max(rain_total - float(state.inflow_volume), 0.0) / max(n_spawnable, 1)
        rain_per_cell = rain_per_cell if rain_per_cell > 0.0 else rain_total / max(n_spawnable, 1)
        if float(ep.disc_saturation_cells) > 0.0:
            disc_sat = float(ep.disc_saturation_cells) * rain_per_cell
        if float(ep.momentum_saturation_cells) > 0.0:
            mom_scale = volume0 / (float(ep.momentum_saturation_cells) * rain_per_cell)
    iter_deposit = cell_units(ep, "iter_deposit", state.height_unit_m)
    if float(ep.slope_limit_deposit) > 0.0:
        iter_deposit = min(iter_deposit, float(ep.slope_limit_deposit) * math.sqrt(2.0) * 0.3)
    w = default_wave(ep, Ptot) if wave is None else int(wave)
    if tape is not None:
        apply, precision, w = _lib.APPLY_WAVE, _lib.PREC_F64, min(w, Ptot)
    prm = make_params(state, ep, volume0, Ptot, w, precision, mom_scale, disc_sat, iter_deposit, threads_per_block, blocks_per_sm,
                      apply, trace_lanes, apply_lanes)
    ecap = _erode_cap(state, ep, prm)
    if events is not None:
        events[0].record()
    if tape is not None:
        if ecap is not None:
            raise ValueError("the adjoint's tape does not cover erosion.slope_limit_erode")
        tp = tape(Ptot, max_steps, -(-Ptot // w), state.height.numel())
        check(L.pge_trace_apply_tape(ctypes.byref(g), ctypes.byref(s), ctypes.byref(spawns), ctypes.byref(prm), ctypes.byref(tp),
                                     _ptr(stats_d), _ptr(ws), ws.numel(), st), "pge_trace_apply_tape")
        stats["adjoint"] = {"spawns": PgeSpawns.from_buffer_copy(spawns), "params": PgeParams.from_buffer_copy(prm), "tape": tp}
    else:
        check(L.pge_trace_apply(ctypes.byref(g), ctypes.byref(s), ctypes.byref(spawns), ctypes.byref(prm), ecap, _ptr(stats_d),
                                _ptr(ws), ws.numel(), st), "pge_trace_apply")
    if events is not None:
        events[1].record()
    hst = sp["host_stats"]
    hst.copy_(stats_d, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    r = PgeStats.from_buffer_copy(hst.numpy().tobytes())
    if r.errors:
        raise _lib.PgeError("ordered apply: a cell hand-off wait gave up; the pass is invalid")
    fx = _lib.FX_MASS
    stats.update({"particles": Ptot, "entries": int(r.entries), "steps_mean": r.entries / max(Ptot, 1), "volume": volume0,
                  "seconds": time.time() - t0, "droplet_steps": int(r.droplet_steps)})
    stats["deaths"] = {n: int(r.deaths[k]) for k, n in enumerate(_lib.DEATH_NAMES)}
    stats["clamped"] = int(r.clamped)
    stats["to_pending"] = r.to_pending_fx / fx
    stats["released"] = r.released_fx / fx
    stats["pending_total"] = r.to_pending_fx / fx
    stats["deficit_out"] = r.deficit_out_fx / fx
    stats["lost_offshore"] = r.lost_offshore_fx / fx
    stats["overflow"] = int(r.overflow)
    stats["eroded"] = r.eroded_fx / fx
    stats["deposited"] = r.deposited_fx / fx
    stats["chunk"] = int(w)
    stats["apply"] = "ordered" if apply == _lib.APPLY_ORDERED else "wave"
    stats["n_pending"] = int(n_pend)
    if parks:  # the loads the lakes took this pass (the rest of a park went on with its droplet)
        stats["parked"] = float(state.lake_load.sum() - parked0)
    stats["disc_saturation"] = disc_sat
    stats["mom_scale"] = mom_scale
    if log is not None:
        log(f"  particles {Ptot} volume {volume0:.3f} mean steps {stats['steps_mean']:.1f} deaths {stats['deaths']} "
            f"clamped {stats['clamped']} pending {stats['pending_total']:.1f} ({stats['seconds']:.2f}s)")
    return stats


def _erode_cap(state: ErosionState, ep, prm: PgeParams):
    """soillib's pit-free erosion cap of this iteration's start terrain
    (maps.py:922-927) when ``erosion.slope_limit_erode > 0``: computed on the
    device, switched on in ``prm``; returns the pointer for pge_trace_apply
    (None when off)."""
    if float(ep.slope_limit_erode) <= 0.0:
        return None
    if state._erode_cap is None or state._erode_cap.shape != state.height.shape:
        state._erode_cap = torch.empty_like(state.height)
    check(_lib.load().pge_slope_erode_cap(ctypes.byref(state.pge_grid()), ctypes.byref(state.pge_state()),
                                          float(ep.slope_limit_erode), float(ep.slope_limit_exit), _ptr(state._erode_cap),
                                          _stream()), "pge_slope_erode_cap")
    prm.use_erode_cap = 1
    return _ptr(state._erode_cap)


def _ensure_workspace(state: ErosionState, ep=None) -> None:
    if state.workspace is None:
        state.reserve(max(state.max_droplets, 1), max(state.max_steps, list_steps_of(ep, state.N) if ep is not None else 1))


def thermal_erosion(state: ErosionState, params) -> None:
    """Talus pass, then the creep pass (maps.py:1050-1085)."""
    ep = erosion_group(params)
    _ensure_workspace(state, ep)
    L = _lib.load()
    u = state.height_unit_m
    check(L.pge_thermal(ctypes.byref(state.pge_grid()), ctypes.byref(state.pge_state()), float(ep.thermal_rate),
                        float(ep.creep_rate), cell_units(ep, "thermal_max", u), float(ep.talus_slope_soft),
                        float(ep.talus_slope_hard), cell_units(ep, "dep_floor_m", u), _ptr(state.workspace),
                        state.workspace.numel(), _stream()), "pge_thermal")


def uplift_cap(state: ErosionState, ep) -> float | None:
    if not state.spherical or float(getattr(ep, "uplift_max_m", 0.0)) <= 0.0:
        return None
    return cell_units(ep, "uplift_max_m", state.height_unit_m)


def apply_uplift(state: ErosionState, cap: float | None = None, scale: float = 1.0) -> None:
    """height += min(uplift, cap) - mean over the active interior (maps.py:1088-1147)."""
    _ensure_workspace(state)
    L = _lib.load()
    check(L.pge_uplift(ctypes.byref(state.pge_grid()), ctypes.byref(state.pge_state()), -1.0 if cap is None else float(cap),
                       float(scale), _ptr(state.workspace), state.workspace.numel(), _stream()), "pge_uplift")


def hold_datum(state: ErosionState, land_fraction: float, level: float = 0.0) -> float:
    """Rigid shift holding round(land_fraction * M) interior cells at or
    above ``level`` (maps.py:1446-1508); returns the shift (cell units)."""
    _ensure_workspace(state)
    L = _lib.load()
    scal = state._spawn["scal"]
    check(L.pge_hold_datum(ctypes.byref(state.pge_grid()), ctypes.byref(state.pge_state()), float(land_fraction), float(level),
                           ctypes.c_void_p(scal.data_ptr() + 8), _ptr(state.workspace), state.workspace.numel(), _stream()),
          "pge_hold_datum")
    q = float(scal[1].item())
    if state.route is not None and q != 0.0:  # the routing surface stays registered with the terrain (maps.py:1498-1499)
        state.route -= q
    return q


def glacial_carve(state: ErosionState, params) -> dict:
    """One glacial pass (erosion/glacial.py:162-257) with the ice line read
    from the evaporation field (``evap <= erosion.ice_evap``; the state
    carries no temperature): the bed under ice lowered, the spoil put on the
    ice margin as moraine, the excess parked as stockpile; the halos
    refreshed.  Returns the reference's statistics."""
    ep = erosion_group(params)
    _ensure_workspace(state, ep)
    u = state.height_unit_m
    sticky = bool(getattr(ep, "glacial_sticky", False))
    if sticky and state.ice_prev is None:
        state.ice_prev = torch.zeros(state.height.shape, dtype=torch.uint8, device=state.height.device)
    out = (ctypes.c_double * 5)()
    check(_lib.load().pge_glacial(ctypes.byref(state.pge_grid()), ctypes.byref(state.pge_state()),
                                  _ptr(state.ice_prev) if sticky else None, cell_units(ep, "glacial_rate", u),
                                  cell_units(ep, "glacial_max", u), int(ep.glacial_ramp), float(ep.ice_evap),
                                  float(ep.disc_saturation), float(getattr(ep, "moraine_frac", 1.0)), cell_units(ep, "iter_deposit", u),
                                  out, _ptr(state.workspace), state.workspace.numel(), _stream()), "pge_glacial")
    if out[1] > 0.0:
        state.exchange_halos()
    return {"ice_cells": int(out[0]), "carved": float(out[1]), "moraine_cells": int(out[2]), "max_carve": float(out[3]),
            "outwash": float(out[4])}


def ocean_min_fraction(params) -> float:
    """``hydro.ocean_min_fraction`` when the params carry a hydro group, else
    the bake's default 0.02 (maps.py:770-774)."""
    hydro = getattr(params, "hydro", None)
    return float(getattr(hydro, "ocean_min_fraction", 0.02)) if hydro is not None else 0.02


def fill_basins(state: ErosionState, params) -> dict | None:
    """``erosion.basin_fill_grade`` > 0 (maps.py:1278-1326): lay sediment into
    the closed basins the bedrock arrives with, up to a plain rising
    ``basin_fill_grade`` (m per km) from each basin's outlet along the flood
    tree, on cells the flood leaves more than ``basin_fill_min_m`` under its
    fill and off the open ocean (``pge_basin_fill``, a host pass: the flood's
    pop order is serial).  Call once on a fresh state after
    :func:`start_replay`; returns the reference's statistics, or None when
    off, on a window or without a world group."""
    ep = erosion_group(params)
    grade = float(getattr(ep, "basin_fill_grade", 0.0))
    if grade <= 0.0 or not state.spherical or getattr(params, "world", None) is None:
        return None
    inter = state.interior
    sb, labels = state._sea_base(ocean_min_fraction(params))
    sea = (labels >= 0) & (sb[inter] == 0.0)  # the open ocean of the current surface
    host = lambda t: np.ascontiguousarray(t.detach().cpu().numpy())
    surf = host((state.height + state.sediment)[inter].float())
    ocean = host(sea.to(torch.uint8))
    owner = host(state.owner_table())
    F, N = state.F, state.N
    add = np.empty((F, N, N), np.float64)
    basin = np.empty((F, N, N), np.uint8)
    nb = ctypes.c_int64(0)
    unit = state.height_unit_m
    step = grade * (float(state.grid.cell_size_m) / 1000.0) / unit  # cell units per cell
    check(_lib.load().pge_basin_fill(ctypes.byref(state.pge_grid()), owner.ctypes.data, surf.ctypes.data, ocean.ctypes.data,
                                     float(step), float(getattr(ep, "basin_fill_min_m", 1.0)) / unit, add.ctypes.data,
                                     basin.ctypes.data, ctypes.byref(nb)), "pge_basin_fill")
    state.sediment[inter] += torch.as_tensor(add, device=state.height.device)
    state.exchange_halos()
    area = host(state._sea_tables()[0])
    b = basin.astype(bool)
    return {"basin_cells": int(nb.value), "basin_area_km2": float(area[b].sum() / 1e6),
            "fill_km3": float((add * unit * area).sum() / 1e9),
            "fill_mean_m": float(add[b].mean() * unit) if b.any() else 0.0, "fill_max_m": float(add.max() * unit)}


def lake_min_depth(params) -> float:
    """``hydro.lake_min_depth`` (m) when the params carry a hydro group, else
    the bake's 0.5 (maps.py:1564)."""
    hydro = getattr(params, "hydro", None)
    return float(getattr(hydro, "lake_min_depth", 0.5)) if hydro is not None else 0.5


def held_land_fraction(state: ErosionState, params) -> float:
    if state.land_target is not None:
        return float(state.land_target)
    if float(getattr(getattr(params, "tectonics", None), "shelf_fraction", 0.0) or 0.0) > 0.0:
        raise ValueError("shelf mode holds the bedrock's land fraction: set state.land_target")
    return float(params.world.land_fraction)


def start_replay(state: ErosionState, params) -> dict | None:
    """``uplift_mode = 'replay'``: lower the start by the run's total applied
    uplift, refresh the halos and hold the datum (maps.py:1178-1213)."""
    ep = erosion_group(params)
    if not state.spherical or str(getattr(ep, "uplift_mode", "stack")) != "replay":
        return None
    _ensure_workspace(state, ep)
    apply_uplift(state, uplift_cap(state, ep), scale=-float(int(ep.iterations)))
    state.exchange_halos()
    info = {"datum_shift": 0.0}
    if hasattr(params, "world"):
        info["datum_shift"] = hold_datum(state, held_land_fraction(state, params))
    return info


def lake_fill_args(state: ErosionState, params):
    """refresh_lakes' ``fill`` (maps.py:1248-1258): (the lake plain's grade in
    cell units per cell, ice_evap, the plain's rise above the water in cell
    units, the share of the fill that is isostatic load) with
    erosion.lake_fill and lake_balance on the planet, else None."""
    ep = erosion_group(params)
    if not (state.spherical and bool(getattr(ep, "lake_fill", False)) and bool(getattr(ep, "lake_balance", False))):
        return None
    cell_km = float(state.grid.cell_size_m) / 1000.0
    return (float(getattr(ep, "basin_fill_grade", 0.0)) * cell_km / state.height_unit_m, float(getattr(ep, "ice_evap", 0.0)),
            float(getattr(ep, "lake_fill_rise_m", 1.0)) / state.height_unit_m, float(getattr(ep, "lake_fill_load", 0.55)))


def settle_lakes(state: ErosionState, params) -> dict | None:
    """The lakes lay what the last iterations parked on them (maps.py:1261-1275,
    a run ends between two refreshes): the sea mask and the route refreshed,
    one lake refresh with the fill, halos exchanged.  None without lake_fill."""
    fill = lake_fill_args(state, params)
    if fill is None or not hasattr(params, "world"):
        return None
    ep = erosion_group(params)
    if int(getattr(ep, "sea_mask_every", 0)) > 0:
        state.refresh_base(ocean_min_fraction(params))
    state.refresh_route(cell_units(ep, "route_eps", state.height_unit_m))
    hydro = getattr(params, "hydro", None)
    st = state.refresh_lakes(float(getattr(hydro, "lake_evap", 6.0)), lake_min_depth(params) / state.height_unit_m,
                             ocean_min_fraction(params), float(getattr(hydro, "land_evap", 3.0)), fill=fill)
    state.exchange_halos()
    return st


def step(state: ErosionState, params, iteration_key, log=None, **kw) -> dict:
    """One plain iteration (maps.py:1516-1617): particles, thermal erosion,
    uplift, isostasy (when ``erosion.isostasy > 0``: the surface change of
    the particles and the mass wasting is the load, applied every
    ``isostasy_every`` iterations, maps.py:1570-1603), datum hold, halo
    exchange; increments ``state.iteration``."""
    ep = erosion_group(params)
    t0 = time.time()
    sea_every = int(getattr(ep, "sea_mask_every", 0))
    st_base = None
    if state.spherical and sea_every > 0 and (state.base_at is None or state.iteration % sea_every == 0):
        # the sea mask before the route: the flood seeds on the sea (maps.py:1546-1551)
        st_base = state.refresh_base(ocean_min_fraction(params))
    flood = int(getattr(ep, "flood_every", 0))
    if flood > 0 and (state.route is None or state.iteration % flood == 0):
        # the routing surface the particles steer on (maps.py:1553-1554)
        state.refresh_route(cell_units(ep, "route_eps", state.height_unit_m))
    st_lake = None
    if state.spherical and bool(getattr(ep, "lake_balance", False)) and flood > 0 and \
            (state.lake_flag is None or state.iteration % flood == 0):
        # the planet's lakes, after the base (rebuilt from scratch) and the route (maps.py:1555-1562)
        hydro = getattr(params, "hydro", None)
        st_lake = state.refresh_lakes(float(getattr(hydro, "lake_evap", 6.0)), lake_min_depth(params) / state.height_unit_m,
                                      ocean_min_fraction(params), float(getattr(hydro, "land_evap", 3.0)),
                                      fill=lake_fill_args(state, params))
    elif not state.spherical and bool(getattr(ep, "window_lakes", False)) and flood > 0 and \
            (state.lake_flag is None or state.iteration % flood == 0):
        # a window's lakes, after the route they are read off (maps.py:1563-1566)
        st_lake = state.refresh_lakes_window(lake_min_depth(params) / state.height_unit_m,
                                             float(getattr(ep, "window_lake_evap", 0.0)))
    t_route = time.time()
    iso = state.spherical and float(getattr(ep, "isostasy", 0.0)) > 0.0
    if iso:
        if state.iso_acc is None:
            state.iso_acc = torch.zeros_like(state.height)
        s0 = state.height + state.sediment
    st = run_iteration(state, params, iteration_key, log=log, **kw)
    t1 = time.time()
    thermal_erosion(state, params)
    if iso:
        # only what surface processes moved: uplift and the datum shift are not loads
        state.iso_acc += (state.height + state.sediment) - s0
    apply_uplift(state, uplift_cap(state, ep))
    ge = int(getattr(ep, "glacial_every", 0))
    if state.spherical and ge > 0 and (state.iteration + 1) % ge == 0 and \
            (state.iteration + 1) >= float(ep.glacial_from) * int(ep.iterations):
        # glacial carving: the one pass that may leave a closed depression (maps.py:1580-1590)
        if iso:
            s1 = state.height + state.sediment
        st["glacial"] = glacial_carve(state, params)
        if iso:
            state.iso_acc += (state.height + state.sediment) - s1
    if iso and (state.iteration + 1) % max(int(getattr(ep, "isostasy_every", 10)), 1) == 0:
        from .isostasy import apply_isostasy

        st["isostasy"] = apply_isostasy(state, params)
    if state.spherical and hasattr(params, "world"):
        st["datum_shift"] = hold_datum(state, held_land_fraction(state, params))
    state.exchange_halos()
    state.iteration += 1
    if st_base is not None:
        st["sea"] = st_base
    if st_lake is not None:
        st["lakes"] = st_lake
    st["seconds_route"] = t_route - t0
    st["seconds_particles"] = t1 - t_route
    st["seconds_total"] = time.time() - t0
    return st


def trace_changelist(state: ErosionState, params, sp_face, sp_x, sp_y, sp_sed, sp_dir, volume0: float, conc_scale: float,
                     precision: int = _lib.PREC_F64, wave: int | None = None, parks: bool = False) -> dict:
    """Parity hook: trace and apply the given droplets in one wave (or waves
    of ``wave``) on the current state, recording each droplet's change list
    in the reference layout (particle.py:275-818) and returning it with the
    pass's accumulators.  The state's terrain is left unchanged.  With
    ``parks`` (the lake parks, on the state's lake_id / lake_room) the lists
    are recorded only: the accumulators stay zero."""
    ep = erosion_group(params)
    P = int(len(sp_face))
    max_steps = max_steps_of(ep, state.N)
    state.reserve(P, list_steps_of(ep, state.N), 1, wave_tables=True)
    L = _lib.load()
    dev = state.height.device
    cap = list_steps_of(ep, state.N) + 2 * 8 + 1 + 8 + 8  # change_list_cap: the reference's row width
    face = torch.as_tensor(np.asarray(sp_face, np.int32), device=dev)
    xs = [torch.as_tensor(np.asarray(a, np.float64), device=dev) for a in (sp_x, sp_y, sp_sed, sp_dir)]
    spawns = PgeSpawns(face=_ptr(face), x=_ptr(xs[0]), y=_ptr(xs[1]), sed=_ptr(xs[2]), dir=_ptr(xs[3]), count=P,
                       volume0=float(volume0))
    w = P if wave is None else int(wave)
    prm = make_params(state, ep, volume0, P, w, precision, apply=_lib.APPLY_WAVE)
    prm.conc_scale = float(conc_scale)
    out = {"cl_cell": torch.zeros(P * cap, dtype=torch.int32, device=dev), "cl_delta": torch.zeros(P * cap, dtype=torch.float64, device=dev),
           "cl_vol": torch.zeros(P * cap, dtype=torch.float32, device=dev), "cl_mom": torch.zeros(P * cap * 2, dtype=torch.float32, device=dev),
           "cl_count": torch.zeros(P, dtype=torch.int64, device=dev), "sp_death": torch.zeros(P, dtype=torch.int8, device=dev)}
    stats_d = torch.zeros(_lib.STATS_WORDS, dtype=torch.int64, device=dev)
    ws = state.workspace
    st = _stream()
    if parks:
        state.ensure_lake_parks()
    g, s = state.pge_grid(), state.pge_state(parks)
    check(L.pge_trace_changelist(ctypes.byref(g), ctypes.byref(s), ctypes.byref(spawns), ctypes.byref(prm), _ptr(out["cl_cell"]),
                                 _ptr(out["cl_delta"]), _ptr(out["cl_vol"]), _ptr(out["cl_mom"]), _ptr(out["cl_count"]),
                                 _ptr(out["sp_death"]), _ptr(stats_d), _ptr(ws), ws.numel(), st), "pge_trace_changelist")
    acc = torch.zeros_like(state.height)
    dtr = torch.zeros_like(state.height)
    mtr = torch.zeros_like(state.momentum)
    pend = torch.zeros_like(state.height)
    check(L.pge_read_accumulators(ctypes.byref(g), _ptr(acc), _ptr(dtr), _ptr(mtr), _ptr(pend), _ptr(ws), ws.numel(), st),
          "pge_read_accumulators")
    torch.cuda.synchronize()
    res = {k: v.cpu().numpy() for k, v in out.items()}
    res["cl_mom"] = res["cl_mom"].reshape(-1, 2)
    res.update(acc=acc.cpu().numpy(), disch_track=dtr.cpu().numpy(), mom_track=mtr.cpu().numpy(), pending=pend.cpu().numpy(),
               cap=cap)
    r = PgeStats.from_buffer_copy(stats_d.cpu().numpy().tobytes())
    fx = _lib.FX_MASS
    res["apply_out"] = np.array([float(r.clamped), r.to_pending_fx / fx, r.deficit_out_fx / fx, r.lost_offshore_fx / fx])
    res["droplet_steps"] = int(r.droplet_steps)
    return res


def apply_spawns(state: ErosionState, params, sp_face, sp_x, sp_y, sp_sed, sp_dir, volume0: float, n_rain: int | None = None,
                 wave: int | None = None, precision: int = _lib.PREC_F64, apply: int = _lib.APPLY_ORDERED, tape=None,
                 parks: bool = False, conc_scale: float | None = None) -> dict:
    """One droplet pass over explicitly given spawns (no random draws): pack,
    waves, apply, fold and EMA, exactly as :func:`run_iteration` does after
    spawning.  ``n_rain`` is the rain count the concurrency divisor is
    computed with (the reference divides by the whole spawn count).
    ``parks``: the lake parks on the state's lake_id / lake_room;
    ``conc_scale``: the concurrency divisor's scale in place of the wave's."""
    ep = erosion_group(params)
    P = int(len(sp_face))
    max_steps = max_steps_of(ep, state.N)
    w = max(1, default_wave(ep, P) if wave is None else int(wave))  # (no spawns: one empty wave)
    state.reserve(max(P, 1), list_steps_of(ep, state.N), w if apply == _lib.APPLY_ORDERED else 1,
                  wave_tables=apply == _lib.APPLY_WAVE)
    L = _lib.load()
    dev = state.height.device
    sp = state._spawn
    sp["face"][:P].copy_(torch.as_tensor(np.asarray(sp_face, np.int32)))
    for k, a in (("x", sp_x), ("y", sp_y), ("sed", sp_sed), ("dir", sp_dir)):
        sp[k][:P].copy_(torch.as_tensor(np.asarray(a, np.float64)))
    spawns = PgeSpawns(face=_ptr(sp["face"]), x=_ptr(sp["x"]), y=_ptr(sp["y"]), sed=_ptr(sp["sed"]), dir=_ptr(sp["dir"]), count=P,
                       volume0=float(volume0))
    iter_deposit = cell_units(ep, "iter_deposit", state.height_unit_m)
    if float(ep.slope_limit_deposit) > 0.0:
        iter_deposit = min(iter_deposit, float(ep.slope_limit_deposit) * math.sqrt(2.0) * 0.3)
    prm = make_params(state, ep, volume0, P, w, precision, iter_deposit=iter_deposit, apply=apply)
    if conc_scale is not None:
        prm.conc_scale = float(conc_scale)
    ecap = _erode_cap(state, ep, prm)
    stats_d = sp["stats"]
    stats_d.zero_()
    ws = state.workspace
    out = {}
    if parks:
        state.ensure_lake_parks()
    pst = state.pge_state(parks)
    if tape is not None:  # the pass recorded for the adjoint (float64 wave apply; see run_iteration)
        tp = tape(P, max_steps, -(-P // w), state.height.numel())
        check(L.pge_trace_apply_tape(ctypes.byref(state.pge_grid()), ctypes.byref(state.pge_state()), ctypes.byref(spawns),
                                     ctypes.byref(prm), ctypes.byref(tp), _ptr(stats_d), _ptr(ws), ws.numel(), _stream()),
              "pge_trace_apply_tape")
        out["adjoint"] = {"spawns": PgeSpawns.from_buffer_copy(spawns), "params": PgeParams.from_buffer_copy(prm), "tape": tp}
    else:
        check(L.pge_trace_apply(ctypes.byref(state.pge_grid()), ctypes.byref(pst), ctypes.byref(spawns),
                                ctypes.byref(prm), ecap, _ptr(stats_d), _ptr(ws), ws.numel(), _stream()), "pge_trace_apply")
    r = PgeStats.from_buffer_copy(stats_d.cpu().numpy().tobytes())
    if r.errors:
        raise _lib.PgeError("ordered apply: a cell hand-off wait gave up; the pass is invalid")
    fx = _lib.FX_MASS
    out.update({"droplets": int(r.droplets), "droplet_steps": int(r.droplet_steps), "entries": int(r.entries),
                "clamped": int(r.clamped), "deaths": [int(v) for v in r.deaths], "to_pending": r.to_pending_fx / fx,
                "lost_offshore": r.lost_offshore_fx / fx, "deficit_out": r.deficit_out_fx / fx, "eroded": r.eroded_fx / fx,
                "deposited": r.deposited_fx / fx})
    return out
