"""Parameters and random streams of the erosion stage, mirrored from the bake.

The drop-in reads its knobs by attribute (``params.erosion.friction``,
``params.world.seed``, ``params.rng("erosion", it)``), so the bake's own
``globe.config.WorldParams`` can be handed in unchanged.  This module
provides a self-contained stand-in with the same names, defaults and
random-stream keys for callers (tests, the benchmark) that run without the
bake installed.

Reference interface (paths within the bake project):

* ``ErosionParams`` -- ``bake/globe/config.py:487-583`` (field names and
  defaults below are the same; lengths in metres, ``LENGTH_PARAMS_M``
  ``config.py:603-605``).
* ``cell_units`` -- ``config.py:608-610``.
* ``WorldParams.rng`` -- ``config.py:830-842``: ``np.random.default_rng``
  seeded with ``[(seed + stage_offset) mod 2^64, len(keys), *keys mod 2^64]``.
* stage seed offsets -- ``config.py:23-33``.
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field

import numpy as np

STAGE_SEED_OFFSETS = {
    "tectonics": 1000,
    "climate": 2000,
    "erosion": 3000,
    "hydro": 4000,
    "watersheds": 5000,
    "refine": 6000,
    "derive": 7000,
    "tiles": 8000,
    "stub": 9000,
}

#: erosion knobs that are lengths in metres (converted to cell units at use)
LENGTH_PARAMS_M = ("cover_depth", "max_erode", "iter_erode", "iter_deposit",
                   "thermal_max", "fan_room", "route_eps",
                   "glacial_rate", "glacial_max", "uplift_max_m")


@dataclass
class ErosionParams:
    """The erosion group: same field names and defaults as the bake."""

    iterations: int = 800
    particles_per_cell: float = 0.25
    dt: float = 1.2
    density: float = 1.0
    friction: float = 0.25
    deposition_rate: float = 0.1
    evap_rate: float = 0.001
    k_mom: float = 1.0
    k_disc: float = 1.0
    ema: float = 0.1
    thermal_rate: float = 0.5
    creep_rate: float = 0.02
    thermal_max: float = 50.0
    talus_slope_soft: float = 0.6
    talus_slope_hard: float = 1.2
    min_volume: float = 0.5
    min_volume_frac: float = 5e-5
    max_steps: int = 0
    checkpoint_every: int = 50
    quicklook_every: int = 50
    slope_gain: float = 2.0
    slope_saturation: float = 0.0
    erodibility: float = 0.2
    cover_depth: float = 5.0
    height_unit_m: float = 0.0
    disc_saturation: float = 32.0
    disc_exponent: float = 0.5
    disc_saturation_cells: float = 0.0
    momentum_saturation_cells: float = 0.0
    slope_limit_erode: float = 0.0
    slope_limit_deposit: float = 0.0
    slope_limit_exit: float = 0.02
    max_erode: float = 12.5
    iter_erode: float = 25.0
    iter_deposit: float = 50.0
    ocean_deposition_rate: float = 0.3
    ocean_steps: int = 64
    fan_room: float = 50.0
    fan_slope: float = 0.05
    offshore_writeoff: float = 0.25
    glacial_every: int = 10
    ice_evap: float = 0.0
    glacial_from: float = 0.75
    glacial_rate: float = 6.0
    glacial_ramp: int = 4
    glacial_max: float = 20.0
    glacial_sticky: bool = True
    moraine_frac: float = 1.0
    climate_at_surface: bool = True
    ice_age_c: float = 8.0
    ice_history: bool = True
    ice_sheet: bool = True
    ice_sea_share: float = 0.0
    isostasy: float = 0.8
    flexure_km: float = 60.0
    isostasy_every: int = 20
    uplift_max_m: float = 0.0
    uplift_mode: str = "replay"
    resume: bool = True
    sea_mask_every: int = 10
    basin_fill_grade: float = 0.1
    basin_fill_min_m: float = 1.0
    lake_balance: bool = True
    lateral_rate: float = 0.0
    window_lakes: bool = False
    window_lake_evap: float = 0.0
    lake_fill: bool = True
    lake_trap: float = 0.9
    lake_fill_rise_m: float = 1.0
    lake_fill_load: float = 0.55
    dep_floor_m: float = 1.0
    flood_every: int = 10
    route_eps: float = 0.05
    pit_steps: int = 16
    chunk: int = 2048
    backend: str = "cpu"
    #: no counterpart in the reference (its particles write one cell a step): the wave apply's
    #: erode / deposit brush radius in cells, 0..4 (PgeParams.brush_radius)
    brush_radius: int = 0


@dataclass
class WorldGroup:
    seed: int = 0
    N_c: int = 1024
    cell_size_m: float = 9773.0
    land_fraction: float = 0.30
    halo: int = 4


@dataclass
class TectonicsGroup:
    shelf_fraction: float = 0.0


@dataclass
class HydroGroup:
    """The hydro knobs the erosion stage reads (the bake's ``hydro`` group,
    defaults as there): the lakes' open-water evaporation and the land's
    (the evaporation balance), the depth a lake must reach, and the share of
    the globe a below-sea body needs to count as open ocean."""

    lake_evap: float = 6.0
    land_evap: float = 3.0
    lake_min_depth: float = 0.5
    ocean_min_fraction: float = 0.02


@dataclass
class WorldParams:
    """Minimal stand-in for the bake's ``WorldParams``: the world, erosion
    and hydro groups plus the deterministic random streams."""

    world: WorldGroup = field(default_factory=WorldGroup)
    erosion: ErosionParams = field(default_factory=ErosionParams)
    tectonics: TectonicsGroup = field(default_factory=TectonicsGroup)
    hydro: HydroGroup = field(default_factory=HydroGroup)

    def rng(self, stage: str, *extra: int) -> np.random.Generator:
        if stage not in STAGE_SEED_OFFSETS:
            raise KeyError(f"unknown stage {stage!r}")
        mask = (1 << 64) - 1
        key = [(int(self.world.seed) + STAGE_SEED_OFFSETS[stage]) & mask, len(extra), *[int(e) & mask for e in extra]]
        return np.random.default_rng(key)

    def with_erosion(self, **kw) -> "WorldParams":
        return dataclasses.replace(self, erosion=dataclasses.replace(self.erosion, **kw))


def erosion_group(params) -> ErosionParams:
    """The erosion group of a WorldParams (ours or the bake's), or the
    argument itself when it already is one."""
    return params.erosion if hasattr(params, "erosion") else params


def cell_units(ep, name: str, cell_size_m: float) -> float:
    """One length parameter (metres) in the kernel's cell units."""
    return float(getattr(ep, name)) / float(cell_size_m)


def max_steps_of(ep, N: int) -> int:
    """``erosion.max_steps``, 0 meaning ``2 N`` (maps.py:777-778)."""
    return int(ep.max_steps) if ep.max_steps > 0 else 2 * int(N)


#: an iteration is split into at least this many chunks (maps.py:783)
MIN_CHUNKS = 16


def chunk_size(ep, n_particles: int) -> int:
    """Particles per chunk of the reference's serial apply (maps.py:786-787)."""
    return max(1, min(int(ep.chunk), -(-int(n_particles) // MIN_CHUNKS)))


def plain_knobs() -> dict:
    """The erosion knobs that switch off every host-refreshed process (routing
    flood, sea mask, lakes, glacial, isostasy, ice, basin fill, lateral cut):
    the plain particle path this library implements."""
    return dict(flood_every=0, sea_mask_every=0, lake_balance=False, lake_fill=False,
                glacial_every=0, isostasy=0.0, basin_fill_grade=0.0,
                ice_sheet=False, ice_history=False, climate_at_surface=False,
                ice_age_c=0.0, lateral_rate=0.0)


def check_plain(ep) -> None:
    """Raise ``ValueError`` when a knob asks for a process this library does
    not run: the ice sheet.  The bank cut (``lateral_rate``), the basin
    fill, isostasy, the routing surface (``flood_every``), the sea mask
    (``sea_mask_every``), the glacial pass (``glacial_every``, the ice line
    of the evaporation field), the planet's lake balance (``lake_balance``)
    with the lake parks (``lake_fill``, the exact apply only) and the lakes
    of a window (``window_lakes``, balanced with ``window_lake_evap > 0``)
    are supported."""
    bad = []
    if bool(getattr(ep, "ice_sheet", False)):
        bad.append("ice_sheet")
    if bad:
        raise ValueError("the b200 erosion backend runs the plain particle path only; switch off: " + ", ".join(bad))
