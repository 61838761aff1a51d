"""ctypes binding of libpgerosion.so (declarations: include/pgerosion.h).

The shared library is built in place next to this file (``csrc/Makefile``).
There is no fallback: if it is missing or fails to load, every entry point
raises, so the product path can only ever run the CUDA kernels.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libpgerosion.so"

PGE_OK, PGE_E_ARG, PGE_E_WORKSPACE, PGE_E_CUDA, PGE_E_UNSUPPORTED = 0, -1, -2, -3, -4
PREC_F64, PREC_F32 = 0, 1
APPLY_ORDERED, APPLY_WAVE = 0, 1
FX_MASS = float(2 ** 40)
FX_TRACK = float(2 ** 32)
N_DEATHS = 6
DEATH_NAMES = ("age", "ocean", "exit", "pit", "evap", "stop")

#: every function include/pgerosion.h declares
EXPORTS = (
    "pge_version", "pge_last_error", "pge_workspace_bytes", "pge_spawn_rain", "pge_count_pending",
    "pge_collect_pending", "pge_trace_apply", "pge_trace_changelist", "pge_read_accumulators", "pge_thermal",
    "pge_uplift", "pge_hold_datum", "pge_halo_gather", "pge_thermal_noalloc", "pge_slope_erode_cap",
    "pge_smooth_step", "pge_trace_apply_tape", "pge_adjoint_pass", "pge_halo_adjoint", "pge_route_flood", "pge_sea_base", "pge_glacial",
    "pge_window_lakes", "pge_lake_balance", "pge_lake_balance_fill", "pge_basin_fill",
    "pge_window_lake_balance", "pge_cubesphere_map", "pge_crmath", "pge_crmath_host",
)
#: cells the workspace-free thermal entry point accepts (include/pgerosion.h)
NOALLOC_MAX_CELLS = 262144
#: the erode / deposit brush (PgeParams.brush_radius, include/pgerosion.h)
BRUSH_MAX_RADIUS = 4
BRUSH_SCALE = 1024

c_i32, c_i64, c_f64, c_vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p


class PgeGrid(ctypes.Structure):
    _fields_ = [("F", c_i32), ("N", c_i32), ("H", c_i32), ("spherical", c_i32), ("deposit_on_exit", c_i32),
                ("metric_shared", c_i32), ("max_steps", c_i32), ("wave_tables", c_i32), ("max_droplets", c_i64),
                ("max_wave", c_i64), ("max_threads", c_i64)]


class PgeState(ctypes.Structure):
    _fields_ = [(n, c_vp) for n in ("height", "sediment", "discharge", "momentum", "pending", "base", "uplift",
                                    "hardness", "precip", "evap", "mask", "metric", "metric_inv", "erodibility", "route",
                                    "lake_flag", "roots", "lake_load", "lake_id", "lake_room")] + [("lakes", c_i64)]


class PgeSpawns(ctypes.Structure):
    _fields_ = [("face", c_vp), ("x", c_vp), ("y", c_vp), ("sed", c_vp), ("dir", c_vp), ("count", c_i64), ("volume0", c_f64)]


PARAM_DOUBLES = ("dt", "density", "friction", "deposition_rate", "evap_rate", "k_mom", "mom_scale", "k_disc",
                 "disc_saturation", "disc_exponent", "slope_gain", "slope_sat", "erodibility", "cover_depth",
                 "min_volume", "max_erode", "conc_scale", "ocean_rate", "fan_room", "dep_floor", "iter_erode",
                 "iter_deposit", "fan_slope", "offshore_writeoff", "ema", "lake_trap", "lateral_rate")
PARAM_INTS = ("max_steps", "pit_steps", "ocean_steps", "wave", "precision", "apply", "use_erode_cap", "threads_per_block",
              "blocks_per_sm", "trace_lanes", "apply_lanes", "brush_radius")


class PgeParams(ctypes.Structure):
    _fields_ = [(n, c_f64) for n in PARAM_DOUBLES] + [(n, c_i32) for n in PARAM_INTS]


class PgeStats(ctypes.Structure):
    _fields_ = [("droplets", c_i64), ("droplet_steps", c_i64), ("entries", c_i64), ("deaths", c_i64 * N_DEATHS),
                ("clamped", c_i64), ("overflow", c_i64), ("to_pending_fx", c_i64), ("deficit_out_fx", c_i64),
                ("lost_offshore_fx", c_i64), ("released_fx", c_i64), ("eroded_fx", c_i64), ("deposited_fx", c_i64),
                ("errors", c_i64)]


STATS_WORDS = ctypes.sizeof(PgeStats) // 8


class PgeTape(ctypes.Structure):
    _fields_ = [("state", c_vp), ("bits", c_vp), ("entry", c_vp), ("count", c_vp), ("droplets", c_i64), ("steps", c_i32),
                ("entries", c_i32), ("wave_acc", c_vp), ("waves", c_i64)]


#: ledger entries a droplet can make beyond its steps (its final deposits)
TAPE_EXTRA_ENTRIES = 8


class PgeLakeInfo(ctypes.Structure):
    _fields_ = [(n, c_i64) for n in ("lake_cells", "lake_cells_closed", "depressions", "overflowing", "closed", "dry")]


class PgeLakeFill(ctypes.Structure):
    _fields_ = ([(n, c_f64) for n in ("grade", "ice_evap", "rise")]
                + [(n, c_vp) for n in ("evap", "centres", "height", "sediment", "lake_load", "lake_id", "lay", "pending", "lake_room")]
                + [("lake_room_cap", c_i64), ("lakes", c_i64)] + [(n, c_f64) for n in ("parked", "laid", "stray", "room")])


class PgeHalo(ctypes.Structure):
    _fields_ = [("K", c_i64), ("dst", c_vp), ("src", c_vp), ("w", c_vp), ("rot", c_vp)]


class PgeError(RuntimeError):
    pass


_LIB = None


def load(path: str | os.PathLike | None = None):
    """Load the library (once) and declare the signatures."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise PgeError(f"{p} is not built: run `make -C procedural-generation_b200/csrc` (or __graft_entry__.build())")
    L = ctypes.CDLL(str(p))
    P = ctypes.POINTER
    L.pge_version.restype = ctypes.c_int
    L.pge_version.argtypes = []
    L.pge_last_error.restype = ctypes.c_int
    L.pge_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.pge_workspace_bytes.restype = ctypes.c_size_t
    L.pge_workspace_bytes.argtypes = [P(PgeGrid)]
    L.pge_spawn_rain.argtypes = [P(PgeGrid), P(PgeState), c_vp, c_vp, c_i64, P(PgeSpawns), c_vp, c_vp, c_vp, ctypes.c_size_t, c_vp]
    L.pge_count_pending.argtypes = [P(PgeGrid), P(PgeState), c_vp, c_vp, ctypes.c_size_t, c_vp]
    L.pge_collect_pending.argtypes = [P(PgeGrid), P(PgeState), P(PgeSpawns), c_i64, c_vp, c_vp, ctypes.c_size_t, c_vp]
    L.pge_trace_apply.argtypes = [P(PgeGrid), P(PgeState), P(PgeSpawns), P(PgeParams), c_vp, c_vp, c_vp, ctypes.c_size_t, c_vp]
    L.pge_trace_changelist.argtypes = [P(PgeGrid), P(PgeState), P(PgeSpawns), P(PgeParams), c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                       c_vp, c_vp, ctypes.c_size_t, c_vp]
    L.pge_read_accumulators.argtypes = [P(PgeGrid), c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.c_size_t, c_vp]
    L.pge_slope_erode_cap.argtypes = [P(PgeGrid), P(PgeState), c_f64, c_f64, c_vp, c_vp]
    L.pge_smooth_step.argtypes = [P(PgeGrid), c_vp, c_vp, c_vp, c_vp, c_f64, c_i32, c_f64, c_vp]
    L.pge_thermal.argtypes = [P(PgeGrid), P(PgeState), c_f64, c_f64, c_f64, c_f64, c_f64, c_f64, c_vp, ctypes.c_size_t, c_vp]
    L.pge_uplift.argtypes = [P(PgeGrid), P(PgeState), c_f64, c_f64, c_vp, ctypes.c_size_t, c_vp]
    L.pge_hold_datum.argtypes = [P(PgeGrid), P(PgeState), c_f64, c_f64, c_vp, c_vp, ctypes.c_size_t, c_vp]
    L.pge_halo_gather.argtypes = [P(PgeHalo), c_vp, c_i32, c_vp]
    L.pge_thermal_noalloc.argtypes = [P(PgeGrid), P(PgeState), c_f64, c_f64, c_f64, c_f64, c_f64, c_f64, c_vp]
    L.pge_trace_apply_tape.argtypes = [P(PgeGrid), P(PgeState), P(PgeSpawns), P(PgeParams), P(PgeTape), c_vp, c_vp,
                                       ctypes.c_size_t, c_vp]
    L.pge_adjoint_pass.argtypes = [P(PgeGrid), P(PgeState), P(PgeSpawns), P(PgeParams), P(PgeTape), c_i32, c_vp, c_vp, c_vp,
                                   c_vp, c_vp, c_vp, ctypes.c_size_t, c_vp]
    L.pge_halo_adjoint.argtypes = [P(PgeHalo), c_vp, c_vp]
    L.pge_route_flood.argtypes = [P(PgeGrid), P(PgeState), c_vp, c_f64, c_vp, c_i64, P(c_i64), c_vp, ctypes.c_size_t, c_vp]
    L.pge_window_lakes.argtypes = [P(PgeGrid), P(PgeState), c_f64, c_vp, c_vp, c_vp]
    L.pge_window_lake_balance.argtypes = [P(PgeGrid), c_vp, c_vp, c_vp, c_vp, c_f64, c_f64, c_vp, c_vp, c_vp]
    L.pge_basin_fill.argtypes = [P(PgeGrid), c_vp, c_vp, c_vp, c_f64, c_f64, c_vp, c_vp, P(c_i64)]
    L.pge_lake_balance.argtypes = [P(PgeGrid), c_vp, c_vp, c_vp, c_f64, c_vp, c_vp, c_vp, c_vp, c_f64, c_f64, c_f64, c_vp, c_vp, c_vp,
                                   P(PgeLakeInfo)]
    L.pge_lake_balance_fill.argtypes = [P(PgeGrid), c_vp, c_vp, c_vp, c_f64, c_vp, c_vp, c_vp, c_vp, c_f64, c_f64, c_f64, c_vp, c_vp,
                                        c_vp, P(PgeLakeFill), P(PgeLakeInfo)]
    L.pge_glacial.argtypes = [P(PgeGrid), P(PgeState), c_vp, c_f64, c_f64, c_i32, c_f64, c_f64, c_f64, c_f64, c_vp, c_vp,
                              ctypes.c_size_t, c_vp]
    L.pge_sea_base.argtypes = [P(PgeGrid), P(PgeState), c_vp, c_vp, c_f64, c_vp, c_vp, c_i64, P(c_i64), c_vp, ctypes.c_size_t, c_vp]
    L.pge_cubesphere_map.argtypes = [c_i32, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp]
    L.pge_crmath.argtypes = [c_i32, c_i64, c_vp, c_vp, c_vp]
    L.pge_crmath_host.argtypes = [c_i32, c_i64, c_vp, c_vp]
    for n in EXPORTS:
        if n not in ("pge_version", "pge_last_error", "pge_workspace_bytes"):
            getattr(L, n).restype = ctypes.c_int
    if path is None:
        _LIB = L
    return L


def last_error() -> str:
    buf = ctypes.create_string_buffer(512)
    load().pge_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(rc: int, what: str) -> None:
    if rc != PGE_OK:
        raise PgeError(f"{what} failed ({rc}): {last_error()}")
