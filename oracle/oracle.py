"""CPU oracle of the bake's plain particle-erosion path (test infrastructure).

Only the tests, the smoke check and the benchmark's CPU-baseline leg import
this module; the product never does.  It drives the C restatement in
``erosion_oracle.c`` with the reference's own control flow, in numpy:

* :class:`OracleState` -- ``ErosionState`` (bake/globe/erosion/maps.py:56-191)
* :func:`spawn_particles` -- maps.py:793-833
* :func:`run_iteration` -- maps.py:839-1047: rain spawns by inverse CDF on
  sorted uniforms, pending re-injection, packed samples, the chunk loop
  (trace on frozen samples, serial apply on the live terrain), fold, EMA
* :func:`thermal_erosion` -- maps.py:1050-1085
* :func:`apply_uplift` -- maps.py:1088-1147 (mean-free over the active interior)
* :func:`start_replay` -- maps.py:1159-1213
* :func:`hold_datum` -- maps.py:1446-1508
* :func:`apply_isostasy` -- maps.py:1331-1410 (the Laplace-Beltrami smoother
  of field.py:179-188, 372-404 restated in numpy)
* :func:`step` -- maps.py:1516-1617, plain path (plus isostasy, the
  routing surface, :func:`refresh_route` / :func:`priority_flood_eps`,
  maps.py:351-358 and route.py:31-125, and the sea mask,
  :func:`refresh_base`, maps.py:360-420 with hydro/run.py:64-83, and the
  glacial pass, :func:`glacial_carve`, erosion/glacial.py:162-257)

Every random number comes from ``params.rng("erosion", iteration)`` exactly
as in the reference, so a GPU run and this oracle see the same spawns.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liberosion_oracle.so"

MASK_OUTSIDE, MASK_ACTIVE, MASK_FROZEN = 0, 1, 2
DEATH_NAMES = ("age", "ocean", "exit", "pit", "evap", "stop")
SPREAD, LAKE_PARKS = 8, 8
NS = 16
S_SURF, S_ROUTE, S_SED, S_RFLAG, S_BASE = 0, 1, 7, 14, 15


def build() -> Path:
    """Compile the C oracle in place (gcc) and return the library path."""
    src = HERE / "erosion_oracle.c"
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_change_list_cap.restype = ctypes.c_int
        L.orc_change_list_cap.argtypes = [ctypes.c_int, ctypes.c_int]
        L.orc_set_threads(int(os.environ.get("PGE_ORACLE_THREADS", os.cpu_count() or 1)))
        _LIB = L
    return _LIB


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


class TraceParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "dt", "density", "friction", "deposition_rate", "evap_rate", "k_mom", "mom_scale", "k_disc",
        "disc_saturation", "disc_exponent", "slope_gain", "slope_sat", "erodibility", "cover_depth",
        "min_volume", "max_erode", "conc_scale", "ocean_rate", "fan_room", "dep_floor", "lake_trap", "lateral_rate",
        "lake_park")] + [
        (n, ctypes.c_int32) for n in ("max_steps", "pit_steps", "ocean_steps", "deposit_on_exit", "N", "H", "spherical", "F",
                                      "use_route", "pad")] + [("roots", ctypes.c_void_p)]


class ApplyParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("iter_erode", "iter_deposit", "fan_slope", "dep_floor", "offshore_writeoff")] + [
        ("use_erode_cap", ctypes.c_int32), ("use_route", ctypes.c_int32)]


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be contiguous"
    return ctypes.c_void_p(a.ctypes.data)


def libm(op: int, x) -> np.ndarray:
    """The C library's tan / atan / sin / cos (op 0..3) of a float64 array."""
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty_like(x)
    lib().orc_libm(ctypes.c_int(int(op)), ctypes.c_int64(x.size), _p(x), _p(y))
    return y


def brush_weights(r: int) -> np.ndarray:
    """The brush's integer weights (2r+1, 2r+1): 1024 x max(0, r + 1 - |(di, dj)|), rounded."""
    d = np.arange(-r, r + 1, dtype=np.float64)
    v = (r + 1) - np.sqrt(d[:, None] ** 2 + d[None, :] ** 2)
    return np.where(v > 0.0, np.floor(1024.0 * v + 0.5), 0.0).astype(np.int64)


def brush_spread(acc, mask, N, H, r, spherical=True):
    """A net change field (F, NE, NE) spread by the erode / deposit brush of the
    library's wave apply (no reference counterpart): every cell's change goes
    to the active cells of its face within distance < r + 1 (the interior ones
    on the sphere), in proportion to the weights; float64, no rounding to
    fixed point.  Linear, so spreading each entry's change or each cell's sum
    is the same up to the library's 2^-40 truncation."""
    if r <= 0:
        return acc.copy()
    NE = acc.shape[1]
    q = brush_weights(r)
    lo, hi = (H, H + N) if spherical else (0, NE)
    act = mask == MASK_ACTIVE
    valid = np.zeros_like(act)
    valid[:, lo:hi, lo:hi] = act[:, lo:hi, lo:hi]
    Q = np.zeros(acc.shape)  # each cell's total weight over its valid footprint (the cell itself always counts)
    for di in range(-r, r + 1):
        for dj in range(-r, r + 1):
            w = q[di + r, dj + r]
            if w == 0:
                continue
            if di == 0 and dj == 0:
                Q += w
                continue
            sh = np.zeros_like(valid)
            i0, i1 = max(0, -di), min(NE, NE - di)
            j0, j1 = max(0, -dj), min(NE, NE - dj)
            sh[:, i0:i1, j0:j1] = valid[:, i0 + di:i1 + di, j0 + dj:j1 + dj]
            Q += w * sh
    out = np.zeros_like(acc)
    src = np.where(acc != 0.0, acc / np.where(Q > 0, Q, 1.0), 0.0)
    for di in range(-r, r + 1):
        for dj in range(-r, r + 1):
            w = q[di + r, dj + r]
            if w == 0:
                continue
            if di == 0 and dj == 0:
                out += w * src
                continue
            i0, i1 = max(0, -di), min(NE, NE - di)
            j0, j1 = max(0, -dj), min(NE, NE - dj)
            part = np.zeros_like(acc)
            part[:, i0 + di:i1 + di, j0 + dj:j1 + dj] = w * src[:, i0:i1, j0:j1]
            out += np.where(valid, part, 0.0)
    return out


def change_list_cap(max_steps: int, lateral: bool = False) -> int:
    return int(lib().orc_change_list_cap(int(max_steps), int(bool(lateral))))


# --------------------------------------------------------------------------
# geometry wrappers (golden-vector tests)
# --------------------------------------------------------------------------
def to_sphere(face, u, v) -> np.ndarray:
    face = np.ascontiguousarray(face, np.int32)
    u = np.ascontiguousarray(u, np.float64)
    v = np.ascontiguousarray(v, np.float64)
    out = np.empty((face.size, 3))
    lib().orc_to_sphere_batch(ctypes.c_int64(face.size), _p(face), _p(u), _p(v), _p(out))
    return out


def from_sphere(xyz):
    xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
    n = xyz.shape[0]
    f = np.empty(n, np.int32)
    u = np.empty(n)
    v = np.empty(n)
    lib().orc_from_sphere_batch(ctypes.c_int64(n), _p(xyz), _p(f), _p(u), _p(v))
    return f, u, v


def transfer_velocity(face, u, v, a, b):
    face = np.ascontiguousarray(face, np.int32)
    uvab = np.ascontiguousarray(np.stack([u, v, a, b], -1), np.float64)
    n = face.size
    f2 = np.empty(n, np.int32)
    out = np.empty((n, 4))
    lib().orc_transfer_velocity_batch(ctypes.c_int64(n), _p(face), _p(uvab), _p(f2), _p(out))
    return f2, out[:, 0], out[:, 1], out[:, 2], out[:, 3]


# --------------------------------------------------------------------------
# state
# --------------------------------------------------------------------------
def _cu(ep, name, unit):
    return float(getattr(ep, name)) / float(unit)


@dataclass
class OracleState:
    height: np.ndarray
    sediment: np.ndarray
    discharge: np.ndarray
    momentum: np.ndarray
    hardness: np.ndarray
    precip: np.ndarray
    evap: np.ndarray
    uplift: np.ndarray
    mask: np.ndarray
    metric: np.ndarray
    metric_inv: np.ndarray
    N: int
    H: int
    spherical: bool
    height_unit_m: float
    grid: object = None
    base: np.ndarray = None
    pending: np.ndarray = None
    iteration: int = 0
    route: np.ndarray = None  # the epsilon-filled routing surface (refresh_route) or None
    #: overflowing lakes (uint8, 1 a lake, 2 a lake with room for its rivers' load; maps.py:87), set by the caller or
    #: by refresh_lakes_window; read with the routing surface only
    lake_flag: np.ndarray = None
    #: the share of the exchange the plants hold back (float32 (F, NE, NE), erosion.vegetation) or None
    roots: np.ndarray = None
    #: the lake parks' bookkeeping (erosion.lake_fill, maps.py:105-107): float64 load parked per cell, int32 lake of
    #: each cell (-1: none), float64 room left per lake; None: no lake keeps a load
    lake_load: np.ndarray = None
    lake_id: np.ndarray = None
    lake_room: np.ndarray = None
    base_at: int = None  # iteration of the last sea-mask refresh (refresh_base)
    ice_prev: np.ndarray = None  # the last glacial pass's ice (erosion.glacial_sticky)
    land_target: float | None = None
    deposit_on_exit: bool = False
    inflow_volume: float = 0.0  # window mode: spawn weight flowing in across the edge, not rain on the window
    samp: np.ndarray = field(default=None, repr=False)
    acc: np.ndarray = field(default=None, repr=False)
    disch_track: np.ndarray = field(default=None, repr=False)
    mom_track: np.ndarray = field(default=None, repr=False)
    iso_acc: np.ndarray = field(default=None, repr=False)

    def __post_init__(self):
        F, NE = self.height.shape[0], self.height.shape[1]
        z = lambda *s: np.zeros((F, NE, NE) + s, dtype=np.float64)
        self.samp = np.zeros((F, NE, NE, NS), np.float32) if self.samp is None else self.samp
        self.acc = z() if self.acc is None else self.acc
        self.pending = z() if self.pending is None else self.pending
        self.base = z() if self.base is None else self.base
        self.disch_track = z() if self.disch_track is None else self.disch_track
        self.mom_track = z(2) if self.mom_track is None else self.mom_track

    @classmethod
    def from_world(cls, world, params) -> "OracleState":
        """Global six-face state from a synthetic world (metres -> cell units),
        as ``ErosionState.from_grid`` builds it."""
        grid = world.grid
        unit = grid.cell_size_m
        F, NE = 6, grid.NE
        c = lambda a, dt: np.ascontiguousarray(np.asarray(a), dtype=dt)
        return cls(
            height=c(world.bedrock, np.float64) / unit,
            sediment=np.zeros((F, NE, NE)),
            discharge=np.zeros((F, NE, NE)),
            momentum=np.zeros((F, NE, NE, 2)),
            hardness=c(world.hardness, np.float32),
            precip=c(world.precip, np.float32),
            evap=c(world.evap, np.float32),
            uplift=c(world.uplift, np.float64) / unit,
            mask=np.ones((F, NE, NE), np.uint8),
            metric=np.ascontiguousarray(np.broadcast_to(grid.metric_face, (F, NE, NE, 3)), np.float32),
            metric_inv=np.ascontiguousarray(np.broadcast_to(grid.metric_inv_face, (F, NE, NE, 3)), np.float32),
            N=grid.N, H=grid.H, spherical=True, height_unit_m=unit, grid=grid,
            land_target=float(world.land_fraction),
        )

    @property
    def F(self):
        return self.height.shape[0]

    @property
    def NE(self):
        return self.height.shape[1]

    @property
    def interior(self):
        H, N = self.H, self.N
        return (slice(None), slice(H, H + N), slice(H, H + N))

    def surface(self):
        return self.height + self.sediment

    def total_mass(self) -> float:
        act = self.mask[self.interior] == MASK_ACTIVE
        return float(np.sum((self.height + self.sediment + self.pending)[self.interior][act]))

    def pack(self):
        n = self.height.size
        lib().orc_pack(ctypes.c_int64(n), _p(self.samp), _p(self.height), _p(self.sediment), _p(self.discharge),
                       _p(self.momentum), _p(self.evap), _p(self.hardness), _p(self.metric), _p(self.metric_inv),
                       _p(self.base), None if getattr(self, "route", None) is None else _p(self.route),
                       None if getattr(self, "lake_flag", None) is None else _p(self.lake_flag))

    def exchange_halos(self):
        if not self.spherical:
            return
        from pgerosion.geometry import exchange_halos as xh

        for a in (self.height, self.sediment, self.discharge):
            xh(self.grid, a)
        xh(self.grid, self.momentum, vector=True)


# --------------------------------------------------------------------------
# the iteration
# --------------------------------------------------------------------------
def _ep(params):
    return params.erosion if hasattr(params, "erosion") else params


def max_steps_of(ep, N):
    return int(ep.max_steps) if ep.max_steps > 0 else 2 * int(N)


def chunk_size(ep, n):
    return max(1, min(int(ep.chunk), -(-int(n) // 16)))


def spawn_weights(state):
    F, NE = state.F, state.NE
    inter = np.zeros((F, NE, NE), dtype=bool)
    inter[state.interior] = True
    ok = inter & (state.mask == MASK_ACTIVE) & (state.height + state.sediment >= state.base) & (state.precip > 0)
    idx = np.flatnonzero(ok)
    return idx, state.precip.reshape(-1)[idx].astype(np.float64)


def spawn_particles(state, n_particles, rng):
    idx, w = spawn_weights(state)
    if idx.size == 0 or n_particles <= 0:
        return None
    total = float(w.sum())
    if total <= 0.0:
        return None
    cdf = np.cumsum(w)
    u = np.sort(rng.random(n_particles))
    off = rng.random((n_particles, 2))
    k = np.empty(n_particles, np.int64)
    lib().orc_spawn_cells(ctypes.c_int64(cdf.size), _p(cdf), ctypes.c_int64(n_particles), _p(u), _p(k))
    flat = idx[k]
    NE = state.NE
    f = flat // (NE * NE)
    rem = flat - f * NE * NE
    ei = rem // NE
    ej = rem - ei * NE
    x = (ei - state.H).astype(np.float64) + off[:, 0]
    y = (ej - state.H).astype(np.float64) + off[:, 1]
    return f.astype(np.int64), x, y, total / n_particles


def trace_params(state, ep, volume0, conc_scale, mom_scale=1.0, disc_sat=None) -> TraceParams:
    u = state.height_unit_m
    return TraceParams(
        dt=float(ep.dt), density=float(ep.density), friction=float(ep.friction), deposition_rate=float(ep.deposition_rate),
        evap_rate=float(ep.evap_rate), k_mom=float(ep.k_mom), mom_scale=float(mom_scale), k_disc=float(ep.k_disc),
        disc_saturation=float(ep.disc_saturation if disc_sat is None else disc_sat), disc_exponent=float(ep.disc_exponent),
        slope_gain=float(ep.slope_gain), slope_sat=float(ep.slope_saturation), erodibility=float(ep.erodibility),
        cover_depth=_cu(ep, "cover_depth", u), min_volume=float(ep.min_volume_frac) * float(volume0),
        max_erode=_cu(ep, "max_erode", u), conc_scale=float(conc_scale), ocean_rate=float(ep.ocean_deposition_rate),
        fan_room=_cu(ep, "fan_room", u), dep_floor=_cu(ep, "dep_floor_m", u), lake_trap=float(getattr(ep, "lake_trap", 0.9)),
        lateral_rate=float(getattr(ep, "lateral_rate", 0.0)),
        lake_park=1.0 if (state.spherical and bool(getattr(ep, "lake_fill", False)) and bool(getattr(ep, "lake_balance", False)))
        else 0.0,
        max_steps=max_steps_of(ep, state.N), pit_steps=int(ep.pit_steps), ocean_steps=int(ep.ocean_steps),
        deposit_on_exit=int(bool(state.deposit_on_exit)), N=int(state.N), H=int(state.H), spherical=int(bool(state.spherical)),
        F=int(state.F), use_route=int(getattr(state, "route", None) is not None),
        roots=None if getattr(state, "roots", None) is None else _p(state.roots))


def apply_params(state, ep, iter_deposit) -> ApplyParams:
    u = state.height_unit_m
    return ApplyParams(iter_erode=_cu(ep, "iter_erode", u), iter_deposit=float(iter_deposit), fan_slope=float(ep.fan_slope),
                       dep_floor=_cu(ep, "dep_floor_m", u), offshore_writeoff=float(ep.offshore_writeoff),
                       use_erode_cap=int(float(ep.slope_limit_erode) > 0.0),
                       use_route=int(getattr(state, "route", None) is not None))


def trace(state, tp: TraceParams, sp_face, sp_x, sp_y, sp_sed, sp_dir, volume0):
    """Trace particles on the current packed samples; returns the change list
    ``(cl_cell, cl_delta, cl_vol, cl_mom, cl_count, cl_lo, cl_hi, sp_death)``."""
    P = int(sp_face.shape[0])
    cap = change_list_cap(tp.max_steps, tp.lateral_rate > 0.0)
    cl_cell = np.zeros(P * cap, np.int32)
    cl_delta = np.zeros(P * cap)
    cl_vol = np.zeros(P * cap, np.float32)
    cl_mom = np.zeros((P * cap, 2), np.float32)
    cnt = np.zeros(P, np.int64)
    lo = np.zeros(P, np.int64)
    hi = np.zeros(P, np.int64)
    death = np.zeros(P, np.int8)
    c = lambda a, dt: np.ascontiguousarray(a, dt)
    lib().orc_trace(ctypes.byref(tp), _p(state.samp), _p(state.mask), ctypes.c_int64(P), _p(c(sp_face, np.int64)),
                    _p(c(sp_x, np.float64)), _p(c(sp_y, np.float64)), _p(c(sp_sed, np.float64)), _p(c(sp_dir, np.float64)),
                    ctypes.c_double(volume0), _p(cl_cell), _p(cl_delta), _p(cl_vol), _p(cl_mom), _p(cnt), _p(lo), _p(hi),
                    _p(death))
    return cl_cell, cl_delta, cl_vol, cl_mom, cnt, lo, hi, death


def apply(state, ap: ApplyParams, cl, cap, ecap=None):
    cl_cell, cl_delta, cl_vol, cl_mom, cnt = cl[:5]
    out4 = np.zeros(4)
    ecap = np.zeros(1) if ecap is None else ecap
    lib().orc_apply(ctypes.byref(ap), _p(cl_cell), _p(cl_delta), _p(cl_vol), _p(cl_mom), ctypes.c_int64(cnt.size),
                    _p(np.ascontiguousarray(cnt)), ctypes.c_int(cap), _p(state.height), _p(state.sediment), _p(state.acc),
                    _p(state.pending), _p(state.samp), _p(state.disch_track), _p(state.mom_track), _p(state.mask), _p(ecap),
                    _p(out4), *((None, None, None) if getattr(state, "lake_id", None) is None else
                                (_p(state.lake_load), _p(state.lake_id), _p(state.lake_room))))
    return int(out4[0]), float(out4[1]), float(out4[2]), float(out4[3])


def run_iteration(state, params, iteration_key, n_particles=None, particles_per_cell=None, rng_stage="erosion", chunk=None) -> dict:
    """One particle pass with the reference's chunked serial-apply semantics.
    ``chunk`` overrides ``erosion.chunk`` (particles per chunk)."""
    ep = _ep(params)
    key = iteration_key if isinstance(iteration_key, (tuple, list)) else (int(iteration_key),)
    rng = params.rng(rng_stage, *key)
    t0 = time.time()
    n_cells = int(np.count_nonzero(state.mask[state.interior] == MASK_ACTIVE))
    if n_particles is None:
        ppc = ep.particles_per_cell if particles_per_cell is None else particles_per_cell
        n_particles = max(1, int(round(ppc * n_cells)))
    sp = spawn_particles(state, n_particles, rng)
    stats = {"particles": 0, "entries": 0, "steps_mean": 0.0}
    if sp is None:
        return stats
    sp_face, sp_x, sp_y, volume0 = sp
    sp_sed = np.zeros(sp_face.shape[0])
    sp_dir = np.zeros(sp_face.shape[0])
    pend_cells = np.flatnonzero(state.pending.reshape(-1) > 0.0)
    released = 0.0
    if pend_cells.size:
        NE = state.NE
        pf = pend_cells // (NE * NE)
        rem = pend_cells - pf * NE * NE
        pei = rem // NE
        pej = rem - pei * NE
        loads = state.pending.reshape(-1)[pend_cells]
        released = float(loads.sum())
        sp_face = np.concatenate([sp_face, pf.astype(np.int64)])
        sp_x = np.concatenate([sp_x, (pei - state.H) + 0.5])
        sp_y = np.concatenate([sp_y, (pej - state.H) + 0.5])
        sp_sed = np.concatenate([sp_sed, loads])
        sp_dir = np.concatenate([sp_dir, rng.random(pend_cells.size) * (2.0 * np.pi)])
        state.pending.reshape(-1)[pend_cells] = 0.0
    state.pack()
    state.acc[...] = 0.0
    disc_sat = float(ep.disc_saturation)
    mom_scale = 1.0
    if float(ep.disc_saturation_cells) > 0.0 or float(ep.momentum_saturation_cells) > 0.0:
        total = float(volume0) * float(n_particles)
        n_rain = max(int(spawn_weights(state)[0].size), 1)
        rain_per_cell = max(total - float(getattr(state, "inflow_volume", 0.0)), 0.0) / n_rain  # maps.py:913-917
        rain_per_cell = rain_per_cell if rain_per_cell > 0.0 else total / n_rain
        if float(ep.disc_saturation_cells) > 0.0:
            disc_sat = float(ep.disc_saturation_cells) * rain_per_cell
        if float(ep.momentum_saturation_cells) > 0.0:
            mom_scale = float(volume0) / (float(ep.momentum_saturation_cells) * rain_per_cell)
    use_ecap = float(ep.slope_limit_erode) > 0.0
    ecap = None
    if use_ecap:
        ecap = np.empty_like(state.height)
        lib().orc_slope_erode_cap(ctypes.c_int(state.F), ctypes.c_int(state.NE), _p(state.height), _p(state.sediment),
                                  _p(state.mask), ctypes.c_double(float(ep.slope_limit_erode)),
                                  ctypes.c_double(float(ep.slope_limit_exit)), _p(ecap))
    iter_deposit = _cu(ep, "iter_deposit", state.height_unit_m)
    if float(ep.slope_limit_deposit) > 0.0:
        iter_deposit = min(iter_deposit, float(ep.slope_limit_deposit) * math.sqrt(2.0) * 0.3)
    max_steps = max_steps_of(ep, state.N)
    cap = change_list_cap(max_steps, float(getattr(ep, "lateral_rate", 0.0)) > 0.0)
    P = sp_face.shape[0]
    chunk = chunk_size(ep, P) if chunk is None else int(chunk)
    tp = trace_params(state, ep, volume0, chunk / (volume0 * P), mom_scale, disc_sat)
    ap = apply_params(state, ep, iter_deposit)
    deaths = np.zeros(len(DEATH_NAMES), np.int64)
    entries = steps = n_clamp = 0
    to_pending = lost = lost_offshore = 0.0
    t_trace = t_apply = 0.0
    for c0 in range(0, P, chunk):
        c1 = min(P, c0 + chunk)
        t1 = time.time()
        cl = trace(state, tp, sp_face[c0:c1], sp_x[c0:c1], sp_y[c0:c1], sp_sed[c0:c1], sp_dir[c0:c1], volume0)
        t2 = time.time()
        nc, tpd, lo, lo_off = apply(state, ap, cl, cap, ecap)
        t_trace += t2 - t1
        t_apply += time.time() - t2
        n_clamp += nc
        to_pending += tpd
        lost += lo
        lost_offshore += lo_off
        cnt = cl[4]
        entries += int(cnt.sum())
        steps += _count_steps(cl[2], cnt, cap)
        deaths += np.bincount(cl[7], minlength=deaths.size)
    lib().orc_fold(ctypes.c_int64(state.height.size), _p(state.height), _p(state.sediment), _p(state.acc), _p(state.mask))
    lib().orc_ema(ctypes.c_int64(state.height.size), _p(state.discharge), _p(state.momentum), _p(state.disch_track),
                  _p(state.mom_track), _p(state.mask), ctypes.c_double(float(ep.ema)))
    stats.update({"particles": int(P), "entries": entries, "steps_mean": entries / max(P, 1), "volume": float(volume0),
                  "seconds": time.time() - t0, "droplet_steps": steps})
    stats["deaths"] = {n: int(c) for n, c in zip(DEATH_NAMES, deaths)}
    stats["clamped"] = n_clamp
    stats["to_pending"] = to_pending
    stats["released"] = released
    stats["pending_total"] = float(state.pending[state.interior].sum())
    stats["deficit_out"] = lost
    stats["lost_offshore"] = lost_offshore
    stats["seconds_trace"] = t_trace
    stats["seconds_apply"] = t_apply
    stats["chunk"] = int(chunk)
    return stats


def _count_steps(cl_vol, cnt, cap) -> int:
    """Droplet-steps: change-list entries with volume >= 0."""
    P = cnt.size
    idx = np.arange(cap)[None, :] < cnt[:, None]
    return int(np.count_nonzero((cl_vol[: P * cap].reshape(P, cap) >= 0.0) & idx))


def thermal_erosion(state, params):
    ep = _ep(params)
    hard = state.hardness
    talus = (np.float32(ep.talus_slope_soft) + np.float32(ep.talus_slope_hard - ep.talus_slope_soft) * hard).astype(np.float64)
    dep_floor = _cu(ep, "dep_floor_m", state.height_unit_m)
    cap = _cu(ep, "thermal_max", state.height_unit_m)
    _mass_wasting(state, talus, float(ep.thermal_rate), cap, state.mask, dep_floor)
    if ep.creep_rate > 0.0:
        cmask = np.where(state.height + state.sediment < state.base, np.uint8(MASK_FROZEN), state.mask).astype(np.uint8)
        _mass_wasting(state, np.zeros_like(talus), float(ep.creep_rate), cap, cmask, dep_floor)


def _mass_wasting(state, talus, rate, cap, mask, dep_floor):
    sh = state.height.shape
    scratch = [np.empty(sh) for _ in range(5)]
    lib().orc_mass_wasting(ctypes.c_int(state.F), ctypes.c_int(state.NE), _p(state.height), _p(state.sediment),
                           _p(state.metric), _p(np.ascontiguousarray(talus)), _p(np.ascontiguousarray(mask)),
                           ctypes.c_double(rate), ctypes.c_double(cap), ctypes.c_double(dep_floor), *[_p(s) for s in scratch])


def _applied_uplift(state, cap=None):
    u = state.uplift if cap is None else np.minimum(state.uplift, float(cap))
    mean = 0.0
    if state.spherical:
        iact = state.mask[state.interior] == MASK_ACTIVE
        mean = float(u[state.interior][iact].mean()) if iact.any() else 0.0
    return u, mean


def apply_uplift(state, cap=None):
    act = state.mask == MASK_ACTIVE
    u, mean = _applied_uplift(state, cap)
    state.height[act] += u[act] - mean


def start_replay(state, params):
    ep = _ep(params)
    if not state.spherical or str(getattr(ep, "uplift_mode", "stack")) != "replay":
        return None
    u, mean = _applied_uplift(state, None)
    act = state.mask == MASK_ACTIVE
    total = np.zeros_like(state.height)
    total[act] = float(int(ep.iterations)) * (u[act] - mean)
    state.height -= total
    state.exchange_halos()
    shift = hold_datum(state, state.land_target)
    return {"datum_shift": shift}


def hold_datum(state, land_fraction, level=0.0):
    surf = (state.height[state.interior] + state.sediment[state.interior]).ravel()
    M = surf.size
    n_land = min(max(int(round(float(land_fraction) * M)), 0), M)
    if n_land == 0:
        q = float(surf.max()) + 1.0
    elif n_land == M:
        q = float(surf.min())
    else:
        k = M - n_land
        q = float(np.partition(surf, k)[k])
    q -= float(level)
    if q != 0.0:
        state.height -= q
        np.subtract(state.base, q, out=state.base, where=state.base < 0.0)
        if state.route is not None:  # registered with the terrain (maps.py:1498-1499)
            state.route -= q
    return q


def refresh_route(state, eps):
    """maps.py:351-358: the routing surface of the current terrain, then the
    linear halo exchange."""
    from pgerosion.geometry import exchange_halos as xh

    owner = state.grid.owner if state.spherical else np.arange(state.height.size, dtype=np.int64).reshape(state.height.shape)
    state.route = priority_flood_eps(state.height + state.sediment, state.mask, owner, state.H, state.N, float(eps), state.base)
    if state.spherical:
        xh(state.grid, state.route, linear=True)


#: hydro.lake_min_depth's default (m): the depth a window lake must reach to be one
LAKE_MIN_DEPTH_M = 0.5


def _window_lake_balance(state, surf, min_depth, lake_evap):
    """maps.py:675-736: a window's depressions settled against evaporation --
    the flat flood (hydro/priority_flood.py:193-270) draining to the inactive
    cells and the array's border, the rain accumulated down the flood tree
    (zoom/bake.py:323-330), each depression (scipy's 8-connected labels)
    where its inflow meets lake_evap x evap over the water; returns (lake
    (NE, NE) bool, counts) and lowers the route to the water on the lakes."""
    import heapq

    from scipy import ndimage

    s = np.ascontiguousarray(surf[0], np.float32)
    W = s.shape[0]
    active = state.mask[0] == MASK_ACTIVE
    drain = ~active
    drain[0, :] = drain[-1, :] = drain[:, 0] = drain[:, -1] = True
    sf, df = s.reshape(-1), drain.reshape(-1)
    M = sf.size
    filled = sf.copy()
    visited = np.zeros(M, bool)
    parent = np.full(M, -1, np.int64)
    pop_seq, heap, fifo, seq = [], [], [], 0

    def nbrs(c):
        i, j = divmod(c, W)
        for k in range(8):
            i2, j2 = i + _D8_DI[k], j + _D8_DJ[k]
            if 0 <= i2 < W and 0 <= j2 < W:
                yield i2 * W + j2

    for c in range(M):
        if df[c]:
            visited[c] = True
            if any(not df[n] for n in nbrs(c)):
                heapq.heappush(heap, (float(sf[c]), seq, c))
                seq += 1
    head = 0
    while head < len(fifo) or heap:
        if head < len(fifo):
            c = fifo[head]
            head += 1
        else:
            c = heapq.heappop(heap)[2]
        lvl = filled[c]
        pop_seq.append(c)
        for n in nbrs(c):
            if visited[n]:
                continue
            visited[n] = True
            parent[n] = c
            if sf[n] <= lvl:
                filled[n] = lvl
                fifo.append(n)
            else:
                filled[n] = sf[n]
                heapq.heappush(heap, (float(sf[n]), seq, n))
                seq += 1
    acc = np.ascontiguousarray(state.precip[0], np.float64).ravel().copy()
    for c in reversed(pop_seq):
        if parent[c] >= 0:
            acc[parent[c]] += acc[c]
    filled = filled.reshape(s.shape)
    acc = acc.reshape(s.shape)
    dep = (filled > s + np.float32(1e-6)) & active
    lab, n = ndimage.label(dep, structure=np.ones((3, 3), bool))
    counts = {"depressions": int(n), "overflowing": 0, "closed": 0, "dry": 0}
    out = np.zeros(s.shape, bool)
    if n == 0:
        return out, counts
    cells = np.flatnonzero(lab.ravel() > 0)
    cells = cells[np.lexsort((s.ravel()[cells], lab.ravel()[cells]))]
    lab_s = lab.ravel()[cells].astype(np.int64)
    ptr = np.searchsorted(lab_s, np.arange(1, n + 2))
    demand = np.cumsum(lake_evap * np.maximum(state.evap[0].ravel()[cells].astype(np.float64), 0.0))
    z = s.ravel()[cells].astype(np.float64)
    spill = np.atleast_1d(ndimage.maximum(filled, lab, np.arange(1, n + 1)))
    inflow = np.atleast_1d(ndimage.maximum(acc, lab, np.arange(1, n + 1)))
    level = np.zeros(n)
    for k in range(n):
        a, b = ptr[k], ptr[k + 1]
        if b <= a:
            continue
        need, before = float(inflow[k]), (demand[a - 1] if a > 0 else 0.0)
        loss = demand[a:b] - before
        if need <= 0.0:
            level[k] = z[a] - 1.0
            counts["dry"] += 1
        elif loss[-1] <= need:
            level[k] = float(spill[k])
            counts["overflowing"] += 1
        else:
            i = int(np.searchsorted(loss, need))
            level[k] = float(z[a + min(i, b - a - 1)])
            counts["closed"] += 1
    lv = np.zeros(n + 1)
    lv[1:] = level
    water = np.where(lab > 0, lv[lab], s)
    out = (water - s > min_depth) & active
    r = state.route[0]
    r[out] = np.minimum(r[out], water[out])
    return out, counts


def refresh_lakes_window(state, min_depth, lake_evap=0.0) -> dict:
    """maps.py:629-673: every depression the routing flood fills more than
    ``min_depth`` (cell units) deep is an overflowing lake, flagged on the
    interior's active cells (the halos stay 0); with ``lake_evap > 0`` each
    settles where its inflow meets its evaporation instead (and the route is
    lowered to the water on the lakes)."""
    flag = np.zeros(state.height.shape, np.uint8)
    if state.route is None:
        state.lake_flag = flag
        return {"lake_cells": 0}
    surf = state.height + state.sediment
    lake = ((state.route - surf) > float(min_depth)) & (state.mask == MASK_ACTIVE)
    st = {}
    if float(lake_evap) > 0.0:
        out, st = _window_lake_balance(state, surf, float(min_depth), float(lake_evap))
        lake = out[None]
    inter = state.interior
    flag[inter] = lake[inter]
    state.lake_flag = flag
    return {"lake_cells": int(lake[inter].sum()), **st}


def laplacian(state, d):
    """FaceField.laplacian (field.py:179-188, 372-404): the flux-form
    Laplace-Beltrami operator at extended indices 1..NE-2 (0 on the outer
    ring), per m^2, as the float32 field the reference returns."""
    from pgerosion.isostasy import sqrt_det_metric

    grid = state.grid
    gi = grid.metric_inv_face.astype(np.float64)[None]
    sq = sqrt_det_metric(grid).astype(np.float64)[None]
    C = slice(1, -1)
    P = slice(2, None)
    M = slice(None, -2)
    fj_c = 0.5 * (d[:, C, P] - d[:, C, M])
    fj_p = 0.5 * (d[:, P, P] - d[:, P, M])
    fj_m = 0.5 * (d[:, M, P] - d[:, M, M])
    fi_c = 0.5 * (d[:, P, C] - d[:, M, C])
    fi_p = 0.5 * (d[:, P, P] - d[:, M, P])
    fi_m = 0.5 * (d[:, P, M] - d[:, M, M])
    gii = 0.5 * (gi[:, C, C, 0] + gi[:, P, C, 0])
    gij = 0.5 * (gi[:, C, C, 1] + gi[:, P, C, 1])
    sv = 0.5 * (sq[:, C, C] + sq[:, P, C])
    Fi_p = sv * (gii * (d[:, P, C] - d[:, C, C]) + gij * 0.5 * (fj_c + fj_p))
    gii = 0.5 * (gi[:, C, C, 0] + gi[:, M, C, 0])
    gij = 0.5 * (gi[:, C, C, 1] + gi[:, M, C, 1])
    sv = 0.5 * (sq[:, C, C] + sq[:, M, C])
    Fi_m = sv * (gii * (d[:, C, C] - d[:, M, C]) + gij * 0.5 * (fj_c + fj_m))
    gjj = 0.5 * (gi[:, C, C, 2] + gi[:, C, P, 2])
    gij = 0.5 * (gi[:, C, C, 1] + gi[:, C, P, 1])
    sv = 0.5 * (sq[:, C, C] + sq[:, C, P])
    Fj_p = sv * (gjj * (d[:, C, P] - d[:, C, C]) + gij * 0.5 * (fi_c + fi_p))
    gjj = 0.5 * (gi[:, C, C, 2] + gi[:, C, M, 2])
    gij = 0.5 * (gi[:, C, C, 1] + gi[:, C, M, 1])
    sv = 0.5 * (sq[:, C, C] + sq[:, C, M])
    Fj_m = sv * (gjj * (d[:, C, C] - d[:, C, M]) + gij * 0.5 * (fi_c + fi_m))
    out = np.zeros_like(d)
    out[:, C, C] = (Fi_p - Fi_m + Fj_p - Fj_m) / sq[:, C, C]
    out /= grid.cell_size_m ** 2
    return out.astype(np.float32)


_KAPPA_CACHE: dict = {}


def smoothing_kappa(state) -> float:
    """maps._smoothing_kappa (maps.py:1331-1363): 0.9 / lambda_max by 40 steps
    of power iteration from default_rng(0) noise; cached per grid."""
    from pgerosion.geometry import exchange_halos as xh

    grid = state.grid
    key = (grid.N, grid.H, float(grid.cell_size_m))
    if key not in _KAPPA_CACHE:
        rng = np.random.default_rng(0)
        H, N, NE = grid.H, grid.N, grid.NE
        f = np.zeros((6, NE, NE))
        f[:, H:H + N, H:H + N] = rng.standard_normal((6, N, N))
        xh(grid, f)
        c2, lam = float(grid.cell_size_m) ** 2, 8.0
        for _ in range(40):
            xh(grid, f, linear=True)
            Lv = laplacian(state, f).astype(np.float64) * c2
            num = float(np.sqrt((Lv[:, H:-H, H:-H] ** 2).sum()))
            den = float(np.sqrt((f[:, H:-H, H:-H] ** 2).sum()))
            if num <= 0.0 or den <= 0.0:
                break
            lam = num / den
            f = Lv / num
        _KAPPA_CACHE[key] = 0.9 / max(lam, 1e-6)
    return _KAPPA_CACHE[key]


def apply_isostasy(state, params) -> dict:
    """maps.apply_isostasy (maps.py:1366-1410): -isostasy x iso_acc, spread by
    ceil(sigma^2 / (2 kappa)) explicit Laplace-Beltrami steps (linear halos
    before each), added mean-free over the active interior; zeroes iso_acc."""
    from pgerosion.geometry import exchange_halos as xh

    ep = _ep(params)
    d = state.iso_acc
    k = float(ep.isostasy)
    load = (-k * d).astype(np.float64)
    cell = float(state.height_unit_m)
    sig = float(ep.flexure_km) * 1000.0 / cell
    sig = min(sig, state.N / 8.0)
    kappa = smoothing_kappa(state)
    n = int(np.ceil(sig * sig / (2.0 * kappa))) if sig >= 0.5 else 0
    f = load.copy()
    for _ in range(n):
        xh(state.grid, f, linear=True)
        f += kappa * laplacian(state, f).astype(np.float64) * (cell * cell)
    xh(state.grid, f, linear=True)
    act = state.mask == MASK_ACTIVE
    iact = state.mask[state.interior] == MASK_ACTIVE
    mean = float(f[state.interior][iact].mean()) if iact.any() else 0.0
    state.height[act] += (f[act] - mean)
    moved = float(np.abs(d[state.interior]).sum())
    state.iso_acc[...] = 0.0
    return {"sigma_cells": sig, "diffusion_steps": n, "kappa": kappa, "load_abs_cells": moved,
            "rebound_max": float((f[state.interior] - mean).max()), "rebound_min": float((f[state.interior] - mean).min())}


def interior_cell_area(grid) -> np.ndarray:
    """(6, N, N) float32 cell areas in m^2 (cubesphere.py:505-517: the
    float32 sqrt det g times the cell size squared, rounded to float32)."""
    g = grid.metric_face.astype(np.float64)
    sq = np.sqrt(g[..., 0] * g[..., 2] - g[..., 1] ** 2).astype(np.float32)
    a = (sq.astype(np.float64) * float(grid.cell_size_m) ** 2).astype(np.float32)
    H, N = grid.H, grid.N
    return np.broadcast_to(a[H:H + N, H:H + N], (6, N, N)).copy()


def below_sea_components(surf32, grid, min_fraction):
    """hydro/run.py:64-83 with hydro/lakes.py:19-46: the interior cells
    under the waterline, their 8-connected components (a walk from the
    lowest unlabelled cell along the owner table's D8 neighbours), and which
    components are open ocean (area >= min_fraction of the globe, and the
    largest)."""
    N, H = grid.N, grid.H
    NE = N + 2 * H
    below = (np.asarray(surf32) < 0.0).reshape(-1)
    if not below.any():
        return below, None, None
    owner = grid.owner.reshape(-1)
    labels = np.full(below.size, -1, np.int32)
    n = 0
    for s0 in range(below.size):
        if not below[s0] or labels[s0] >= 0:
            continue
        labels[s0] = n
        stack = [s0]
        while stack:
            c = stack.pop()
            f, rem = divmod(c, N * N)
            i, j = divmod(rem, N)
            for di, dj in D8:
                o = int(owner[(f * NE + i + H + di) * NE + j + H + dj])
                f2, r2 = divmod(o, NE * NE)
                q = (f2 * N + r2 // NE - H) * N + r2 % NE - H
                if below[q] and labels[q] < 0:
                    labels[q] = n
                    stack.append(q)
        n += 1
    area = interior_cell_area(grid).reshape(-1).astype(np.float64)
    per = np.bincount(labels[below], weights=area[below], minlength=max(n, 1))
    keep = per >= float(min_fraction) * float(area.sum())
    keep[int(np.argmax(per))] = True
    return below, labels, keep


def refresh_base(state, min_fraction) -> dict:
    """maps.py:360-420: the base level -- 0 on the open ocean and on land,
    a closed below-sea basin's deepest surface on its cells; halos copied
    from their nearest interior source."""
    base = np.zeros_like(state.height)
    info = {"closed_cells": 0, "closed_basins": 0, "sea_cells": 0, "deepest_basin_floor": 0.0}
    inter = state.interior
    surf = (state.height[inter] + state.sediment[inter]).astype(np.float64)
    below, labels, keep = below_sea_components(surf.astype(np.float32), state.grid, float(min_fraction))
    if labels is not None:
        sea = below & keep[np.maximum(labels, 0)]
        closed = below & ~sea
        info["sea_cells"] = int(sea.sum())
        info["closed_cells"] = int(closed.sum())
        if closed.any():
            lab = labels[closed]
            floor = np.zeros(keep.size, dtype=np.float64)
            np.minimum.at(floor, lab, surf.reshape(-1)[closed])
            inner = np.zeros(surf.size, dtype=np.float64)
            inner[closed] = floor[lab]
            base[inter] = inner.reshape(surf.shape)
            info["closed_basins"] = int(np.unique(lab).size)
            info["deepest_basin_floor"] = float(floor.min())
    hm = state.grid.halo
    flat = base.reshape(-1, 1)
    flat[hm.dst] = flat[hm.nearest]
    state.base = base
    state.base_at = state.iteration
    state.sea = None if labels is None else (below & keep[np.maximum(labels, 0)]).reshape(surf.shape)
    return info


# --------------------------------------------------------------------------
# the planet's lake refresh (maps.py:422-479 with erosion.lake_fill off), restated
# --------------------------------------------------------------------------
_D8_DI = np.array([1, 1, 0, -1, -1, -1, 0, 1])
_D8_DJ = np.array([0, 1, 1, 1, 0, -1, -1, -1])


def _cell_neighbors(grid) -> np.ndarray:
    """(M, 8) cell ids of every interior cell's D8 neighbours through the
    owner table (hydro/d8.py:70-77)."""
    N, H, NE = grid.N, grid.H, grid.NE
    f, i, j = np.meshgrid(np.arange(6), np.arange(N), np.arange(N), indexing="ij")
    out = np.empty((6 * N * N, 8), np.int64)
    for k in range(8):
        o = grid.owner[f, i + H + _D8_DI[k], j + H + _D8_DJ[k]].reshape(-1).astype(np.int64)
        f2, r = o // (NE * NE), o % (NE * NE)
        out[:, k] = (f2 * N + r // NE - H) * N + r % NE - H
    return out


def hydro_flood(surf32, ocean, nbr, N):
    """hydro/priority_flood.py:127-191, 294-318: the whole-sphere priority
    flood from the ocean drains (the lowest cell when there is none), a FIFO
    for cells at or below the current level and a (level, push order) heap
    for the rest; returns (filled float32, parent, order, pop_seq)."""
    import heapq

    M = surf32.size
    drain = np.asarray(ocean, bool).reshape(-1).copy()
    if not drain.any():
        drain[int(np.argmin(surf32))] = True
    filled = surf32.copy()
    visited = np.zeros(M, bool)
    parent = np.full(M, -1, np.int64)
    order = np.full(M, -1, np.int64)
    pop_seq = []
    heap, fifo, seq = [], [], 0
    for c in range(M):
        if drain[c]:
            visited[c] = True
            if (~drain[nbr[c]]).any():
                heapq.heappush(heap, (float(surf32[c]), seq, c))
                seq += 1
    head = 0
    NN = N * N
    while head < len(fifo) or heap:
        if head < len(fifo):
            c = fifo[head]
            head += 1
        else:
            c = heapq.heappop(heap)[2]
        lvl = filled[c]
        order[c] = len(pop_seq)
        pop_seq.append(c)
        for n in nbr[c]:
            if visited[n]:
                continue
            if n // NN != c // NN and c not in nbr[n]:
                continue  # a one-sided link across a face edge
            visited[n] = True
            parent[n] = c
            if surf32[n] <= lvl:
                filled[n] = lvl
                fifo.append(n)
            else:
                filled[n] = surf32[n]
                heapq.heappush(heap, (float(surf32[n]), seq, n))
                seq += 1
    return filled, parent, order, np.array(pop_seq, np.int64)


def flow_down(filled, ocean, parent, nbr, metric_face, N, H):
    """hydro/routing.py:28-90 + d8.py:123-136: each land cell's downstream
    cell, by the steepest physical descent on the filled surface (the float32
    height difference over the float64 step length), flats to their flood
    parent."""
    M = filled.size
    down = np.full(M, -1, np.int64)
    oc = np.asarray(ocean, bool).reshape(-1)
    for c in range(M):
        if oc[c]:
            continue
        i, j = (c % (N * N)) // N, c % N
        g = metric_face[i + H, j + H]
        best, best_s = -1, 0.0
        for k in range(8):
            hn = filled[nbr[c, k]]
            if hn < filled[c]:
                di, dj = float(_D8_DI[k]), float(_D8_DJ[k])
                d2 = float(g[0]) * di * di + 2.0 * float(g[1]) * di * dj + float(g[2]) * dj * dj
                sl = float(np.float32(filled[c] - hn)) / math.sqrt(d2)
                if sl > best_s:
                    best, best_s = k, sl
        if best < 0 and parent[c] >= 0:
            hit = np.flatnonzero(nbr[c] == parent[c])
            best = int(hit[0]) if hit.size else -1
        if best < 0:
            raise RuntimeError("a land cell has no D8 direction")
        down[c] = nbr[c, best]
    return down


def _label_level(mask, level, nbr):
    """hydro/lakes.py:18-46: 8-connected components joining only cells of
    one level, numbered by their lowest cell id."""
    M = mask.size
    lab = np.full(M, -1, np.int64)
    n = 0
    for s0 in range(M):
        if not mask[s0] or lab[s0] >= 0:
            continue
        lab[s0] = n
        stack = [s0]
        while stack:
            c = stack.pop()
            for q in nbr[c]:
                if mask[q] and lab[q] < 0 and level[q] == level[c]:
                    lab[q] = n
                    stack.append(q)
        n += 1
    return lab, n


def balance_lakes(surf32, filled, ocean, order, down, topo, precip, pet, area, cell_size_m, nbr, lake_evap, land_evap):
    """hydro/balance.py:63-108, 159-284: every depression lowered to the level
    where its inflow meets its evaporation, in one upstream-first pass;
    returns (water float32 (M,), info)."""
    M = surf32.size
    oc = np.asarray(ocean, bool).reshape(-1)
    w = np.asarray(precip, np.float64).reshape(-1)
    dep = (filled > surf32) & ~oc
    info = {"depressions": 0, "overflowing": 0, "closed": 0, "dry": 0}
    if (float(lake_evap) <= 0.0 and float(land_evap) <= 0.0) or not dep.any():
        return filled.copy(), info
    lab, n = _label_level(dep, filled, nbr)
    cells = np.flatnonzero(lab >= 0)
    cells = cells[np.lexsort((surf32[cells], lab[cells]))]
    lab_s = lab[cells]
    ptr = np.searchsorted(lab_s, np.arange(n + 1))
    z = surf32[cells].astype(np.float64)
    af = np.asarray(area, np.float64).reshape(-1) / (float(cell_size_m) ** 2)
    ev = np.asarray(pet, np.float64).reshape(-1)
    wr = w
    k_lake = float(lake_evap)
    if float(land_evap) > 0.0:
        rain = w / af
        pe = float(land_evap) * ev
        a = np.maximum(pe / np.maximum(rain, 1e-9), 1e-9)
        et = rain * np.sqrt(a * np.tanh(1.0 / a) * (1.0 - np.exp(-a)))
        wr = (rain - et) * af
        per = (pe[cells] - et[cells]) * af[cells]
        k_lake = 1.0
    else:
        per = ev[cells] * af[cells]
    csum = np.cumsum(per)
    before = np.zeros(n)
    before[1:] = csum[ptr[1:n] - 1]
    cum = csum - before[lab_s]
    ordv = order[cells]
    best = np.full(n, np.iinfo(np.int64).max)
    np.minimum.at(best, lab_s, ordv)
    sel = ordv == best[lab_s]
    outlet = np.zeros(n, np.int64)
    outlet[lab_s[sel]] = cells[sel]
    outlet_lake = np.full(M, -1, np.int64)
    outlet_lake[outlet] = np.arange(n)
    spill = filled[outlet].astype(np.float64)
    level = np.zeros(n)
    outflow = np.zeros(n)
    acc = w.copy()
    run = wr.copy()
    for c in topo:
        L = outlet_lake[c]
        if L >= 0:
            inflow = run[c]
            lo, hi = ptr[L], ptr[L + 1]
            if inflow <= 0.0:
                level[L], outflow[L] = z[lo], 0.0
            else:
                i = int(np.searchsorted(cum[lo:hi], inflow / k_lake))
                if i >= hi - lo:
                    level[L], outflow[L] = spill[L], inflow - k_lake * cum[hi - 1]
                else:
                    level[L], outflow[L] = z[lo + i], 0.0
            if float(land_evap) > 0.0:
                acc[c] = acc[c] * (outflow[L] / inflow) if inflow > 0.0 else 0.0
            else:
                acc[c] = outflow[L]
            run[c] = outflow[L]
        d = down[c]
        if d >= 0:
            acc[d] += acc[c]
            run[d] += run[c]
    water = surf32.copy()
    np.maximum.at(water, cells, level[lab_s].astype(np.float32))
    water[oc] = filled[oc]
    closed = outflow <= 0.0
    wet = level > z[ptr[:n]]
    info.update(depressions=int(n), overflowing=int((~closed).sum()), closed=int((closed & wet).sum()),
                dry=int((closed & ~wet).sum()))
    return water, info


def fill_basins(state, params) -> dict | None:
    """maps.py:1216-1229, 1278-1326: sediment into the closed basins of a
    fresh state, up to the flood's surface graded ``basin_fill_grade`` (m per
    km) up from each basin's outlet along the flood tree, where the flood
    leaves more than ``basin_fill_min_m`` off the open ocean."""
    ep = _ep(params)
    grade = float(getattr(ep, "basin_fill_grade", 0.0))
    if grade <= 0.0 or not state.spherical or not hasattr(params, "world"):
        return None
    grid = state.grid
    N = grid.N
    inter = state.interior
    surf = np.ascontiguousarray((state.height + state.sediment)[inter], np.float32)
    below, labels, keep = below_sea_components(surf, grid, _ocean_min_fraction(params))
    ocean = np.zeros(surf.size, bool) if labels is None else (below & keep[np.maximum(labels, 0)]).reshape(-1)
    if getattr(state, "_nbr", None) is None:
        state._nbr = _cell_neighbors(grid)
    s32 = surf.reshape(-1)
    filled, parent, order, pop_seq = hydro_flood(s32, ocean, state._nbr, N)
    step = grade * (float(grid.cell_size_m) / 1000.0) / state.height_unit_m
    g = s32.astype(np.float64)
    for c in pop_seq:
        q = parent[c]
        if q >= 0 and g[q] + step > g[c]:
            g[c] = g[q] + step
    basin = ((filled - s32) > np.float32(float(ep.basin_fill_min_m) / state.height_unit_m)) & ~ocean
    add = np.where(basin, np.maximum(g - s32, 0.0), 0.0)
    sed = state.sediment[inter].reshape(-1) + add
    state.sediment[inter] = sed.reshape(surf.shape)
    state.exchange_halos()
    return {"basin_cells": int(basin.sum())}


def _lake_plain(water, lab, parent, pop_seq, grade):
    """maps.py:1232-1245: the plain a lake fills towards -- its water level at
    the outlet, ``grade`` higher with every flood step inside the same lake
    (pop order: a parent is done before its children)."""
    g = water.copy()
    for c in pop_seq:
        if lab[c] >= 0:
            q = parent[c]
            if q >= 0 and lab[q] == lab[c]:
                g[c] = g[q] + grade
    return g


def settle_lake_loads(state, lake, water, surf, flood, grade, ice_evap, rise=0.0, load_share=1.0):
    """maps.py:490-628: lay what the lakes kept (``lake_load``) over their
    floors and give every lake its room until the next refresh.  A load goes
    to the lake of this refresh that holds its cell, else to the heir of the
    lake it was parked in (the new lake covering most of it), else on as a
    stockpile; each lake fills towards a plain graded from its outlet, at
    most ``rise`` above the water, farthest cells from the outlet first; its
    room left is what that plain would still take (0 for a frozen lake).
    Returns (volumes, takes)."""
    grid = state.grid
    N, H = grid.N, grid.H
    inter = state.interior
    filled, parent, order, pop_seq = flood
    load = state.lake_load[inter]
    out = {"parked": float(load.sum()), "laid": 0.0, "stray": 0.0, "room": 0.0, "lakes": 0}
    takes = np.zeros(lake.size, bool)
    lake_id = np.full(lake.size, -1, np.int32)
    state.lake_room = np.zeros(1)

    def add(arr, flat_cells, values):
        f, i, j = np.unravel_index(flat_cells, (6, N, N))
        arr[f, i + H, j + H] += values  # distinct cells

    lab, n = _label_level(lake.reshape(-1), np.asarray(water, np.float32).reshape(-1), state._nbr)
    lflat = load.reshape(-1)
    held = np.flatnonzero(lflat > 0.0)
    have = np.zeros(max(n, 1))
    if held.size:
        was = state.lake_id[inter].reshape(-1)
        n_was = int(was.max()) + 1 if was.size else 0
        heir = np.full(max(n_was, 1), -1, np.int64)
        both = np.flatnonzero((was >= 0) & (lab >= 0))
        if both.size and n > 0:
            key, cnt = np.unique(was[both].astype(np.int64) * n + lab[both], return_counts=True)
            o = np.lexsort((cnt, key // n))
            k_old = (key // n)[o]
            last = np.r_[k_old[1:] != k_old[:-1], True]
            heir[k_old[last]] = (key % n)[o][last]
        to = np.where(lab[held] >= 0, lab[held], np.where(was[held] >= 0, heir[np.maximum(was[held], 0)], -1))
        ok = to >= 0
        np.add.at(have, to[ok], lflat[held[ok]])
        if (~ok).any():
            add(state.pending, held[~ok], lflat[held[~ok]])
            out["stray"] = float(lflat[held[~ok]].sum())
    cells = np.flatnonzero(lab >= 0)
    if cells.size:
        s64 = np.asarray(surf, np.float64).reshape(-1)
        w64 = np.asarray(water, np.float64).reshape(-1)
        plain = _lake_plain(w64, lab, parent, pop_seq, float(grade))
        room = np.maximum(np.minimum(plain[cells], w64[cells] + float(rise)) - s64[cells], 0.0)
        order_f = order[cells]
        first = np.full(n, np.iinfo(np.int64).max)
        np.minimum.at(first, lab[cells], order_f)
        outlet = np.zeros(n, np.int64)
        at = order_f == first[lab[cells]]
        outlet[lab[cells][at]] = cells[at]
        if getattr(state, "_centres", None) is None:
            state._centres = np.ascontiguousarray(grid.centers()[:, H:H + N, H:H + N].reshape(-1, 3))
        centres = state._centres
        far = np.linalg.norm(centres[cells] - centres[outlet[lab[cells]]], axis=1)
        o = np.lexsort((-far, lab[cells]))
        cells, room = cells[o], room[o]
        L = lab[cells].astype(np.int64)
        ptr = np.searchsorted(L, np.arange(n))
        csum = np.cumsum(room)
        before = csum - room - (csum[ptr] - room[ptr])[L]
        lay = np.clip(have[L] - before, 0.0, room)
        add(state.sediment, cells, lay)
        if getattr(state, "iso_acc", None) is not None:
            add(state.iso_acc, cells, float(load_share) * lay)
        left = np.bincount(L, weights=room - lay, minlength=n)
        over = have - np.bincount(L, weights=lay, minlength=n)
        spill = over > 1e-9
        if spill.any():
            add(state.pending, cells[ptr[spill]], over[spill])
            out["stray"] += float(over[spill].sum())
        warm = np.ones(n, bool)
        cold = (state.evap[inter] <= float(ice_evap)).reshape(-1)[cells]
        warm[np.unique(L[cold])] = False
        open_ = warm & (left > 0.0)
        takes[cells[open_[L]]] = True
        ids = np.cumsum(open_) - 1
        lake_id[cells[open_[L]]] = ids[L[open_[L]]].astype(np.int32)
        if open_.any():
            state.lake_room = np.ascontiguousarray(left[open_], np.float64)
        out.update(laid=float(lay.sum()), room=float(left[open_].sum()), lakes=int(open_.sum()))
    state.lake_load[inter] = 0.0
    full = np.full(state.height.shape, -1, np.int32)
    full[inter] = lake_id.reshape(6, N, N)
    state.lake_id = full
    return out, takes


def lake_fill_args(state, params):
    """maps.py:1248-1258: refresh_lakes' ``fill`` -- (grade in cell units per
    cell, ice_evap, the plain's rise above the water in cell units, the load
    share) with erosion.lake_fill and lake_balance on the planet, else None."""
    ep = _ep(params)
    if not (state.spherical and bool(getattr(ep, "lake_fill", False)) and bool(getattr(ep, "lake_balance", False))):
        return None
    cell_km = float(state.grid.cell_size_m) / 1000.0
    return (float(getattr(ep, "basin_fill_grade", 0.0)) * cell_km / state.height_unit_m, float(getattr(ep, "ice_evap", 0.0)),
            float(getattr(ep, "lake_fill_rise_m", 1.0)) / state.height_unit_m, float(getattr(ep, "lake_fill_load", 0.55)))


def refresh_lakes(state, lake_evap, min_depth, min_fraction, land_evap=0.0, fill=None) -> dict:
    """maps.py:422-479 (erosion.lake_fill off): the planet's lakes on the
    current surface -- overflowing lakes deeper than ``min_depth`` flagged,
    a lake drawn below its rim a closed sea at its level in ``base``; flags
    and base halos copied from their nearest interior cell."""
    grid = state.grid
    N, H = grid.N, grid.H
    inter = state.interior
    surf = np.ascontiguousarray((state.height + state.sediment)[inter], np.float32)
    sea = getattr(state, "sea", None)
    if sea is None:
        below, labels, keep = below_sea_components(surf, grid, float(min_fraction))
        sea = np.zeros(surf.shape, bool) if labels is None else (below & keep[np.maximum(labels, 0)]).reshape(surf.shape)
    ocean = np.asarray(sea, bool).reshape(-1)
    if getattr(state, "_nbr", None) is None:
        state._nbr = _cell_neighbors(grid)
    nbr = state._nbr
    s32 = surf.reshape(-1)
    filled, parent, order, pop_seq = hydro_flood(s32, ocean, nbr, N)
    down = flow_down(filled, ocean, parent, nbr, grid.metric_face, N, H)
    topo = pop_seq[::-1]
    topo = topo[~ocean[topo]]
    pet = getattr(state, "lake_pet", None)
    pet = (state.evap if pet is None else pet)[inter]
    water, bal = balance_lakes(s32, filled, ocean, order, down, topo, state.precip[inter], pet, interior_cell_area(grid),
                               grid.cell_size_m, nbr, lake_evap, land_evap)
    lake = ((water - s32) > np.float32(min_depth)) & ~ocean
    closed = lake & (water < filled - np.float32(1e-4))
    flag = np.zeros(state.height.shape, np.uint8)
    settled = {}
    if fill is not None:
        if state.lake_load is None:
            state.lake_load = np.zeros_like(state.height)
            state.lake_id = np.full(state.height.shape, -1, np.int32)
            state.lake_room = np.zeros(1)
        settled, takes = settle_lake_loads(state, lake & ~closed, water, s32, (filled, parent, order, pop_seq), *fill)
        s32 = np.ascontiguousarray((state.height + state.sediment)[inter], np.float32).reshape(-1)
        lake &= (water - s32) > np.float32(min_depth)  # what the load raised to its plain is ground again
        flag[inter] = ((lake & ~closed).astype(np.uint8) + (takes & lake & ~closed)).reshape(surf.shape)
    else:
        flag[inter] = (lake & ~closed).reshape(surf.shape)
    if closed.any():
        b = state.base[inter].reshape(-1).copy()
        b[closed] = water[closed]
        state.base[inter] = b.reshape(surf.shape)
    hm = grid.halo
    for arr in (flag, state.base):
        flat = arr.reshape(-1, 1)
        flat[hm.dst] = flat[hm.nearest]
    state.lake_flag = flag
    return {"lake_cells": int(lake.sum()), "lake_cells_closed": int((closed & lake).sum()), **bal,
            **{f"load_{k}": v for k, v in settled.items()}}


def _ocean_min_fraction(params) -> float:
    """hydro.ocean_min_fraction when the params carry a hydro group, else the bake's 0.02 (maps.py:770-774)."""
    hydro = getattr(params, "hydro", None)
    return float(getattr(hydro, "ocean_min_fraction", OCEAN_MIN_FRACTION)) if hydro is not None else OCEAN_MIN_FRACTION


def step(state, params, iteration_key, n_particles=None, chunk=None) -> dict:
    ep = _ep(params)
    sea_every = int(getattr(ep, "sea_mask_every", 0))
    st_base = None
    if state.spherical and sea_every > 0 and (state.base_at is None or state.iteration % sea_every == 0):
        st_base = refresh_base(state, _ocean_min_fraction(params))  # maps.py:1546-1551, before the route
    if int(getattr(ep, "flood_every", 0)) > 0 and (state.route is None or state.iteration % int(ep.flood_every) == 0):
        refresh_route(state, _cu(ep, "route_eps", state.height_unit_m))  # maps.py:1553-1554
    st_lake = None
    if state.spherical and bool(getattr(ep, "lake_balance", False)) and int(getattr(ep, "flood_every", 0)) > 0 and \
            (getattr(state, "lake_flag", None) is None or state.iteration % int(ep.flood_every) == 0):
        hydro = getattr(params, "hydro", None)
        depth_m = float(getattr(hydro, "lake_min_depth", LAKE_MIN_DEPTH_M)) if hydro is not None else LAKE_MIN_DEPTH_M
        st_lake = refresh_lakes(state, float(getattr(hydro, "lake_evap", 6.0)), depth_m / state.height_unit_m,
                                _ocean_min_fraction(params), float(getattr(hydro, "land_evap", 3.0)),
                                lake_fill_args(state, params))  # maps.py:1555-1562
    elif not state.spherical and bool(getattr(ep, "window_lakes", False)) and int(getattr(ep, "flood_every", 0)) > 0 and \
            (state.lake_flag is None or state.iteration % int(ep.flood_every) == 0):
        hydro = getattr(params, "hydro", None)
        depth_m = float(getattr(hydro, "lake_min_depth", LAKE_MIN_DEPTH_M)) if hydro is not None else LAKE_MIN_DEPTH_M
        st_lake = refresh_lakes_window(state, depth_m / state.height_unit_m,
                                       float(getattr(ep, "window_lake_evap", 0.0)))  # maps.py:1563-1566
    iso = state.spherical and float(getattr(ep, "isostasy", 0.0)) > 0.0
    if iso:
        if getattr(state, "iso_acc", None) is None:
            state.iso_acc = np.zeros_like(state.height)
        s0 = state.height + state.sediment
    st = run_iteration(state, params, iteration_key, n_particles=n_particles, chunk=chunk)
    thermal_erosion(state, params)
    if iso:
        state.iso_acc += (state.height + state.sediment) - s0
    apply_uplift(state, None)
    ge = int(getattr(ep, "glacial_every", 0))
    if state.spherical and ge > 0 and (state.iteration + 1) % ge == 0 and \
            (state.iteration + 1) >= float(ep.glacial_from) * int(ep.iterations):
        if iso:
            s1 = state.height + state.sediment
        st["glacial"] = glacial_carve(state, params)  # maps.py:1580-1590
        if iso:
            state.iso_acc += (state.height + state.sediment) - s1
    if iso and (state.iteration + 1) % max(int(getattr(ep, "isostasy_every", 10)), 1) == 0:
        st["isostasy"] = apply_isostasy(state, params)
    if state.spherical:
        st["datum_shift"] = hold_datum(state, state.land_target)
    state.exchange_halos()
    state.iteration += 1
    if st_base is not None:
        st["sea"] = st_base
    if st_lake is not None:
        st["lakes"] = st_lake
    return st


#: the deposit floor of the glacial pass's room (particle.py:99), cell units
GLACIAL_DEP_FLOOR = 0.02


def _ring(a: np.ndarray) -> np.ndarray:
    """The eight D8 neighbours of every cell of each face's extended array,
    wrapping at the array's edges (np.roll, as the reference's passes do)."""
    out = []
    for di in (-1, 0, 1):
        for dj in (-1, 0, 1):
            if di or dj:
                out.append(np.roll(np.roll(a, di, axis=1), dj, axis=2))
    return out


def glacial_carve(state, params) -> dict:
    """erosion/glacial.py:162-257 (the ice line of the evaporation field:
    no ice sheet, no surface temperature): the bed under ice lowered by
    glacial_rate sqrt(discharge / disc_saturation) (1 - 0.5 hardness) times
    the taper of :func:`_ice_depth`, capped, down to the cell's base level;
    the spoil spread over the ice margin by discharge, capped per cell at
    iter_deposit, the rest parked as stockpile."""
    ep = _ep(params)
    u = state.height_unit_m
    rate = _cu(ep, "glacial_rate", u)
    cap = _cu(ep, "glacial_max", u)
    stats = {"ice_cells": 0, "carved": 0.0, "moraine_cells": 0, "max_carve": 0.0, "outwash": 0.0}
    if rate <= 0.0:
        return stats
    active = state.mask == MASK_ACTIVE
    cold = state.evap <= float(ep.ice_evap)
    ice = active & cold & (state.height + state.sediment > 0.0)
    sticky = bool(getattr(ep, "glacial_sticky", False))
    if sticky and state.ice_prev is not None:
        ice = ice | (state.ice_prev & active & cold)
    if not ice.any():
        return stats
    state.exchange_halos()
    if sticky:
        state.ice_prev = ice.copy()
    sat = max(float(ep.disc_saturation), 1e-9)
    q = np.maximum(state.discharge, 0.0) / sat
    ramp = int(ep.glacial_ramp)
    if ramp <= 0:
        taper = ice.astype(np.float64)
    else:
        inner = ice.copy()
        depth = ice.astype(np.float64)
        for _ in range(ramp):
            shrunk = inner.copy()
            for nb in _ring(inner):
                shrunk &= nb
            state.exchange_halos()
            inner = shrunk
            depth += inner
        state.exchange_halos()
        taper = np.clip(depth / float(ramp + 1), 0.0, 1.0)
    dz = rate * np.sqrt(q) * (1.0 - 0.5 * state.hardness) * taper
    np.clip(dz, 0.0, cap, out=dz)
    dz = np.where(ice, dz, 0.0)
    room = np.maximum(state.height + state.sediment + GLACIAL_DEP_FLOOR - state.base, 0.0)
    dz = np.minimum(dz, room)
    inter = state.interior
    carved = float(dz[inter].sum())
    if carved <= 0.0:
        return stats
    state.height -= dz
    near = np.zeros_like(ice)
    for nb in _ring(ice):
        near |= nb
    margin = near & ~ice & active & (state.height + state.sediment > state.base)
    frac = float(ep.moraine_frac)
    parked = 0.0
    if margin.any() and frac > 0.0:
        w = np.where(margin, np.maximum(state.discharge, 0.0) + 1e-6, 0.0)
        wsum = float(w[inter].sum())
        if wsum > 0.0:
            add = (w / wsum) * (carved * frac)
            placed = np.minimum(add, _cu(ep, "iter_deposit", u))
            state.sediment += placed
            state.pending += add - placed
            parked = float((add - placed)[inter].sum())
    state.exchange_halos()
    stats.update(ice_cells=int(ice[inter].sum()), carved=carved, moraine_cells=int(margin[inter].sum()),
                 max_carve=float(dz[inter].max()), outwash=parked)
    return stats


#: hydro.ocean_min_fraction, the bake's default (the share of the globe a below-sea body needs to be open ocean)
OCEAN_MIN_FRACTION = 0.02


# --------------------------------------------------------------------------
# routing surface (globe/erosion/route.py:31-125), for the refresh_route tests
# --------------------------------------------------------------------------
D8 = ((1, 0), (1, 1), (0, 1), (-1, 1), (-1, 0), (-1, -1), (0, -1), (1, -1))


def priority_flood_eps(surface, mask, owner, H, N, eps, base):
    """The epsilon-filled surface by a heap priority flood, in the
    reference's order (route.py:31-125): cells outside the mask and on the
    array border are never entered; seeds are interior cells with
    surface < 0 and surface <= base, or a D8 neighbour (through ``owner``)
    outside the mask or not interior; popping the lowest (value, cell), each
    unvisited neighbour takes max(its surface, value + eps)."""
    import heapq

    F, NE, _ = surface.shape
    s = np.asarray(surface, np.float64).reshape(-1)
    b = np.asarray(base, np.float64).reshape(-1)
    m = np.asarray(mask).reshape(-1)
    o = np.asarray(owner, np.int64).reshape(-1)
    filled = s.copy()
    visited = np.zeros(s.size, bool)
    idx = np.arange(s.size).reshape(F, NE, NE)
    border = np.zeros((F, NE, NE), bool)
    border[:, 0, :] = border[:, -1, :] = border[:, :, 0] = border[:, :, -1] = True
    visited[(m == MASK_OUTSIDE) | border.reshape(-1)] = True
    heap = []
    for f in range(F):
        for ei in range(H, H + N):
            for ej in range(H, H + N):
                c = int(idx[f, ei, ej])
                if visited[c]:
                    continue
                seed = s[c] < 0.0 and s[c] <= b[c]
                if not seed:
                    for di, dj in D8:
                        n = int(o[idx[f, ei + di, ej + dj]])
                        if m[n] == MASK_OUTSIDE:
                            seed = True
                            break
                        rem = n % (NE * NE)
                        if not (H <= rem // NE < H + N and H <= rem % NE < H + N):
                            seed = True
                            break
                if seed:
                    visited[c] = True
                    heapq.heappush(heap, (s[c], c))
    while heap:
        h, c = heapq.heappop(heap)
        f, rem = divmod(c, NE * NE)
        ei, ej = divmod(rem, NE)
        for di, dj in D8:
            n = int(o[idx[f, ei + di, ej + dj]])
            if visited[n]:
                continue
            visited[n] = True
            v = s[n]
            if v < h + eps:
                v = h + eps
            filled[n] = v
            heapq.heappush(heap, (v, n))
    return filled.reshape(F, NE, NE)
