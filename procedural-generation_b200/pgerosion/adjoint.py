"""Gradients of a heightfield loss through the particle erosion: the
calibration workload (a per-cell erodibility field and the erodibility,
deposition, evaporation and friction rates fitted to a target heightfield).

The reference has no gradients; its parameters are tuned by grid sweeps.
This module adds, beside the plain path:

* ``Calibration``: the forward -- ``iterations`` plain iterations
  (particles, thermal erosion, uplift, datum hold, halo exchange, as
  ``maps.step``) with the particle pass run as the order-free wave apply
  (by default one wave per iteration: every droplet traced against the
  iteration's start terrain and its changes applied against that terrain
  plus its own, summed as int64 fixed point: deterministic, droplets
  independent), and a checkpoint of the state every ``checkpoint_every``
  iterations;
* its reverse (``Calibration.backward``): per block of iterations, from the
  block's checkpoint, the forward is recomputed with each pass taped
  (``pge_trace_apply_tape``; bit-identical to the forward), then the
  iterations are reversed last to first: the halo exchange (transpose of the
  gather, ``pge_halo_adjoint``), the datum hold (a rigid shift by the
  order-statistic cell's height), and the particle pass
  (``pge_adjoint_pass``: each droplet's cell path and branches held fixed);
* ``erode``: the same as a ``torch.autograd.Function`` of the erodibility
  field and the four rates.

Held fixed in the reverse (no gradient flows through them): the droplets'
cell paths and branches, the discharge and momentum tracks, sediment cover,
stockpiles, the base level's shift, the thermal / creep pass (its change is
treated as a constant: its derivative is taken as the identity on the
surface) and the droplet's own earlier changes inside its ledger's bounds.
Two switches choose how far derivatives are carried.  ``carry_path``: the
droplets' positions and directions differentiated along their whole paths
(the exact derivative of each pass on its path), or only each step's own move
(see ``pge_adjoint_pass``).  ``carry_terrain``: the terrain's adjoint carried
back through every iteration (the exact derivative of the run on its paths),
or each iteration's change taken to reach the final terrain unaltered (the
gradient is then the sum over iterations of each pass's own response).

The defaults are both off.  The erosion is chaotic at the scale of the
workload: a droplet's path turns on float32 samples of the terrain, and the
final terrain's response to a parameter, measured by central differences, is
rough at any step size; the exact derivative along the recorded paths is
right for each pass (checked against path-frozen differences) but grows
without bound when chained over tens of iterations.  The truncated gradient
stays bounded and is a descent direction of the loss.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np
import torch

from . import _lib
from ._lib import PgeHalo, PgeStats, PgeTape, check
from .maps import (ErosionState, _ptr, _stream, apply_uplift, held_land_fraction, hold_datum, run_iteration, thermal_erosion,
                   uplift_cap)
from .params import ErosionParams, WorldGroup, WorldParams, check_plain, erosion_group, plain_knobs

#: the rates differentiated, in PgeParams' names and units (erosion group fields of the same names)
RATES = ("erodibility", "deposition_rate", "evap_rate", "friction")
#: a wave at least as large as any pass: every droplet of an iteration traced against its start terrain
ONE_WAVE = 1 << 30
#: state arrays a pass reads and changes (restored for the reverse)
PASS_FIELDS = ("height", "sediment", "discharge", "momentum", "pending", "base")


class TapeStore:
    """Device arrays of the tapes of one block of passes."""

    def __init__(self, device):
        self.device = device
        self.kept = []

    def __call__(self, n: int, max_steps: int, waves: int, cells: int) -> PgeTape:
        d = self.device
        S, E = int(max_steps), int(max_steps) + _lib.TAPE_EXTRA_ENTRIES
        n, waves = max(int(n), 1), max(int(waves), 1)
        t = {"state": torch.empty((n, S + 1, 6), dtype=torch.float64, device=d),
             "bits": torch.empty((n, S + 1), dtype=torch.int32, device=d),
             "entry": torch.empty((n, E, 4), dtype=torch.int32, device=d),
             "count": torch.zeros((n, 2), dtype=torch.int32, device=d),
             "wave_acc": torch.empty((waves, int(cells)), dtype=torch.int64, device=d)}
        self.kept.append(t)
        return PgeTape(state=_ptr(t["state"]), bits=_ptr(t["bits"]), entry=_ptr(t["entry"]), count=_ptr(t["count"]), droplets=n,
                       steps=S, entries=E, wave_acc=_ptr(t["wave_acc"]), waves=waves)

    def clear(self) -> None:
        self.kept.clear()


def surface(state: ErosionState) -> torch.Tensor:
    """Height + sediment (cell units), (F, NE, NE) float64."""
    return state.height + state.sediment


def snapshot(state: ErosionState) -> dict:
    return {k: getattr(state, k).clone() for k in PASS_FIELDS} | {"iteration": state.iteration}


def restore(state: ErosionState, snap: dict) -> None:
    for k in PASS_FIELDS:
        getattr(state, k).copy_(snap[k])
    state.iteration = snap["iteration"]


def with_rates(params, rates) -> object:
    """``params`` with the four rates replaced (host floats)."""
    vals = [float(v) for v in rates]
    return dataclasses.replace(params, erosion=dataclasses.replace(erosion_group(params), **dict(zip(RATES, vals))))


def calib_step(state: ErosionState, params, iteration_key, n_particles: int, tape=None, wave: int | None = None) -> dict:
    """One plain iteration with the particle pass as the wave apply (waves of
    ``wave`` droplets, None: the reference's chunk), in the order of
    ``maps.step`` (particles, thermal, uplift, datum, halos).
    With ``tape`` (a ``TapeStore``) the pass is taped and the datum's
    order-statistic cell is located; both come back under ``"adjoint"``."""
    ep = erosion_group(params)
    check_plain(ep)
    if state.spherical and float(getattr(ep, "isostasy", 0.0)) > 0.0:
        raise ValueError("the calibration path has no isostasy (erosion.isostasy = 0)")
    if int(getattr(ep, "flood_every", 0)) > 0 or state.route is not None:
        raise ValueError("the calibration path has no routing surface (erosion.flood_every = 0)")
    st = run_iteration(state, params, iteration_key, n_particles=n_particles, apply=_lib.APPLY_WAVE, wave=wave, tape=tape)
    thermal_erosion(state, params)
    apply_uplift(state, uplift_cap(state, ep))
    datum_cell = None
    if state.spherical and hasattr(params, "world"):
        pre = surface(state) if tape is not None else None
        shift = hold_datum(state, held_land_fraction(state, params))
        st["datum_shift"] = shift
        if pre is not None:
            # the shift is (the order statistic) - level with level 0: find the cell holding it
            inter = torch.zeros_like(pre, dtype=torch.bool)
            inter[state.interior] = True
            hit = torch.nonzero(((pre == shift) & inter).reshape(-1))
            datum_cell = int(hit[0].item()) if hit.numel() else None
    state.exchange_halos()
    state.iteration += 1
    if tape is not None and "adjoint" in st:
        st["adjoint"]["datum_cell"] = datum_cell
    return st


class Calibration:
    """The calibration run: ``iterations`` plain iterations of ``n_particles``
    droplets from the state's current contents (kept as the start), with the
    per-cell erodibility field and the rates as inputs.  After ``backward``
    the state holds an intermediate iteration's contents: call ``run`` again
    before reading it."""

    def __init__(self, state: ErosionState, params, iterations: int, n_particles: int, checkpoint_every: int = 5,
                 first_key: int = 0, carry_path: bool = False, carry_terrain: bool = False, wave: int | None = ONE_WAVE):
        if not state.spherical:
            raise ValueError("the calibration path runs on the sphere")
        self.state = state
        self.params = params
        self.iterations = int(iterations)
        self.n_particles = int(n_particles)
        self.k = max(int(checkpoint_every), 1)
        self.first_key = int(first_key)
        self.carry_path = bool(carry_path)
        self.carry_terrain = bool(carry_terrain)
        self.wave = wave
        self.start = snapshot(state)
        self.ckpt: dict[int, dict] = {}
        self._params = params
        self.stats: list[dict] = []

    def _set(self, erod: torch.Tensor | None, rates) -> None:
        st = self.state
        st.erodibility = None if erod is None else erod.to(device=st.height.device, dtype=torch.float32).contiguous()
        self._params = with_rates(self.params, [float(v) for v in rates])

    def run(self, erod: torch.Tensor | None, rates) -> torch.Tensor:
        """The forward: the final surface (F, NE, NE) float64, cell units."""
        self._set(erod, rates)
        st = self.state
        restore(st, self.start)
        self.ckpt.clear()
        self.stats = []
        for it in range(self.iterations):
            if it % self.k == 0:
                self.ckpt[it] = snapshot(st)
            self.stats.append(calib_step(st, self._params, self.first_key + it, self.n_particles, wave=self.wave))
        return surface(st).clone()

    def backward(self, zbar: torch.Tensor):
        """dL/d(erodibility field) (F, NE, NE) float64 and dL/d(rates) (4,)
        float64, both on the device, from ``zbar`` = dL/d(final surface) of
        the last ``run``."""
        st = self.state
        dev = st.height.device
        L = _lib.load()
        s_ = _stream()
        lam = zbar.to(device=dev, dtype=torch.float64).contiguous()
        zb = lam.clone()
        zb2 = torch.empty_like(zb)
        ebar = torch.zeros_like(zb)
        pbar = torch.zeros(4, dtype=torch.float64, device=dev)
        stats_d = torch.zeros(_lib.STATS_WORDS, dtype=torch.int64, device=dev)
        dst, src, w, rot = st.halo_tables()
        halo = PgeHalo(K=int(dst.shape[0]), dst=_ptr(dst), src=_ptr(src), w=_ptr(w), rot=_ptr(rot))
        tapes = TapeStore(dev)
        for b0 in sorted(self.ckpt, reverse=True):
            b1 = min(b0 + self.k, self.iterations)
            restore(st, self.ckpt[b0])
            tapes.clear()
            recs = []
            for it in range(b0, b1):
                snap = snapshot(st)
                s = calib_step(st, self._params, self.first_key + it, self.n_particles, tape=tapes, wave=self.wave)
                recs.append((snap, s.get("adjoint")))
            for snap, rec in reversed(recs):
                if not self.carry_terrain:  # this iteration's change reaches the final terrain unaltered
                    zb.copy_(lam)
                # the halo exchange, then the datum shift z -= z[k*] - level on every cell
                check(L.pge_halo_adjoint(ctypes.byref(halo), _ptr(zb), s_), "pge_halo_adjoint")
                if rec is not None and rec.get("datum_cell") is not None:
                    zb.view(-1)[rec["datum_cell"]] -= zb.sum()
                # uplift adds a terrain-independent field and the thermal pass is held fixed: zb passes through
                if rec is None:  # no droplets: the pass changed nothing
                    continue
                restore(st, snap)
                check(L.pge_adjoint_pass(ctypes.byref(st.pge_grid()), ctypes.byref(st.pge_state()), ctypes.byref(rec["spawns"]),
                                         ctypes.byref(rec["params"]), ctypes.byref(rec["tape"]), 1 if self.carry_path else 0,
                                         _ptr(zb), _ptr(zb2), _ptr(ebar), _ptr(pbar), _ptr(stats_d), _ptr(st.workspace),
                                         st.workspace.numel(), s_), "pge_adjoint_pass")
                zb, zb2 = zb2, zb
            tapes.clear()
        r = PgeStats.from_buffer_copy(stats_d.cpu().numpy().tobytes())
        if r.errors:
            raise _lib.PgeError(f"adjoint: a tape disagreed with its steps (code {int(r.errors)})")
        self.zbar_start = zb
        return ebar, pbar


class _ErosionFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, erod, rates, calib):
        z = calib.run(erod.detach(), rates.detach().cpu().tolist())
        ctx.calib = calib
        ctx.erod_dtype = erod.dtype
        ctx.rates_meta = (rates.device, rates.dtype)
        return z

    @staticmethod
    def backward(ctx, zbar):
        ebar, pbar = ctx.calib.backward(zbar)
        dev, dt = ctx.rates_meta
        return ebar.to(ctx.erod_dtype), pbar.to(device=dev, dtype=dt), None


def erode(erod: torch.Tensor, rates: torch.Tensor, calib: Calibration) -> torch.Tensor:
    """The final surface of ``calib``'s run as a differentiable function of
    the per-cell erodibility field (F, NE, NE) and the rates (4,)
    (erodibility, deposition_rate, evap_rate, friction)."""
    return _ErosionFn.apply(erod, rates, calib)


def land_loss(z: torch.Tensor, target: torch.Tensor, land: torch.Tensor, unit_m: float) -> torch.Tensor:
    """Mean squared difference in metres of the surface and the target over
    the land cells."""
    d = (z - target) * float(unit_m)
    return (d[land] ** 2).mean()


def block_loss(z: torch.Tensor, target: torch.Tensor, land: torch.Tensor, unit_m: float, N: int, H: int,
               block: int = 8) -> torch.Tensor:
    """Mean squared difference in metres of the surface's and the target's
    means over ``block`` x ``block`` cell blocks of each face's interior,
    over the blocks that are land in the majority: the shape of the valleys
    and ranges without the cell-scale placement of single channels, which
    moves chaotically with any change of the rates."""
    pool = lambda a: torch.nn.functional.avg_pool2d(a[:, None, H:H + N, H:H + N], block)[:, 0]
    d = (pool(z) - pool(target)) * float(unit_m)
    keep = pool(land.to(z.dtype)) > 0.5
    return (d[keep] ** 2).mean()


# --------------------------------------------------------------------------
# the calibration workload
# --------------------------------------------------------------------------
#: the workload's sizes: N_c, droplets per iteration, iterations, checkpoint interval
CALIB_N, CALIB_DROPLETS, CALIB_ITERATIONS, CALIB_CHECKPOINT = 256, 1 << 17, 50, 5


def calibration_params(seed: int = 0, N: int = CALIB_N, iterations: int = CALIB_ITERATIONS, jitter: float = 0.0,
                       jitter_seed: int = 1, cell_size_m: float | None = None) -> WorldParams:
    """Plain Earth-like parameters at N_c = ``N`` (the same planet at every
    resolution unless ``cell_size_m`` is given); with ``jitter`` > 0 the four
    rates scaled by U(1 - jitter, 1 + jitter) drawn from ``jitter_seed``
    (the target's parameters come from another seed)."""
    base = ErosionParams()
    f = np.ones(4)
    if jitter > 0.0:
        f = 1.0 + jitter * (2.0 * np.random.default_rng([jitter_seed, 4]).random(4) - 1.0)
    ep = ErosionParams(iterations=iterations, max_steps=0, uplift_mode="replay", **plain_knobs(),
                       **{k: getattr(base, k) * float(f[i]) for i, k in enumerate(RATES)})
    cell = 9773.0 * 1024.0 / N if cell_size_m is None else float(cell_size_m)
    return WorldParams(world=WorldGroup(seed=seed, N_c=N, cell_size_m=cell, land_fraction=0.29, halo=2), erosion=ep)


def calibration_state(params: WorldParams, device="cuda") -> ErosionState:
    """The synthetic world of ``params`` (fBm bedrock with ridges, banded
    rain, seeded uplift) with the uplift replay started."""
    from .maps import start_replay
    from .synth import earth_world

    w = params.world
    world = earth_world(seed=int(w.seed), N=int(w.N_c), cell_size_m=float(w.cell_size_m), land_fraction=float(w.land_fraction))
    st = ErosionState.from_world(world, device=device)
    start_replay(st, params)
    return st


def erodibility_init(state: ErosionState, seed: int = 0, spread: float = 0.2) -> torch.Tensor:
    """The field's start: 1 + U(-spread, spread) per cell (seeded), float32."""
    rng = np.random.default_rng([seed, 17])
    e = 1.0 + spread * (2.0 * rng.random(tuple(state.height.shape)) - 1.0)
    return torch.as_tensor(e.astype(np.float32), device=state.height.device)


def rates_of(params) -> torch.Tensor:
    ep = erosion_group(params)
    return torch.tensor([float(getattr(ep, k)) for k in RATES], dtype=torch.float64)


def calibrate(calib: Calibration, target: torch.Tensor, land: torch.Tensor, erod0: torch.Tensor, rates0: torch.Tensor,
              steps: int = 10, lr_rates: float = 0.05, lr_field: float = 0.02, field: bool = True, method: str = "line",
              loss_fn=None, eta0: float = 0.1, eta_min: float = 1e-3) -> dict:
    """Gradient-based calibration in place of the grid sweep of the rates
    (docs/erosion-tuning.md's procedure), each step one forward run of
    ``calib`` and its adjoint.

    ``method`` "line" (the default): the four rates in log space move along
    the normalised negative gradient by a backtracking line search (step
    ``eta0``, halved until the loss falls, down to ``eta_min``; the next step
    starts from twice the accepted one); the field stays at ``erod0``.  The
    loss falls or the run stops, whatever the roughness of the loss surface
    (the gradient is the truncated one along the recorded paths: a descent
    direction for small steps, not a model of the loss at large ones).
    ``method`` "adam": Adam on the log-rates (``lr_rates``) and, with
    ``field``, on the per-cell erodibility field (``lr_field``).

    ``loss_fn(z)`` is the loss of a final surface (default: ``land_loss``
    against ``target`` over ``land``).  Returns the loss before every step
    and after the last (for "line", the steps taken), the rates after each step (for "line" also the
    accepted step sizes and the numbers of forward and adjoint runs), and the
    field."""
    dev = calib.state.height.device
    unit = calib.state.height_unit_m
    if loss_fn is None:
        loss_fn = lambda z: land_loss(z, target, land, unit)
    logr = torch.log(rates0.detach().to(dev, torch.float64)).clone().requires_grad_(True)
    losses, rates_hist = [], []
    if method == "line":
        erod = erod0.detach().clone()
        etas, forwards, adjoints = [], 1, 0
        eta = float(eta0)
        loss = loss_fn(erode(erod, torch.exp(logr), calib))
        for _ in range(int(steps)):
            logr.grad = None
            loss.backward()
            adjoints += 1
            cur = float(loss.detach())
            losses.append(cur)
            g = logr.grad.detach()
            gn = float(g.norm())
            if not np.isfinite(gn) or gn == 0.0:
                losses.pop()
                break
            accepted = None
            while eta >= eta_min:
                with torch.no_grad():
                    trial = (logr - eta * g / gn).detach()
                trial.requires_grad_(True)
                tl = loss_fn(erode(erod, torch.exp(trial), calib))
                forwards += 1
                if float(tl.detach()) < cur:
                    accepted = (trial, tl)
                    break
                eta *= 0.5
            if accepted is None:  # no step lowered the loss: the run ends where it is
                losses.pop()
                break
            logr, loss = accepted
            etas.append(eta)
            rates_hist.append(torch.exp(logr).detach().cpu().tolist())
            eta = min(2.0 * eta, float(eta0))
        losses.append(float(loss.detach()))
        return {"loss": losses, "rates": rates_hist, "field": erod, "eta": etas, "forwards": forwards, "adjoints": adjoints}
    if method != "adam":
        raise ValueError(f"calibrate: method {method!r} is neither 'line' nor 'adam'")
    erod = erod0.detach().clone().requires_grad_(field)
    groups = [{"params": [logr], "lr": lr_rates}]
    if field:
        groups.append({"params": [erod], "lr": lr_field})
    opt = torch.optim.Adam(groups)
    for _ in range(int(steps)):
        opt.zero_grad()
        loss = loss_fn(erode(erod, torch.exp(logr), calib))
        loss.backward()
        losses.append(float(loss.detach()))
        opt.step()
        with torch.no_grad():
            erod.clamp_(0.05, 5.0)
        rates_hist.append(torch.exp(logr).detach().cpu().tolist())
    with torch.no_grad():
        final = loss_fn(erode(erod, torch.exp(logr), calib))
    losses.append(float(final))
    return {"loss": losses, "rates": rates_hist, "field": erod.detach()}
