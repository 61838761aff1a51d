"""Flexural isostasy on the device: the reference's ``apply_isostasy`` and
``_smoothing_kappa`` (bake/globe/erosion/maps.py:1331-1410).

The load is ``-isostasy x`` the surface change the particles and the mass
wasting made since the last call (``state.iso_acc``); it is spread by
explicit diffusion with the metric-aware Laplace-Beltrami operator
(FaceField.laplacian, bake/globe/field.py:179-188, 372-404) over
``ceil(sigma^2 / (2 kappa))`` steps, the halos refreshed with the monotone
linear weights before each, and added to the active cells mean-free over the
active interior.  ``kappa`` is 0.9 over the largest eigenvalue of the
operator, estimated once per grid by 40 steps of power iteration on the
reference's seeded noise.

Each step is one ``pge_smooth_step`` launch (the operator rounds its result
to float32, as the reference's float32 field does) plus one linear halo
gather; the mean-free add is ``pge_uplift`` on the smoothed field.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from .params import erosion_group

_KAPPA: dict = {}
_SQDET: dict = {}


def sqrt_det_metric(grid) -> np.ndarray:
    """float32 sqrt(det g) of the face-shared metric (cubesphere.py:505-507)."""
    g = grid.metric_face.astype(np.float64)
    return np.sqrt(g[..., 0] * g[..., 2] - g[..., 1] ** 2).astype(np.float32)


def _sqdet(state) -> torch.Tensor:
    key = (state.N, state.H, float(state.height_unit_m), str(state.height.device))
    t = _SQDET.get(key)
    if t is None:
        t = _SQDET[key] = torch.as_tensor(np.ascontiguousarray(sqrt_det_metric(state.grid)), device=state.height.device)
    return t


def _step(state, src: torch.Tensor, dst: torch.Tensor, kappa: float, keep: bool) -> None:
    from .maps import _ptr, _stream

    _lib.check(_lib.load().pge_smooth_step(ctypes.byref(state.pge_grid()), _ptr(state.metric_inv), _ptr(_sqdet(state)), _ptr(src),
                                           _ptr(dst), float(kappa), 1 if keep else 0, float(state.height_unit_m), _stream()),
               "pge_smooth_step")


def smoothing_kappa(state) -> float:
    """Largest monotone explicit step of the smoother (maps.py:1331-1363):
    0.9 / lambda_max of -L in cell units, by power iteration from the
    reference's noise (``default_rng(0).standard_normal``), cached per grid."""
    key = (state.N, state.H, float(state.height_unit_m))
    if key not in _KAPPA:
        N, H = state.N, state.H
        noise = np.random.default_rng(0).standard_normal((6, N, N))
        f = torch.zeros_like(state.height)
        f[:, H:H + N, H:H + N] = torch.as_tensor(noise, device=f.device)
        state.exchange_field(f)  # FaceField.from_interior exchanges with the cubic weights
        lv = torch.empty_like(f)
        lam = 8.0
        for _ in range(40):
            state.exchange_field(f, linear=True)
            _step(state, f, lv, 1.0, keep=False)  # the Laplacian in cell units
            num = float(torch.sqrt((lv[:, H:-H, H:-H] ** 2).sum()))
            den = float(torch.sqrt((f[:, H:-H, H:-H] ** 2).sum()))
            if num <= 0.0 or den <= 0.0:
                break
            lam = num / den
            f = lv / num
        _KAPPA[key] = 0.9 / max(lam, 1e-6)
    return _KAPPA[key]


def apply_isostasy(state, params) -> dict:
    """The flexural isostatic response to ``state.iso_acc`` (maps.py:1366-1410);
    zeroes ``iso_acc``.  Global pass only."""
    from .maps import _ensure_workspace, _ptr, _stream

    ep = erosion_group(params)
    d = state.iso_acc
    k = float(ep.isostasy)
    load = -k * d
    cell = float(state.height_unit_m)
    sig = float(ep.flexure_km) * 1000.0 / cell
    sig = min(sig, state.N / 8.0)
    kappa = smoothing_kappa(state)
    n = int(math.ceil(sig * sig / (2.0 * kappa))) if sig >= 0.5 else 0
    f, g = load, torch.empty_like(load)
    for _ in range(n):
        state.exchange_field(f, linear=True)
        _step(state, f, g, kappa, keep=True)
        f, g = g, f
    state.exchange_field(f, linear=True)
    inter = (slice(None), slice(state.H, state.H + state.N), slice(state.H, state.H + state.N))
    # height[active] += f - mean(f over the active interior): the uplift pass's mean-free add
    _ensure_workspace(state, ep)
    s = state.pge_state()
    s.uplift = _ptr(f)
    _lib.check(_lib.load().pge_uplift(ctypes.byref(state.pge_grid()), ctypes.byref(s), -1.0, 1.0, _ptr(state.workspace),
                                      state.workspace.numel(), _stream()), "pge_uplift")
    fi = f[inter]
    if state.mask is not None:
        act = state.mask[inter] == 1
        mean = float(fi[act].mean()) if bool(act.any()) else 0.0
    else:
        mean = float(fi.mean())
    moved = float(d[inter].abs().sum())
    state.iso_acc.zero_()
    return {"sigma_cells": sig, "diffusion_steps": n, "kappa": kappa, "load_abs_cells": moved,
            "rebound_max": float((fi - mean).max()), "rebound_min": float((fi - mean).min())}
