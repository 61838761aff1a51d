"""The erosion stage driver on the GPU: the drop-in for the bake's
``globe.erosion.run`` plain path (bake/globe/erosion/run.py).

Same contract: ``OUTPUTS`` and ``run(store, params, log) -> info``
(run.py:63, 374-551).  The stage's inputs are the coarse fields ``bedrock``,
``hardness``, ``uplift``, ``precip``, ``evap``; its outputs ``height``,
``sediment``, ``discharge``, ``momentum`` as float32 metres (maps.py:738-752).
Checkpoints keep the bake's format (run.py:100-225): ``erosion_iterNNNN.npz``
with the float64 cell-unit arrays ``height, sediment, discharge, momentum,
pending, lake_load`` (plus the refreshed state: routing surface, base level,
isostatic load, sticky ice, and the lake flags with ``lake_id, lake_room``),
written to ``.tmp`` then renamed, then a ``.json`` with
the iteration and the parameter hash; the two newest checkpoints of a hash
family are kept; a run resumes from the newest matching checkpoint at or
below its end.  The hash adds this backend's token and apply mode, because
its float results are not the CPU backend's bit for bit.

``store`` is duck-typed: anything with ``load_field(name, grid)`` (returning
an object with ``.data`` or an array), ``save_field(name, array)`` and a
``checkpoint_dir`` path works -- the bake's ``WorldStore`` through a thin
adapter, or :class:`LocalStore` below (the bake's ``coarse/<name>.f{k}.npy``
layout).
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import re
import time
from pathlib import Path

import numpy as np

from . import _lib
from . import maps as gm
from .geometry import exchange_halos, get_grid
from .params import check_plain, erosion_group

OUTPUTS = ["height", "sediment", "discharge", "momentum"]
#: bumped whenever a change alters this backend's results (part of the checkpoint hash)
BACKEND_VERSION = 1
_CKPT_RE = re.compile(r"erosion_iter(\d+)\.npz$")


class LocalStore:
    """A world directory with the bake's field layout: interior faces in
    ``coarse/<name>.f{k}.npy``, checkpoints in ``checkpoints/``."""

    def __init__(self, root):
        self.root = Path(root)
        self.coarse = self.root / "coarse"
        self.checkpoint_dir = self.root / "checkpoints"

    def save_field(self, name: str, arr: np.ndarray, H: int) -> None:
        self.coarse.mkdir(parents=True, exist_ok=True)
        for k in range(6):
            np.save(self.coarse / f"{name}.f{k}.npy", np.ascontiguousarray(arr[k, H:-H, H:-H]))

    def has_field(self, name: str) -> bool:
        return (self.coarse / f"{name}.f0.npy").exists()

    def stage_info(self, stage: str) -> dict | None:
        """The stage's entry in ``manifest.json`` (``{"stages": {stage: {...,
        "hash": ...}}}``, the bake's WorldStore.stage_info,
        world_store.py:93-94), or None without one."""
        m = self.root / "manifest.json"
        if not m.exists():
            return None
        try:
            return json.loads(m.read_text()).get("stages", {}).get(stage)
        except json.JSONDecodeError:
            return None

    def load_field(self, name: str, grid, vector: bool = False) -> np.ndarray:
        """The six faces with their halos filled by the grid's cubic exchange
        (FaceField.load, bake/globe/field.py:327-338)."""
        faces = np.stack([np.load(self.coarse / f"{name}.f{k}.npy") for k in range(6)])
        H, NE = grid.H, grid.NE
        out = np.zeros((6, NE, NE) + faces.shape[3:], dtype=faces.dtype)
        out[:, H:H + grid.N, H:H + grid.N] = faces
        exchange_halos(grid, out, vector=vector)
        return out


def _field(store, name, grid):
    v = store.load_field(name, grid)
    return np.asarray(getattr(v, "data", v))


def _group_dict(g) -> dict:
    return dataclasses.asdict(g) if dataclasses.is_dataclass(g) else dict(vars(g))


def _short_hash(obj) -> str:
    return hashlib.sha256(json.dumps(obj, sort_keys=True, default=str).encode()).hexdigest()[:16]


#: the upstream stages whose parameters and outputs a checkpoint depends on (run.py:89-96)
UPSTREAM_STAGES = ("tectonics", "climate")


def ckpt_hash(params, apply: int, store=None) -> str:
    """Everything a checkpoint depends on, as run.py:68-97 hashes it: the
    world and erosion groups (run-control knobs normalised out; the iteration
    count kept in replay mode, where the start state depends on it), the
    tectonics and climate groups, and -- with a ``store`` that answers
    ``stage_info(stage)`` (the bake's ``WorldStore``, world_store.py:93-94)
    -- the manifest hashes of the tectonics and climate outputs, so that a
    re-baked upstream stage with unchanged parameters invalidates the
    checkpoint.  Then this backend's token, its version (the counterpart of
    ``particle.KERNEL_VERSION``) and the apply mode."""
    ep = erosion_group(params)
    e = _group_dict(ep)
    replay = str(e.get("uplift_mode", "stack")) == "replay"
    for k in ("checkpoint_every", "quicklook_every", "resume"):
        e.pop(k, None)
    if not replay:
        e["iterations"] = 0
    own = _short_hash({"world": _group_dict(params.world), "erosion": e})
    groups = {s: _group_dict(getattr(params, s)) for s in UPSTREAM_STAGES if getattr(params, s, None) is not None}
    up = ""
    info_of = getattr(store, "stage_info", None) if store is not None else None
    if info_of is not None:
        for s in UPSTREAM_STAGES:
            up += ":" + str((info_of(s) or {}).get("hash", ""))
    return own + ":" + _short_hash(groups) + up + f":b200v{BACKEND_VERSION}:apply{apply}"


#: the evolving arrays a checkpoint holds (run.py:100-139); iso_acc only while isostasy is on
CKPT_FIELDS = ("height", "sediment", "discharge", "momentum", "pending")


def _state_fields(state) -> list:
    """The arrays a checkpoint holds beyond CKPT_FIELDS, as the reference's
    (run.py:104-116): the routing surface (refreshed every flood_every), the
    base level once the sea mask has run, an isostatic load not yet applied,
    and the sticky glacial ice."""
    out = []
    if state.route is not None:
        out.append("route")
    if state.base_at is not None:
        out.append("base")
    if state.iso_acc is not None:
        out.append("iso_acc")
    if state.ice_prev is not None:
        out.append("ice_prev")
    if state.lake_flag is not None:
        out.append("lake_flag")
    if state.lake_load is not None:  # the lake parks' bookkeeping (run.py:107, 127-128)
        out += ["lake_load", "lake_id", "lake_room"]
    return out


def _lake_arrays(arrays: dict) -> None:
    """The lake arrays the reference's checkpoints always hold (run.py:104-128;
    its state has lake flags from the first pack on): the flags (zeros when
    the state has none) and the parked-load bookkeeping, at its initial
    values (nothing parked, lake_id -1, one zero room) when the run has no
    parks."""
    if "lake_flag" not in arrays:
        arrays["lake_flag"] = np.zeros(arrays["height"].shape, np.uint8)
    if "lake_id" not in arrays:
        arrays["lake_id"] = np.full(arrays["height"].shape, -1, np.int32)
        arrays["lake_room"] = np.zeros(1, np.float64)


def _write_checkpoint(d: Path, it: int, arrays: dict, meta: dict) -> Path:
    """npz to ``.tmp``, renamed, then the ``.json`` (a crash in between leaves
    the previous checkpoint for :func:`find_checkpoint`), then pruning."""
    p = d / f"erosion_iter{it:04d}.npz"
    tmp = p.with_suffix(".npz.tmp")
    with open(tmp, "wb") as fh:
        np.savez(fh, **arrays)
    tmp.replace(p)
    with open(p.with_suffix(".json"), "w") as fh:
        json.dump(meta, fh, indent=1)
    prune_checkpoints(d, meta["params_hash"], keep=2)
    return p


def _ckpt_meta(state, params, apply, store=None) -> dict:
    return {"iteration": state.iteration, "params_hash": ckpt_hash(params, apply, store), "height_unit_m": state.height_unit_m,
            "time": time.strftime("%Y-%m-%dT%H:%M:%S")}


def save_checkpoint(store, state: gm.ErosionState, params, apply: int) -> Path:
    d = Path(store.checkpoint_dir)
    d.mkdir(parents=True, exist_ok=True)
    a = state.to_numpy()
    arrays = {k: a[k] for k in CKPT_FIELDS}
    arrays["lake_load"] = np.zeros_like(a["height"])
    for k in _state_fields(state):
        arrays[k] = getattr(state, k).detach().cpu().numpy()
    _lake_arrays(arrays)
    return _write_checkpoint(d, state.iteration, arrays, _ckpt_meta(state, params, apply, store))


class CheckpointWriter:
    """Checkpoints written while the iterations go on: ``submit`` snapshots
    the state's arrays on the device (a device-to-device copy on the current
    stream, ordered with the iterations), copies the snapshot to pinned host
    buffers on a side stream and hands the file writing to a background
    thread; the next iterations run meanwhile.  The files are those of
    :func:`save_checkpoint`, byte for byte.  One checkpoint is in flight at
    a time (a new ``submit`` first waits for the previous one); ``wait``
    before reading the files."""

    def __init__(self, store):
        import torch
        from concurrent.futures import ThreadPoolExecutor

        self.dir = Path(store.checkpoint_dir)
        self.store = store
        self._ex = ThreadPoolExecutor(max_workers=1)
        self._pending = None
        self._snap: dict = {}
        self._host: dict = {}
        self._stream = torch.cuda.Stream()

    def submit(self, state: gm.ErosionState, params, apply: int) -> None:
        import torch

        self.wait()
        self.dir.mkdir(parents=True, exist_ok=True)
        extra = _state_fields(state)
        names = list(CKPT_FIELDS) + extra
        for k in names:  # the snapshot, on the stream the iterations run on
            src = getattr(state, k)
            if k not in self._snap or self._snap[k].shape != src.shape:
                self._snap[k] = torch.empty_like(src)
                self._host[k] = torch.empty(src.shape, dtype=src.dtype, pin_memory=True)
            self._snap[k].copy_(src)
        ready = torch.cuda.Event()
        ready.record()
        with torch.cuda.stream(self._stream):
            self._stream.wait_event(ready)
            for k in names:
                self._host[k].copy_(self._snap[k], non_blocking=True)
            copied = torch.cuda.Event()
            copied.record()
        meta = _ckpt_meta(state, params, apply, self.store)
        it = state.iteration

        def write():
            copied.synchronize()
            arrays = {k: self._host[k].numpy() for k in CKPT_FIELDS}
            arrays["lake_load"] = np.zeros_like(arrays["height"])
            for k in extra:
                arrays[k] = self._host[k].numpy()
            _lake_arrays(arrays)
            # the writer reads the pinned buffers only until np.savez returns
            return _write_checkpoint(self.dir, it, arrays, meta)

        self._pending = self._ex.submit(write)

    def wait(self) -> Path | None:
        if self._pending is None:
            return None
        p = self._pending.result()
        self._pending = None
        return p

    def close(self) -> None:
        self.wait()
        self._ex.shutdown(wait=True)


def prune_checkpoints(d: Path, params_hash: str, keep: int = 2) -> None:
    """Keep the ``keep`` newest checkpoints of one hash family (run.py:140-164)."""
    mine = []
    for q in Path(d).glob("erosion_iter*.npz"):
        m = _CKPT_RE.search(q.name)
        jq = q.with_suffix(".json")
        if not m or not jq.exists():
            continue
        try:
            if json.loads(jq.read_text()).get("params_hash") != params_hash:
                continue
        except json.JSONDecodeError:
            continue
        mine.append((int(m.group(1)), q))
    for _, q in sorted(mine)[: max(0, len(mine) - keep)]:
        q.unlink(missing_ok=True)
        q.with_suffix(".json").unlink(missing_ok=True)


def find_checkpoint(store, params, apply: int, max_iteration: int | None = None):
    """Newest checkpoint with a matching hash at or below ``max_iteration``
    (run.py:167-192); a truncated ``.json`` is skipped."""
    d = Path(store.checkpoint_dir)
    if not d.exists():
        return None
    want = ckpt_hash(params, apply, store)
    best = None
    for p in d.glob("erosion_iter*.npz"):
        if not _CKPT_RE.search(p.name):
            continue
        jp = p.with_suffix(".json")
        if not jp.exists():
            continue
        try:
            meta = json.loads(jp.read_text())
        except json.JSONDecodeError:
            continue
        if meta.get("params_hash") != want:
            continue
        it = int(meta.get("iteration", -1))
        if max_iteration is not None and it > max_iteration:
            continue
        if best is None or it > best[1]["iteration"]:
            best = (p, meta)
    return best


def load_checkpoint(state: gm.ErosionState, path: Path, meta: dict) -> None:
    import torch

    with np.load(path) as z:
        for k in ("height", "sediment", "discharge", "momentum"):
            getattr(state, k).copy_(torch.as_tensor(z[k]))
        state.pending.copy_(torch.as_tensor(z["pending"]) if "pending" in z.files else torch.zeros_like(state.pending))
        dev = state.height.device
        state.iso_acc = torch.as_tensor(z["iso_acc"], device=dev) if "iso_acc" in z.files else None
        state.route = torch.as_tensor(z["route"], device=dev) if "route" in z.files else None
        if "base" in z.files:  # a resume sees the sea mask the continuous run had
            state.base = torch.as_tensor(z["base"], device=dev)
            state.base_at = int(meta["iteration"])
        else:
            state.base_at = None
        state.ice_prev = torch.as_tensor(np.asarray(z["ice_prev"], np.uint8), device=dev) if "ice_prev" in z.files else None
        state.lake_flag = torch.as_tensor(np.asarray(z["lake_flag"], np.uint8), device=dev) if "lake_flag" in z.files else None
        if "lake_id" in z.files:  # the loads parked since the last refresh, the lakes' numbers and rooms (run.py:202, 222-224)
            state.lake_load = torch.as_tensor(np.asarray(z["lake_load"], np.float64), device=dev) if "lake_load" in z.files \
                else torch.zeros_like(state.height)
            state.lake_id = torch.as_tensor(np.asarray(z["lake_id"], np.int32), device=dev)
            state.lake_room = torch.as_tensor(np.asarray(z["lake_room"], np.float64), device=dev)
    state.iteration = int(meta["iteration"])


#: the active volcanic edifices tectonics hands over (run.py:229)
VOLCANO_FIELD = "volcano_active"


def active_volcanoes(store, grid) -> np.ndarray | None:
    """The cones (m, extended) of the edifices active at the end of tectonics,
    or None when the store has none (run.py:232-234)."""
    has = getattr(store, "has_field", None)
    return _field(store, VOLCANO_FIELD, grid) if has is not None and has(VOLCANO_FIELD) else None


def datum_land_fraction(params, bedrock_interior) -> float:
    """The land fraction the datum hold keeps (maps.py:1413-1430):
    ``world.land_fraction``, or in shelf mode (``tectonics.shelf_fraction``
    > 0, where the land area is an output of tectonics) the share of cells
    whose bedrock stands at or above 0."""
    if float(getattr(getattr(params, "tectonics", None), "shelf_fraction", 0.0) or 0.0) > 0.0:
        return float(np.mean(np.asarray(bedrock_interior) >= 0))
    return float(params.world.land_fraction)


def build_state(store, params, device="cuda") -> gm.ErosionState:
    """The iteration-0 state from the stage inputs (run.py:237-296): the
    bedrock with the active volcanic cones taken off (the stage erodes the
    ground under them; :func:`run` puts them back at its end), the held land
    fraction of :func:`datum_land_fraction`."""
    w = params.world
    grid = get_grid(int(w.N_c), int(w.halo), float(w.cell_size_m))
    bed = _field(store, "bedrock", grid)
    cone = active_volcanoes(store, grid)
    if cone is not None:
        bed = bed - cone
    st = gm.ErosionState.from_grid(grid, bed, _field(store, "hardness", grid), _field(store, "precip", grid),
                                   _field(store, "evap", grid), _field(store, "uplift", grid), device=device)
    H, N = grid.H, grid.N
    st.land_target = datum_land_fraction(params, np.asarray(bed)[:, H:H + N, H:H + N])
    return st


def restore_volcanoes(state: gm.ErosionState, cone) -> dict:
    """Put the active edifices back on top of the eroded surface (run.py:299-311)."""
    import torch

    if cone is None:
        return {}
    add = np.asarray(cone).astype(np.float64) / state.height_unit_m
    state.height += torch.as_tensor(add, device=state.height.device)
    c = np.asarray(cone)[state.interior]
    surf = (state.height + state.sediment)[state.interior].cpu().numpy()
    on = c > 0.0
    return {"volcano_cells": int(on.sum()), "volcano_max_m": float(c.max()) if on.any() else 0.0,
            "volcano_land_cells": int((on & (surf >= 0.0)).sum())}


def write_outputs(store, state: gm.ErosionState) -> None:
    """float32 metres, as ErosionState.fields (maps.py:738-752)."""
    a = state.to_numpy()
    u = state.height_unit_m
    H = state.H
    store.save_field("height", (a["height"] * u).astype(np.float32), H)
    store.save_field("sediment", (a["sediment"] * u).astype(np.float32), H)
    store.save_field("discharge", a["discharge"].astype(np.float32), H)
    store.save_field("momentum", a["momentum"].astype(np.float32), H)


def run(store, params, log=print, apply: int = _lib.APPLY_ORDERED, wave: int | None = None,
        async_checkpoints: bool = True) -> dict:
    """The erosion stage (run.py:374-551, plain path) on the GPU.  With
    ``async_checkpoints`` the checkpoint files are written in the background
    while the next iterations run (:class:`CheckpointWriter`)."""
    ep = erosion_group(params)
    check_plain(ep)
    n_iter = int(ep.iterations)
    state = build_state(store, params)
    land0 = float((state.surface()[state.interior] >= 0).float().mean().item())
    rep = gm.start_replay(state, params)
    # the basins the bedrock arrives with become sedimentary plains (run.py:383-385); a resume
    # overwrites this with the checkpoint's sediment, which already carries it
    fill = gm.fill_basins(state, params)
    if fill is not None:
        log(f"[erosion] basin fill: {fill['basin_cells']} cells, {fill['fill_km3']:.1f} km3, mean {fill['fill_mean_m']:.1f} m")
    ck = find_checkpoint(store, params, apply, max_iteration=n_iter) if ep.resume else None
    if ck is not None:
        load_checkpoint(state, *ck)
        log(f"[erosion] resumed from {ck[0].name} (iteration {state.iteration})")
    times, clamped, lost_offshore, datum = [], 0, 0.0, 0.0
    writer = CheckpointWriter(store) if async_checkpoints and ep.checkpoint_every > 0 else None
    # each iteration's rain draws made on the host one iteration ahead, while the device runs the current one
    n_particles = max(1, int(round(float(ep.particles_per_cell) * state.n_active_interior())))
    feeder = gm.SpawnFeeder(params, n_particles, device=state.height.device) if state.iteration < n_iter else None
    while state.iteration < n_iter:
        it = state.iteration
        t0 = time.time()
        rng, u, off, _ = feeder.get((it,))
        st = gm.step(state, params, it, apply=apply, wave=wave, n_particles=n_particles, predrawn=(rng, u, off))
        times.append(time.time() - t0)
        clamped += int(st.get("clamped", 0))
        lost_offshore += float(st.get("lost_offshore", 0.0))
        datum += float(st.get("datum_shift", 0.0))
        d = st.get("deaths", {})
        log(f"[erosion] iter {it + 1}/{n_iter}: {st['particles']} particles, mean {st['steps_mean']:.0f} steps, "
            f"deaths ocean {d.get('ocean', 0)} pit {d.get('pit', 0)} age {d.get('age', 0)}, clamped {st.get('clamped', 0)}, "
            f"pending {st.get('pending_total', 0.0):.1f}, {times[-1]:.2f}s")
        done = state.iteration
        if ep.checkpoint_every > 0 and (done % ep.checkpoint_every == 0 or done == n_iter):
            if writer is not None:
                writer.submit(state, params, apply)
                log(f"[erosion] checkpoint -> erosion_iter{done:04d}.npz (writing)")
            else:
                p = save_checkpoint(store, state, params, apply)
                log(f"[erosion] checkpoint -> {p.name}")
    if writer is not None:
        writer.close()
    if feeder is not None:
        feeder.close()
    # the lakes lay what the last iterations brought them: a run ends between two lake refreshes (run.py:476-483)
    lakes_end = gm.settle_lakes(state, params)
    if lakes_end is not None:
        log(f"[erosion] lakes at the end: {lakes_end['lake_cells']} cells, "
            f"{lakes_end.get('load_laid', 0.0) * state.height_unit_m:,.0f} m-cells laid of "
            f"{lakes_end.get('load_parked', 0.0) * state.height_unit_m:,.0f} their rivers left")
    # the active volcanic edifices go back on top of what the stage made of the ground under them (run.py:495-499)
    volc = restore_volcanoes(state, active_volcanoes(store, state.grid))
    if volc:
        log(f"[erosion] active volcanoes back on top: {volc['volcano_cells']} cells, max {volc['volcano_max_m']:.0f} m, "
            f"{volc['volcano_land_cells']} of them land")
    write_outputs(store, state)
    a = state.to_numpy()
    inter = state.interior
    surf = (a["height"] + a["sediment"])[inter]
    u = state.height_unit_m
    info = {"iterations": n_iter, "height_unit_m": u, "seconds_per_iteration": float(np.mean(times)) if times else 0.0,
            "land_fraction": float(np.mean(surf >= 0)), "land_fraction_bedrock": land0,
            "max_discharge": float(a["discharge"][inter].max()), "sediment_mean_m": float(a["sediment"][inter].mean() * u),
            "pending_total_m": float(a["pending"][inter].sum() * u), "clamped_entries": clamped,
            "datum_drift_m": datum * u, "lost_offshore_m": lost_offshore * u, "uplift_mode": str(ep.uplift_mode),
            "backend": "b200", "apply": "ordered" if apply == _lib.APPLY_ORDERED else "wave"}
    if rep is not None:
        info["replay_datum_start_m"] = rep["datum_shift"] * u
    if fill is not None:
        info["basin_fill"] = fill
    if lakes_end is not None:
        info["lakes_end"] = lakes_end
    info.update(volc)
    return info
