"""The adjoint of the particle pass against finite differences of the
float64 forward.

A droplet pass is piecewise smooth: while no droplet changes cell path or
branch, its result is a smooth function of the rates, the erodibility field
and the terrain, and pge_adjoint_pass with carry_path = 1 is that function's
exact gradient.  In the one-wave pass droplets do not interact, so the checks
run on a set of droplets from which every droplet whose path or branches a
perturbation changes (compared through the tapes) has been removed: the
differences are then path-frozen differences of the forward itself.

* the taped forward equals the plain wave-apply pass bit for bit;
* path-frozen central differences of the four rates, a direction of the
  erodibility field and a direction of the terrain against the adjoint --
  and per cell of the field on 1024 sampled cells (the float64 reference
  gradient);
* the two carry_path modes agree where positions do not enter (erodibility,
  deposition rate, field);
* the halo transpose against the gather (<G x, y> = <x, G^T y>);
* the multi-iteration reverse as a torch.autograd.Function: its gradient
  equals the reverse called directly, is finite, and the truncated and the
  exact gradients agree in sign for the erodibility, deposition and
  evaporation rates.

Tolerances: rates and field 1e-4 relative plus the bound of the int64
fixed point (each applied change is rounded to 2^-40 cell units, so two runs'
difference of sum(lambda z) is off by at most sum over entries of
|lambda[cell]| 2^-40; steps of 1e-4 relative, 1e-2 for the evaporation rate,
whose small value would otherwise leave the difference below that bound);
the terrain direction 2e-3 (the pass samples the terrain in float32, which
the adjoint differentiates as exact: the differences carry that rounding).  This file runs after the other GPU
tests.
"""
import ctypes
import dataclasses
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "procedural-generation_b200"))

pytestmark = pytest.mark.gpu


def _world(N=32, cell=20000.0, seed=3, warm=600):
    from pgerosion import adjoint as adj

    params = adj.calibration_params(seed=seed, N=N, iterations=10, cell_size_m=cell)
    # the erosion cap off, so most erosion steps run the capacity law
    params = dataclasses.replace(params, erosion=dataclasses.replace(params.erosion, max_erode=1e6))
    st = adj.calibration_state(params)
    for it in range(2):
        adj.calib_step(st, params, 100 + it, warm)
    return st, params


def _spawns(st, n, seed=9):
    """n rain droplets at random positions of random land cells."""
    z = (st.height + st.sediment)[st.interior].cpu().numpy()
    f, i, j = np.nonzero(z > 0.0)
    rng = np.random.default_rng(seed)
    k = rng.choice(len(f), n, replace=False)
    return {"face": f[k].astype(np.int32), "x": i[k] + rng.random(n), "y": j[k] + rng.random(n), "sed": np.zeros(n),
            "dir": np.zeros(n)}


def _pass(st, snap, params, rates, erod, sp, rows, height=None):
    from pgerosion import _lib
    from pgerosion import adjoint as adj
    from pgerosion import maps as gm

    adj.restore(st, snap)
    if height is not None:
        st.height.copy_(height)
    st.erodibility = erod
    tapes = adj.TapeStore(st.height.device)
    r = np.asarray(rows)
    s = gm.apply_spawns(st, adj.with_rates(params, rates), sp["face"][r], sp["x"][r], sp["y"][r], sp["sed"][r], sp["dir"][r], 1.0,
                        wave=len(r), apply=_lib.APPLY_WAVE, tape=tapes)
    return adj.surface(st).clone(), s, tapes.kept[-1]


def _structure(t):
    cnt = t["count"].cpu().numpy()
    bits = t["bits"].cpu().numpy()
    ent = t["entry"].cpu().numpy()
    return [(int(cnt[r, 0]), int(cnt[r, 1]), bits[r, :cnt[r, 0]].tobytes(), ent[r, :cnt[r, 1], :3].tobytes())
            for r in range(cnt.shape[0])]


def _adjoint(st, snap, rec, lam, carry):
    from pgerosion import _lib
    from pgerosion import adjoint as adj
    from pgerosion.maps import _ptr, _stream

    adj.restore(st, snap)
    zb = torch.empty_like(lam)
    eb = torch.zeros_like(lam)
    pb = torch.zeros(4, dtype=torch.float64, device=lam.device)
    stats = torch.zeros(_lib.STATS_WORDS, dtype=torch.int64, device=lam.device)
    _lib.check(_lib.load().pge_adjoint_pass(ctypes.byref(st.pge_grid()), ctypes.byref(st.pge_state()), ctypes.byref(rec["spawns"]),
                                            ctypes.byref(rec["params"]), ctypes.byref(rec["tape"]), int(carry), _ptr(lam), _ptr(zb),
                                            _ptr(eb), _ptr(pb), _ptr(stats), _ptr(st.workspace), st.workspace.numel(), _stream()),
               "pge_adjoint_pass")
    torch.cuda.synchronize()
    assert int(stats[-1]) == 0, "tape and steps disagree"
    return zb, eb, pb


#: relative steps of the rates and the field direction; absolute step of the terrain direction (cell units)
RATE_STEPS, FIELD_STEP, TERRAIN_STEP = (1e-4, 1e-4, 1e-2, 1e-4), 1e-4, 1e-3
FX_MASS_ULP = 2.0 ** -40


def _perturbations(case):
    """name -> ((+ run kwargs), (- run kwargs), divisor of the difference)."""
    rates, erod, d_e, d_z = case["rates"], case["erod"], case["d_erod"], case["d_z"]
    out = {}
    for i in range(4):
        h = RATE_STEPS[i] * rates[i]
        up, dn = list(rates), list(rates)
        up[i] += h
        dn[i] -= h
        out[f"rate{i}"] = ({"rates": up}, {"rates": dn}, 2 * h)
    ep = (erod.double() + FIELD_STEP * d_e).float()
    em = (erod.double() - FIELD_STEP * d_e).float()
    out["field"] = ({"erod": ep}, {"erod": em}, 1.0)
    h0 = case["snap"]["height"]
    out["terrain"] = ({"height": h0 + TERRAIN_STEP * d_z}, {"height": h0 - TERRAIN_STEP * d_z}, 2 * TERRAIN_STEP)
    return out


def _run(case, rows, rates=None, erod=None, height=None):
    return _pass(case["st"], case["snap"], case["params"], case["rates"] if rates is None else rates,
                 case["erod"] if erod is None else erod, case["sp"], rows, height)


@pytest.fixture(scope="module")
def case(cuda):
    from pgerosion import adjoint as adj

    st, params = _world()
    snap = adj.snapshot(st)
    g = torch.Generator().manual_seed(5)
    shape = st.height.shape
    erod = (1.0 + 0.2 * (2 * torch.rand(shape, generator=g, dtype=torch.float64) - 1)).float().cuda()
    lam = torch.zeros_like(st.height)
    lam[st.interior] = torch.randn(lam[st.interior].shape, generator=g, dtype=torch.float64).cuda()
    d_z = torch.zeros_like(st.height)
    d_z[st.interior] = (2 * torch.rand(d_z[st.interior].shape, generator=g, dtype=torch.float64) - 1).cuda()
    c = {"st": st, "params": params, "snap": snap, "rates": adj.rates_of(params).tolist(), "erod": erod, "lam": lam,
         "d_erod": (2 * torch.rand(shape, generator=g, dtype=torch.float64) - 1).cuda(), "d_z": d_z, "sp": _spawns(st, 1000)}
    # drop every droplet whose path or branches one of the perturbations changes, until none does
    rows = list(range(1000))
    for _ in range(6):
        base = _structure(_run(c, rows)[2])
        keep = np.ones(len(rows), bool)
        for plus, minus, _div in _perturbations(c).values():
            for kw in (plus, minus):
                other = _structure(_run(c, rows, **kw)[2])
                keep &= np.array([a == b for a, b in zip(base, other)])
        if keep.all():
            break
        rows = [r for r, k in zip(rows, keep) if k]
    else:
        pytest.fail("the droplet set did not settle")
    print(f"{len(rows)} of 1000 droplets keep their paths under every perturbation")
    assert len(rows) >= 100, len(rows)
    c["rows"] = rows
    z0, s0, t0 = _run(c, rows)
    c["z0"], c["rec"], c["base"] = z0, s0["adjoint"], _structure(t0)
    # sum over the pass's entries of |lambda[cell]|: the fixed point's bound on a difference of two runs
    ent, cnt = t0["entry"].cpu().numpy(), t0["count"].cpu().numpy()
    lam_h = lam.cpu().numpy().reshape(-1)
    c["quant"] = FX_MASS_ULP * float(sum(np.abs(lam_h[ent[r, :cnt[r, 1], 0]]).sum() for r in range(cnt.shape[0])))
    c["adj"] = {k: _adjoint(st, snap, s0["adjoint"], lam, k) for k in (0, 1)}
    return c


def test_taped_pass_equals_the_plain_wave_pass(case):
    from pgerosion import _lib
    from pgerosion import adjoint as adj
    from pgerosion import maps as gm

    st, snap, params, sp = case["st"], case["snap"], case["params"], case["sp"]
    r = np.arange(1000)
    for wave in (400, 64):  # one wave, and waves with refreshes between them
        adj.restore(st, snap)
        st.erodibility = case["erod"]
        tapes = adj.TapeStore(st.height.device)
        s1 = gm.apply_spawns(st, params, sp["face"][r], sp["x"][r], sp["y"][r], sp["sed"][r], sp["dir"][r], 1.0, wave=wave,
                             apply=_lib.APPLY_WAVE, tape=tapes)
        taped = {k: getattr(st, k).clone() for k in adj.PASS_FIELDS}
        adj.restore(st, snap)
        st.erodibility = case["erod"]
        s2 = gm.apply_spawns(st, params, sp["face"][r], sp["x"][r], sp["y"][r], sp["sed"][r], sp["dir"][r], 1.0, wave=wave,
                             apply=_lib.APPLY_WAVE)
        for k in adj.PASS_FIELDS:
            assert torch.equal(taped[k], getattr(st, k)), (wave, k)
        assert s1["droplet_steps"] == s2["droplet_steps"] and s1["entries"] == s2["entries"]
    # the field really enters the pass
    adj.restore(st, snap)
    st.erodibility = None
    gm.apply_spawns(st, params, sp["face"][r], sp["x"][r], sp["y"][r], sp["sed"][r], sp["dir"][r], 1.0, wave=64, apply=_lib.APPLY_WAVE)
    assert not torch.equal(taped["height"] + taped["sediment"], adj.surface(st))


def test_path_frozen_differences_match_the_adjoint(case):
    lam = case["lam"]
    zb, eb, pb = case["adj"][1]
    fails = []
    for name, (plus, minus, div) in _perturbations(case).items():
        zp, _, tp = _run(case, case["rows"], **plus)
        zm, _, tm = _run(case, case["rows"], **minus)
        assert _structure(tp) == case["base"] and _structure(tm) == case["base"], name
        fd = float(((zp - zm) * lam).sum()) / div
        quant = case["quant"] / div
        if name.startswith("rate"):
            ad, tol = float(pb[int(name[-1])]), 1e-4
        elif name == "field":
            e0 = case["erod"].double()
            ad, tol = float((eb * ((e0 + FIELD_STEP * case["d_erod"]).float().double() -
                                   (e0 - FIELD_STEP * case["d_erod"]).float().double())).sum()), 1e-4
        else:
            ad, tol = float((zb * case["d_z"]).sum()), 2e-3
        print(f"{name}: path-frozen difference {fd:.9e} adjoint {ad:.9e} (fixed-point bound {quant:.2e})")
        if not abs(fd - ad) <= tol * max(abs(fd), abs(ad)) + quant:
            fails.append((name, fd, ad))
    assert not fails, fails


def test_modes_agree_where_positions_do_not_enter(case):
    """Positions and directions do not depend on the erodibility, the
    deposition rate or the field: both carry_path modes give the same
    gradients for them."""
    _, e0, p0 = case["adj"][0]
    _, e1, p1 = case["adj"][1]
    for i in (0, 1):
        assert abs(float(p0[i]) - float(p1[i])) <= 1e-12 * abs(float(p1[i])), i
    torch.testing.assert_close(e0, e1, rtol=1e-12, atol=1e-14 * float(e1.abs().max()))


def test_reference_gradient_on_1024_sampled_cells(case):
    """Per-cell central differences of the float64 forward on 1024 cells of
    the erodibility field (the cells the pass's capacity law reads first),
    each checked path-frozen; a cell whose difference changes a path is
    counted and skipped."""
    lam, rows = case["lam"], case["rows"]
    _, eb, _ = case["adj"][1]
    ebn = eb.cpu().numpy().reshape(-1)
    inter = np.zeros(case["st"].height.shape, bool)
    inter[case["st"].interior] = True
    touched = np.flatnonzero(ebn != 0.0)
    quiet = np.flatnonzero((ebn == 0.0) & inter.reshape(-1))
    rng = np.random.default_rng(2)
    n_t = min(len(touched), 768)
    assert n_t >= 256, n_t
    cells = np.concatenate([rng.choice(touched, n_t, replace=False), rng.choice(quiet, 1024 - n_t, replace=False)])
    fd = np.full(len(cells), np.nan)
    erod = case["erod"]
    for n, c in enumerate(cells):
        e0 = erod.view(-1)[c].item()
        ep, em = erod.clone(), erod.clone()
        ep.view(-1)[c] = e0 + 2.0 ** -12  # exact float32 offsets around 1
        em.view(-1)[c] = e0 - 2.0 ** -12
        zp, _, tp = _run(case, rows, erod=ep)
        zm, _, tm = _run(case, rows, erod=em)
        if _structure(tp) == case["base"] and _structure(tm) == case["base"]:
            fd[n] = float(((zp - zm) * lam).sum()) / (ep.view(-1)[c].item() - em.view(-1)[c].item())
    ad = ebn[cells]
    ok = ~np.isnan(fd)
    err = np.abs(fd - ad)
    scale = np.abs(ad).max()
    print(f"1024 cells ({n_t} the pass reads): {ok.sum()} path-frozen; max |difference - adjoint| {np.nanmax(err):.3e} "
          f"of max |gradient| {scale:.3e}")
    assert ok.sum() >= 900
    bad = ok & ~(err <= 1e-4 * np.abs(ad) + 1e-6 * scale)
    assert not bad.any(), list(zip(cells[bad][:8], fd[bad][:8], ad[bad][:8]))
    assert np.all(fd[n_t:][ok[n_t:]] == 0.0)


def test_halo_transpose(cuda):
    from pgerosion import _lib
    from pgerosion import maps as gm
    from pgerosion.maps import _ptr, _stream
    from pgerosion.synth import plain_small_world

    st = gm.ErosionState.from_world(plain_small_world(seed=1, N=24))
    dst, src, w, rot = st.halo_tables()
    halo = _lib.PgeHalo(K=int(dst.shape[0]), dst=_ptr(dst), src=_ptr(src), w=_ptr(w), rot=_ptr(rot))
    g = torch.Generator().manual_seed(4)
    x = torch.randn(st.height.shape, generator=g, dtype=torch.float64).cuda()
    y = torch.randn(st.height.shape, generator=g, dtype=torch.float64).cuda()
    gx = x.clone()
    st.exchange_field(gx)
    gty = y.clone()
    _lib.check(_lib.load().pge_halo_adjoint(ctypes.byref(halo), _ptr(gty), _stream()), "pge_halo_adjoint")
    torch.cuda.synchronize()
    lhs, rhs = float((gx * y).sum()), float((x * gty).sum())
    assert abs(lhs - rhs) <= 1e-12 * float((gx.abs() * y.abs()).sum())
    assert float(gty.reshape(-1)[dst.long()].abs().max()) == 0.0


def _calibration_case():
    from pgerosion import adjoint as adj

    st, params = _world(N=32, cell=20000.0, seed=5)
    calib = adj.Calibration(st, params, 6, 800, checkpoint_every=2, first_key=200)
    target = calib.run(None, (adj.rates_of(params) * torch.tensor([1.25, 0.8, 1.2, 0.85], dtype=torch.float64)).tolist())
    land = torch.zeros_like(target, dtype=torch.bool)
    land[st.interior] = target[st.interior] > 0.0
    return st, params, calib, target, land


def test_autograd_function_matches_the_reverse(cuda):
    """Six iterations, checkpoints every 2: the torch.autograd.Function's
    gradients equal Calibration.backward called directly (both switches) and
    are finite; the truncated and the exact gradients agree in sign for the
    erodibility, deposition and evaporation rates."""
    from pgerosion import adjoint as adj

    st, params, calib, target, land = _calibration_case()
    unit = st.height_unit_m
    grads = {}
    for carry_path, carry_terrain in ((False, False), (True, True)):
        calib.carry_path, calib.carry_terrain = carry_path, carry_terrain
        erod = adj.erodibility_init(st, seed=0).requires_grad_(True)
        rates = adj.rates_of(params).cuda().requires_grad_(True)
        loss = adj.land_loss(adj.erode(erod, rates, calib), target, land, unit)
        loss.backward()
        z = calib.run(erod.detach(), adj.rates_of(params).tolist()).requires_grad_(True)
        adj.land_loss(z, target, land, unit).backward()
        eb, pb = calib.backward(z.grad)
        torch.testing.assert_close(rates.grad, pb, rtol=1e-9, atol=0.0)
        torch.testing.assert_close(erod.grad.double(), eb.float().double(), rtol=1e-6, atol=1e-30)
        assert bool(torch.isfinite(pb).all()) and bool(torch.isfinite(eb).all())
        print(f"carry_path {carry_path} carry_terrain {carry_terrain}: loss {float(loss):.6e} rate gradient {pb.tolist()}")
        grads[carry_path] = pb.cpu().numpy()
    assert np.all(np.sign(grads[False][:3]) == np.sign(grads[True][:3])), grads


def test_line_search_calibration_lowers_the_loss(cuda):
    """Three steps of the line-search calibration from the base rates toward
    the target of rates x (1.25, 0.8, 1.2, 0.85): the truncated gradient is a
    descent direction (at least one step accepted, the loss lower at the end
    than at the start, never higher after a step), for the land loss and the
    4 x 4-block loss."""
    from pgerosion import adjoint as adj

    st, params, calib, target, land = _calibration_case()
    unit, N, H = st.height_unit_m, st.N, st.H
    for name, fn in (("land", None), ("block4", lambda z: adj.block_loss(z, target, land, unit, N, H, block=4))):
        cal = adj.calibrate(calib, target, land, adj.erodibility_init(st, seed=0), adj.rates_of(params), steps=3,
                            method="line", loss_fn=fn, eta0=0.2, eta_min=1e-3)
        L = cal["loss"]
        print(f"{name}: loss {L} steps {cal['eta']} forwards {cal['forwards']} rates {cal['rates'][-1] if cal['rates'] else None}")
        assert len(cal["eta"]) >= 1, "no step lowered the loss"
        assert all(b < a for a, b in zip(L[:-1], L[1:])), L
