"""Generate the golden fixtures in this directory from the reference itself.

Run from the repository root where the bake project is available::

    NUMBA_CACHE_DIR=/tmp/numba python tests/golden/gen_golden.py /path/to/bake

It imports the bake's own numba code (``globe.cubesphere``,
``globe.erosion.particle``, ``globe.erosion.maps``) and records what it
computes on seeded synthetic inputs built by ``pgerosion.synth``:

* ``cubesphere_vectors.npz`` -- to_sphere / from_sphere / transfer_velocity
  of the scalar functions the particle kernel uses (cubesphere.py:70-220),
  on uniform points plus points within 1e-4 of face edges and corners.
* ``cubesphere_ref_vectors.npz`` -- the bake's own vector file
  (tests/data/cubesphere_vectors.bin: to_sphere / from_sphere records its
  scalar functions reproduce bit for bit), copied into an npz.
* ``halo_N8_H2.npz`` -- the Grid's halo tables, owner and metric at N=8, H=2,
  and SHA-256 digests of the tables at two larger grids.
* ``trace_isolated.npz`` -- a six-face N=48 world after three reference
  iterations, a set of droplets whose touched cells (plus a one-cell ring)
  are pairwise disjoint, and the reference ``trace_particles`` change lists
  and ``apply_changes`` results for them (particle.py:275-1042).
* ``trace_isolated_c1.npz``, ``trace_isolated_n1024.npz`` -- isolated
  droplets on the fresh N_c = 128 small world and N_c = 1024 Earth-default
  world (rebuilt from seed 0 by the tests), with the reference's change
  lists and accumulators for them under those workloads' knobs.
* ``window_trace.npz`` -- one face of that N=48 world cut out as a window
  (``spherical=False``, F = 1; mask: an active basin inside a frozen
  margin inside an outside ring; ``deposit_on_exit``), loaded and unloaded
  droplets sharing cells, the reference ``trace_particles`` change lists
  and the serial ``apply_changes`` results for all of them.
* ``isostasy_tiny.npz`` -- the same kind of N=32 world run through the
  reference ``maps.step`` with isostasy on (0.8, every 2 iterations): the
  smoother's step bound and every iteration's isostasy statistics, and the
  final state.
* ``step_tiny.npz`` -- a six-face N=32 world run through the reference
  ``maps.step`` (plain knobs, uplift replay) for a few iterations: the
  initial state, the final state and the per-iteration stats.
* ``route_flood.npz`` -- the reference's routing flood
  (``route.priority_flood_eps``) on a six-face N=32 world after two
  iterations (with one basin given its own base level) and on a one-face
  window of it.
* ``step_route.npz`` -- as ``step_tiny.npz`` with the routing surface on
  (``erosion.flood_every = 2``): particles steer on the flood.
* ``step_sea.npz`` -- a world with closed below-sea basins: the reference's
  sea mask (``refresh_base``) of its start, and steps with the sea mask and
  the routing flood on (``sea_mask_every = flood_every = 2``).
* ``step_glacial.npz`` -- steps with the glacial pass on (every 2
  iterations from the start) on a world frozen poleward of 50 degrees.

The fixtures are small (well under a few MB) and committed; the tests never
import the bake.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT / "procedural-generation_b200"))


def _ref(bake: str):
    sys.path.insert(0, bake)
    import globe.cubesphere as cs
    import globe.erosion.maps as maps
    import globe.erosion.particle as pk
    from globe.config import WorldParams

    return cs, maps, pk, WorldParams


def gen_vectors(cs):
    rng = np.random.default_rng(20261203)
    K = 3000
    face = rng.integers(0, 6, K)
    u = rng.random(K)
    v = rng.random(K)
    e = K // 4
    i1 = rng.choice(K, e, replace=False)
    u[i1] = np.where(rng.random(e) < 0.5, rng.random(e) * 1e-4, 1.0 - rng.random(e) * 1e-4)
    i2 = rng.choice(K, e, replace=False)
    v[i2] = np.where(rng.random(e) < 0.5, rng.random(e) * 1e-4, 1.0 - rng.random(e) * 1e-4)
    xyz = np.array([cs.to_sphere(int(f), float(a), float(b)) for f, a, b in zip(face, u, v)])
    back = [cs.from_sphere(*p) for p in xyz]
    f2 = np.array([b[0] for b in back], np.int32)
    u2 = np.array([b[1] for b in back])
    v2 = np.array([b[2] for b in back])
    # transfer_velocity on points just outside an edge (the particle crossing)
    T = 2000
    tf = rng.integers(0, 6, T)
    tu = rng.random(T)
    tv = rng.random(T)
    side = rng.integers(0, 4, T)
    d = rng.random(T) * 0.02 + 1e-6
    tu = np.where(side == 0, -d, np.where(side == 1, 1.0 + d, tu))
    tv = np.where(side == 2, -d, np.where(side == 3, 1.0 + d, tv))
    ta, tb = rng.normal(size=(2, T))
    tr = np.array([cs.transfer_velocity(int(f), float(a), float(b), float(c), float(g)) for f, a, b, c, g in zip(tf, tu, tv, ta, tb)])
    np.savez_compressed(HERE / "cubesphere_vectors.npz", face=face.astype(np.int32), u=u, v=v, xyz=xyz, face2=f2, u2=u2, v2=v2,
                        t_face=tf.astype(np.int32), t_u=tu, t_v=tv, t_a=ta, t_b=tb, t_face2=tr[:, 0].astype(np.int32),
                        t_out=tr[:, 1:].astype(np.float64))


def gen_ref_vectors(bake: str):
    """The bake's own checked-in vector file (tests/data/cubesphere_vectors.bin:
    "CSV2", a count, then records of face, u, v, x, y, z, face2, u2, v2 that
    its scalar to_sphere / from_sphere reproduce bit for bit,
    bake/tests/test_cubesphere.py:376-402), kept as an npz so the device
    tests can read it where the bake is not mounted."""
    import struct

    rec_t = np.dtype([("face", "<i4"), ("u", "<f8"), ("v", "<f8"), ("x", "<f8"), ("y", "<f8"), ("z", "<f8"), ("face2", "<i4"),
                      ("u2", "<f8"), ("v2", "<f8")])
    with open(Path(bake) / "tests" / "data" / "cubesphere_vectors.bin", "rb") as fh:
        assert fh.read(4) == b"CSV2"
        (K,) = struct.unpack("<i", fh.read(4))
        rec = np.frombuffer(fh.read(), dtype=rec_t)
    assert rec.shape[0] == K
    np.savez_compressed(HERE / "cubesphere_ref_vectors.npz", face=rec["face"].astype(np.int32), u=rec["u"], v=rec["v"],
                        xyz=np.stack([rec["x"], rec["y"], rec["z"]], 1), face2=rec["face2"].astype(np.int32), u2=rec["u2"],
                        v2=rec["v2"])


def gen_halo(cs):
    g = cs.Grid(8, 2, 50.0)
    hm = g.halo
    dig = {}
    for N, H, c in ((16, 2, 50.0), (32, 4, 9773.0)):
        gg = cs.Grid(N, H, c)
        h = gg.halo
        for k in ("dst", "src", "w", "w_lin", "rot", "nearest"):
            dig[f"{N}_{H}_{k}"] = hashlib.sha256(np.ascontiguousarray(getattr(h, k)).tobytes()).hexdigest()
        dig[f"{N}_{H}_owner"] = hashlib.sha256(np.ascontiguousarray(gg.owner).tobytes()).hexdigest()
        dig[f"{N}_{H}_metric"] = hashlib.sha256(np.ascontiguousarray(gg.metric[0]).tobytes()).hexdigest()
    np.savez_compressed(HERE / "halo_N8_H2.npz", dst=hm.dst, src=hm.src, w=hm.w, w_lin=hm.w_lin, rot=hm.rot, nearest=hm.nearest,
                        owner=g.owner, metric=g.metric[0], metric_inv=g.metric_inv[0], digests=json.dumps(dig))


def _world_params(WorldParams, N, H, cell, seed, land, **erosion):
    from pgerosion.params import plain_knobs

    p = WorldParams.tiny_world(seed)
    kn = plain_knobs()
    kn.update(erosion)
    return p.with_overrides(world={"N_c": N, "halo": H, "cell_size_m": cell, "land_fraction": land, "T": N, "R": 2}, erosion=kn)


def _ref_state(cs, maps, world, p):
    grid = cs.get_grid(world.grid.N, world.grid.H, world.grid.cell_size_m)
    st = maps.ErosionState.from_grid(grid, world.bedrock, world.hardness, world.precip, world.evap, world.uplift, p.erosion)
    st.land_target = float(world.land_fraction)
    return st


def gen_trace(cs, maps, pk, WorldParams):
    from pgerosion import synth

    world = synth.earth_world(seed=3, N=48, H=2, cell_size_m=50.0, land_fraction=0.35)
    p = _world_params(WorldParams, 48, 2, 50.0, 3, 0.35, iterations=10, max_steps=64, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="stack")
    st = _ref_state(cs, maps, world, p)
    for it in range(3):
        maps.step(st, p, it)
    st.pack()
    ep = p.erosion
    NE, H, N = st.NE, st.H, st.N
    rng = np.random.default_rng(77)
    # candidates: rain on land plus loaded droplets (a re-injected stockpile) on land and sea cells
    idx, w = maps.spawn_weights(st)
    nc = 3000
    pick = idx[rng.integers(0, idx.size, nc)]
    f = pick // (NE * NE)
    rem = pick - f * NE * NE
    ei, ej = rem // NE, rem % NE
    x = (ei - H) + rng.random(nc)
    y = (ej - H) + rng.random(nc)
    sed = np.zeros(nc)
    dirs = np.zeros(nc)
    nl = 600
    allc = np.flatnonzero(np.ones(st.height.shape, bool) & (np.pad(np.ones((6, N, N), bool), ((0, 0), (H, H), (H, H)))))
    lp = allc[rng.integers(0, allc.size, nl)]
    lf = lp // (NE * NE)
    lrem = lp - lf * NE * NE
    f = np.concatenate([f, lf])
    x = np.concatenate([x, (lrem // NE - H) + 0.5])
    y = np.concatenate([y, (lrem % NE - H) + 0.5])
    sed = np.concatenate([sed, rng.random(nl) * 0.5 + 1e-3])
    dirs = np.concatenate([dirs, rng.random(nl) * 2 * np.pi])
    P = f.size
    volume0 = float(w.sum()) / 2048.0
    max_steps = maps.max_steps_of(ep, N)
    cap = int(pk.change_list_cap(max_steps, False))

    def trace(ff, xx, yy, ss, dd, conc):
        n = ff.size
        out = dict(cl_cell=np.zeros(n * cap, np.int32), cl_delta=np.zeros(n * cap), cl_vol=np.zeros(n * cap, np.float32),
                   cl_mom=np.zeros((n * cap, 2), np.float32), cl_count=np.zeros(n, np.int64), cl_lo=np.zeros(n, np.int64),
                   cl_hi=np.zeros(n, np.int64), sp_death=np.zeros(n, np.int8))
        cu = lambda k: float(getattr(ep, k)) / st.height_unit_m
        pk.trace_particles(ff.astype(np.int64), xx, yy, ss, dd, volume0, st.samp, False, st.mask, N, H, True,
                           float(ep.dt), float(ep.density), float(ep.friction), float(ep.deposition_rate), float(ep.evap_rate),
                           float(ep.k_mom), 1.0, float(ep.k_disc), float(ep.disc_saturation), float(ep.disc_exponent),
                           float(ep.slope_gain), float(ep.slope_saturation), float(ep.erodibility), cu("cover_depth"),
                           float(ep.min_volume_frac) * volume0, int(max_steps), cu("max_erode"), conc, int(ep.pit_steps), False,
                           float(ep.ocean_deposition_rate), int(ep.ocean_steps), cu("fan_room"), cu("dep_floor_m"),
                           float(ep.lake_trap), 0.0, 0.0, np.zeros((1, 1, 1), np.float32), False,
                           out["cl_cell"], out["cl_delta"], out["cl_vol"], out["cl_mom"], out["cl_count"], out["cl_lo"],
                           out["cl_hi"], out["sp_death"])
        return out

    conc = 1.0 / volume0
    allt = trace(f, x, y, sed, dirs, conc)
    own = st.grid.owner.reshape(-1)
    taken = np.zeros(st.height.size, bool)
    keep = []
    for q in range(P):
        cells = allt["cl_cell"][q * cap: q * cap + allt["cl_count"][q]].astype(np.int64)
        fi = int(f[q])
        c0 = (fi * NE + int(np.floor(x[q])) + H) * NE + int(np.floor(y[q])) + H
        cells = np.unique(np.concatenate([cells, [c0]]))
        cf = cells // (NE * NE)
        cr = cells - cf * NE * NE
        ci, cj = cr // NE, cr % NE
        ring = []
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                ii = np.clip(ci + di, 0, NE - 1)
                jj = np.clip(cj + dj, 0, NE - 1)
                ring.append(own[(cf * NE + ii) * NE + jj])
        ring = np.unique(np.concatenate(ring))
        if taken[ring].any():
            continue
        taken[ring] = True
        keep.append(q)
    keep = np.array(keep)
    f, x, y, sed, dirs = f[keep], x[keep], y[keep], sed[keep], dirs[keep]
    res = trace(f, x, y, sed, dirs, conc)
    acc = np.zeros_like(st.height)
    pending = np.zeros_like(st.height)
    dtr = np.zeros_like(st.height)
    mtr = np.zeros_like(st.momentum)
    samp = st.samp.copy()
    cu = lambda k: float(getattr(ep, k)) / st.height_unit_m
    ap = pk.apply_changes(res["cl_cell"], res["cl_delta"], res["cl_vol"], res["cl_mom"], res["cl_count"], cap,
                          st.height, st.sediment, acc, pending, samp, dtr, mtr, st.mask, cu("iter_erode"), cu("iter_deposit"),
                          float(ep.fan_slope), False, cu("dep_floor_m"), float(ep.offshore_writeoff), np.zeros(1), False,
                          st.lake_load, st.lake_id, st.lake_room)
    np.savez_compressed(
        HERE / "trace_isolated.npz", N=N, H=H, height=st.height, sediment=st.sediment, discharge=st.discharge,
        momentum=st.momentum, hardness=st.hardness, evap=st.evap, base=st.base, mask=st.mask,
        sp_face=f.astype(np.int64), sp_x=x, sp_y=y, sp_sed=sed, sp_dir=dirs, volume0=volume0, conc_scale=conc, cap=cap,
        max_steps=max_steps, params=json.dumps({k: getattr(ep, k) for k in ep.__dataclass_fields__}),
        cell_size_m=st.height_unit_m, **res, acc=acc, pending=pending, disch_track=dtr, mom_track=mtr,
        apply_out=np.array([float(a) for a in ap]))
    print(f"trace_isolated: {keep.size} isolated droplets of {P}; deaths {np.bincount(res['sp_death'], minlength=6)}")


def gen_isolated_configs(cs, maps, pk, WorldParams, which=("c1", "n1024")):
    """Gate 1 on the benchmarked worlds: isolated droplets (paths plus a
    one-cell ring pairwise disjoint) on the fresh N_c = 128 small world and
    the fresh N_c = 1024 Earth-default world (the ones ``synth`` builds from
    seed 0), traced by the reference's ``trace_particles`` and applied by its
    ``apply_changes`` with those workloads' knobs, volume and concurrency
    divisor.  The worlds are rebuilt by the tests from their seed and checked
    against the bedrock digest stored here; the change lists are stored
    compacted (``cl_count`` entries per droplet) and the accumulators as
    their nonzero cells."""
    from pgerosion import synth

    for name in which:
        if name == "c1":
            world = synth.plain_small_world(0)
            ours, P = synth.config_params("small")
        else:
            world = synth.earth_world(seed=0, N=1024, device="cpu")
            ours, P = synth.config_params("earth")
        N, H, cell = world.grid.N, world.grid.H, world.grid.cell_size_m
        eo = ours.erosion
        p = _world_params(WorldParams, N, H, cell, 0, world.land_fraction, iterations=int(eo.iterations),
                          max_steps=int(eo.max_steps), friction=float(eo.friction), erodibility=float(eo.erodibility),
                          deposition_rate=float(eo.deposition_rate), evap_rate=float(eo.evap_rate), uplift_mode=str(eo.uplift_mode))
        st = _ref_state(cs, maps, world, p)
        st.pack()
        ep = p.erosion
        NE = st.NE
        rng = np.random.default_rng(4242 + N)
        idx, w = maps.spawn_weights(st)
        total = float(w.sum())
        volume0 = total / P
        chunk = maps.chunk_size(ep, P)
        conc = chunk / (volume0 * P)
        nc, nl = 1400, 200
        pick = idx[np.searchsorted(np.cumsum(w), rng.random(nc) * total, side="right").clip(0, idx.size - 1)]
        f = pick // (NE * NE)
        rem = pick - f * NE * NE
        x = (rem // NE - H) + rng.random(nc)
        y = (rem % NE - H) + rng.random(nc)
        inter = np.flatnonzero(np.pad(np.ones((6, N, N), bool), ((0, 0), (H, H), (H, H))).reshape(-1))
        lp = inter[rng.integers(0, inter.size, nl)]
        lf = lp // (NE * NE)
        lrem = lp - lf * NE * NE
        f = np.concatenate([f, lf])
        x = np.concatenate([x, (lrem // NE - H) + 0.5])
        y = np.concatenate([y, (lrem % NE - H) + 0.5])
        sed = np.concatenate([np.zeros(nc), rng.random(nl) * 0.02 + 1e-4])
        dirs = np.concatenate([np.zeros(nc), rng.random(nl) * 2 * np.pi])
        max_steps = maps.max_steps_of(ep, N)
        cap = int(pk.change_list_cap(max_steps, False))
        allt = _ref_trace(pk, ep, st.samp, st.mask, N, H, True, False, f, x, y, sed, dirs, volume0, conc, max_steps, cap,
                          st.height_unit_m)
        own = st.grid.owner.reshape(-1)
        taken = np.zeros(st.height.size, bool)
        keep = []
        for q in range(f.size):
            cells = allt["cl_cell"][q * cap: q * cap + allt["cl_count"][q]].astype(np.int64)
            c0 = (int(f[q]) * NE + int(np.floor(x[q])) + H) * NE + int(np.floor(y[q])) + H
            cells = np.unique(np.concatenate([cells, [c0]]))
            cf = cells // (NE * NE)
            cr = cells - cf * NE * NE
            ci, cj = cr // NE, cr % NE
            ring = np.unique(np.concatenate([own[(cf * NE + np.clip(ci + di, 0, NE - 1)) * NE + np.clip(cj + dj, 0, NE - 1)]
                                             for di in (-1, 0, 1) for dj in (-1, 0, 1)]))
            if taken[ring].any():
                continue
            taken[ring] = True
            keep.append(q)
        keep = np.array(keep)
        f, x, y, sed, dirs = f[keep], x[keep], y[keep], sed[keep], dirs[keep]
        res = _ref_trace(pk, ep, st.samp, st.mask, N, H, True, False, f, x, y, sed, dirs, volume0, conc, max_steps, cap,
                         st.height_unit_m)
        acc = np.zeros_like(st.height)
        pending = np.zeros_like(st.height)
        dtr = np.zeros_like(st.height)
        mtr = np.zeros_like(st.momentum)
        samp = st.samp.copy()
        cu = lambda k: float(getattr(ep, k)) / st.height_unit_m
        pk.apply_changes(res["cl_cell"], res["cl_delta"], res["cl_vol"], res["cl_mom"], res["cl_count"], cap,
                         st.height, st.sediment, acc, pending, samp, dtr, mtr, st.mask, cu("iter_erode"), cu("iter_deposit"),
                         float(ep.fan_slope), False, cu("dep_floor_m"), float(ep.offshore_writeoff), np.zeros(1), False,
                         st.lake_load, st.lake_id, st.lake_room)
        n = keep.size
        sel = np.concatenate([np.arange(q * cap, q * cap + res["cl_count"][q]) for q in range(n)])
        touched = np.flatnonzero((acc != 0) | (pending != 0) | (dtr != 0) | (mtr[..., 0] != 0) | (mtr[..., 1] != 0))
        np.savez_compressed(
            HERE / f"trace_isolated_{name}.npz", world=name, N=N, H=H, cell_size_m=cell, P=P,
            bedrock_sha=hashlib.sha256(np.ascontiguousarray(world.bedrock).tobytes()).hexdigest(),
            sp_face=f.astype(np.int64), sp_x=x, sp_y=y, sp_sed=sed, sp_dir=dirs, volume0=volume0, conc_scale=conc, cap=cap,
            max_steps=max_steps, params=json.dumps({k: getattr(ep, k) for k in ep.__dataclass_fields__}),
            cl_count=res["cl_count"], sp_death=res["sp_death"], cl_cell=res["cl_cell"][sel], cl_delta=res["cl_delta"][sel],
            cl_vol=res["cl_vol"][sel], cl_mom=res["cl_mom"][sel], touched=touched, acc=acc.reshape(-1)[touched],
            pending=pending.reshape(-1)[touched], disch_track=dtr.reshape(-1)[touched],
            mom_track=mtr.reshape(-1, 2)[touched])
        print(f"trace_isolated_{name}: {n} isolated droplets of {nc + nl} candidates; deaths "
              f"{np.bincount(res['sp_death'], minlength=6)}; entries {sel.size}")


def _ref_trace(pk, ep, st_samp, mask, N, H, spherical, deposit_on_exit, f, x, y, sed, dirs, volume0, conc, max_steps, cap, unit,
               use_route=False, roots=None, lateral=0.0, lake_park=0.0):
    n = f.size
    out = dict(cl_cell=np.zeros(n * cap, np.int32), cl_delta=np.zeros(n * cap), cl_vol=np.zeros(n * cap, np.float32),
               cl_mom=np.zeros((n * cap, 2), np.float32), cl_count=np.zeros(n, np.int64), cl_lo=np.zeros(n, np.int64),
               cl_hi=np.zeros(n, np.int64), sp_death=np.zeros(n, np.int8))
    cu = lambda k: float(getattr(ep, k)) / unit
    pk.trace_particles(f.astype(np.int64), x, y, sed, dirs, volume0, st_samp, bool(use_route), mask, N, H, spherical,
                       float(ep.dt), float(ep.density), float(ep.friction), float(ep.deposition_rate), float(ep.evap_rate),
                       float(ep.k_mom), 1.0, float(ep.k_disc), float(ep.disc_saturation), float(ep.disc_exponent),
                       float(ep.slope_gain), float(ep.slope_saturation), float(ep.erodibility), cu("cover_depth"),
                       float(ep.min_volume_frac) * volume0, int(max_steps), cu("max_erode"), conc, int(ep.pit_steps),
                       bool(deposit_on_exit), float(ep.ocean_deposition_rate), int(ep.ocean_steps), cu("fan_room"),
                       cu("dep_floor_m"), float(ep.lake_trap), float(lake_park), float(lateral),
                       np.zeros((1, 1, 1), np.float32) if roots is None else roots, roots is not None,
                       out["cl_cell"], out["cl_delta"], out["cl_vol"], out["cl_mom"], out["cl_count"], out["cl_lo"],
                       out["cl_hi"], out["sp_death"])
    return out


def gen_window(cs, maps, pk, WorldParams):
    """A single-face window (spherical=False) cut from the evolved N=48 world."""
    from pgerosion import synth

    world = synth.earth_world(seed=3, N=48, H=2, cell_size_m=50.0, land_fraction=0.35)
    p = _world_params(WorldParams, 48, 2, 50.0, 3, 0.35, iterations=10, max_steps=64, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="stack")
    st = _ref_state(cs, maps, world, p)
    for it in range(3):
        maps.step(st, p, it)
    ep = p.erosion
    NE, H, N = st.NE, st.H, st.N
    land = [(st.height[k][H:H + N, H:H + N] + st.sediment[k][H:H + N, H:H + N] >= 0).mean() for k in range(6)]
    fw = int(np.argsort(land)[3])  # a face with land and sea
    sl = slice(fw, fw + 1)
    w = {k: np.ascontiguousarray(getattr(st, k)[sl]) for k in ("height", "sediment", "discharge", "momentum", "evap", "hardness",
                                                                "base", "metric", "metric_inv")}
    # mask: outside ring (2 cells), frozen margin (3 cells), active basin
    mask = np.zeros((1, NE, NE), np.uint8)
    mask[0, 2:NE - 2, 2:NE - 2] = 2
    mask[0, 5:NE - 5, 5:NE - 5] = 1
    samp = np.zeros((1, NE, NE, st.samp.shape[-1]), np.float32)
    pk.pack_samples(samp, w["height"], w["sediment"], w["height"], False, w["discharge"], w["momentum"], w["evap"], w["hardness"],
                    w["metric"], w["metric_inv"], w["base"], np.zeros((1, NE, NE), np.uint8))
    rng = np.random.default_rng(91)
    act = np.flatnonzero(mask.reshape(-1) == 1)
    n_rain, n_load = 1200, 250
    pick = act[rng.integers(0, act.size, n_rain + n_load)]
    ei, ej = pick // NE, pick % NE
    x = (ei - H) + np.concatenate([rng.random(n_rain), np.full(n_load, 0.5)])
    y = (ej - H) + np.concatenate([rng.random(n_rain), np.full(n_load, 0.5)])
    sed = np.concatenate([np.zeros(n_rain), rng.random(n_load) * 0.5 + 1e-3])
    dirs = np.concatenate([np.zeros(n_rain), rng.random(n_load) * 2 * np.pi])
    f = np.zeros(x.size, np.int64)
    volume0 = 0.02
    conc = 1.0 / (volume0 * x.size)
    max_steps = maps.max_steps_of(ep, N)
    cap = int(pk.change_list_cap(max_steps, False))
    res = _ref_trace(pk, ep, samp, mask, N, H, False, True, f, x, y, sed, dirs, volume0, conc, max_steps, cap, st.height_unit_m)
    acc = np.zeros_like(w["height"])
    pending = np.zeros_like(w["height"])
    dtr = np.zeros_like(w["height"])
    mtr = np.zeros_like(w["momentum"])
    samp_after = samp.copy()
    cu = lambda k: float(getattr(ep, k)) / st.height_unit_m
    z = np.zeros((1, NE, NE))
    ap = pk.apply_changes(res["cl_cell"], res["cl_delta"], res["cl_vol"], res["cl_mom"], res["cl_count"], cap,
                          w["height"], w["sediment"], acc, pending, samp_after, dtr, mtr, mask, cu("iter_erode"), cu("iter_deposit"),
                          float(ep.fan_slope), False, cu("dep_floor_m"), float(ep.offshore_writeoff), np.zeros(1), False,
                          z.copy(), np.zeros((1, NE, NE), np.int32), np.zeros(1))
    np.savez_compressed(
        HERE / "window_trace.npz", N=N, H=H, face=fw, **w, mask=mask, sp_face=f, sp_x=x, sp_y=y, sp_sed=sed, sp_dir=dirs,
        volume0=volume0, conc_scale=conc, cap=cap, max_steps=max_steps, deposit_on_exit=True,
        params=json.dumps({k: getattr(ep, k) for k in ep.__dataclass_fields__}), cell_size_m=st.height_unit_m, **res, acc=acc,
        pending=pending, disch_track=dtr, mom_track=mtr, apply_out=np.array([float(a) for a in ap]))
    print(f"window_trace: face {fw}, {x.size} droplets, entries {int(res['cl_count'].sum())}, deaths "
          f"{np.bincount(res['sp_death'], minlength=6)}, clamped {ap[0]}")


def gen_step(cs, maps, pk, WorldParams):
    from pgerosion import synth

    world = synth.earth_world(seed=5, N=32, H=2, cell_size_m=50.0, land_fraction=0.3)
    iters = 6
    p = _world_params(WorldParams, 32, 2, 50.0, 5, 0.3, iterations=iters, max_steps=48, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="replay")
    st = _ref_state(cs, maps, world, p)
    init = dict(bedrock=world.bedrock, hardness=world.hardness, precip=world.precip, evap=world.evap, uplift=world.uplift)
    maps.start_replay(st, p)
    h_start = st.height.copy()
    stats = []
    for it in range(iters):
        s = maps.step(st, p, it, n_particles=4096)
        stats.append({k: s[k] for k in ("particles", "entries", "clamped", "to_pending", "released", "pending_total",
                                         "deficit_out", "lost_offshore", "deaths", "datum_shift")})
    np.savez_compressed(HERE / "step_tiny.npz", N=32, H=2, cell_size_m=50.0, land_fraction=0.3, seed=5, iterations=iters,
                        n_particles=4096, params=json.dumps({k: getattr(p.erosion, k) for k in p.erosion.__dataclass_fields__}),
                        h_start=h_start, height=st.height, sediment=st.sediment, discharge=st.discharge, momentum=st.momentum,
                        pending=st.pending, stats=json.dumps(stats), **init)
    print("step_tiny:", stats[-1])


def gen_step_route(cs, maps, pk, WorldParams):
    """gen_step with the routing surface on (erosion.flood_every = 2): the
    reference's maps.step refreshes route.priority_flood_eps before the
    particle pass and the kernel steers on it."""
    from pgerosion import synth

    world = synth.earth_world(seed=7, N=32, H=2, cell_size_m=50.0, land_fraction=0.45)
    iters = 5
    p = _world_params(WorldParams, 32, 2, 50.0, 7, 0.45, iterations=iters, max_steps=48, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="replay", flood_every=2)
    st = _ref_state(cs, maps, world, p)
    init = dict(bedrock=world.bedrock, hardness=world.hardness, precip=world.precip, evap=world.evap, uplift=world.uplift)
    maps.start_replay(st, p)
    h_start = st.height.copy()
    stats = []
    routes = []
    for it in range(iters):
        s = maps.step(st, p, it, n_particles=4096)
        stats.append({k: s[k] for k in ("particles", "entries", "clamped", "to_pending", "released", "pending_total",
                                         "deficit_out", "lost_offshore", "deaths", "datum_shift")})
        routes.append(int((st.route > st.height + st.sediment).sum()))
    np.savez_compressed(HERE / "step_route.npz", N=32, H=2, cell_size_m=50.0, land_fraction=0.45, seed=7, iterations=iters,
                        n_particles=4096, params=json.dumps({k: getattr(p.erosion, k) for k in p.erosion.__dataclass_fields__}),
                        h_start=h_start, height=st.height, sediment=st.sediment, discharge=st.discharge, momentum=st.momentum,
                        pending=st.pending, route=st.route, stats=json.dumps(stats), **init)
    print("step_route: cells under the route", routes, stats[-1])


def gen_sea(cs, maps, pk, WorldParams):
    """The reference's sea mask (ErosionState.refresh_base: below-sea
    components, open ocean by area, closed basins at their floor) on a
    six-face N=32 world with closed basins, and steps with the sea mask and
    the routing flood on (sea_mask_every = flood_every = 2)."""
    from pgerosion import synth

    world = synth.earth_world(seed=7, N=32, H=2, cell_size_m=50.0, land_fraction=0.45)
    iters = 5
    p = _world_params(WorldParams, 32, 2, 50.0, 7, 0.45, iterations=iters, max_steps=48, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="replay", flood_every=2, sea_mask_every=2)
    st = _ref_state(cs, maps, world, p)
    init = dict(bedrock=world.bedrock, hardness=world.hardness, precip=world.precip, evap=world.evap, uplift=world.uplift)
    mf = float(p.hydro.ocean_min_fraction)
    b_height, b_sediment = st.height.copy(), st.sediment.copy()
    info0 = st.refresh_base(mf)
    base0 = st.base.copy()
    maps.start_replay(st, p)
    h_start = st.height.copy()
    stats = []
    for it in range(iters):
        s = maps.step(st, p, it, n_particles=4096)
        stats.append({k: s[k] for k in ("particles", "entries", "clamped", "deaths", "datum_shift")})
        if "sea" in s:
            stats[-1]["sea"] = s["sea"]
    np.savez_compressed(HERE / "step_sea.npz", N=32, H=2, cell_size_m=50.0, land_fraction=0.45, seed=7, iterations=iters,
                        n_particles=4096, ocean_min_fraction=mf,
                        params=json.dumps({k: getattr(p.erosion, k) for k in p.erosion.__dataclass_fields__}),
                        b_height=b_height, b_sediment=b_sediment, b_base=base0, b_info=json.dumps(info0),
                        h_start=h_start, height=st.height, sediment=st.sediment, discharge=st.discharge, momentum=st.momentum,
                        pending=st.pending, base=st.base, route=st.route, stats=json.dumps(stats), **init)
    print("step_sea: first refresh", info0, "last", stats[-1])


def gen_glacial(cs, maps, pk, WorldParams):
    """Steps with the glacial pass on (glacial_every = 2 from the start,
    erosion/glacial.py carve): a world whose high latitudes are frozen
    (evaporation multiplier 0 poleward of 50 degrees, the reference's ice line
    at ice_evap = 0), run through the reference's maps.step."""
    from pgerosion import synth

    world = synth.earth_world(seed=17, N=32, H=2, cell_size_m=50.0, land_fraction=0.4)
    world.evap[...] = np.where(np.abs(world.grid.latitude()) > np.radians(50.0), 0.0, 1.0).astype(np.float32)
    iters = 4
    p = _world_params(WorldParams, 32, 2, 50.0, 17, 0.4, iterations=iters, max_steps=48, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="replay", glacial_every=2, glacial_from=0.0)
    st = _ref_state(cs, maps, world, p)
    init = dict(bedrock=world.bedrock, hardness=world.hardness, precip=world.precip, evap=world.evap, uplift=world.uplift)
    maps.start_replay(st, p)
    h_start = st.height.copy()
    stats = []
    pre = None
    for it in range(iters):
        if (it + 1) % 2 == 0 and pre is None:
            pre = {k: getattr(st, k).copy() for k in ("height", "sediment", "discharge", "momentum", "pending", "base")}
        s = maps.step(st, p, it, n_particles=4096)
        stats.append({k: s[k] for k in ("particles", "entries", "clamped", "deaths", "datum_shift")})
        if "glacial" in s:
            stats[-1]["glacial"] = s["glacial"]
    np.savez_compressed(HERE / "step_glacial.npz", N=32, H=2, cell_size_m=50.0, land_fraction=0.4, seed=17, iterations=iters,
                        n_particles=4096, params=json.dumps({k: getattr(p.erosion, k) for k in p.erosion.__dataclass_fields__}),
                        h_start=h_start, height=st.height, sediment=st.sediment, discharge=st.discharge, momentum=st.momentum,
                        pending=st.pending, stats=json.dumps(stats), **init)
    print("step_glacial:", [x.get("glacial") for x in stats])


def gen_isostasy(cs, maps, pk, WorldParams):
    from pgerosion import synth

    world = synth.earth_world(seed=9, N=32, H=2, cell_size_m=50.0, land_fraction=0.3)
    iters = 4
    p = _world_params(WorldParams, 32, 2, 50.0, 9, 0.3, iterations=iters, max_steps=48, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="replay", isostasy=0.8, isostasy_every=2)
    st = _ref_state(cs, maps, world, p)
    init = dict(bedrock=world.bedrock, hardness=world.hardness, precip=world.precip, evap=world.evap, uplift=world.uplift)
    maps.start_replay(st, p)
    stats = []
    for it in range(iters):
        s = maps.step(st, p, it, n_particles=4096)
        stats.append({k: s[k] for k in ("particles", "entries", "clamped", "datum_shift")})
        if "isostasy" in s:
            stats[-1]["isostasy"] = s["isostasy"]
    np.savez_compressed(HERE / "isostasy_tiny.npz", N=32, H=2, cell_size_m=50.0, land_fraction=0.3, seed=9, iterations=iters,
                        n_particles=4096, params=json.dumps({k: getattr(p.erosion, k) for k in p.erosion.__dataclass_fields__}),
                        kappa=maps._smoothing_kappa(st.grid), height=st.height, sediment=st.sediment, discharge=st.discharge,
                        momentum=st.momentum, pending=st.pending, stats=json.dumps(stats), **init)
    print("isostasy_tiny:", [x.get("isostasy") for x in stats])


def gen_route(cs, maps, pk, WorldParams):
    """The reference's routing flood (route.priority_flood_eps) on a
    six-face N=32 world after two reference iterations, and on a window of
    one of its faces (identity owner, a mask with an outside ring)."""
    from globe.erosion import route as rt
    from pgerosion import synth

    world = synth.earth_world(seed=13, N=32, H=2, cell_size_m=50.0, land_fraction=0.35)
    p = _world_params(WorldParams, 32, 2, 50.0, 13, 0.35, iterations=10, max_steps=48, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="stack")
    st = _ref_state(cs, maps, world, p)
    for it in range(2):
        maps.step(st, p, it, n_particles=3000)
    eps = 0.05 / 50.0
    surf = st.height + st.sediment
    base = np.zeros_like(surf)
    base[:, 8:12, 8:12] = surf[:, 8:12, 8:12].min()  # a basin with its own base level: its low point seeds
    mask = np.ones(surf.shape, np.uint8)
    owner = np.ascontiguousarray(st.grid.owner, dtype=np.int64)
    route = rt.priority_flood_eps(surf, mask, owner, st.H, st.N, eps, base)
    NE = st.NE
    wmask = np.zeros((1, NE, NE), np.uint8)
    wmask[0, 3:NE - 3, 3:NE - 3] = 1
    wsurf = np.ascontiguousarray(surf[2:3])
    wowner = rt.window_owner(1, NE)
    wroute = rt.priority_flood_eps(wsurf, wmask, wowner, st.H, st.N, eps, np.zeros_like(wsurf))
    np.savez_compressed(HERE / "route_flood.npz", N=32, H=2, eps=eps, height=st.height, sediment=st.sediment, base=base, mask=mask,
                        owner=owner, route=route, w_height=np.ascontiguousarray(st.height[2:3]),
                        w_sediment=np.ascontiguousarray(st.sediment[2:3]), w_mask=wmask, w_owner=wowner, w_route=wroute)
    print(f"route_flood: filled cells {(route > surf).sum()}, window filled {(wroute > wsurf).sum()}")


def _window_of_evolved(cs, maps, pk, WorldParams):
    """One face (with land and sea) of the N=48 world after three reference
    iterations, as a window: an outside ring of 2 cells, a frozen margin of
    3, the active basin inside."""
    from pgerosion import synth

    world = synth.earth_world(seed=3, N=48, H=2, cell_size_m=50.0, land_fraction=0.35)
    p = _world_params(WorldParams, 48, 2, 50.0, 3, 0.35, iterations=10, max_steps=64, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="stack")
    st = _ref_state(cs, maps, world, p)
    for it in range(3):
        maps.step(st, p, it)
    NE, H, N = st.NE, st.H, st.N
    land = [(st.height[k][H:H + N, H:H + N] + st.sediment[k][H:H + N, H:H + N] >= 0).mean() for k in range(6)]
    fw = int(np.argsort(land)[3])
    sl = slice(fw, fw + 1)
    w = {k: np.ascontiguousarray(getattr(st, k)[sl]) for k in ("height", "sediment", "discharge", "momentum", "evap", "hardness",
                                                                "base", "metric", "metric_inv")}
    mask = np.zeros((1, NE, NE), np.uint8)
    mask[0, 2:NE - 2, 2:NE - 2] = 2
    mask[0, 5:NE - 5, 5:NE - 5] = 1
    return st, p, fw, w, mask


def gen_lake_trace(cs, maps, pk, WorldParams):
    """Lakes on a window (erosion.window_lakes): the reference's
    ErosionState.refresh_route and refresh_lakes_window (maps.py:629-673) on
    a window of the evolved N=48 world, then one trace + serial apply with
    the routing surface and the lake flags packed (particle.py:186-190: flag
    2 on a lake cell; 626-636: no exchange while crossing, the load dropped
    at the shore; 763: no pit count on a lake; 952-956: the bed never eroded
    below the water; 1010-1012: lake flags kept)."""
    st, p, fw, w, mask = _window_of_evolved(cs, maps, pk, WorldParams)
    ep = p.erosion
    NE, H, N = st.NE, st.H, st.N
    unit = st.height_unit_m
    ws = maps.ErosionState(height=w["height"].copy(), sediment=w["sediment"].copy(), discharge=w["discharge"].copy(),
                           momentum=w["momentum"].copy(), hardness=w["hardness"], precip=np.ones((1, NE, NE), np.float32),
                           evap=w["evap"], uplift=np.zeros((1, NE, NE)), mask=mask, metric=w["metric"], metric_inv=w["metric_inv"],
                           N=N, H=H, spherical=False, height_unit_m=unit, base=w["base"].copy(), deposit_on_exit=True)
    eps = float(ep.route_eps) / unit
    min_depth = float(p.hydro.lake_min_depth) / unit
    ws.refresh_route(eps)
    info = ws.refresh_lakes_window(min_depth, 0.0)
    samp = np.zeros((1, NE, NE, pk.NS), np.float32)
    pk.pack_samples(samp, w["height"], w["sediment"], ws.route, True, w["discharge"], w["momentum"], w["evap"], w["hardness"],
                    w["metric"], w["metric_inv"], w["base"], ws.lake_flag)
    rng = np.random.default_rng(93)
    act = np.flatnonzero(mask.reshape(-1) == 1)
    lakec = np.flatnonzero((ws.lake_flag.reshape(-1) > 0) & (mask.reshape(-1) == 1))
    n_rain, n_load, n_lake = 1200, 250, 300
    pick = np.concatenate([act[rng.integers(0, act.size, n_rain + n_load)], lakec[rng.integers(0, lakec.size, n_lake)]])
    ei, ej = pick // NE, pick % NE
    x = (ei - H) + np.concatenate([rng.random(n_rain), np.full(n_load, 0.5), rng.random(n_lake)])
    y = (ej - H) + np.concatenate([rng.random(n_rain), np.full(n_load, 0.5), rng.random(n_lake)])
    sed = np.concatenate([np.zeros(n_rain), rng.random(n_load) * 0.5 + 1e-3, rng.random(n_lake) * 0.2])
    dirs = np.concatenate([np.zeros(n_rain), rng.random(n_load + n_lake) * 2 * np.pi])
    f = np.zeros(x.size, np.int64)
    volume0 = 0.02
    conc = 1.0 / (volume0 * x.size)
    max_steps = maps.max_steps_of(ep, N)
    cap = int(pk.change_list_cap(max_steps, False))
    res = _ref_trace(pk, ep, samp, mask, N, H, False, True, f, x, y, sed, dirs, volume0, conc, max_steps, cap, unit, use_route=True)
    acc = np.zeros_like(w["height"])
    pending = np.zeros_like(w["height"])
    dtr = np.zeros_like(w["height"])
    mtr = np.zeros_like(w["momentum"])
    samp_after = samp.copy()
    cu = lambda k: float(getattr(ep, k)) / unit
    ap = pk.apply_changes(res["cl_cell"], res["cl_delta"], res["cl_vol"], res["cl_mom"], res["cl_count"], cap,
                          w["height"], w["sediment"], acc, pending, samp_after, dtr, mtr, mask, cu("iter_erode"), cu("iter_deposit"),
                          float(ep.fan_slope), True, cu("dep_floor_m"), float(ep.offshore_writeoff), np.zeros(1), False,
                          np.zeros((1, NE, NE)), np.zeros((1, NE, NE), np.int32), np.zeros(1))
    np.savez_compressed(
        HERE / "lake_trace.npz", N=N, H=H, face=fw, **w, mask=mask, route=ws.route, lake_flag=ws.lake_flag, eps=eps,
        min_depth=min_depth, sp_face=f, sp_x=x, sp_y=y, sp_sed=sed, sp_dir=dirs, volume0=volume0, conc_scale=conc, cap=cap,
        max_steps=max_steps, deposit_on_exit=True, params=json.dumps({k: getattr(ep, k) for k in ep.__dataclass_fields__}),
        cell_size_m=unit, **res, acc=acc, pending=pending, disch_track=dtr, mom_track=mtr,
        rflag_after=samp_after[..., pk.S_RFLAG], apply_out=np.array([float(a) for a in ap]))
    print(f"lake_trace: face {fw}, lakes {info}, {x.size} droplets, entries {int(res['cl_count'].sum())}, deaths "
          f"{np.bincount(res['sp_death'], minlength=6)}, clamped {ap[0]}")


def gen_step_lake(cs, maps, pk, WorldParams):
    """Full steps on the sphere with lake flags set by the caller (the
    kernel side of erosion.lake_balance, whose hydro-stage balance is not
    run here: ErosionState.lake_flag = 1 where the routing surface stands
    more than hydro.lake_min_depth over the terrain of the first refresh, 2
    on faces 0-2 (a lake with room, packed as 3), halos copied from the
    nearest interior cell as refresh_lakes does, maps.py:471-479); the
    routing flood refreshed every 2 iterations (flood_every = 2)."""
    from pgerosion import synth

    world = synth.earth_world(seed=7, N=32, H=2, cell_size_m=50.0, land_fraction=0.45)
    iters = 5
    p = _world_params(WorldParams, 32, 2, 50.0, 7, 0.45, iterations=iters, max_steps=48, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="replay", flood_every=2)
    st = _ref_state(cs, maps, world, p)
    init = dict(bedrock=world.bedrock, hardness=world.hardness, precip=world.precip, evap=world.evap, uplift=world.uplift)
    maps.start_replay(st, p)
    h_start = st.height.copy()
    unit = st.height_unit_m
    st.refresh_route(float(p.erosion.route_eps) / unit)
    H, N = st.H, st.N
    inter = (slice(None), slice(H, H + N), slice(H, H + N))
    lake = (st.route - (st.height + st.sediment)) > float(p.hydro.lake_min_depth) / unit
    flag = np.zeros(st.height.shape, np.uint8)
    flag[inter] = lake[inter]
    flag[:3][flag[:3] > 0] = 2
    hm = st.grid.halo
    flat = flag.reshape(-1, 1)
    flat[hm.dst] = flat[hm.nearest]
    st.lake_flag = flag
    planted = flag.copy()
    stats = []
    for it in range(iters):
        s = maps.step(st, p, it, n_particles=4096)
        stats.append({k: s[k] for k in ("particles", "entries", "clamped", "to_pending", "released", "pending_total",
                                         "deficit_out", "lost_offshore", "deaths", "datum_shift")})
    np.savez_compressed(HERE / "step_lake.npz", N=32, H=2, cell_size_m=50.0, land_fraction=0.45, seed=7, iterations=iters,
                        n_particles=4096, params=json.dumps({k: getattr(p.erosion, k) for k in p.erosion.__dataclass_fields__}),
                        h_start=h_start, lake_flag=planted, height=st.height, sediment=st.sediment, discharge=st.discharge,
                        momentum=st.momentum, pending=st.pending, route=st.route, stats=json.dumps(stats), **init)
    print("step_lake: lake cells", int((planted[inter] > 0).sum()), "of which with room", int((planted[inter] > 1).sum()),
          "last", stats[-1])


def gen_lake_balance(cs, maps, pk, WorldParams):
    """The planet's lake refresh (ErosionState.refresh_lakes, maps.py:422-479,
    erosion.lake_fill off): on a six-face N=32 world after two reference
    iterations, the refresh with the land's evaporation (hydro.land_evap = 3,
    Budyko's curve) and without it (lake_evap alone), recording the flags, the
    base level and the water surface; then full steps with lake_balance on,
    the sea mask and the routing flood every 2 iterations."""
    from pgerosion import synth

    world = synth.earth_world(seed=11, N=32, H=2, cell_size_m=50.0, land_fraction=0.45)
    iters = 5
    p = _world_params(WorldParams, 32, 2, 50.0, 11, 0.45, iterations=iters, max_steps=48, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="replay", flood_every=2, sea_mask_every=2,
                      lake_balance=True, lake_fill=False)
    p = p.with_overrides(hydro={"land_evap": 3.0, "lake_evap": 6.0, "pet_t0": 0.0})
    st = _ref_state(cs, maps, world, p)
    init = dict(bedrock=world.bedrock, hardness=world.hardness, precip=world.precip, evap=world.evap, uplift=world.uplift)
    mf = float(p.hydro.ocean_min_fraction)
    unit = st.height_unit_m
    depth = float(p.hydro.lake_min_depth) / unit
    # two plain iterations first (no refreshes) so the surface has the pits erosion makes
    q = p.with_overrides(erosion={"flood_every": 0, "sea_mask_every": 0, "lake_balance": False})
    for it in range(2):
        maps.step(st, q, it, n_particles=4096)
    st.iteration = 0
    u_height, u_sediment = st.height.copy(), st.sediment.copy()
    st.refresh_base(mf)
    st.refresh_route(float(p.erosion.route_eps) / unit)
    sea = st.sea.copy()
    base_before = st.base.copy()
    unit_out = {}
    for tag, le in (("budyko", 3.0), ("plain", 0.0)):
        st.base = base_before.copy()
        st.lake_flag = None
        info = st.refresh_lakes(float(p.hydro.lake_evap), depth, mf, None, le)
        unit_out[f"{tag}_flag"] = st.lake_flag.copy()
        unit_out[f"{tag}_base"] = st.base.copy()
        unit_out[f"{tag}_water"] = np.asarray(st.lake_level, np.float32).copy()
        unit_out[f"{tag}_info"] = json.dumps(info)
        print("lake_balance", tag, info)
    st2 = _ref_state(cs, maps, world, p)
    maps.start_replay(st2, p)
    h_start = st2.height.copy()
    stats = []
    for it in range(iters):
        s = maps.step(st2, p, it, n_particles=4096)
        stats.append({k: s[k] for k in ("particles", "entries", "clamped", "deaths", "datum_shift")})
        if s.get("lakes") is not None:
            stats[-1]["lakes"] = s["lakes"]
    np.savez_compressed(HERE / "lake_balance.npz", N=32, H=2, cell_size_m=50.0, land_fraction=0.45, seed=11, iterations=iters,
                        n_particles=4096, ocean_min_fraction=mf, min_depth=depth, lake_evap=float(p.hydro.lake_evap),
                        params=json.dumps({k: getattr(p.erosion, k) for k in p.erosion.__dataclass_fields__}),
                        u_height=u_height, u_sediment=u_sediment, u_sea=sea, u_base=base_before, u_route=st.route, **unit_out,
                        h_start=h_start, height=st2.height, sediment=st2.sediment, discharge=st2.discharge, momentum=st2.momentum,
                        pending=st2.pending, base=st2.base, lake_flag=st2.lake_flag, route=st2.route, stats=json.dumps(stats),
                        **init)
    print("lake_balance steps:", stats[-1])


def gen_basin_fill(cs, maps, pk, WorldParams):
    """The reference's fill_basins (maps.py:1278-1326) on a fresh six-face
    N=32 world after start_replay: the sediment it lays and its statistics."""
    from pgerosion import synth

    world = synth.earth_world(seed=11, N=32, H=2, cell_size_m=50.0, land_fraction=0.45)
    p = _world_params(WorldParams, 32, 2, 50.0, 11, 0.45, iterations=5, max_steps=48, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="replay", basin_fill_grade=0.1, basin_fill_min_m=1.0)
    st = _ref_state(cs, maps, world, p)
    maps.start_replay(st, p)
    h0, s0 = st.height.copy(), st.sediment.copy()
    info = maps.fill_basins(st, p)
    np.savez_compressed(HERE / "basin_fill.npz", N=32, H=2, cell_size_m=50.0, land_fraction=0.45, seed=11,
                        params=json.dumps({k: getattr(p.erosion, k) for k in p.erosion.__dataclass_fields__}),
                        h_start=h0, s_start=s0, height=st.height, sediment=st.sediment, info=json.dumps(info),
                        bedrock=world.bedrock, hardness=world.hardness, precip=world.precip, evap=world.evap, uplift=world.uplift)
    print("basin_fill:", info)


def gen_roots_trace(cs, maps, pk, WorldParams):
    """Roots (erosion.vegetation, particle.py:615-618: the exchange rate on
    land scaled by 1 - roots) on the window of the evolved N=48 world: one
    trace + serial apply of the reference with a seeded roots field."""
    st, p, fw, w, mask = _window_of_evolved(cs, maps, pk, WorldParams)
    ep = p.erosion
    NE, H, N = st.NE, st.H, st.N
    unit = st.height_unit_m
    rng = np.random.default_rng(97)
    roots = (rng.random((1, NE, NE)) * 0.9).astype(np.float32)
    samp = np.zeros((1, NE, NE, pk.NS), np.float32)
    pk.pack_samples(samp, w["height"], w["sediment"], w["height"], False, w["discharge"], w["momentum"], w["evap"], w["hardness"],
                    w["metric"], w["metric_inv"], w["base"], np.zeros((1, NE, NE), np.uint8))
    act = np.flatnonzero(mask.reshape(-1) == 1)
    n_rain, n_load = 1200, 250
    pick = act[rng.integers(0, act.size, n_rain + n_load)]
    ei, ej = pick // NE, pick % NE
    x = (ei - H) + np.concatenate([rng.random(n_rain), np.full(n_load, 0.5)])
    y = (ej - H) + np.concatenate([rng.random(n_rain), np.full(n_load, 0.5)])
    sed = np.concatenate([np.zeros(n_rain), rng.random(n_load) * 0.5 + 1e-3])
    dirs = np.concatenate([np.zeros(n_rain), rng.random(n_load) * 2 * np.pi])
    f = np.zeros(x.size, np.int64)
    volume0 = 0.02
    conc = 1.0 / (volume0 * x.size)
    max_steps = maps.max_steps_of(ep, N)
    cap = int(pk.change_list_cap(max_steps, False))
    res = _ref_trace(pk, ep, samp, mask, N, H, False, True, f, x, y, sed, dirs, volume0, conc, max_steps, cap, unit, roots=roots)
    acc = np.zeros_like(w["height"])
    pending = np.zeros_like(w["height"])
    dtr = np.zeros_like(w["height"])
    mtr = np.zeros_like(w["momentum"])
    samp_after = samp.copy()
    cu = lambda k: float(getattr(ep, k)) / unit
    ap = pk.apply_changes(res["cl_cell"], res["cl_delta"], res["cl_vol"], res["cl_mom"], res["cl_count"], cap,
                          w["height"], w["sediment"], acc, pending, samp_after, dtr, mtr, mask, cu("iter_erode"), cu("iter_deposit"),
                          float(ep.fan_slope), False, cu("dep_floor_m"), float(ep.offshore_writeoff), np.zeros(1), False,
                          np.zeros((1, NE, NE)), np.zeros((1, NE, NE), np.int32), np.zeros(1))
    np.savez_compressed(
        HERE / "roots_trace.npz", N=N, H=H, face=fw, **w, mask=mask, roots=roots, sp_face=f, sp_x=x, sp_y=y, sp_sed=sed,
        sp_dir=dirs, volume0=volume0, conc_scale=conc, cap=cap, max_steps=max_steps, deposit_on_exit=True,
        params=json.dumps({k: getattr(ep, k) for k in ep.__dataclass_fields__}), cell_size_m=unit, **res, acc=acc,
        pending=pending, disch_track=dtr, mom_track=mtr, apply_out=np.array([float(a) for a in ap]))
    print(f"roots_trace: {x.size} droplets, entries {int(res['cl_count'].sum())}, clamped {ap[0]}")


def gen_window_steps(cs, maps, pk, WorldParams):
    """Full reference steps on a window (maps.step with spherical=False):
    the window of the evolved N=48 world with its masks, the cell-count
    discharge scales on (disc_saturation_cells, momentum_saturation_cells)
    and part of the spawn weight declared as inflow across the window's edge
    (ErosionState.inflow_volume, maps.py:913-917)."""
    st, p, fw, w, mask = _window_of_evolved(cs, maps, pk, WorldParams)
    NE, H, N = st.NE, st.H, st.N
    unit = st.height_unit_m
    rng = np.random.default_rng(101)
    precip = (0.5 + rng.random((1, NE, NE))).astype(np.float32)
    q = p.with_overrides(erosion={"disc_saturation_cells": 40.0, "momentum_saturation_cells": 15.0, "uplift_mode": "stack"})
    ws = maps.ErosionState(height=w["height"].copy(), sediment=w["sediment"].copy(), discharge=w["discharge"].copy(),
                           momentum=w["momentum"].copy(), hardness=w["hardness"], precip=precip, evap=w["evap"],
                           uplift=np.zeros((1, NE, NE)), mask=mask, metric=w["metric"], metric_inv=w["metric_inv"], N=N, H=H,
                           spherical=False, height_unit_m=unit, base=w["base"].copy(), deposit_on_exit=True)
    ws.inflow_volume = float(0.3 * maps.spawn_weights(ws)[1].sum())  # 30 % of the spawn weight flows in
    h0 = {k: getattr(ws, k).copy() for k in ("height", "sediment", "discharge", "momentum")}
    stats = []
    for it in range(3):
        s_ = maps.step(ws, q, it, n_particles=1500)
        stats.append({k: s_[k] for k in ("particles", "entries", "clamped", "deaths")})
    np.savez_compressed(HERE / "window_steps.npz", N=N, H=H, cell_size_m=unit, seed=int(q.world.seed), land_fraction=0.35,
                        mask=mask, precip=precip, evap=w["evap"],
                        hardness=w["hardness"], base=w["base"], metric=w["metric"], metric_inv=w["metric_inv"],
                        inflow_volume=ws.inflow_volume, n_particles=1500, iterations=3,
                        params=json.dumps({k: getattr(q.erosion, k) for k in q.erosion.__dataclass_fields__}),
                        **{f"start_{k}": v for k, v in h0.items()}, height=ws.height, sediment=ws.sediment,
                        discharge=ws.discharge, momentum=ws.momentum, pending=ws.pending, stats=json.dumps(stats))
    print("window_steps:", stats[-1])


def gen_lateral(cs, maps, pk, WorldParams):
    """The bank cut on the outside of bends (erosion.lateral_rate,
    particle.py:699-738; entries of volume -2 applied under the erosion caps,
    particle.py:934-1018): one reference trace + serial apply on the window
    of the evolved N=48 world, and full reference steps on a six-face N=32
    world with lateral_rate = 0.5."""
    st, p, fw, w, mask = _window_of_evolved(cs, maps, pk, WorldParams)
    ep = p.erosion
    NE, H, N = st.NE, st.H, st.N
    unit = st.height_unit_m
    rate = 0.5
    samp = np.zeros((1, NE, NE, pk.NS), np.float32)
    pk.pack_samples(samp, w["height"], w["sediment"], w["height"], False, w["discharge"], w["momentum"], w["evap"], w["hardness"],
                    w["metric"], w["metric_inv"], w["base"], np.zeros((1, NE, NE), np.uint8))
    rng = np.random.default_rng(103)
    act = np.flatnonzero(mask.reshape(-1) == 1)
    n_rain, n_load = 1200, 250
    pick = act[rng.integers(0, act.size, n_rain + n_load)]
    ei, ej = pick // NE, pick % NE
    x = (ei - H) + np.concatenate([rng.random(n_rain), np.full(n_load, 0.5)])
    y = (ej - H) + np.concatenate([rng.random(n_rain), np.full(n_load, 0.5)])
    sed = np.concatenate([np.zeros(n_rain), rng.random(n_load) * 0.5 + 1e-3])
    dirs = np.concatenate([np.zeros(n_rain), rng.random(n_load) * 2 * np.pi])
    f = np.zeros(x.size, np.int64)
    volume0 = 0.02
    conc = 1.0 / (volume0 * x.size)
    max_steps = maps.max_steps_of(ep, N)
    cap = int(pk.change_list_cap(max_steps, True))
    res = _ref_trace(pk, ep, samp, mask, N, H, False, True, f, x, y, sed, dirs, volume0, conc, max_steps, cap, unit, lateral=rate)
    acc = np.zeros_like(w["height"])
    pending = np.zeros_like(w["height"])
    dtr = np.zeros_like(w["height"])
    mtr = np.zeros_like(w["momentum"])
    samp_after = samp.copy()
    cu = lambda k: float(getattr(ep, k)) / unit
    ap = pk.apply_changes(res["cl_cell"], res["cl_delta"], res["cl_vol"], res["cl_mom"], res["cl_count"], cap,
                          w["height"], w["sediment"], acc, pending, samp_after, dtr, mtr, mask, cu("iter_erode"), cu("iter_deposit"),
                          float(ep.fan_slope), False, cu("dep_floor_m"), float(ep.offshore_writeoff), np.zeros(1), False,
                          np.zeros((1, NE, NE)), np.zeros((1, NE, NE), np.int32), np.zeros(1))
    banks = int((res["cl_vol"] == -2.0).sum())
    np.savez_compressed(
        HERE / "lateral_trace.npz", N=N, H=H, face=fw, **w, mask=mask, lateral_rate=rate, sp_face=f, sp_x=x, sp_y=y, sp_sed=sed,
        sp_dir=dirs, volume0=volume0, conc_scale=conc, cap=cap, max_steps=max_steps, deposit_on_exit=True,
        params=json.dumps({**{k: getattr(ep, k) for k in ep.__dataclass_fields__}, "lateral_rate": rate}), cell_size_m=unit,
        **res, acc=acc, pending=pending, disch_track=dtr, mom_track=mtr, apply_out=np.array([float(a) for a in ap]))
    print(f"lateral_trace: {x.size} droplets, entries {int(res['cl_count'].sum())}, bank entries {banks}, clamped {ap[0]}")

    from pgerosion import synth

    world = synth.earth_world(seed=5, N=32, H=2, cell_size_m=50.0, land_fraction=0.3)
    iters = 4
    p2 = _world_params(WorldParams, 32, 2, 50.0, 5, 0.3, iterations=iters, max_steps=48, friction=0.05, erodibility=0.3,
                       deposition_rate=0.3, evap_rate=0.01, uplift_mode="replay", lateral_rate=rate)
    st2 = _ref_state(cs, maps, world, p2)
    init = dict(bedrock=world.bedrock, hardness=world.hardness, precip=world.precip, evap=world.evap, uplift=world.uplift)
    maps.start_replay(st2, p2)
    h_start = st2.height.copy()
    stats = []
    for it in range(iters):
        s_ = maps.step(st2, p2, it, n_particles=4096)
        stats.append({k: s_[k] for k in ("particles", "entries", "clamped", "deaths", "datum_shift")})
    np.savez_compressed(HERE / "step_lateral.npz", N=32, H=2, cell_size_m=50.0, land_fraction=0.3, seed=5, iterations=iters,
                        n_particles=4096, params=json.dumps({k: getattr(p2.erosion, k) for k in p2.erosion.__dataclass_fields__}),
                        h_start=h_start, height=st2.height, sediment=st2.sediment, discharge=st2.discharge,
                        momentum=st2.momentum, pending=st2.pending, stats=json.dumps(stats), **init)
    print("step_lateral:", stats[-1])


def gen_window_lake_balance(cs, maps, pk, WorldParams):
    """A window's lakes settled against evaporation (ErosionState.
    refresh_lakes_window with window_lake_evap > 0, maps.py:629-736) on the
    window of the evolved N=48 world with a seeded rain field: the flags, the
    lowered routing surface and the counts, for two evaporation rates."""
    st, p, fw, w, mask = _window_of_evolved(cs, maps, pk, WorldParams)
    NE, H, N = st.NE, st.H, st.N
    unit = st.height_unit_m
    rng = np.random.default_rng(107)
    precip = (0.2 + rng.random((1, NE, NE))).astype(np.float32)
    out = {}
    for tag, le in (("a", 5.0), ("b", 60.0)):
        ws = maps.ErosionState(height=w["height"].copy(), sediment=w["sediment"].copy(), discharge=w["discharge"].copy(),
                               momentum=w["momentum"].copy(), hardness=w["hardness"], precip=precip, evap=w["evap"],
                               uplift=np.zeros((1, NE, NE)), mask=mask, metric=w["metric"], metric_inv=w["metric_inv"], N=N, H=H,
                               spherical=False, height_unit_m=unit, base=w["base"].copy(), deposit_on_exit=True)
        eps = float(p.erosion.route_eps) / unit
        depth = float(p.hydro.lake_min_depth) / unit
        ws.refresh_route(eps)
        route0 = ws.route.copy()
        info = ws.refresh_lakes_window(depth, le)
        out[f"{tag}_route0"] = route0
        out[f"{tag}_route"] = ws.route.copy()
        out[f"{tag}_flag"] = ws.lake_flag.copy()
        out[f"{tag}_info"] = json.dumps(info)
        out[f"{tag}_lake_evap"] = le
        print("window_lake_balance", tag, le, info)
    np.savez_compressed(HERE / "window_lake_balance.npz", N=N, H=H, cell_size_m=unit, height=w["height"], sediment=w["sediment"],
                        mask=mask, precip=precip, evap=w["evap"], min_depth=float(p.hydro.lake_min_depth) / unit, **out)


def gen_lake_parks(cs, maps, pk, WorldParams):
    """Lake parks (erosion.lake_fill: particle.py:626-636, 672-696 in the
    trace, 912-933 and 1019 in the apply): the lake window of
    gen_lake_trace with every lake flagged 2 (room for its rivers' load),
    each lake numbered (lake_id) with a small room (lake_room) so that the
    serial countdown refuses some loads; one reference trace with lake_park
    on and one serial apply, recording the parked loads and the rooms left."""
    from scipy import ndimage

    st, p, fw, w, mask = _window_of_evolved(cs, maps, pk, WorldParams)
    ep = p.erosion
    NE, H, N = st.NE, st.H, st.N
    unit = st.height_unit_m
    ws = maps.ErosionState(height=w["height"].copy(), sediment=w["sediment"].copy(), discharge=w["discharge"].copy(),
                           momentum=w["momentum"].copy(), hardness=w["hardness"], precip=np.ones((1, NE, NE), np.float32),
                           evap=w["evap"], uplift=np.zeros((1, NE, NE)), mask=mask, metric=w["metric"], metric_inv=w["metric_inv"],
                           N=N, H=H, spherical=False, height_unit_m=unit, base=w["base"].copy(), deposit_on_exit=True)
    ws.refresh_route(float(ep.route_eps) / unit)
    ws.refresh_lakes_window(float(p.hydro.lake_min_depth) / unit, 0.0)
    lab, n = ndimage.label(ws.lake_flag[0] > 0, structure=np.ones((3, 3), bool))
    flag = (ws.lake_flag > 0).astype(np.uint8) * 2
    lake_id = np.full((1, NE, NE), -1, np.int32)
    lake_id[0][lab > 0] = lab[lab > 0] - 1
    lake_room = np.full(max(n, 1), 0.02, np.float64)
    samp = np.zeros((1, NE, NE, pk.NS), np.float32)
    pk.pack_samples(samp, w["height"], w["sediment"], ws.route, True, w["discharge"], w["momentum"], w["evap"], w["hardness"],
                    w["metric"], w["metric_inv"], w["base"], flag)
    rng = np.random.default_rng(109)
    act = np.flatnonzero(mask.reshape(-1) == 1)
    n_rain, n_load = 1500, 400
    pick = act[rng.integers(0, act.size, n_rain + n_load)]
    ei, ej = pick // NE, pick % NE
    x = (ei - H) + np.concatenate([rng.random(n_rain), np.full(n_load, 0.5)])
    y = (ej - H) + np.concatenate([rng.random(n_rain), np.full(n_load, 0.5)])
    sed = np.concatenate([np.zeros(n_rain), rng.random(n_load) * 0.5 + 1e-3])
    dirs = np.concatenate([np.zeros(n_rain), rng.random(n_load) * 2 * np.pi])
    f = np.zeros(x.size, np.int64)
    volume0 = 0.02
    conc = 1.0 / (volume0 * x.size)
    max_steps = maps.max_steps_of(ep, N)
    cap = int(pk.change_list_cap(max_steps, False))
    res = _ref_trace(pk, ep, samp, mask, N, H, False, True, f, x, y, sed, dirs, volume0, conc, max_steps, cap, unit,
                     use_route=True, lake_park=1.0)
    acc = np.zeros_like(w["height"])
    pending = np.zeros_like(w["height"])
    dtr = np.zeros_like(w["height"])
    mtr = np.zeros_like(w["momentum"])
    samp_after = samp.copy()
    lake_load = np.zeros((1, NE, NE))
    room_after = lake_room.copy()
    cu = lambda k: float(getattr(ep, k)) / unit
    ap = pk.apply_changes(res["cl_cell"], res["cl_delta"], res["cl_vol"], res["cl_mom"], res["cl_count"], cap,
                          w["height"], w["sediment"], acc, pending, samp_after, dtr, mtr, mask, cu("iter_erode"), cu("iter_deposit"),
                          float(ep.fan_slope), True, cu("dep_floor_m"), float(ep.offshore_writeoff), np.zeros(1), False,
                          lake_load, lake_id, room_after)
    parks = int((res["cl_vol"] == -3.0).sum())
    np.savez_compressed(
        HERE / "lake_parks.npz", N=N, H=H, face=fw, **w, mask=mask, route=ws.route, lake_flag=flag, lake_id=lake_id,
        lake_room=lake_room, sp_face=f, sp_x=x, sp_y=y, sp_sed=sed, sp_dir=dirs, volume0=volume0, conc_scale=conc, cap=cap,
        max_steps=max_steps, deposit_on_exit=True, params=json.dumps({k: getattr(ep, k) for k in ep.__dataclass_fields__}),
        cell_size_m=unit, **res, acc=acc, pending=pending, disch_track=dtr, mom_track=mtr, lake_load=lake_load,
        room_after=room_after, apply_out=np.array([float(a) for a in ap]))
    print(f"lake_parks: {n} lakes, {x.size} droplets, park entries {parks}, parked {lake_load.sum():.4f}, rooms left {room_after}")


def gen_lake_fill_steps(cs, maps, pk, WorldParams):
    """Full reference steps with the bake's default lakes: lake_balance and
    lake_fill on (the loads rivers bring a lake parked in it and laid over
    its floor at each refresh, maps.py:490-628), the sea mask and the routing
    flood every 2 iterations, on the six-face N=32 world of gen_lake_balance."""
    from pgerosion import synth

    world = synth.earth_world(seed=11, N=32, H=2, cell_size_m=50.0, land_fraction=0.45)
    iters = 7
    p = _world_params(WorldParams, 32, 2, 50.0, 11, 0.45, iterations=iters, max_steps=48, friction=0.05, erodibility=0.3,
                      deposition_rate=0.3, evap_rate=0.01, uplift_mode="replay", flood_every=2, sea_mask_every=2,
                      lake_balance=True, lake_fill=True, basin_fill_grade=0.1)
    p = p.with_overrides(hydro={"land_evap": 3.0, "lake_evap": 6.0, "pet_t0": 0.0})
    st = _ref_state(cs, maps, world, p)
    maps.start_replay(st, p)
    h_start = st.height.copy()
    stats = []
    for it in range(iters):
        s_ = maps.step(st, p, it, n_particles=4096)
        stats.append({k: s_[k] for k in ("particles", "entries", "clamped", "deaths", "datum_shift")})
        if s_.get("lakes") is not None:
            stats[-1]["lakes"] = s_["lakes"]
    np.savez_compressed(HERE / "lake_fill_steps.npz", N=32, H=2, cell_size_m=50.0, land_fraction=0.45, seed=11, iterations=iters,
                        n_particles=4096, params=json.dumps({k: getattr(p.erosion, k) for k in p.erosion.__dataclass_fields__}),
                        h_start=h_start, height=st.height, sediment=st.sediment, discharge=st.discharge, momentum=st.momentum,
                        pending=st.pending, base=st.base, lake_flag=st.lake_flag, lake_load=st.lake_load, lake_id=st.lake_id,
                        lake_room=st.lake_room, route=st.route, stats=json.dumps(stats), bedrock=world.bedrock,
                        hardness=world.hardness, precip=world.precip, evap=world.evap, uplift=world.uplift)
    print("lake_fill_steps:", [s_.get("lakes") for s_ in stats])


def main(bake: str, only: str | None = None):
    cs, maps, pk, WorldParams = _ref(bake)
    gens = {"vectors": lambda: gen_vectors(cs), "ref_vectors": lambda: gen_ref_vectors(bake), "halo": lambda: gen_halo(cs),
            "trace": lambda: gen_trace(cs, maps, pk, WorldParams),
            "isolated_configs": lambda: gen_isolated_configs(cs, maps, pk, WorldParams), "window": lambda: gen_window(cs, maps, pk, WorldParams),
            "isostasy": lambda: gen_isostasy(cs, maps, pk, WorldParams),
            "step": lambda: gen_step(cs, maps, pk, WorldParams), "route": lambda: gen_route(cs, maps, pk, WorldParams),
            "step_route": lambda: gen_step_route(cs, maps, pk, WorldParams), "sea": lambda: gen_sea(cs, maps, pk, WorldParams),
            "glacial": lambda: gen_glacial(cs, maps, pk, WorldParams),
            "lake_trace": lambda: gen_lake_trace(cs, maps, pk, WorldParams),
            "step_lake": lambda: gen_step_lake(cs, maps, pk, WorldParams),
            "lake_balance": lambda: gen_lake_balance(cs, maps, pk, WorldParams),
            "basin_fill": lambda: gen_basin_fill(cs, maps, pk, WorldParams),
            "roots_trace": lambda: gen_roots_trace(cs, maps, pk, WorldParams),
            "window_steps": lambda: gen_window_steps(cs, maps, pk, WorldParams),
            "lateral": lambda: gen_lateral(cs, maps, pk, WorldParams),
            "window_lake_balance": lambda: gen_window_lake_balance(cs, maps, pk, WorldParams),
            "lake_parks": lambda: gen_lake_parks(cs, maps, pk, WorldParams),
            "lake_fill_steps": lambda: gen_lake_fill_steps(cs, maps, pk, WorldParams)}
    for name, g in gens.items():
        if only is None or name == only:
            g()


if __name__ == "__main__":
    import os

    bake = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PGE_BAKE_DIR")
    if not bake:
        sys.exit("usage: gen_golden.py <bake checkout> [fixture]   (or set PGE_BAKE_DIR)")
    main(bake, sys.argv[2] if len(sys.argv) > 2 else None)
