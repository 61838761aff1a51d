"""Cube-sphere geometry tables for the erosion kernels (host side, numpy).

The bake's grid is an equi-angular cube-sphere: face ``f`` has an
orthonormal basis ``(right, up, normal)`` (OpenGL cube-map order +X, -X, +Y,
-Y, +Z, -Z), a face coordinate ``(u, v)`` maps to the unit vector
``normalize(normal + tan((u-1/2) pi/2) right + tan((v-1/2) pi/2) up)``.
Arrays are extended with a halo of ``H`` cells: ``NE = N + 2H``.

What the kernels need from the geometry, computed here once per grid:

* the dimensionless metric ``(g_ii, g_ij, g_jj)`` and its inverse in cell
  units, float32 -- bake/globe/cubesphere.py:477-502.  The metric does not
  depend on the face, so one ``(NE, NE, 3)`` table serves all six faces
  (the device kernels index it by ``(ei, ej)`` only).
* the halo gather tables -- cubesphere.py:540-662: every halo cell is a
  16-source weighted sum of interior cells.  Edge blocks use a 4x4 cubic
  Lagrange stencil on the neighbouring face, corner blocks a least-squares
  quadratic fit over the 16 nearest interior cells; vector fields are
  rotated into the destination face's components with exact
  ``transfer_vector`` matrices.
* the owner table -- cubesphere.py:664-674: flat index of the interior cell
  that owns each extended cell (the nearest halo source).

Unlike the bake's ``Grid``, nothing here materialises a ``(6, NE, NE, 3)``
table of cell centres, so an N = 8192 grid costs only its halo rows.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from functools import cached_property

import numpy as np

#: face bases (right, up, normal), cube-map order +X, -X, +Y, -Y, +Z, -Z
BASES = np.array(
    [
        [[0.0, 0.0, -1.0], [0.0, -1.0, 0.0], [1.0, 0.0, 0.0]],
        [[0.0, 0.0, 1.0], [0.0, -1.0, 0.0], [-1.0, 0.0, 0.0]],
        [[1.0, 0.0, 0.0], [0.0, 0.0, 1.0], [0.0, 1.0, 0.0]],
        [[1.0, 0.0, 0.0], [0.0, 0.0, -1.0], [0.0, -1.0, 0.0]],
        [[1.0, 0.0, 0.0], [0.0, -1.0, 0.0], [0.0, 0.0, 1.0]],
        [[-1.0, 0.0, 0.0], [0.0, -1.0, 0.0], [0.0, 0.0, -1.0]],
    ],
    dtype=np.float64,
)
HALF_PI = math.pi / 2.0
TWO_OVER_PI = 2.0 / math.pi


def planet_radius(N: int, cell_size_m: float) -> float:
    """Radius at which a face edge is exactly N cells of ``cell_size_m``."""
    return N * cell_size_m * 4.0 / (2.0 * math.pi)


# --------------------------------------------------------------------------
# vectorised mapping
# --------------------------------------------------------------------------
def face_point(face, u, v) -> np.ndarray:
    """(face, u, v) -> unit vectors (..., 3); (u, v) may leave [0, 1)."""
    face = np.asarray(face, dtype=np.int64)
    s = np.tan((np.asarray(u, dtype=np.float64) - 0.5) * HALF_PI)
    t = np.tan((np.asarray(v, dtype=np.float64) - 0.5) * HALF_PI)
    B = BASES[face]
    q = B[..., 2, :] + s[..., None] * B[..., 0, :] + t[..., None] * B[..., 1, :]
    return q / np.linalg.norm(q, axis=-1, keepdims=True)


def point_face(p) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Unit vectors -> (face, u, v); the face is the dominant axis, ties
    resolved X before Y before Z; u, v in the closed interval [0, 1]."""
    p = np.asarray(p, dtype=np.float64)
    a = np.abs(p)
    xdom = (a[..., 0] >= a[..., 1]) & (a[..., 0] >= a[..., 2])
    ydom = ~xdom & (a[..., 1] >= a[..., 2])
    face = np.where(xdom, np.where(p[..., 0] >= 0, 0, 1),
                    np.where(ydom, np.where(p[..., 1] >= 0, 2, 3), np.where(p[..., 2] >= 0, 4, 5))).astype(np.int64)
    B = BASES[face]
    d = np.sum(p * B[..., 2, :], axis=-1)
    u = np.arctan(np.sum(p * B[..., 0, :], axis=-1) / d) * TWO_OVER_PI + 0.5
    v = np.arctan(np.sum(p * B[..., 1, :], axis=-1) / d) * TWO_OVER_PI + 0.5
    return face, u, v


def tangents(face, u, v) -> tuple[np.ndarray, np.ndarray]:
    """dp/du and dp/dv on the unit sphere, each (..., 3)."""
    face = np.asarray(face, dtype=np.int64)
    s = np.tan((np.asarray(u, dtype=np.float64) - 0.5) * HALF_PI)
    t = np.tan((np.asarray(v, dtype=np.float64) - 0.5) * HALF_PI)
    B = BASES[face]
    q = B[..., 2, :] + s[..., None] * B[..., 0, :] + t[..., None] * B[..., 1, :]
    ql = np.linalg.norm(q, axis=-1, keepdims=True)
    p = q / ql
    du = B[..., 0, :] * (HALF_PI * (1.0 + s * s))[..., None]
    dv = B[..., 1, :] * (HALF_PI * (1.0 + t * t))[..., None]
    ju = (du - p * np.sum(p * du, axis=-1, keepdims=True)) / ql
    jv = (dv - p * np.sum(p * dv, axis=-1, keepdims=True)) / ql
    return ju, jv


def reexpress(face_src, u_src, v_src, ab, face_dst, u_dst, v_dst) -> np.ndarray:
    """Tangent vector components ``ab`` (..., 2) at a point of one face into
    the components of another face at the same point (2x2 normal equations)."""
    ju, jv = tangents(face_src, u_src, v_src)
    w = ab[..., :1] * ju + ab[..., 1:] * jv
    ku, kv = tangents(face_dst, u_dst, v_dst)
    guu = np.sum(ku * ku, -1)
    guv = np.sum(ku * kv, -1)
    gvv = np.sum(kv * kv, -1)
    ru = np.sum(ku * w, -1)
    rv = np.sum(kv * w, -1)
    det = guu * gvv - guv * guv
    return np.stack([(gvv * ru - guv * rv) / det, (guu * rv - guv * ru) / det], axis=-1)


def cubic_weights(t) -> np.ndarray:
    """Cubic Lagrange weights on nodes -1, 0, 1, 2 at offset ``t`` (..., 4)."""
    t = np.asarray(t, dtype=np.float64)
    return np.stack([-t * (t - 1) * (t - 2) / 6.0, (t + 1) * (t - 1) * (t - 2) / 2.0,
                     -(t + 1) * t * (t - 2) / 2.0, (t + 1) * t * (t - 1) / 6.0], axis=-1)


def linear_weights(t) -> np.ndarray:
    """Two-node linear weights laid on the 4-node stencil -1..2."""
    t = np.asarray(t, dtype=np.float64)
    w = np.zeros(t.shape + (4,), dtype=np.float64)
    lo = np.clip(np.floor(t).astype(np.int64), -1, 1)
    frac = np.clip(t - lo, 0.0, 1.0)
    np.put_along_axis(w, (lo + 1)[..., None], (1 - frac)[..., None], axis=-1)
    np.put_along_axis(w, (lo + 2)[..., None], frac[..., None], axis=-1)
    return w


@dataclass(frozen=True)
class HaloTables:
    """Halo gather tables: ``dst`` (K,) flat halo indices, ``src`` (K, 16)
    flat interior sources, ``w`` (K, 16) cubic / quadratic-fit weights,
    ``w_lin`` (K, 16) monotone weights, ``rot`` (K, 16, 2, 2) source-to-
    destination vector rotations, ``nearest`` (K,) best single source."""

    dst: np.ndarray
    src: np.ndarray
    w: np.ndarray
    w_lin: np.ndarray
    rot: np.ndarray
    nearest: np.ndarray


class Grid:
    """Geometry of one cube-sphere resolution (N cells per face edge, halo
    H, nominal cell size in metres)."""

    SOURCES = 16

    def __init__(self, N: int, H: int = 4, cell_size_m: float = 50.0, R_planet: float | None = None):
        if N < 2 * H:
            raise ValueError("N must be at least 2H")
        self.N = int(N)
        self.H = int(H)
        self.NE = self.N + 2 * self.H
        self.cell_size_m = float(cell_size_m)
        self.R_planet = float(R_planet) if R_planet is not None else planet_radius(N, cell_size_m)

    # -- coordinates ----------------------------------------------------------
    def cell_uv(self, ei, ej):
        return (np.asarray(ei) - self.H + 0.5) / self.N, (np.asarray(ej) - self.H + 0.5) / self.N

    def flat_index(self, face, ei, ej):
        return (np.asarray(face) * self.NE + np.asarray(ei)) * self.NE + np.asarray(ej)

    def centers_of(self, face, ei, ej) -> np.ndarray:
        u, v = self.cell_uv(ei, ej)
        return face_point(np.broadcast_to(np.asarray(face), np.shape(u)), u, v)

    # -- metric ---------------------------------------------------------------
    @cached_property
    def metric_face(self) -> np.ndarray:
        """(NE, NE, 3) float32 metric (g_ii, g_ij, g_jj) in cell units; the
        same on every face."""
        e = np.arange(self.NE)
        U, V = np.meshgrid((e - self.H + 0.5) / self.N, (e - self.H + 0.5) / self.N, indexing="ij")
        ju, jv = tangents(np.zeros(U.shape, dtype=np.int64), U, V)
        g = np.stack([np.sum(ju * ju, -1), np.sum(ju * jv, -1), np.sum(jv * jv, -1)], axis=-1)
        k = (self.R_planet / (self.N * self.cell_size_m)) ** 2
        return (g * k).astype(np.float32)

    @cached_property
    def metric_inv_face(self) -> np.ndarray:
        g = self.metric_face.astype(np.float64)
        det = g[..., 0] * g[..., 2] - g[..., 1] ** 2
        inv = np.stack([g[..., 2] / det, -g[..., 1] / det, g[..., 0] / det], axis=-1)
        return inv.astype(np.float32)

    @property
    def metric(self) -> np.ndarray:
        """(6, NE, NE, 3) broadcast view of :attr:`metric_face`."""
        return np.broadcast_to(self.metric_face, (6,) + self.metric_face.shape)

    @property
    def metric_inv(self) -> np.ndarray:
        return np.broadcast_to(self.metric_inv_face, (6,) + self.metric_inv_face.shape)

    # -- halo -----------------------------------------------------------------
    @cached_property
    def _edge_corner(self):
        H, N, NE = self.H, self.N, self.NE
        halo = np.ones((NE, NE), dtype=bool)
        halo[H:H + N, H:H + N] = False
        corner = np.zeros((NE, NE), dtype=bool)
        corner[:H, :H] = corner[:H, NE - H:] = corner[NE - H:, :H] = corner[NE - H:, NE - H:] = True
        return halo & ~corner, corner

    @cached_property
    def halo(self) -> HaloTables:
        N, H, S = self.N, self.H, self.SOURCES
        edge, corner = self._edge_corner
        parts = [self._edge_rows(f, *np.nonzero(edge)) for f in range(6)]
        ci, cj = np.nonzero(corner)
        tree, cand = self._corner_candidates()
        parts += [self._corner_rows(f, ci, cj, tree, cand) for f in range(6)]
        return HaloTables(*(np.concatenate([p[k] for p in parts]) for k in range(6)))

    def _edge_rows(self, f, ei, ej):
        N, H, S = self.N, self.H, self.SOURCES
        K = ei.size
        u, v = self.cell_uv(ei, ej)
        faces = np.full(K, f)
        sf, su, sv = point_face(face_point(faces, u, v))
        fi = su * N - 0.5 + H
        fj = sv * N - 0.5 + H
        i0 = np.clip(np.floor(fi).astype(np.int64), H + 1, H + N - 3)
        j0 = np.clip(np.floor(fj).astype(np.int64), H + 1, H + N - 3)
        ti, tj = fi - i0, fj - j0
        offs = np.arange(-1, 3)
        src = self.flat_index(sf[:, None, None], (i0[:, None] + offs)[:, :, None], (j0[:, None] + offs)[:, None, :]).reshape(K, S)
        w = (cubic_weights(ti)[:, :, None] * cubic_weights(tj)[:, None, :]).reshape(K, S)
        wl = (linear_weights(ti)[:, :, None] * linear_weights(tj)[:, None, :]).reshape(K, S)
        near = src[np.arange(K), np.argmax(wl, axis=1)]
        e1 = reexpress(sf, su, sv, np.tile([[1.0, 0.0]], (K, 1)), faces, u, v)
        e2 = reexpress(sf, su, sv, np.tile([[0.0, 1.0]], (K, 1)), faces, u, v)
        R = np.stack([e1, e2], axis=-1)  # columns: images of the source unit vectors
        rot = np.broadcast_to(R[:, None], (K, S, 2, 2)).copy()
        return self.flat_index(f, ei, ej), src, w, wl, rot, near

    def _corner_candidates(self):
        """Interior cells within H + 3 cells of any face corner and a k-d tree
        over their centres (the pool corner halo cells fit over)."""
        from scipy.spatial import cKDTree

        N, H = self.N, self.H
        M = H + 3
        cf, ci, cj = [], [], []
        for f in range(6):
            for a0, b0 in ((H, H), (H, H + N - M), (H + N - M, H), (H + N - M, H + N - M)):
                ii, jj = np.meshgrid(np.arange(a0, a0 + M), np.arange(b0, b0 + M), indexing="ij")
                cf.append(np.full(ii.size, f))
                ci.append(ii.ravel())
                cj.append(jj.ravel())
        cf, ci, cj = np.concatenate(cf), np.concatenate(ci), np.concatenate(cj)
        pos = self.centers_of(cf, ci, cj)
        cu, cv = self.cell_uv(ci, cj)
        return cKDTree(pos), (cf, ci, cj, pos, cu, cv, self.flat_index(cf, ci, cj))

    def _corner_rows(self, f, ci, cj, tree, cand):
        S = self.SOURCES
        cf_, _ci, _cj, cpos, cu_, cv_, cflat = cand
        K = ci.size
        u, v = self.cell_uv(ci, cj)
        faces = np.full(K, f)
        p = face_point(faces, u, v)
        _, idx = tree.query(p, k=S)
        src = cflat[idx]
        near = cflat[idx[:, 0]]
        ax = np.where(np.abs(p[:, :1]) < 0.9, np.array([[1.0, 0.0, 0.0]]), np.array([[0.0, 1.0, 0.0]]))
        e1 = ax - p * np.sum(ax * p, axis=1, keepdims=True)
        e1 /= np.linalg.norm(e1, axis=1, keepdims=True)
        e2 = np.cross(p, e1)
        q = cpos[idx]
        wl = np.zeros((K, S))
        d = np.linalg.norm(q[:, :4] - p[:, None, :], axis=2)
        inv = 1.0 / (d * d)
        wl[:, :4] = inv / inv.sum(axis=1, keepdims=True)
        dq = q / np.sum(q * p[:, None, :], axis=2, keepdims=True) - p[:, None, :]
        x = np.sum(dq * e1[:, None, :], axis=2)
        y = np.sum(dq * e2[:, None, :], axis=2)
        A = np.stack([np.ones_like(x), x, y, x * x, x * y, y * y], axis=2)
        w = np.linalg.pinv(A)[:, 0, :]
        ff = np.repeat(faces[:, None], S, axis=1)
        uu = np.repeat(u[:, None], S, axis=1)
        vv = np.repeat(v[:, None], S, axis=1)
        r1 = reexpress(cf_[idx], cu_[idx], cv_[idx], np.broadcast_to([1.0, 0.0], (K, S, 2)), ff, uu, vv)
        r2 = reexpress(cf_[idx], cu_[idx], cv_[idx], np.broadcast_to([0.0, 1.0], (K, S, 2)), ff, uu, vv)
        rot = np.stack([r1, r2], axis=-1)
        return self.flat_index(f, ci, cj), src, w, wl, rot, near

    @cached_property
    def owner(self) -> np.ndarray:
        """(6, NE, NE) int64: flat index of the interior cell owning each cell."""
        own = np.arange(6 * self.NE * self.NE, dtype=np.int64)
        hm = self.halo
        own[hm.dst] = hm.nearest
        return own.reshape(6, self.NE, self.NE)

    def latitude(self) -> np.ndarray:
        """(6, NE, NE) latitude in radians (+Z is the pole)."""
        e = np.arange(self.NE)
        EI, EJ = np.meshgrid(e, e, indexing="ij")
        out = np.empty((6, self.NE, self.NE))
        for f in range(6):
            out[f] = np.arcsin(np.clip(self.centers_of(f, EI, EJ)[..., 2], -1.0, 1.0))
        return out

    def centers(self) -> np.ndarray:
        """(6, NE, NE, 3) float64 cell centres (materialised on request only)."""
        e = np.arange(self.NE)
        EI, EJ = np.meshgrid(e, e, indexing="ij")
        return np.stack([self.centers_of(f, EI, EJ) for f in range(6)])


_GRIDS: dict = {}


def get_grid(N: int, H: int = 4, cell_size_m: float = 50.0) -> Grid:
    key = (int(N), int(H), float(cell_size_m))
    g = _GRIDS.get(key)
    if g is None:
        g = _GRIDS[key] = Grid(N, H, cell_size_m)
    return g


def exchange_halos(grid: Grid, arr: np.ndarray, vector: bool = False, linear: bool = False) -> np.ndarray:
    """Fill the halo cells of a (6, NE, NE[, 2]) array in place from the
    interior (bake/globe/field.py:104-125): scalars as the weighted sum of
    their 16 sources, vectors rotated into the destination face first."""
    hm = grid.halo
    flat = arr.reshape(6 * grid.NE * grid.NE, -1)
    w = (hm.w_lin if linear else hm.w).astype(flat.dtype)
    srcv = flat[hm.src]  # (K, 16, C)
    if vector:
        rot = hm.rot.astype(flat.dtype)
        g = np.einsum("ks,ksab,ksb->ka", w, rot, srcv)
    else:
        g = np.einsum("ks,ksc->kc", w, srcv)
    flat[hm.dst] = g
    return arr
