"""Shared-node table of a continuous quadratic slip (the ``layout="continuous"``
source axis), host-side geometry with mhs's numbering (mhs/shared.py:80-273).

Vertices are welded by rounding to ``WELD_TOL_OVER_H`` x the shortest edge,
within a group (a fault network passes its fault ids so faults meeting along
a line keep separate nodes there); the nodes are the welded vertices in
lexicographic key order, then one midpoint per unique edge in lexicographic
(sorted vertex pair) order.  Element ``s``'s nodes are ``ids[s]`` in the
kernels' order ``v1 v2 v3 m12 m23 m31``.  The numbering has to equal mhs's so
that a matrix's columns mean the same nodes in both libraries.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import defaults, tdcs

#: The one order the continuous layout exists for.
CONTINUOUS_ORDER = 2
LAYOUTS = ("discontinuous", "continuous")


@dataclasses.dataclass(frozen=True)
class SharedNodes:
    """Nodes of a continuous P2 slip: ``coords`` (n, 3) vertices then edge
    midpoints, ``ids`` (n_tri, 6), upward ``normals`` (n, 3), ``boundary``
    (rim nodes), ``weights`` (exact quadratic integration), ``group``."""

    coords: np.ndarray
    ids: np.ndarray
    normals: np.ndarray
    boundary: np.ndarray
    weights: np.ndarray
    group: np.ndarray
    n_vertices: int
    tol: float

    @property
    def n(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_tri(self) -> int:
        return int(self.ids.shape[0])

    @property
    def n_edges(self) -> int:
        return self.n - self.n_vertices

    @property
    def frames(self) -> np.ndarray:
        """``(n, 3, 3)`` [strike, dip, tensile] rows on each node normal."""
        return tdcs.frame_from_normals(self.normals)

    @property
    def trace(self) -> np.ndarray:
        """Boundary nodes on the free surface."""
        return self.boundary & (self.coords[:, 2] >= -self.tol)

    @property
    def front(self) -> np.ndarray:
        """Boundary nodes inside the body (crack fronts, rooted edges)."""
        return self.boundary & ~self.trace

    def expand(self, values) -> np.ndarray:
        """Nodal values (n, ...) -> element-major (n_tri * 6, ...)."""
        v = np.asarray(values)
        if v.shape[0] != self.n:
            raise ValueError(f"expected {self.n} nodal values, got {v.shape[0]}")
        return v[self.ids].reshape((self.n_tri * 6,) + v.shape[1:])

    def integrate(self, values) -> np.ndarray:
        """Exact integral of a quadratic nodal field over the surface."""
        v = np.asarray(values, float)
        if v.shape[0] != self.n:
            raise ValueError(f"expected {self.n} nodal values, got {v.shape[0]}")
        return np.tensordot(self.weights, v, axes=(0, 0))

    def element_mean(self, values) -> np.ndarray:
        """Per-element mean by the three-midpoint rule."""
        v = np.asarray(values, float)
        return v[self.ids[:, 3:]].mean(axis=1)


def shared_nodes(tris, *, groups=None, tol_over_h: float = defaults.WELD_TOL_OVER_H) -> SharedNodes:
    """Build the :class:`SharedNodes` of ``tris (n_tri, 3, 3)``; refuses
    non-manifold tilings, inconsistent winding and unconnected soups."""
    t = np.ascontiguousarray(np.asarray(tris, dtype=np.float64))
    if t.ndim != 3 or t.shape[1:] != (3, 3) or t.shape[0] == 0:
        raise ValueError(f"tris must have shape (n_tri, 3, 3), got {t.shape}")
    if not np.all(np.isfinite(t)):
        raise ValueError("tris must be finite")
    n_tri = t.shape[0]
    grp = (np.zeros(n_tri, dtype=np.int64) if groups is None
           else np.asarray(groups).reshape(-1).astype(np.int64))
    if grp.shape[0] != n_tri:
        raise ValueError(f"groups has {grp.shape[0]} entries for {n_tri} triangles")
    edge_len = np.linalg.norm(t - np.roll(t, 1, axis=1), axis=2)
    h_min = float(edge_len.min())
    if not h_min > 0.0:
        raise ValueError("a triangle has a zero-length edge")
    tol = float(tol_over_h) * h_min

    # --- weld: integer keys (rounded coordinates, group), unique in key order
    pts = t.reshape(-1, 3)
    keys = np.empty((pts.shape[0], 4), dtype=np.int64)
    keys[:, :3] = np.round(pts / tol).astype(np.int64)
    keys[:, 3] = np.repeat(grp, 3)
    _, vid = np.unique(keys, axis=0, return_inverse=True)
    vid = vid.reshape(-1)
    n_v = int(vid.max()) + 1
    cnt = np.bincount(vid, minlength=n_v).astype(float)
    verts = np.zeros((n_v, 3))
    np.add.at(verts, vid, pts)
    verts /= cnt[:, None]
    tv = vid.reshape(-1, 3)
    if np.any(tv[:, 0] == tv[:, 1]) or np.any(tv[:, 1] == tv[:, 2]) or np.any(tv[:, 2] == tv[:, 0]):
        raise ValueError(f"a triangle has two vertices within the weld tolerance {tol:.3e}: "
                         f"degenerate, or tol_over_h too loose for this mesh")

    # --- edges 12, 23, 31 of every element, unique in sorted-pair order
    loc = np.stack([tv[:, [0, 1]], tv[:, [1, 2]], tv[:, [2, 0]]], axis=1).reshape(-1, 2)
    pairs = np.sort(loc, axis=1)
    edges, eid, ecount = np.unique(pairs, axis=0, return_inverse=True, return_counts=True)
    eid = eid.reshape(-1)
    if np.any(ecount > 2):
        bad = int(np.argmax(ecount))
        raise ValueError(f"non-manifold: edge {edges[bad].tolist()} is shared by "
                         f"{int(ecount[bad])} triangles, so a node on it has no single "
                         f"tangent plane. The continuous layout needs a manifold tiling.")
    if n_tri > 1 and not np.any(ecount == 2):
        raise ValueError(f"nothing is shared: {n_tri} triangles and no common edge. A soup "
                         f"of separate elements wants the discontinuous layout; the "
                         f"continuous one welds vertices at {tol:.3e} (tol_over_h "
                         f"{tol_over_h:g} x the shortest edge {h_min:.3e}).")
    forward = (loc[:, 0] < loc[:, 1]).astype(float)
    n_fwd = np.bincount(eid, weights=forward, minlength=edges.shape[0])
    bad_wind = (ecount == 2) & (n_fwd != 1)
    if np.any(bad_wind):
        bad = int(np.argmax(bad_wind))
        raise ValueError(f"inconsistent winding: the two triangles on edge {edges[bad].tolist()} "
                         f"traverse it the same way, so their vertex-order normals disagree "
                         f"and one Cartesian slip at a shared node would mean opposite jumps "
                         f"on the two sides. Wind the mesh consistently (every normal up is "
                         f"the usual choice).")

    n_e = edges.shape[0]
    coords = np.concatenate([verts, 0.5 * (verts[edges[:, 0]] + verts[edges[:, 1]])])
    ids = np.concatenate([tv, n_v + eid.reshape(-1, 3)], axis=1)

    boundary = np.zeros(n_v + n_e, bool)
    rim = ecount == 1
    boundary[n_v + np.flatnonzero(rim)] = True
    boundary[edges[rim].reshape(-1)] = True

    up = tdcs.unit_normals(t)
    area = 0.5 * np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), axis=1)
    normals = np.zeros((n_v + n_e, 3))
    np.add.at(normals, ids.reshape(-1), np.repeat(area[:, None] * up, 6, axis=0))
    normals /= np.linalg.norm(normals, axis=1, keepdims=True)
    weights = np.zeros(n_v + n_e)
    np.add.at(weights, ids[:, 3:].reshape(-1), np.repeat(area / 3.0, 3))
    group = np.zeros(n_v + n_e, dtype=np.int64)
    group[ids.reshape(-1)] = np.repeat(grp, 6)
    return SharedNodes(coords=coords, ids=ids, normals=normals, boundary=boundary,
                       weights=weights, group=group, n_vertices=int(n_v), tol=tol)


def check_layout(layout: str) -> str:
    if layout not in LAYOUTS:
        raise ValueError(f"layout must be one of {LAYOUTS}, got {layout!r}")
    return layout
