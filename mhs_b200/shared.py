"""The shared-node table of a continuous quadratic slip: the column axis of
``layout="continuous"`` matrices, built on the host.

The columns must mean the same nodes as mhs's (mhs/shared.py:80-273), so
the numbering follows its rules: vertices are welded by rounding their
coordinates to ``tol_over_h`` x the shortest edge, with the group id as a
fourth key (faults of a network that meet along a line keep separate nodes
there); welded vertices are numbered in lexicographic order of those keys,
then come the edge midpoints in lexicographic order of their sorted vertex
pairs.  Element ``s`` names its nodes ``ids[s]`` in the kernels' order
``v1 v2 v3 m12 m23 m31``.  Tilings that cannot carry one slip per node are
refused with mhs's messages: a collapsed triangle, an edge on three or more
triangles, a soup with no shared edge, and neighbours wound opposite ways.

Both numberings come from one helper, ``_rank_rows``: a lexicographic sort
of integer key rows and a dense rank per distinct row.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import defaults, tdcs

#: The one order the continuous layout exists for.
CONTINUOUS_ORDER = 2
LAYOUTS = ("discontinuous", "continuous")
_LOCAL_EDGES = ((0, 1), (1, 2), (2, 0))   # m12, m23, m31


@dataclasses.dataclass(frozen=True)
class SharedNodes:
    """Nodes of a continuous P2 slip on one triangulated surface.

    ``coords`` (n, 3): the welded vertices, then the edge midpoints;
    ``ids`` (n_tri, 6): each element's nodes; ``normals`` (n, 3): unit,
    upward, the area-weighted mean of the adjoining elements' normals;
    ``boundary`` (n,): nodes on edges that belong to one triangle only;
    ``weights`` (n,): the exact quadrature of a quadratic field (area / 3 at
    each edge midpoint, zero at the vertices); ``group`` (n,): the group a
    node was welded in; ``n_vertices``; ``tol``: the weld tolerance."""

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
        """Number of nodes (vertices + edges)."""
        return len(self.coords)

    @property
    def n_tri(self) -> int:
        return len(self.ids)

    @property
    def n_edges(self) -> int:
        return self.n - self.n_vertices

    @property
    def frames(self) -> np.ndarray:
        """``(n, 3, 3)`` cutde frames (rows strike, dip, tensile) on the node
        normals (mhs.tdcs)."""
        return tdcs.frame_from_normals(self.normals)

    @property
    def trace(self) -> np.ndarray:
        """Boundary nodes that lie on the free surface z = 0 (within tol)."""
        return self.boundary & (self.coords[:, 2] >= -self.tol)

    @property
    def front(self) -> np.ndarray:
        """Boundary nodes below the surface: crack fronts and rooted edges."""
        return self.boundary & ~self.trace

    def _nodal(self, values, dtype=None) -> np.ndarray:
        v = np.asarray(values, dtype=dtype)
        if len(v) != self.n:
            raise ValueError(f"expected {self.n} nodal values, got {v.shape[0]}")
        return v

    def expand(self, values) -> np.ndarray:
        """Nodal values (n, ...) as the element-major source axis of the
        discontinuous layout (n_tri * 6, ...), node index fastest."""
        v = self._nodal(values)
        return v[self.ids.ravel()]

    def integrate(self, values) -> np.ndarray:
        """Integral of a quadratic nodal field over the whole surface."""
        return np.tensordot(self.weights, self._nodal(values, float), axes=(0, 0))

    def element_mean(self, values) -> np.ndarray:
        """Mean of a nodal field over each element (its three midpoints)."""
        return np.asarray(values, float)[self.ids[:, 3:]].mean(axis=1)


def _rank_rows(keys: np.ndarray):
    """Dense lexicographic rank of each row of an integer matrix, the number
    of rows sharing each rank, and one representative row per rank (in rank
    order)."""
    order = np.lexsort(keys.T[::-1])
    ranked = keys[order]
    starts = np.ones(len(ranked), dtype=bool)
    starts[1:] = np.any(ranked[1:] != ranked[:-1], axis=1)
    rank = np.empty(len(keys), dtype=np.int64)
    rank[order] = np.cumsum(starts) - 1
    return rank, np.bincount(rank), ranked[starts]


def _sum_by(index: np.ndarray, values: np.ndarray, n: int) -> np.ndarray:
    """Per-index sums of the rows of `values` (added in row order)."""
    values = values.reshape(len(index), -1)
    return np.stack([np.bincount(index, weights=values[:, c], minlength=n)
                     for c in range(values.shape[1])], axis=1)


def shared_nodes(tris, *, groups=None, tol_over_h: float = defaults.WELD_TOL_OVER_H) -> SharedNodes:
    """The :class:`SharedNodes` of ``tris`` (n_tri, 3, 3); ``groups``
    (n_tri,) keeps the nodes of different groups (faults) apart."""
    t = np.ascontiguousarray(np.asarray(tris, dtype=np.float64))
    if t.ndim != 3 or t.shape[1:] != (3, 3) or t.shape[0] == 0:
        raise ValueError(f"tris must have shape (n_tri, 3, 3), got {t.shape}")
    if not np.isfinite(t).all():
        raise ValueError("tris must be finite")
    n_tri = len(t)
    grp = np.zeros(n_tri, np.int64) if groups is None else \
        np.asarray(groups).reshape(-1).astype(np.int64)
    if len(grp) != n_tri:
        raise ValueError(f"groups has {grp.shape[0]} entries for {n_tri} triangles")
    h_min = float(np.linalg.norm(t - np.roll(t, 1, axis=1), axis=2).min())
    if not h_min > 0.0:
        raise ValueError("a triangle has a zero-length edge")
    tol = float(tol_over_h) * h_min

    # vertices: weld keys (rounded coordinates, group), ranked
    corners = t.reshape(-1, 3)
    keys = np.column_stack([np.round(corners / tol).astype(np.int64), np.repeat(grp, 3)])
    vid, mult, _ = _rank_rows(keys)
    n_v = len(mult)
    verts = _sum_by(vid, corners, n_v) / mult[:, None]
    tv = vid.reshape(n_tri, 3)
    if any(np.any(tv[:, a] == tv[:, b]) for a, b in _LOCAL_EDGES):
        raise ValueError(f"a triangle has two vertices within the weld tolerance {tol:.3e}: "
                         f"degenerate, or tol_over_h too loose for this mesh")

    # edges: each element's 12, 23, 31 as sorted vertex pairs, ranked
    walked = np.stack([tv[:, [a, b]] for a, b in _LOCAL_EDGES], axis=1).reshape(-1, 2)
    eid, used, edges = _rank_rows(np.sort(walked, axis=1))
    if used.max() > 2:
        bad = int(np.argmax(used))
        raise ValueError(f"non-manifold: edge {edges[bad].tolist()} is shared by "
                         f"{int(used[bad])} triangles, so a node on it has no single "
                         f"tangent plane. The continuous layout needs a manifold tiling.")
    if n_tri > 1 and not (used == 2).any():
        raise ValueError(f"nothing is shared: {n_tri} triangles and no common edge. A soup "
                         f"of separate elements wants the discontinuous layout; the "
                         f"continuous one welds vertices at {tol:.3e} (tol_over_h "
                         f"{tol_over_h:g} x the shortest edge {h_min:.3e}).")
    # an interior edge is walked once in each direction by its two triangles
    ascending = np.bincount(eid, weights=walked[:, 0] < walked[:, 1], minlength=len(edges))
    flipped = (used == 2) & (ascending != 1)
    if flipped.any():
        bad = int(np.argmax(flipped))
        raise ValueError(f"inconsistent winding: the two triangles on edge {edges[bad].tolist()} "
                         f"traverse it the same way, so their vertex-order normals disagree "
                         f"and one Cartesian slip at a shared node would mean opposite jumps "
                         f"on the two sides. Wind the mesh consistently (every normal up is "
                         f"the usual choice).")

    n = n_v + len(edges)
    ids = np.hstack([tv, n_v + eid.reshape(n_tri, 3)])
    coords = np.vstack([verts, 0.5 * (verts[edges[:, 0]] + verts[edges[:, 1]])])
    rim = used == 1
    boundary = np.zeros(n, dtype=bool)
    boundary[edges[rim].ravel()] = True
    boundary[n_v + np.flatnonzero(rim)] = True
    area = 0.5 * np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), axis=1)
    nsum = _sum_by(ids.ravel(), np.repeat(area[:, None] * tdcs.unit_normals(t), 6, axis=0), n)
    normals = nsum / np.linalg.norm(nsum, axis=1, keepdims=True)
    weights = np.bincount(ids[:, 3:].ravel(), weights=np.repeat(area / 3.0, 3), minlength=n)
    group = np.zeros(n, dtype=np.int64)
    group[ids.ravel()] = np.repeat(grp, 6)
    return SharedNodes(coords=coords, ids=ids, normals=normals, boundary=boundary,
                       weights=weights, group=group, n_vertices=int(n_v), tol=tol)


def check_layout(layout: str) -> str:
    if layout not in LAYOUTS:
        raise ValueError(f"layout must be one of {LAYOUTS}, got {layout!r}")
    return layout
