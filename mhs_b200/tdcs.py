"""Per-triangle (strike, dip, tensile) frames in cutde's convention
(mhs/tdcs.py:49-140): tensile is the unit normal turned upward, strike is
``(-n_y, n_x, 0)`` normalised (``(1, 0, 0)`` for a horizontal element), dip
is ``tensile x strike`` and so points up-dip."""
from __future__ import annotations

import numpy as np

#: Order of the frame's rows and of the slip components that pair with them.
COMPONENTS = ("strike", "dip", "tensile")
#: In-plane normal length below which an element counts as horizontal.
FLAT_TOL = 1e-12


def unit_normals(tris) -> np.ndarray:
    """Upward unit normals ``(n, 3)`` from the vertices."""
    t = np.asarray(tris, float).reshape(-1, 3, 3)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    mag = np.linalg.norm(n, axis=1, keepdims=True)
    if not np.all(mag > 0.0):
        bad = int(np.argmin(mag))
        raise ValueError(
            f"tris[{bad}] is degenerate: its vertices are collinear, so it has "
            f"no normal and no frame. Zero-area triangles have to be removed "
            f"by the mesh, not absorbed here.")
    n = n / mag
    return np.where(n[:, 2:3] < 0.0, -n, n)


def frame_from_normals(normals) -> np.ndarray:
    """``(n, 3, 3)`` rows ``[strike, dip, tensile]`` on UPWARD unit normals."""
    n = np.asarray(normals, float).reshape(-1, 3)
    if np.any(n[:, 2] < 0.0):
        raise ValueError("frame_from_normals takes UPWARD normals (n_z >= 0); "
                         "use unit_normals for a mesh's")
    strike = np.stack([-n[:, 1], n[:, 0], np.zeros(len(n))], axis=1)
    mag = np.linalg.norm(strike, axis=1, keepdims=True)
    flat = mag[:, 0] <= FLAT_TOL
    strike = np.where(flat[:, None], np.array([1.0, 0.0, 0.0]),
                      strike / np.where(mag > 0.0, mag, 1.0))
    dip = np.cross(n, strike)
    return np.stack([strike, dip, n], axis=1)


def slip_frame(tris) -> np.ndarray:
    """``(n, 3, 3)`` with rows ``[strike, dip, tensile]`` in Cartesian xyz."""
    return frame_from_normals(unit_normals(tris))


def to_cartesian(tris, slip) -> np.ndarray:
    """(strike, dip, tensile) slip ``(n, 3)`` -> Cartesian ``(n, 3)``."""
    frame = slip_frame(tris)
    slip = np.asarray(slip, float).reshape(-1, 3)
    if slip.shape[0] != frame.shape[0]:
        raise ValueError(f"slip has {slip.shape[0]} rows for {frame.shape[0]} triangles")
    return np.einsum("sab,sa->sb", frame, slip)


def from_cartesian(tris, slip) -> np.ndarray:
    """Cartesian slip ``(n, 3)`` -> (strike, dip, tensile) ``(n, 3)``."""
    frame = slip_frame(tris)
    slip = np.asarray(slip, float).reshape(-1, 3)
    if slip.shape[0] != frame.shape[0]:
        raise ValueError(f"slip has {slip.shape[0]} rows for {frame.shape[0]} triangles")
    return np.einsum("sab,sb->sa", frame, slip)


def component_index(names, allowed=COMPONENTS) -> np.ndarray:
    """Frame row indices of component names; ``normal`` means ``tensile``."""
    if isinstance(names, str):
        names = (names,)
    out = []
    for nm in names:
        key = "tensile" if nm == "normal" else nm
        if key not in allowed:
            raise ValueError(f"unknown component {nm!r}; expected some of "
                             f"{list(allowed)} (or 'normal' for 'tensile')")
        out.append(allowed.index(key))
    if not out:
        raise ValueError("at least one component is required")
    return np.array(out, dtype=int)
