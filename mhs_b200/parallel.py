"""Row sharding of one matrix across GPUs (one process per GPU).

Every (observer, source) pair is independent, so a matrix splits into
contiguous blocks of receiver rows with no exchange between the parts --
mhs's ``by_rows`` (mhs/parallel.py:267), the only legal cut for continuous
columns.  Rows are not equally expensive: a receiver inside a surface-reaching
source's fold band costs a polar-grid quadrature for that source (about
``FOLD_PAIR_COST`` ordinary pairs on a B200), so blocks are balanced by a
per-row cost estimate, not by count.

* ``row_costs(obs, tris, eps)`` -- estimated cost of each receiver row;
* ``row_blocks(costs, world)`` -- contiguous ``(lo, hi)`` per rank, balanced;
* ``interaction_rows(tris, material, eps, rank, world, **kw)`` -- this rank's
  block of ``interaction_matrix`` (rows of the collocation points);
* ``gather_rows(block, lo, hi, n_rows, group=None)`` -- the full matrix on
  every rank from the blocks (``torch.distributed`` all-gather; NCCL over
  NVLink between GPUs, gloo on the CPU), for callers that want it in one
  place.  The assembly itself needs no collective.
"""
from __future__ import annotations

import numpy as np

from . import defaults

#: Cost of one fold band pair in units of one ordinary pair (direct + image
#: terms), measured on the 2,400-triangle interaction workload on a B200:
#: fold 220 ms for 96,121 band pairs against 55 ms for 5.76 M pairs.
FOLD_PAIR_COST = 240.0


def _straddles(tris: np.ndarray, eps: np.ndarray) -> np.ndarray:
    depth = -tris[:, :, 2]
    return depth.min(axis=1) < defaults.FOLD_SOURCE_DEPTH_EPS * eps


def row_costs(obs: np.ndarray, tris: np.ndarray, eps) -> np.ndarray:
    """Estimated cost per receiver row: one unit per source, plus
    FOLD_PAIR_COST for each surface-reaching source whose fold band holds
    the receiver (depth and reach tests of the fold band)."""
    obs = np.asarray(obs, float).reshape(-1, 3)
    tris = np.asarray(tris, float).reshape(-1, 3, 3)
    eps = np.broadcast_to(np.asarray(eps, float), (tris.shape[0],))
    cost = np.full(obs.shape[0], float(tris.shape[0]))
    s = np.flatnonzero(_straddles(tris, eps))
    if s.size:
        e = eps[s]
        near_top = (-tris[s, :, 2]) < defaults.FOLD_SOURCE_DEPTH_EPS * e[:, None]
        top = (tris[s, :, :2] * near_top[:, :, None]).sum(axis=1) / near_top.sum(axis=1)[:, None]
        depth_ok = (-obs[:, 2])[:, None] < defaults.FOLD_BAND_DEPTH_EPS * e[None, :]
        reach = np.hypot(obs[:, None, 0] - top[None, :, 0], obs[:, None, 1] - top[None, :, 1])
        band = depth_ok & (reach < defaults.FOLD_REACH_EPS * e[None, :])
        cost += FOLD_PAIR_COST * band.sum(axis=1)
    return cost


def row_blocks(costs, world: int) -> list:
    """Contiguous (lo, hi) row blocks, one per rank, with nearly equal total
    cost (each cut at the row where the running cost crosses k / world of
    the total); every block is non-empty when there are at least `world`
    rows."""
    costs = np.asarray(costs, float)
    n = costs.size
    if world < 1:
        raise ValueError("world must be >= 1")
    if n < world:
        raise ValueError(f"{n} rows cannot be split across {world} ranks")
    cum = np.cumsum(costs)
    cuts = [0]
    for k in range(1, world):
        c = int(np.searchsorted(cum, cum[-1] * k / world, side="left")) + 1
        c = min(max(c, cuts[-1] + 1), n - (world - k))
        cuts.append(c)
    cuts.append(n)
    return [(cuts[i], cuts[i + 1]) for i in range(world)]


def interaction_rows(tris, material, eps, rank: int, world: int, **kw):
    """This rank's (lo, hi, block) of interaction_matrix(tris, ...): the
    receiver rows of a cost-balanced contiguous split.  Same keywords as
    interaction_matrix (except rows=)."""
    from .matrices import COLLOCATION_SHRINK, collocation_points, interaction_matrix, n_nodes
    if "rows" in kw:
        raise ValueError("interaction_rows chooses the rows itself")
    t = np.asarray(tris.cpu().numpy() if hasattr(tris, "cpu") else tris, float).reshape(-1, 3, 3)
    e = eps.cpu().numpy() if hasattr(eps, "cpu") else eps
    order = kw.get("order", 0)
    if kw.get("layout", "discontinuous") == "continuous":
        sn = kw.get("shared")
        if sn is None:
            from .shared import shared_nodes
            sn = shared_nodes(t)
            kw["shared"] = sn
        pts = sn.coords
    else:
        pts = collocation_points(t if kw.get("obs_tris") is None else kw["obs_tris"], order,
                                 kw.get("shrink", COLLOCATION_SHRINK))
    lo, hi = row_blocks(row_costs(pts, t, e), world)[rank]
    return lo, hi, interaction_matrix(tris, material, eps, rows=(lo, hi), **kw)


def gather_rows(block, lo: int, hi: int, n_rows: int, group=None):
    """Assemble the full matrix on every rank from per-rank row blocks
    (torch tensors of equal trailing shape), by a padded all-gather."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rows = torch.tensor([hi - lo], dtype=torch.int64, device=block.device)
    counts = [torch.zeros_like(rows) for _ in range(world)]
    dist.all_gather(counts, rows, group=group)
    counts = [int(c.item()) for c in counts]
    pad = max(counts)
    buf = torch.zeros((pad,) + tuple(block.shape[1:]), dtype=block.dtype, device=block.device)
    buf[: hi - lo] = block
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    full = torch.cat([p[:c] for p, c in zip(parts, counts)], dim=0)
    if full.shape[0] != n_rows:
        raise ValueError(f"blocks cover {full.shape[0]} rows, expected {n_rows}")
    return full
