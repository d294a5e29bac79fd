"""Byte arithmetic of the matrix forms and the refusal that carries it
(mhs/chunking.py:23-142): bytes per (observer, source dof) pair, an
observer-sliced plan under a ceiling, and a MemoryError that states the
arithmetic.  Device-resident outputs are also held to a fraction of the
device's free memory."""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

from . import defaults

PAIR_SHAPE = {
    "disp": (3, 3),
    "stress": (3, 3, 3),
    "strain": (3, 3, 3),
    "eigenstress": (3, 3, 3),
    "traction": (3, 3),
}


def pair_shape(kind) -> tuple:
    if isinstance(kind, tuple):
        return kind
    if kind not in PAIR_SHAPE:
        raise KeyError(f"unknown output kind {kind!r}; expected one of {sorted(PAIR_SHAPE)}")
    return PAIR_SHAPE[kind]


def pair_bytes(kind, dtype=np.float64, parts: bool = False) -> int:
    n = int(np.prod(pair_shape(kind))) * np.dtype(dtype).itemsize
    return 2 * n if parts else n


def default_ceiling() -> int:
    """``MATRIX_MAX_BYTES``, capped at ``MATRIX_RAM_FRACTION`` of host RAM."""
    cap = int(defaults.MATRIX_MAX_BYTES)
    try:
        total = os.sysconf("SC_PHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError, AttributeError):
        return cap
    return min(cap, int(defaults.MATRIX_RAM_FRACTION * total))


@dataclass(frozen=True)
class ChunkPlan:
    n_obs: int
    n_src: int
    bytes_total: int
    bytes_per_chunk: int
    obs_per_chunk: int
    n_chunks: int


def chunk_plan(n_obs: int, n_src: int, kind="stress", dtype=np.float64, parts: bool = False,
               ceiling: int | None = None) -> ChunkPlan:
    n_obs, n_src = int(n_obs), int(n_src)
    if n_obs < 0 or n_src < 0:
        raise ValueError(f"negative sizes: n_obs={n_obs}, n_src={n_src}")
    per = pair_bytes(kind, dtype, parts)
    row = per * max(n_src, 1)
    total = row * n_obs
    cap = default_ceiling() if ceiling is None else int(ceiling)
    per_chunk = max(1, cap // max(row, 1))
    per_chunk = min(per_chunk, max(n_obs, 1))
    n_chunks = -(-n_obs // per_chunk) if n_obs else 0
    return ChunkPlan(n_obs=n_obs, n_src=n_src, bytes_total=total, bytes_per_chunk=row * per_chunk,
                     obs_per_chunk=per_chunk, n_chunks=n_chunks)


def _gib(n: int) -> str:
    return f"{n / 1024**3:.2f} GiB"


def refuse_if_too_large(n_obs: int, n_src: int, kind, dtype=np.float64, parts: bool = False,
                        ceiling: int | None = None) -> None:
    """Raise MemoryError with the arithmetic if the output exceeds the ceiling."""
    cap = default_ceiling() if ceiling is None else int(ceiling)
    plan = chunk_plan(n_obs, n_src, kind, dtype, parts, ceiling=cap)
    if plan.bytes_total <= cap:
        return
    label = kind if isinstance(kind, str) else f"interaction{pair_shape(kind)}"
    raise MemoryError(
        f"{label} matrix for {n_obs} obs x {n_src} sources would allocate "
        f"{_gib(plan.bytes_total)}{' (parts=True returns two arrays)' if parts else ''}, over the "
        f"{_gib(cap)} ceiling.\n"
        f"  per obs/source pair: {pair_bytes(kind, dtype, parts)} B ({np.dtype(dtype).name})\n"
        f"  largest n_obs that fits at n_src={n_src}: {plan.obs_per_chunk}\n"
        f"  so this is {plan.n_chunks} chunks of {_gib(plan.bytes_per_chunk)}\n"
        f"Escapes: pass out= (a preallocated array, or a float32 buffer to halve it), or "
        f"slice the inputs -- chunking.chunk_plan() reports this arithmetic without "
        f"allocating. The ceiling itself is defaults.MATRIX_MAX_BYTES.")
