"""Output sizes of the matrix forms, and the refusal that states them.

Every output is (observer rows) x (source dof columns) x (a fixed block of
entries per pair), and every layout puts the observer axis first, so any run
of observer rows is one contiguous slab of the matrix.  A single helper,
``_slabs``, turns (rows, bytes per row, budget) into a slab size and count;
the public names below are the ones mhs exposes for the same arithmetic
(mhs/chunking.py:23-142: the per-pair table, ``pair_bytes``, the ceiling,
``chunk_plan`` and the ``MemoryError`` whose text spells the numbers out),
and ``stream_rows`` sizes the device staging slab of a host ``out=``."""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np

from . import defaults

# Entries per (observer, source dof) pair for each named readout; slip is the
# last axis of each.  interaction_matrix passes its own (n_a, n_b) instead.
PAIR_SHAPE = {
    "disp": (3, 3),
    "traction": (3, 3),
    "stress": (3, 3, 3),
    "strain": (3, 3, 3),
    "eigenstress": (3, 3, 3),
}


def pair_shape(kind) -> tuple:
    """Trailing shape of one pair: a readout name or an explicit tuple."""
    if isinstance(kind, tuple):
        return kind
    try:
        return PAIR_SHAPE[kind]
    except KeyError:
        raise KeyError(f"unknown output kind {kind!r}; expected one of {sorted(PAIR_SHAPE)}") \
            from None


def pair_bytes(kind, dtype=np.float64, parts: bool = False) -> int:
    """Bytes one pair costs; ``parts=True`` returns two arrays, so twice."""
    return (2 if parts else 1) * math.prod(pair_shape(kind)) * np.dtype(dtype).itemsize


def default_ceiling() -> int:
    """``defaults.MATRIX_MAX_BYTES``, no more than ``MATRIX_RAM_FRACTION`` of
    the host's RAM when that is known."""
    cap = int(defaults.MATRIX_MAX_BYTES)
    try:
        ram = os.sysconf("SC_PHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except (ValueError, OSError, AttributeError):
        return cap
    return min(cap, int(defaults.MATRIX_RAM_FRACTION * ram))


def _slabs(n_rows: int, row_bytes: int, budget: int) -> tuple[int, int]:
    """(rows per slab, number of slabs): as many whole rows as the budget
    holds, at least one, at most all of them."""
    rows = min(max(1, budget // max(row_bytes, 1)), max(n_rows, 1))
    return rows, (n_rows + rows - 1) // rows if n_rows else 0


@dataclass(frozen=True)
class ChunkPlan:
    """The cost of an observer-sliced assembly; computing it allocates nothing."""

    n_obs: int
    n_src: int
    bytes_total: int
    bytes_per_chunk: int
    obs_per_chunk: int
    n_chunks: int


def chunk_plan(n_obs: int, n_src: int, kind="stress", dtype=np.float64, parts: bool = False,
               ceiling: int | None = None) -> ChunkPlan:
    """Slabs of observer rows that each fit under ``ceiling``."""
    n_obs, n_src = int(n_obs), int(n_src)
    if min(n_obs, n_src) < 0:
        raise ValueError(f"negative sizes: n_obs={n_obs}, n_src={n_src}")
    row = pair_bytes(kind, dtype, parts) * max(n_src, 1)
    rows, n = _slabs(n_obs, row, default_ceiling() if ceiling is None else int(ceiling))
    return ChunkPlan(n_obs, n_src, row * n_obs, row * rows, rows, n)


def stream_rows(n_rows: int, row_bytes: int, free_device_bytes: int, cap_bytes: int) -> int:
    """Rows of the device staging slab that streams a host ``out=``: within
    ``cap_bytes`` and a quarter of the device's free memory."""
    return _slabs(n_rows, row_bytes, min(int(cap_bytes), int(free_device_bytes) // 4))[0]


def _gib(n: int) -> str:
    return f"{n / 2**30:.2f} GiB"


def refuse_if_too_large(n_obs: int, n_src: int, kind, dtype=np.float64, parts: bool = False,
                        ceiling: int | None = None) -> None:
    """MemoryError, with the arithmetic, when the output would pass the ceiling."""
    cap = default_ceiling() if ceiling is None else int(ceiling)
    plan = chunk_plan(n_obs, n_src, kind, dtype, parts, ceiling=cap)
    if plan.bytes_total <= cap:
        return
    label = kind if isinstance(kind, str) else f"interaction{pair_shape(kind)}"
    two = " (parts=True returns two arrays)" if parts else ""
    raise MemoryError(
        f"{label} matrix for {n_obs} obs x {n_src} sources would allocate "
        f"{_gib(plan.bytes_total)}{two}, over the {_gib(cap)} ceiling.\n"
        f"  per obs/source pair: {pair_bytes(kind, dtype, parts)} B ({np.dtype(dtype).name})\n"
        f"  largest n_obs that fits at n_src={n_src}: {plan.obs_per_chunk}\n"
        f"  so this is {plan.n_chunks} chunks of {_gib(plan.bytes_per_chunk)}\n"
        f"Escapes: pass out= (a preallocated numpy array or memmap, which is filled in "
        f"observer-row slabs and may be larger than the device; or a float32 buffer to halve "
        f"it), or slice the inputs -- chunking.chunk_plan() reports this arithmetic without "
        f"allocating. The ceiling itself is defaults.MATRIX_MAX_BYTES.")
