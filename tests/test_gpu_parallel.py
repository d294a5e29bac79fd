"""Row-sharded interaction on one device: the blocks of every rank of a
world of 3, computed one after another, concatenate to the full matrix."""
from __future__ import annotations

import numpy as np
import pytest

from mhs_b200 import parallel, synthetic

pytestmark = pytest.mark.gpu


def test_row_blocks_concatenate_to_the_full_matrix(cuda):
    import mhs_b200 as m
    c = synthetic.config2(seed=4, nu=5, nv=3)
    mat = m.Material(c["mu"], c["lam"])
    full = m.interaction_matrix(c["tris"], mat, c["eps"], order=1)
    parts = [parallel.interaction_rows(c["tris"], mat, c["eps"], r, 3, order=1) for r in range(3)]
    assert parts[0][0] == 0 and parts[-1][1] == full.shape[0]
    assert np.array_equal(np.concatenate([p[2] for p in parts], axis=0), full)
