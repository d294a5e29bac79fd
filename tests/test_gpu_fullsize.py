"""CUDA path against mhs's own outputs at the workloads' full sizes (FP64).

* config 1 in full: 600 observers x 100 triangles, disp and stress;
* config 2 (2,400-triangle rough surface-reaching fault, per-triangle eps,
  fold on): 8 fold-band receiver rows and 8 other rows of the full 3x3
  interaction matrix;
* config 4 (3-fault network, ~6,000 triangles, continuous P2, source =
  (strike, dip)): 4 fold-band rows and 4 other rows.

The fixtures were written by tests/golden/make_golden.py from mhs itself.
Tolerance: relmax <= 1e-12 (max|a - b| / max|b| over the compared rows --
a smaller denominator than the whole matrix's maximum, so a stricter test)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, relmax

pytestmark = pytest.mark.gpu
TOL = 1e-12


def test_config1_full_disp_and_stress(cuda):
    import mhs_b200 as m
    d = golden("c1_full")
    mat = m.Material(float(d["mu"]), float(d["lam"]))
    e = float(d["eps"])
    assert relmax(m.disp_matrix(d["obs"], d["tris"], mat, e), d["disp"]) < TOL
    assert relmax(m.stress_matrix(d["obs"], d["tris"], mat, e), d["stress"]) < TOL


def _rows_of(fn, rows):
    return np.stack([fn((int(r), int(r) + 1))[0] for r in rows])


@pytest.mark.parametrize("part", ["band", "other"])
def test_config2_rows(cuda, part):
    import mhs_b200 as m
    d = golden("c2_rows")
    mat = m.Material(float(d["mu"]), float(d["lam"]))
    nb = int(d["n_band"])
    sel = slice(0, nb) if part == "band" else slice(nb, None)
    rows, ref = d["rows"][sel], d["K"][sel]
    got = _rows_of(lambda r: m.interaction_matrix(d["tris"], mat, d["eps"], rows=r), rows)
    assert relmax(got, ref) < TOL


def test_config2_rows_from_the_whole_matrix(cuda):
    """The same rows read out of one full-matrix assembly (no rows=)."""
    import torch
    import mhs_b200 as m
    d = golden("c2_rows")
    mat = m.Material(float(d["mu"]), float(d["lam"]))
    K = m.interaction_matrix(torch.as_tensor(d["tris"], device=cuda), mat,
                             torch.as_tensor(d["eps"], device=cuda))
    got = K[torch.as_tensor(d["rows"], device=cuda)].cpu().numpy()
    assert relmax(got, d["K"]) < TOL


@pytest.mark.parametrize("part", ["band", "other"])
def test_config4_continuous_p2_rows(cuda, part):
    import mhs_b200 as m
    d = golden("c4_rows")
    mat = m.Material(float(d["mu"]), float(d["lam"]))
    sn = m.shared_nodes(d["tris"], groups=d["groups"])
    assert sn.n == int(d["n_cols"])
    nb = int(d["n_band"])
    sel = slice(0, nb) if part == "band" else slice(nb, None)
    rows, ref = d["rows"][sel], d["K"][sel]
    got = _rows_of(lambda r: m.interaction_matrix(d["tris"], mat, float(d["eps"]), order=2,
                                                  layout="continuous", shared=sn,
                                                  source=("strike", "dip"), rows=r), rows)
    assert relmax(got, ref) < TOL
