"""CUDA path against mhs's own outputs (golden fixtures), FP64.

Tolerance: relmax <= 1e-12 (norm-wise, max|a-b| / max|b|), the parity bar
for the all-float64 form."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, relmax

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _mat(d):
    import mhs_b200 as m
    return m.Material(float(d["mu"]), float(d["lam"]))


def test_c1_subset_disp_stress(cuda):
    import mhs_b200 as m
    d = golden("c1_subset")
    mat = _mat(d)
    assert relmax(m.disp_matrix(d["obs"], d["tris"], mat, float(d["eps"])), d["disp"]) < TOL
    assert relmax(m.stress_matrix(d["obs"], d["tris"], mat, float(d["eps"])), d["stress"]) < TOL
    assert relmax(m.total_stress_matrix(d["obs"], d["tris"], mat, float(d["eps"])),
                  d["total_stress"]) < TOL


@pytest.mark.parametrize("p", [0, 1, 2])
def test_orders(cuda, p):
    import mhs_b200 as m
    d = golden("orders")
    mat = _mat(d)
    e = float(d["eps"])
    assert relmax(m.disp_matrix(d["obs"], d["tris"], mat, e, order=p), d[f"disp_p{p}"]) < TOL
    assert relmax(m.stress_matrix(d["obs"], d["tris"], mat, e, order=p), d[f"stress_p{p}"]) < TOL
    assert relmax(m.total_stress_matrix(d["obs"], d["tris"], mat, e, order=p), d[f"total_p{p}"]) < TOL
    assert relmax(m.traction_matrix(d["obs"], d["normals"], d["tris"], mat, e, order=p),
                  d[f"traction_p{p}"]) < TOL


@pytest.mark.parametrize("p", [0, 1])
def test_eps_per_triangle(cuda, p):
    import mhs_b200 as m
    d = golden("eps_per_tri")
    mat = _mat(d)
    assert relmax(m.disp_matrix(d["obs"], d["tris"], mat, d["eps"], order=p), d[f"disp_p{p}"]) < TOL
    assert relmax(m.stress_matrix(d["obs"], d["tris"], mat, d["eps"], order=p), d[f"stress_p{p}"]) < TOL


def test_interaction(cuda):
    import mhs_b200 as m
    d = golden("interaction")
    mat = _mat(d)
    e = float(d["eps"])
    assert relmax(m.interaction_matrix(d["tris"], mat, e), d["int_p0"]) < TOL
    assert relmax(m.interaction_matrix(d["tris"], mat, e, order=1, receiver=("strike", "dip")),
                  d["int_p1"]) < TOL
    assert relmax(m.interaction_matrix(d["tris"], mat, e, order=2, receiver="strike",
                                       source="strike"), d["int_p2"]) < TOL
    assert relmax(m.interaction_matrix(d["tris"], mat, e, rows=(5, 17)), d["int_p0_rows"]) < TOL
    assert relmax(m.interaction_matrix(d["tris"], mat, e, subtract_eigenstress=False),
                  d["int_p0_noeig"]) < TOL


def test_fold(cuda):
    import mhs_b200 as m
    d = golden("fold")
    mat = _mat(d)
    e = float(d["eps"])
    assert relmax(m.interaction_matrix(d["tris"], mat, e), d["int_p0"]) < TOL
    assert relmax(m.stress_matrix(d["obs"], d["tris"], mat, e), d["stress_p0"]) < TOL
    assert relmax(m.stress_matrix(d["obs"], d["tris"], mat, e, fold=False),
                  d["stress_p0_nofold"]) < TOL
    assert relmax(m.disp_matrix(d["obs"], d["tris"], mat, e), d["disp_p0"]) < TOL
    assert relmax(m.interaction_matrix(d["tris"], mat, e, order=1, receiver=("strike",),
                                       source=("strike", "dip")), d["int_p1"]) < TOL


def test_continuous(cuda):
    import mhs_b200 as m
    d = golden("continuous")
    mat = _mat(d)
    sn = m.shared_nodes(d["tris"], groups=d["groups"])
    assert np.array_equal(sn.ids, d["ids"])
    K = m.interaction_matrix(d["tris"], mat, float(d["eps"]), order=2, layout="continuous",
                             shared=sn, source=("strike", "dip"))
    assert relmax(K, d["int_cont"]) < TOL
    T = m.traction_matrix(d["obs"], d["obs_normals"], d["tris"], mat, float(d["eps"]), order=2,
                          layout="continuous", shared=sn)
    assert relmax(T, d["trac_cont"]) < TOL


def test_rough_surface(cuda):
    import mhs_b200 as m
    d = golden("rough_surface")
    mat = _mat(d)
    assert relmax(m.interaction_matrix(d["tris"], mat, d["eps"]), d["int_p0"]) < TOL
