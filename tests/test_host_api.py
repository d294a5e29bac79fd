"""Host-side semantics of the drop-in API (no GPU): validation refusals with
mhs's conditions, frames, the shared-node table, byte arithmetic, constants."""
from __future__ import annotations

import re

import numpy as np
import pytest

from conftest import ROOT, golden
import mhs_b200 as m
from mhs_b200 import chunking, defaults, tdcs
from oracle import mhs_oracle as O

TRI = np.array([[[0.0, 0.0, -1.0], [1.0, 0.0, -1.0], [0.0, 1.0, -1.5]]])
OBS = np.array([[0.2, 0.3, -0.5]])
MAT = m.Material(30.0, 30.0)


def test_material_rules():
    with pytest.raises(ValueError):
        m.Material(0.0, 1.0)
    with pytest.raises(ValueError):
        m.Material(1.0, -1.0)
    assert m.Material.from_mu_nu(1.0, 0.25).lam == pytest.approx(1.0)
    with pytest.raises(ValueError):
        m.Material.from_mu_nu(1.0, 0.5)


@pytest.mark.parametrize("bad,exc,msg", [
    (dict(material=(30, 30)), TypeError, "Material"),
    (dict(obs=np.zeros((2, 2))), ValueError, "n_obs, 3"),
    (dict(tris=np.zeros((1, 3))), ValueError, "n_src, 3, 3"),
    (dict(obs=np.zeros((0, 3))), ValueError, "nothing to assemble"),
    (dict(obs=np.array([[0, 0, 0.1]])), ValueError, "z <= 0"),
    (dict(tris=TRI * np.array([1, 1, -1])), ValueError, "half space is z <= 0"),
    (dict(eps=0.0), ValueError, "strictly positive"),
    (dict(obs=np.array([[np.nan, 0, -1]])), ValueError, "finite"),
])
def test_coerce_refusals(bad, exc, msg):
    kw = dict(obs=OBS, tris=TRI, material=MAT, eps=0.1)
    kw.update(bad)
    with pytest.raises(exc, match=msg):
        m.disp_matrix(kw["obs"], kw["tris"], kw["material"], kw["eps"])


def test_order_layout_refusals():
    with pytest.raises(ValueError, match="order must be 0, 1 or 2"):
        m.disp_matrix(OBS, TRI, MAT, 0.1, order=3)
    with pytest.raises(ValueError, match="layout must be one of"):
        m.disp_matrix(OBS, TRI, MAT, 0.1, layout="bogus")
    with pytest.raises(ValueError, match="quadratic only"):
        m.disp_matrix(OBS, TRI, MAT, 0.1, layout="continuous", order=1)
    with pytest.raises(ValueError, match="names no plane"):
        m.traction_matrix(OBS, [0.0, 0.0, 0.0], TRI, MAT, 0.1)
    with pytest.raises(ValueError, match="rows="):
        m.interaction_matrix(np.concatenate([TRI, TRI + 2 * np.array([1, 0, -1])]), MAT, 0.1, rows=(1, 1))


def test_ceiling_refusal(monkeypatch):
    monkeypatch.setattr(defaults, "MATRIX_MAX_BYTES", 1000)
    with pytest.raises(MemoryError, match="ceiling"):
        m.stress_matrix(np.zeros((10, 3)) - 1.0, np.repeat(TRI, 10, axis=0), MAT, 0.1)


def test_out_validation():
    with pytest.raises(ValueError, match="out has shape"):
        m.disp_matrix(OBS, TRI, MAT, 0.1, out=np.zeros((1, 3, 2, 3)))
    with pytest.raises(ValueError, match="float64 or float32"):
        m.disp_matrix(OBS, TRI, MAT, 0.1, out=np.zeros((1, 3, 1, 3), dtype=np.int32))


def test_chunking_arithmetic():
    assert chunking.pair_bytes("stress") == 216
    assert chunking.pair_bytes("disp", parts=True) == 144
    assert chunking.pair_bytes((1, 1)) == 8
    p = chunking.chunk_plan(1000, 100, "stress", ceiling=216 * 100 * 30)
    assert (p.obs_per_chunk, p.n_chunks) == (30, 34)


def test_tdcs_frames_match_the_oracle_and_conventions():
    rng = np.random.default_rng(0)
    tris = rng.standard_normal((20, 3, 3)) - np.array([0, 0, 5.0])
    F = tdcs.slip_frame(tris)
    assert np.allclose(F, O.slip_frame(tris), atol=0, rtol=0)
    assert np.allclose(np.einsum("sab,scb->sac", F, F), np.eye(3)[None], atol=1e-14)
    assert np.all(F[:, 2, 2] >= 0) and np.all(F[:, 0, 2] == 0)
    flat = np.array([[[0, 0, -1.0], [1, 0, -1.0], [0, 1, -1.0]]])
    assert np.array_equal(tdcs.slip_frame(flat)[0, 0], [1.0, 0.0, 0.0])
    assert list(tdcs.component_index(("strike", "normal"))) == [0, 2]
    with pytest.raises(ValueError):
        tdcs.component_index("up")
    s = rng.standard_normal((20, 3))
    assert np.allclose(tdcs.from_cartesian(tris, tdcs.to_cartesian(tris, s)), s, atol=1e-14)


def test_shared_nodes_reproduce_mhs_numbering():
    d = golden("continuous")
    sn = m.shared_nodes(d["tris"], groups=d["groups"])
    assert np.array_equal(sn.ids, d["ids"])
    assert np.allclose(sn.coords, d["coords"], rtol=0, atol=1e-15)
    assert np.allclose(sn.normals, d["normals"], rtol=0, atol=1e-15)
    assert sn.n == d["coords"].shape[0]
    v = np.arange(sn.n, dtype=float)
    assert np.array_equal(sn.expand(v).reshape(-1, 6), v[sn.ids])


def test_shared_nodes_refusals():
    t = np.array([[[0, 0, -1.0], [1, 0, -1.0], [0, 1, -1.0]], [[5, 5, -1.0], [6, 5, -1.0], [5, 6, -1.0]]])
    with pytest.raises(ValueError, match="nothing is shared"):
        m.shared_nodes(t)
    a = np.array([[0, 0, -1.0], [1, 0, -1.0], [0, 1, -1.0]])
    b = np.array([[1, 0, -1.0], [0, 1, -1.0], [1, 1, -1.0]])   # same traversal of edge (1,2)
    with pytest.raises(ValueError, match="inconsistent winding"):
        m.shared_nodes(np.stack([a, b]))


def test_collocation_points():
    t = np.array([[[0, 0, -1.0], [3, 0, -1.0], [0, 3, -1.0]]])
    assert np.allclose(m.collocation_points(t), [[1, 1, -1]])
    p1 = m.collocation_points(t, order=1)
    assert np.allclose(p1[0], 0.5 * t[0, 0] + 0.5 * np.array([1, 1, -1]))
    assert np.allclose(p1, O.collocation_points(t, 1))


def test_constants_agree_across_package_engine_and_oracle():
    src = (ROOT / "mhs_b200" / "csrc" / "engine_base.cuh").read_text()
    eng = {k: float(v) for k, v in re.findall(r"constexpr (?:double|int) ([A-Z_0-9]+) = ([0-9.e+-]+);", src)}
    pairs = {"D_STAR": O.D_STAR, "FAR_GAUSS_N": O.FAR_N, "FAR_GAUSS_N_DISTANT": O.FAR_N_DISTANT,
             "D_STAR_DISTANT": O.D_STAR_DISTANT, "SERIES_U_OVER_RHO": O.SERIES_U_OVER_RHO,
             "SERIES_TERMS": O.SERIES_TERMS, "SMALL_U_OVER_RHO": O.SMALL_U_OVER_RHO,
             "IMAGE_Q_BUDGET_C": O.Q_BUDGET_C, "IMAGE_Q_GAUSS_MIN": O.Q_MIN,
             "IMAGE_Q_GAUSS_MAX": O.Q_MAX, "FOLD_SOURCE_DEPTH_EPS": O.FOLD_SRC_EPS,
             "FOLD_BAND_DEPTH_EPS": O.FOLD_BAND_EPS, "FOLD_REACH_EPS": O.FOLD_REACH_EPS,
             "FOLD_N_RADIAL": O.FOLD_NR, "FOLD_N_ANGULAR": O.FOLD_NA,
             "FOLD_CREASE_MARGIN_EPS": O.FOLD_MARGIN_EPS, "FOLD_FINE_SPACING_EPS": O.FOLD_FINE_EPS,
             "FOLD_MEDIUM_SPACING_EPS": O.FOLD_MED_EPS, "FOLD_N_COARSE": O.FOLD_COARSE,
             "FOLD_FINE_SUBPANEL_EPS": O.FOLD_FINE_SUB_EPS,
             "FOLD_MEDIUM_SUBPANEL_EPS": O.FOLD_MED_SUB_EPS, "FOLD_R1_MARGIN_DIAM": O.FOLD_R1_DIAM}
    for k, v in pairs.items():
        assert eng[k] == v, k
        assert getattr(defaults, k) == v, k


def test_serving_admission_rule():
    from mhs_b200.serve import admissible
    assert admissible(10, 80, 3, 100, 4)
    assert not admissible(30, 80, 3, 100, 4)     # bytes
    assert not admissible(1, 0, 4, 100, 4)       # slots
    assert admissible(100, 0, 0, 100, 1)         # exactly the budget
