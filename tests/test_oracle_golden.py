"""Pin the numpy oracle to mhs's own outputs (golden fixtures).

The oracle restates mhs term by term, so on the same inputs it must agree
with mhs's arrays to rounding: relmax <= 1e-13."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, relmax
from oracle import mhs_oracle as O

TOL = 1e-13


def _m(d):
    return float(d["mu"]), float(d["lam"])


def test_c1_subset():
    d = golden("c1_subset")
    mu, lam = _m(d)
    sel = slice(0, 60, 4)
    assert relmax(O.disp_matrix(d["obs"][sel], d["tris"], mu, lam, float(d["eps"])), d["disp"][sel]) < TOL
    assert relmax(O.stress_matrix(d["obs"][sel], d["tris"], mu, lam, float(d["eps"])), d["stress"][sel]) < TOL


@pytest.mark.parametrize("p", [0, 1, 2])
def test_orders(p):
    d = golden("orders")
    mu, lam = _m(d)
    e = float(d["eps"])
    assert relmax(O.disp_matrix(d["obs"], d["tris"], mu, lam, e, p), d[f"disp_p{p}"]) < TOL
    assert relmax(O.stress_matrix(d["obs"], d["tris"], mu, lam, e, p), d[f"stress_p{p}"]) < TOL
    assert relmax(O.total_stress_matrix(d["obs"], d["tris"], mu, lam, e, p), d[f"total_p{p}"]) < TOL
    assert relmax(O.traction_matrix(d["obs"], d["normals"], d["tris"], mu, lam, e, p),
                  d[f"traction_p{p}"]) < TOL


def test_eps_per_triangle():
    d = golden("eps_per_tri")
    mu, lam = _m(d)
    assert relmax(O.stress_matrix(d["obs"], d["tris"], mu, lam, d["eps"], 1), d["stress_p1"]) < TOL


def test_interaction():
    d = golden("interaction")
    mu, lam = _m(d)
    e = float(d["eps"])
    assert relmax(O.self_interaction(d["tris"], mu, lam, e), d["int_p0"]) < TOL
    assert relmax(O.self_interaction(d["tris"], mu, lam, e, subtract_eigenstress=False),
                  d["int_p0_noeig"]) < TOL


def test_fold():
    d = golden("fold")
    mu, lam = _m(d)
    e = float(d["eps"])
    assert relmax(O.self_interaction(d["tris"], mu, lam, e), d["int_p0"]) < TOL
    assert relmax(O.stress_matrix(d["obs"], d["tris"], mu, lam, e, fold=False),
                  d["stress_p0_nofold"]) < TOL


def test_continuous_traction():
    d = golden("continuous")
    mu, lam = _m(d)
    ids = d["ids"]
    n = d["coords"].shape[0]
    T = O.traction_matrix(d["obs"], d["obs_normals"], d["tris"], mu, lam, float(d["eps"]), 2,
                          ids=ids, n_dof=n)
    assert relmax(T, d["trac_cont"]) < TOL


@pytest.mark.parametrize("t", [0, 1])
@pytest.mark.parametrize("p", [0, 1, 2])
def test_fullspace_influence(t, p, monkeypatch):
    """The oracle's full-space kernels -- slip source U, H, E and force source
    G, S -- against mhs.fullspace.api.influence, with the hybrid far field
    and with quadrature everywhere."""
    d = golden("fullspace")
    mu, nu = float(d["mu"]), float(d["nu"])
    lam = 2.0 * mu * nu / (1.0 - 2.0 * nu)
    eps = float(d["eps"][t])
    for ff in ("hybrid", "quadrature"):
        if ff == "quadrature":
            monkeypatch.setattr(O, "D_STAR", -1.0)
        got = O.direct(d["obs"], d["tris"][t], p, mu, lam, eps, ("U", "H", "E", "G", "S"))
        for k in ("U", "H", "E", "G", "S"):
            assert relmax(got[k], d[f"{k}_{t}_{p}_{ff}"]) < 1e-13, (k, ff)
