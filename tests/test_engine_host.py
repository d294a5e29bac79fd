"""The device engine's arithmetic, compiled for the CPU (tests/engine_host),
term by term against the numpy oracle: direct Kelvin-Cortez, image R-family,
image Q-family and the folded image, every order.  Tolerance 1e-12 relmax."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import build_hostcheck, relmax
from oracle import mhs_oracle as O

D = ctypes.POINTER(ctypes.c_double)
TOL = 1e-12


@pytest.fixture(scope="module")
def hc():
    return ctypes.CDLL(str(build_hostcheck()))


def _p(a):
    return a.ctypes.data_as(D)


TRI = np.array([[0.37, -0.81, -1.44], [1.92, 0.11, -2.63], [-0.25, 1.57, -1.22]])
MU, LAM, EPS = 30.0, 20.0, 0.1


def _obs():
    rng = np.random.default_rng(0)
    o = np.concatenate([rng.uniform(-3, 3, (12, 3)), rng.uniform(-40, 40, (6, 3)),
                        rng.uniform(-200, 200, (4, 3))])
    o[:, 2] = -np.abs(o[:, 2])
    return np.ascontiguousarray(o)


def test_gauss_legendre_matches_numpy(hc):
    for n in (1, 4, 6, 8, 12, 37, 192):
        x, w = np.zeros(n), np.zeros(n)
        assert hc.hc_gauss(n, _p(x), _p(w)) == 0
        xr, wr = np.polynomial.legendre.leggauss(n)
        assert np.max(np.abs(x - xr)) < 1e-15 and np.max(np.abs(w - wr)) < 2e-14


@pytest.mark.parametrize("P", [0, 1, 2])
def test_direct(hc, P):
    obs = _obs()
    N, K = obs.shape[0], (P + 1) * (P + 2) // 2
    ref = O.direct(obs, TRI, P, MU, LAM, EPS, ("U", "H", "E"))
    U, H, E = np.zeros((N, K, 3, 3)), np.zeros((N, K, 3, 3, 3)), np.zeros((N, K))
    c = ctypes.c_double
    hc.hc_direct(P, 1, _p(obs), N, _p(TRI.copy()), c(MU), c(LAM), c(EPS), _p(U), None, None)
    hc.hc_direct(P, 6, _p(obs), N, _p(TRI.copy()), c(MU), c(LAM), c(EPS), None, _p(H), _p(E))
    assert relmax(U, ref["U"]) < TOL
    assert relmax(H, ref["H"]) < TOL
    assert relmax(E, ref["E"]) < TOL


@pytest.mark.parametrize("P", [0, 1, 2])
def test_image_r_and_q(hc, P):
    obs = _obs()
    N, K = obs.shape[0], (P + 1) * (P + 2) // 2
    c = ctypes.c_double
    for code, key in ((1, "U"), (2, "H")):
        shape = (N, K, 3, 3) if key == "U" else (N, K, 3, 3, 3)
        A = np.zeros(shape)
        hc.hc_image_r(P, code, _p(obs), N, _p(TRI.copy()), c(MU), c(LAM), c(EPS), _p(A), _p(A))
        assert relmax(A, O.image_r(obs, TRI, P, MU, LAM, EPS, (key,))[key]) < TOL
        B = np.zeros(shape)
        hc.hc_image_q(P, code, _p(obs), N, _p(TRI.copy()), c(MU), c(LAM), c(EPS), 0, _p(B), _p(B), None)
        assert relmax(B, O.image_q(obs, TRI, P, MU, LAM, EPS, (key,))[key]) < TOL


def test_p2_image_closer_to_converged_than_mhs_arithmetic(hc, monkeypatch):
    """Where the closed-form image moments are ill-conditioned (P2, a few L
    from the reflected element), the engine and mhs's arithmetic (the
    oracle) differ by ~1e-12 of the matrix maximum; both are compared with a
    converged 40 x 40 Gauss rule, and the engine must be the closer one."""
    from mhs_b200 import synthetic
    rng = np.random.default_rng(1)
    tris = synthetic.planar_fault(rng.uniform(0, 90), rng.uniform(30, 90), 3.0, 2.0, -0.8, 3, 2)
    obs = np.concatenate([rng.uniform([-3, -3, -3], [3, 3, 0], (10, 3)),
                          rng.uniform([-30, -30, -20], [30, 30, 0], (6, 3))])
    x = np.ascontiguousarray(obs[7:8])
    g = np.abs(O.stress_matrix(obs, tris, MU, 22.0, 0.12, 2)).max()
    oracle = np.stack([O.image_r(x, t, 2, MU, 22.0, 0.12, ("H",))["H"][0] for t in tris])
    eng = []
    for t in tris:
        A = np.zeros((1, 6, 3, 3, 3))
        c = ctypes.c_double
        hc.hc_image_r(2, 2, _p(x), 1, _p(np.ascontiguousarray(t)), c(MU), c(22.0), c(0.12), _p(A), _p(A))
        eng.append(A[0])
    eng = np.stack(eng)
    rule = O._tri_rule
    monkeypatch.setattr(O, "D_STAR", 1e-9)
    monkeypatch.setattr(O, "_tri_rule", lambda n: rule(40))
    truth = np.stack([O.image_r(x, t, 2, MU, 22.0, 0.12, ("H",))["H"][0] for t in tris])
    e_eng = np.abs(eng - truth).max() / g
    e_mhs = np.abs(oracle - truth).max() / g
    assert e_eng < e_mhs and e_eng < 1e-12


@pytest.mark.parametrize("P,key", [(0, "H"), (0, "U"), (1, "H")])
def test_fold_image(hc, P, key):
    tri = np.array([[0.0, 0.0, 0.0], [1.5, 0.2, -0.05], [0.3, 0.9, -1.1]])
    obs = np.array([[0.5, 0.5, -0.3], [2.0, -1.0, -0.05]])
    N, K = obs.shape[0], (P + 1) * (P + 2) // 2
    shape = (N, K, 3, 3) if key == "U" else (N, K, 3, 3, 3)
    A = np.zeros(shape)
    c = ctypes.c_double
    hc.hc_fold_image(P, 1 if key == "U" else 2, _p(obs), N, _p(tri.copy()), c(MU), c(LAM), c(0.12),
                     _p(A), _p(A))
    assert relmax(A, O.fold_image(obs, tri, P, MU, LAM, 0.12, (key,))[key]) < TOL


@pytest.mark.parametrize("P", [0, 1, 2])
def test_surface_load_fast_matches_full_stress(hc, P):
    """The fold's surface load contracts the lifted moments with a per-source
    sigma_zz row instead of assembling and rotating all of H; both forms
    agree at surface points in the closed-form and both quadrature zones."""
    tri = np.array([[0.0, 0.0, 0.0], [1.5, 0.2, -0.05], [0.3, 0.9, -1.1]])
    rng = np.random.default_rng(3)
    pts = np.ascontiguousarray(np.concatenate([rng.uniform(-2, 3, (40, 2)), rng.uniform(-30, 30, (10, 2)),
                                               rng.uniform(-300, 300, (6, 2))]))
    K = (P + 1) * (P + 2) // 2
    c = ctypes.c_double
    out = {}
    for fast in (0, 1):
        s = np.zeros((pts.shape[0], K, 3))
        assert hc.hc_surface_load(P, fast, _p(pts), pts.shape[0], _p(tri.copy()), c(MU), c(LAM),
                                  c(0.12), _p(s)) == 0
        out[fast] = s
    assert np.abs(out[1]).max() > 0
    assert relmax(out[1], out[0]) < 1e-13


@pytest.mark.parametrize("P", [0, 1, 2])
def test_fold_closed_edge_form_matches_plain(hc, P):
    """The fold's closed-form edge integrals (reciprocal radii, products with
    1/rho2) agree with the plain form to rounding on every edge geometry."""
    rng = np.random.default_rng(P)
    c = ctypes.c_double
    worst = 0.0
    for _ in range(300):
        ua, ub = np.sort(rng.uniform(-3, 3, 2))
        rho2 = rng.uniform(0.01, 4.0)
        a, b = np.zeros(40), np.zeros(40)
        hc.hc_edge_closed(P, 0, c(ua), c(ub), c(rho2), _p(a))
        hc.hc_edge_closed(P, 1, c(ua), c(ub), c(rho2), _p(b))
        scale = np.abs(a).max()
        if scale > 0:
            worst = max(worst, np.abs(a - b).max() / scale)
    assert worst < 1e-13


def test_fold_finish_form_matches_plain(hc):
    """The fold's seeds and recursion (reciprocal 1/h, products with 1/h^2)
    agree with the plain form to rounding."""
    rng = np.random.default_rng(9)
    worst = 0.0
    for _ in range(200):
        pr = np.ascontiguousarray(rng.uniform(-2, 2, 6))
        bn = np.ascontiguousarray(rng.uniform(-1, 1, 64))
        h2 = float(rng.uniform(0.01, 3.0))
        a, b = np.zeros(64), np.zeros(64)
        n = hc.hc_closed_finish(0, _p(pr), ctypes.c_double(h2), _p(bn), _p(a))
        hc.hc_closed_finish(1, _p(pr), ctypes.c_double(h2), _p(bn), _p(b))
        worst = max(worst, np.abs(a[:n] - b[:n]).max() / np.abs(a[:n]).max())
    assert worst < 1e-13


@pytest.mark.parametrize("P", [0, 1, 2])
def test_force_source(hc, P, monkeypatch):
    """The force (Kelvin single-layer) kernels G and S of the engine against
    the oracle, with the hybrid split and with quadrature everywhere; and
    against mhs's own fullspace.influence (golden fixture)."""
    from conftest import golden
    c = ctypes.c_double
    obs = _obs()
    N, K = obs.shape[0], (P + 1) * (P + 2) // 2
    for near_l in (10.0, -1.0):
        monkeypatch.setattr(O, "D_STAR", near_l)
        ref = O.direct(obs, TRI, P, MU, LAM, EPS, ("G", "S"))
        G, S = np.zeros((N, K, 3, 3)), np.zeros((N, K, 3, 3, 3))
        assert hc.hc_force(P, 24, _p(obs), N, _p(TRI.copy()), c(MU), c(LAM), c(EPS), c(near_l),
                           _p(G), _p(S)) == 0
        assert relmax(G, ref["G"]) < TOL, near_l
        assert relmax(S, ref["S"]) < TOL, near_l
    d = golden("fullspace")
    mu, nu = float(d["mu"]), float(d["nu"])
    lam = 2.0 * mu * nu / (1.0 - 2.0 * nu)
    for t in (0, 1):
        tri = np.ascontiguousarray(d["tris"][t])
        o = np.ascontiguousarray(d["obs"])
        n = o.shape[0]
        for ff, near_l in (("hybrid", 10.0), ("quadrature", -1.0)):
            G, S = np.zeros((n, K, 3, 3)), np.zeros((n, K, 3, 3, 3))
            hc.hc_force(P, 24, _p(o), n, _p(tri), c(mu), c(lam), c(float(d["eps"][t])),
                        c(near_l), _p(G), _p(S))
            assert relmax(G, d[f"G_{t}_{P}_{ff}"]) < TOL, (t, ff)
            assert relmax(S, d[f"S_{t}_{P}_{ff}"]) < TOL, (t, ff)
