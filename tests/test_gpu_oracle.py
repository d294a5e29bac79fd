"""CUDA path against the numpy oracle on seeded inputs, FP64, relmax <= 1e-12.

Sizes are small enough for the oracle to finish in seconds; every kind,
order, layout and the fold are covered."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import relmax
from mhs_b200 import synthetic
from oracle import mhs_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12
MU, LAM = 30.0, 22.0


def _case(seed, top=-0.8, n=(3, 2)):
    rng = np.random.default_rng(seed)
    tris = synthetic.planar_fault(rng.uniform(0, 90), rng.uniform(30, 90), 3.0, 2.0, top, *n)
    obs = np.concatenate([rng.uniform([-3, -3, -3], [3, 3, 0], (10, 3)),
                          rng.uniform([-30, -30, -20], [30, 30, 0], (6, 3))])
    return tris, obs


#: At P2 the image R-family reads closed-form moments up to n = 9 at degree
#: 7.  Where the observer sits nearly in the reflected element's plane a few
#: widths L away (closed-form regime, D <= D_STAR L, and D / h > 10 with h =
#: sqrt(z^2 + eps^2) its height over that plane), the upward vertical seed
#: I_9 = (E_7 + 5 I_7) / (7 h^2) amplifies last-ulp differences of log1p /
#: pow by ~(D / h)^2 x 1e8, so mhs's own arithmetic (restated by the oracle)
#: carries up to ~1.5e-12 of the matrix maximum there, and this engine lands
#: closer to a converged quadrature than mhs does (tests/test_engine_host.py::
#: test_p2_image_closer_to_converged_than_mhs_arithmetic).  The relaxed P2
#: bound applies to the entries of those (observer, source) pairs only (9 to
#: 30 % of the pairs of these near-field cases); every other entry is held to
#: 1e-12 of the matrix maximum.
TOL_P2_REGION = 5e-12
#: The eigenstress matrix peaks on the element and decays like R^-7, so its
#: far tail -- the blob weight, from the same upward seed I_7 -- is ~1e-5 of
#: its maximum and carries mhs's rounding at ~1e-15 absolute: 1e-11 of the
#: maximum at P2 (the engine is ~30x closer to a converged quadrature there).
TOL_EIGEN_P2_REGION = 3e-11


def _image_closed_pairs(obs, tris, eps):
    """(n_obs, n_src) mask of the ill-conditioned P2 pairs: the reflected
    element's closed form applies (centroid within D_STAR L, eps included:
    mhs/fullspace/moments.py:551-554 on the reflected frame) and the
    observer's height over that element's plane is under a tenth of D."""
    refl = tris * np.array([1.0, 1.0, -1.0])
    c = refl.mean(axis=1)
    n = np.cross(refl[:, 1] - refl[:, 0], refl[:, 2] - refl[:, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    L = np.max(np.linalg.norm(tris - np.roll(tris, 1, axis=1), axis=2), axis=1)
    d = obs[:, None, :] - c[None]
    D = np.sqrt(np.sum(d * d, axis=2) + eps * eps)
    h = np.sqrt(np.einsum("osk,sk->os", d, n) ** 2 + eps * eps)
    return (D <= 10.0 * L[None, :]) & (D > 10.0 * h)


def _check(got, ref, pairs, p, tol_region, what):
    """relmax <= 1e-12 outside the P2 ill-conditioned pairs, <= tol_region
    inside them (both against the whole matrix's maximum); at P0/P1 1e-12
    everywhere."""
    got, ref = np.asarray(got), np.asarray(ref)
    big = np.max(np.abs(ref))
    err = np.abs(got - ref) / big
    if p < 2:
        assert err.max() < TOL, f"{what}: {err.max():.2e}"
        return
    K = 6
    # entry -> (observer, source): obs is axis 0, the source dof axis is -2
    mask = np.repeat(pairs, K, axis=1)                       # (n_obs, n_dof)
    shape = [1] * got.ndim
    shape[0], shape[-2] = mask.shape
    m = np.broadcast_to(mask.reshape(shape), got.shape)
    assert err[~m].max() < TOL, f"{what} outside the region: {err[~m].max():.2e}"
    assert err[m].max() < tol_region, f"{what} in the region: {err[m].max():.2e}"


@pytest.mark.parametrize("p", [0, 1, 2])
@pytest.mark.parametrize("seed", [1, 2])
def test_kinds_against_oracle(cuda, p, seed):
    import mhs_b200 as m
    tris, obs = _case(seed)
    mat = m.Material(MU, LAM)
    eps = 0.12
    pairs = _image_closed_pairs(obs, tris, eps)
    _check(m.disp_matrix(obs, tris, mat, eps, order=p), O.disp_matrix(obs, tris, MU, LAM, eps, p),
           pairs, p, TOL_P2_REGION, "disp")
    _check(m.stress_matrix(obs, tris, mat, eps, order=p), O.stress_matrix(obs, tris, MU, LAM, eps, p),
           pairs, p, TOL_P2_REGION, "stress")
    _check(m.eigenstress_matrix(obs, tris, mat, eps, order=p),
           O.eigenstress_matrix(obs, tris, MU, LAM, eps, p), pairs, p, TOL_EIGEN_P2_REGION, "eigen")
    _check(m.elastic_strain_matrix(obs, tris, mat, eps, order=p),
           O.elastic_strain_matrix(obs, tris, MU, LAM, eps, p), pairs, p, TOL_P2_REGION, "strain")
    nrm = np.random.default_rng(seed).standard_normal(obs.shape)
    _check(m.traction_matrix(obs, nrm, tris, mat, eps, order=p),
           O.traction_matrix(obs, nrm, tris, MU, LAM, eps, p), pairs, p, TOL_P2_REGION, "traction")


def test_p2_region_size():
    """Size of the relaxed region on the seeded P2 cases: the fraction of
    (observer, source) pairs whose image takes the closed form."""
    fr = []
    for seed in (1, 2):
        tris, obs = _case(seed)
        fr.append(_image_closed_pairs(obs, tris, 0.12).mean())
    assert 0.0 < min(fr) and max(fr) < 0.35


def test_fold_and_per_triangle_eps(cuda):
    import mhs_b200 as m
    c = synthetic.config2(seed=5, nu=3, nv=2)
    mat = m.Material(c["mu"], c["lam"])
    K = m.interaction_matrix(c["tris"], mat, c["eps"])
    R = O.self_interaction(c["tris"], c["mu"], c["lam"], c["eps"])
    assert relmax(K, R) < TOL
    rng = np.random.default_rng(3)
    obs = np.column_stack([rng.uniform(-15, 15, 5), rng.uniform(-2, 5, 5), -rng.uniform(0, 2, 5)])
    assert relmax(m.disp_matrix(obs, c["tris"], mat, c["eps"]),
                  O.disp_matrix(obs, c["tris"], c["mu"], c["lam"], c["eps"])) < TOL


def test_continuous_p2_against_oracle(cuda):
    import mhs_b200 as m
    tris = synthetic.planar_fault(20.0, 70.0, 3.0, 2.0, -0.5, 3, 2)
    sn = m.shared_nodes(tris)
    mat = m.Material(MU, LAM)
    K = m.interaction_matrix(tris, mat, 0.1, order=2, layout="continuous", shared=sn,
                             receiver=("strike", "normal"), source=("dip",))
    fr = sn.frames
    R = O.interaction_matrix(sn.coords, fr[:, 2, :], fr[:, [0, 2], :], tris, fr[:, [1], :], MU, LAM,
                             0.1, 2, ids=sn.ids, n_dof=sn.n)
    assert relmax(K, R) < TOL
