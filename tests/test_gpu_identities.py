"""Identities of the assembled matrices on the GPU, at sizes the oracle could
not check directly (mhs's gates, restated on the CUDA path):

* total - eigenstress == stress                      (verify_fullspace_assembly [d])
* traction == stress . n                             (verify_image_kernel part i)
* interaction == stress resolved in both frames      (verify_image_kernel part i)
* uniform nodal P1/P2 slip == P0 at every entry point (verify_image_kernel part g)
* continuous == element columns summed into shared ones (verify_shared_nodes b)
* rows= block == slice of the whole, additivity over sources
* negative self-interaction diagonal (strike/strike)
* float32 out == float64 rounded, torch in/out == numpy in/out
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import relmax
from mhs_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    return synthetic.config1(seed=0)


def _mat(c):
    import mhs_b200 as m
    return m.Material(c["mu"], c["lam"])


def test_total_minus_eigen_is_stress(cuda, c1):
    import mhs_b200 as m
    mat = _mat(c1)
    S = m.stress_matrix(c1["obs"], c1["tris"], mat, c1["eps"])
    T = m.total_stress_matrix(c1["obs"], c1["tris"], mat, c1["eps"])
    E = m.eigenstress_matrix(c1["obs"], c1["tris"], mat, c1["eps"])
    assert relmax(T - E, S) < 1e-14
    S2, E2 = m.stress_matrix(c1["obs"], c1["tris"], mat, c1["eps"], parts=True)
    assert np.array_equal(S2, S) and np.array_equal(E2, E)


def test_traction_and_interaction_are_contracted_stress(cuda):
    import mhs_b200 as m
    c = synthetic.config2(seed=2, nu=8, nv=4)
    mat = _mat(c)
    pts = m.collocation_points(c["tris"])
    fr = m.tdcs.slip_frame(c["tris"])
    S = m.stress_matrix(pts, c["tris"], mat, c["eps"])
    T = m.traction_matrix(pts, fr[:, 2, :], c["tris"], mat, c["eps"])
    assert relmax(T, np.einsum("oijsm,oj->oism", S, fr[:, 2, :])) < 1e-13
    K = m.interaction_matrix(c["tris"], mat, c["eps"])
    Kc = np.einsum("oai,oism,sbm->osab", fr, np.einsum("oijsm,oj->oism", S, fr[:, 2, :]), fr)
    assert relmax(K, Kc) < 1e-13
    # upward-wound mesh: slip relieves its own shear (mhs's gate clause [h])
    for comp in (0, 1):
        assert np.all(np.einsum("ii->i", K[:, :, comp, comp]) < 0)


def test_self_interaction_sign_on_mhs_dipping_patch(cuda):
    import mhs_b200 as m
    dipping = np.array([
        [[0.0, 0.0, -1.0], [1.0, 0.0, -1.0], [0.0, 0.6, -1.8]],
        [[1.0, 0.0, -1.0], [1.0, 0.6, -1.8], [0.0, 0.6, -1.8]],
        [[1.0, 0.0, -1.0], [2.0, 0.0, -1.0], [1.0, 0.6, -1.8]],
    ])
    mat = m.Material(1.0, 1.5)
    for comp in ("strike", "dip"):
        d = np.diag(m.interaction_matrix(dipping, mat, 0.1, receiver=comp, source=comp)[:, :, 0, 0])
        assert np.all(d < 0.0), comp


@pytest.mark.parametrize("p", [1, 2])
def test_uniform_nodal_slip_is_p0(cuda, c1, p):
    import mhs_b200 as m
    mat = _mat(c1)
    obs = c1["obs"][::5]
    K = (p + 1) * (p + 2) // 2
    for fn in (m.disp_matrix, m.stress_matrix, m.total_stress_matrix):
        A0 = fn(obs, c1["tris"], mat, c1["eps"])
        Ap = fn(obs, c1["tris"], mat, c1["eps"], order=p)
        Ap = Ap.reshape(Ap.shape[:-2] + (c1["tris"].shape[0], K, 3)).sum(axis=-2)
        assert relmax(Ap, A0) < 1e-11          # mhs's gate bound for this identity


def test_continuous_equals_summed_element_columns(cuda):
    import mhs_b200 as m
    tris, fid = synthetic.fault_network(length=8.0, depth=3.0, splay_len=4.0, splay_width=3.0,
                                        nu=8, nv=3, nv_splay=3)
    sn = m.shared_nodes(tris, groups=fid)
    mat = m.Material(30.0, 30.0)
    obs = sn.coords[::7] - np.array([0.0, 0.1, 0.05])
    obs[:, 2] = np.minimum(obs[:, 2], 0.0)
    Dd = m.disp_matrix(obs, tris, mat, 0.1, order=2)
    Dc = m.disp_matrix(obs, tris, mat, 0.1, order=2, layout="continuous", shared=sn)
    acc = np.zeros_like(Dc)
    for s in range(tris.shape[0]):
        for k in range(6):
            acc[:, :, sn.ids[s, k], :] += Dd[:, :, 6 * s + k, :]
    assert relmax(Dc, acc) < 1e-13


def test_rows_block_and_source_additivity(cuda):
    import mhs_b200 as m
    c = synthetic.config2(seed=4, nu=6, nv=3)
    mat = _mat(c)
    K = m.interaction_matrix(c["tris"], mat, c["eps"])
    B = m.interaction_matrix(c["tris"], mat, c["eps"], rows=(7, 23))
    assert np.array_equal(B, K[7:23])
    obs = m.collocation_points(c["tris"])
    A = m.disp_matrix(obs, c["tris"], mat, c["eps"])
    A1 = m.disp_matrix(obs, c["tris"][:10], mat, c["eps"][:10])
    A2 = m.disp_matrix(obs, c["tris"][10:], mat, c["eps"][10:])
    assert np.array_equal(A, np.concatenate([A1, A2], axis=2))


def test_float32_out_and_torch_round_trip(cuda, c1):
    import torch
    import mhs_b200 as m
    mat = _mat(c1)
    D = m.disp_matrix(c1["obs"], c1["tris"], mat, c1["eps"])
    out32 = np.empty(D.shape, np.float32)
    m.disp_matrix(c1["obs"], c1["tris"], mat, c1["eps"], out=out32)
    assert np.array_equal(out32, D.astype(np.float32))
    Dt = m.disp_matrix(torch.as_tensor(c1["obs"], device=cuda), torch.as_tensor(c1["tris"], device=cuda),
                       mat, c1["eps"])
    assert isinstance(Dt, torch.Tensor) and Dt.is_cuda
    assert np.array_equal(Dt.cpu().numpy(), D)
    o = torch.empty(D.shape, dtype=torch.float64, device=cuda)
    r = m.disp_matrix(c1["obs"], c1["tris"], mat, c1["eps"], out=o)
    assert r is o and np.array_equal(o.cpu().numpy(), D)


def test_fold_off_equals_lift_outside_band(cuda):
    import mhs_b200 as m
    c = synthetic.config2(seed=6, nu=6, nv=3)
    mat = _mat(c)
    rng = np.random.default_rng(0)
    # below the band of every source: depth beyond FOLD_BAND_DEPTH_EPS x the largest eps
    z0 = 10.0 * float(np.max(c["eps"])) + 1.0
    deep = np.column_stack([rng.uniform(-10, 10, 20), rng.uniform(-5, 5, 20), -z0 - rng.uniform(0, 10, 20)])
    A = m.stress_matrix(deep, c["tris"], mat, c["eps"])
    B = m.stress_matrix(deep, c["tris"], mat, c["eps"], fold=False)
    assert np.array_equal(A, B)


# ------------------------------------------------------------ apply mode
@pytest.mark.parametrize("layout", ["discontinuous", "continuous"])
def test_matvec_equals_matrix_times_slip(cuda, layout):
    """The apply mode (the matrix contracted with a slip vector, never
    stored) against the FP64 matrix contracted on the host."""
    import mhs_b200 as m
    from conftest import golden
    d = golden("continuous")
    mat = m.Material(float(d["mu"]), float(d["lam"]))
    kw = dict(order=2, layout=layout) if layout == "continuous" else dict(order=1)
    rng = np.random.default_rng(3)
    K = m.interaction_matrix(d["tris"], mat, 0.1, source=("strike", "dip"), **kw)
    slip = rng.standard_normal((K.shape[1], 2))
    y = m.interaction_matvec(d["tris"], mat, 0.1, slip, source=("strike", "dip"), **kw)
    ref = np.einsum("rcab,cb->ra", K, slip)
    assert y.shape == ref.shape
    assert relmax(y, ref) < 1e-12
    sl3 = rng.standard_normal((K.shape[1], 3))
    T = m.traction_matrix(d["obs"], d["obs_normals"], d["tris"], mat, 0.1, **kw)
    t = m.traction_matvec(d["obs"], d["obs_normals"], d["tris"], mat, 0.1, sl3, **kw)
    assert relmax(t, np.einsum("oicm,cm->oi", T, sl3)) < 1e-12
    S = m.stress_matrix(d["obs"], d["tris"], mat, 0.1, **kw)
    st = m.stress_matvec(d["obs"], d["tris"], mat, 0.1, sl3, **kw)
    assert relmax(st, np.einsum("oijcm,cm->oij", S, sl3)) < 1e-12
    U = m.disp_matrix(d["obs"], d["tris"], mat, 0.1, **kw)
    u = m.disp_matvec(d["obs"], d["tris"], mat, 0.1, sl3, **kw)
    assert relmax(u, np.einsum("oicm,cm->oi", U, sl3)) < 1e-12


def test_matvec_with_the_fold_and_rows(cuda):
    import mhs_b200 as m
    from conftest import golden
    d = golden("c2_rows")
    mat = m.Material(float(d["mu"]), float(d["lam"]))
    rng = np.random.default_rng(9)
    slip = rng.standard_normal((d["tris"].shape[0], 3))
    r0 = int(d["rows"][0])
    y = m.interaction_matvec(d["tris"], mat, d["eps"], slip, rows=(r0, r0 + 1))
    ref = np.einsum("cab,cb->a", d["K"][0], slip)
    assert relmax(y[0], ref) < 1e-12
