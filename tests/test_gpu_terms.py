"""Single influence terms on the GPU (mhs_debug_terms), one source at a few
observers: the folded image against the numpy oracle, and the fold's
surface load from the contracted sigma_zz row against the full stress
kernel, every order, on the device."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import relmax
from oracle import mhs_oracle as O

pytestmark = pytest.mark.gpu
MU, LAM, EPS = 30.0, 22.0, 0.12
TRI = np.array([[0.0, 0.0, 0.0], [1.5, 0.2, -0.05], [0.3, 0.9, -1.1]])


def _terms(P, term, want_u, obs):
    import torch
    from mhs_b200 import _native as nat
    lib = nat.load()
    K = (P + 1) * (P + 2) // 2
    C = 9 if want_u else 27
    dev = torch.device("cuda")
    o = torch.as_tensor(np.ascontiguousarray(obs, dtype=np.float64), device=dev)
    t = torch.as_tensor(TRI, device=dev)
    coef = torch.zeros(4096, dtype=torch.float64, device=dev)
    out = torch.zeros(obs.shape[0] * (K * C + K), dtype=torch.float64, device=dev)
    rc = lib.mhs_debug_terms(P, term, want_u, obs.shape[0], o.data_ptr(), t.data_ptr(),
                             MU, LAM, EPS, coef.data_ptr(), out.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(obs.shape[0], K * C + K)[:, :K * C], K


@pytest.mark.parametrize("P", [0, 1, 2])
def test_surface_load_row_matches_full_stress(P):
    rng = np.random.default_rng(5)
    pts = np.concatenate([rng.uniform(-2, 3, (48, 2)), rng.uniform(-30, 30, (8, 2)),
                          rng.uniform(-300, 300, (8, 2))])
    obs = np.concatenate([pts, np.zeros((pts.shape[0], 1))], axis=1)
    fast, K = _terms(P, 4, 0, obs)
    full, _ = _terms(P, 5, 0, obs)
    assert np.abs(full[:, :3 * K]).max() > 0
    assert relmax(fast[:, :3 * K], full[:, :3 * K]) < 1e-13


@pytest.mark.parametrize("P,key", [(0, "H"), (1, "H"), (1, "U"), (2, "H")])
def test_fold_term_against_oracle(P, key):
    obs = np.array([[0.5, 0.5, -0.3], [2.0, -1.0, -0.05], [0.8, 0.3, -0.02]])
    A, K = _terms(P, 3, 1 if key == "U" else 0, obs)
    shape = (obs.shape[0], K, 3, 3) if key == "U" else (obs.shape[0], K, 3, 3, 3)
    ref = O.fold_image(obs, TRI, P, MU, LAM, EPS, (key,))[key]
    assert relmax(A.reshape(shape), ref) < (5e-12 if P == 2 else 1e-12)
