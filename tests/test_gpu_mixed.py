"""The mixed form (precision="mixed": far-field quadrature of the direct
term, the fold's surface loads and its mirror in float32 with float32
accumulation; near-field recursions, image terms and the eigenstress
subtraction in float64) against the FP64 oracle: relmax <= 1e-6 for every
matrix and order, and genuinely different from the FP64 path where the far
field contributes."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import relmax
from mhs_b200 import synthetic
from oracle import mhs_oracle as O

pytestmark = pytest.mark.gpu
TOL_MIXED = 1e-6
MU, LAM = 30.0, 22.0


def _case(seed):
    rng = np.random.default_rng(seed)
    tris = synthetic.planar_fault(rng.uniform(0, 90), rng.uniform(30, 90), 3.0, 2.0, -0.8, 3, 2)
    obs = np.concatenate([rng.uniform([-3, -3, -3], [3, 3, 0], (10, 3)),
                          rng.uniform([-60, -60, -40], [60, 60, 0], (10, 3))])
    return tris, obs


@pytest.mark.parametrize("p", [0, 1, 2])
def test_every_matrix_within_1e6_of_the_fp64_oracle(cuda, p):
    import mhs_b200 as m
    tris, obs = _case(7)
    mat = m.Material(MU, LAM)
    eps = 0.12
    nrm = np.random.default_rng(7).standard_normal(obs.shape)
    cases = {
        "disp": (lambda pr: m.disp_matrix(obs, tris, mat, eps, order=p, precision=pr),
                 O.disp_matrix(obs, tris, MU, LAM, eps, p)),
        "stress": (lambda pr: m.stress_matrix(obs, tris, mat, eps, order=p, precision=pr),
                   O.stress_matrix(obs, tris, MU, LAM, eps, p)),
        "total_stress": (lambda pr: m.total_stress_matrix(obs, tris, mat, eps, order=p, precision=pr),
                         O.total_stress_matrix(obs, tris, MU, LAM, eps, p)),
        "eigenstress": (lambda pr: m.eigenstress_matrix(obs, tris, mat, eps, order=p, precision=pr),
                        O.eigenstress_matrix(obs, tris, MU, LAM, eps, p)),
        "traction": (lambda pr: m.traction_matrix(obs, nrm, tris, mat, eps, order=p, precision=pr),
                     O.traction_matrix(obs, nrm, tris, MU, LAM, eps, p)),
    }
    differs = False
    for name, (f, ref) in cases.items():
        mixed = f("mixed")
        err = relmax(mixed, ref)
        assert err < TOL_MIXED, (name, p, err)
        differs |= not np.array_equal(mixed, f("fp64"))
    assert differs, "the mixed form ran the FP64 path"


def test_folded_interaction_within_1e6(cuda):
    import mhs_b200 as m
    c = synthetic.config2(seed=5, nu=3, nv=2)
    mat = m.Material(c["mu"], c["lam"])
    R = O.self_interaction(c["tris"], c["mu"], c["lam"], c["eps"])
    K = m.interaction_matrix(c["tris"], mat, c["eps"], precision="mixed")
    assert relmax(K, R) < TOL_MIXED
    assert not np.array_equal(K, m.interaction_matrix(c["tris"], mat, c["eps"]))
