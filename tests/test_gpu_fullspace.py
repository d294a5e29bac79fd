"""The full-space single-triangle API (mhs_b200.fullspace) against mhs's own
mhs.fullspace.api outputs (golden fixture): nodal influence tensors of the
slip source (U, H, E) and the force source (G, S) at orders 0-2 with the
hybrid and quadrature far fields, and the contracted calls (displacement,
stress, total stress, eigenstress, force displacement, force stress).
Tolerance: relmax <= 1e-12."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, relmax
from oracle import mhs_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("t", [0, 1])
@pytest.mark.parametrize("p", [0, 1, 2])
def test_influence_matches_mhs(cuda, t, p):
    from mhs_b200 import fullspace as fs
    d = golden("fullspace")
    mu, nu, eps = float(d["mu"]), float(d["nu"]), float(d["eps"][t])
    for ff in ("hybrid", "quadrature"):
        inf = fs.influence(d["obs"], d["tris"][t], mu, nu, eps, order=p,
                           want=("U", "H", "E", "G", "S"), far_field=ff)
        for k in ("U", "H", "E", "G", "S"):
            assert relmax(getattr(inf, k), d[f"{k}_{t}_{p}_{ff}"]) < TOL, (k, ff)
        assert inf.nodes.shape == ((p + 1) * (p + 2) // 2, 3)


@pytest.mark.parametrize("t", [0, 1])
@pytest.mark.parametrize("p", [0, 1, 2])
def test_contracted_calls_match_mhs(cuda, t, p):
    from mhs_b200 import fullspace as fs
    d = golden("fullspace")
    mu, nu, eps = float(d["mu"]), float(d["nu"]), float(d["eps"][t])
    obs, tri = d["obs"], d["tris"][t]
    slip, force = d[f"slip_{t}_{p}"], d[f"force_{t}_{p}"]
    assert relmax(fs.displacement(obs, tri, slip, mu, nu, eps), d[f"disp_{t}_{p}"]) < TOL
    assert relmax(fs.stress(obs, tri, slip, mu, nu, eps), d[f"stress_{t}_{p}"]) < TOL
    assert relmax(fs.stress(obs, tri, slip, mu, nu, eps, subtract_eigenstress=False),
                  d[f"total_{t}_{p}"]) < TOL
    assert relmax(fs.eigenstress(obs, tri, slip, mu, nu, eps), d[f"eigen_{t}_{p}"]) < TOL
    assert relmax(fs.force_displacement(obs, tri, force, mu, nu, eps), d[f"fdisp_{t}_{p}"]) < TOL
    assert relmax(fs.force_stress(obs, tri, force, mu, nu, eps), d[f"fstress_{t}_{p}"]) < TOL


def test_device_inputs_single_point_and_analytic(cuda, monkeypatch):
    """CUDA tensors in -> CUDA tensors out; a (3,) point gives unbatched
    results; the analytic far field (closed form everywhere) against the
    oracle with its switch moved out of reach."""
    import torch
    from mhs_b200 import fullspace as fs
    d = golden("fullspace")
    mu, nu, eps = float(d["mu"]), float(d["nu"]), float(d["eps"][0])
    tri = d["tris"][0]
    obs = d["obs"][:30]
    u_dev = fs.force_displacement(torch.as_tensor(obs, device=cuda), tri, d["force_0_1"], mu, nu,
                                  eps)
    assert u_dev.is_cuda
    assert relmax(u_dev.cpu().numpy(), d["fdisp_0_1"][:30]) < TOL
    one = fs.displacement(obs[0], tri, d["slip_0_2"], mu, nu, eps)
    assert one.shape == (3,) and relmax(one, d["disp_0_2"][0]) < TOL
    lam = 2.0 * mu * nu / (1.0 - 2.0 * nu)
    near = d["obs"][:24]                     # within a few element lengths: the closed
    monkeypatch.setattr(O, "D_STAR", np.inf)  # form loses digits with distance
    ref = O.direct(near, tri, 1, mu, lam, eps, ("U", "G"))
    inf = fs.influence(near, tri, mu, nu, eps, order=1, want=("U", "G"), far_field="analytic")
    assert relmax(inf.U, ref["U"]) < 1e-11 and relmax(inf.G, ref["G"]) < 1e-11
