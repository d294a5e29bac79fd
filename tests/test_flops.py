"""The op-counting host build that bench.py's roofline uses: it builds, and
its per-unit counts have the structure of the arithmetic they count."""
from __future__ import annotations

import pytest


@pytest.fixture(scope="module")
def units():
    from mhs_b200 import flops
    return {P: flops.per_unit(P, True) for P in (0, 1, 2)}


def test_units_are_counted(units):
    for P, u in units.items():
        for name, ops in u.items():
            assert ops["flop"] > 0, (P, name)


def test_far_rules_scale_with_their_points(units):
    # the 12 x 12 and 8 x 8 rules differ only in their 144 vs 64 points (the
    # rule is walked once per group of shape nodes: at most 64 of the 22
    # surface-load moments at a time, so P1 in two passes and P2 in three)
    for P, u in units.items():
        passes = {0: 1, 1: 2, 2: 3}[P]
        per_point = (u["far12"]["flop"] - u["far8"]["flop"]) / 80.0
        assert u["far12"]["sqrt"] - u["far8"]["sqrt"] == 80 * passes
        fixed = u["far8"]["flop"] - 64 * per_point   # geometry and the sigma_zz contraction
        assert 0 < fixed < 0.1 * u["far8"]["flop"], P


def test_series_edges_cost_their_32_terms(units):
    # small- and large-|u| series sum 32 terms per (m, k); the closed form
    # is a handful of operations and a few divisions
    for P, u in units.items():
        assert u["edge_small"]["flop"] > 10 * u["edge_closed"]["flop"]
        assert u["edge_large"]["flop"] > 10 * u["edge_closed"]["flop"]
        assert 1 <= u["edge_closed"]["div"] <= 6


def test_order_raises_the_work(units):
    for name in ("near", "far12", "far8", "node", "pair"):
        assert units[0][name]["flop"] < units[1][name]["flop"] < units[2][name]["flop"], name


def test_fold_flops_combines_a_census():
    from mhs_b200 import flops
    census = {"pairs": 2, "panels": 40, "near": 1000, "far12": 400, "far8": 100,
              "edge_closed": 1800, "edge_small": 900, "edge_large": 300}
    u = flops.per_unit(0, True)
    tot = flops.fold_flops(census, 0, True)
    expect = (1000 + 2) * u["near"]["flop"] + 400 * u["far12"]["flop"] + 100 * u["far8"]["flop"] \
        + (1800 + 6) * u["edge_closed"]["flop"] + 900 * u["edge_small"]["flop"] \
        + 300 * u["edge_large"]["flop"] + 1500 * u["node"]["flop"] + 2 * u["pair"]["flop"] \
        + 40 * u["panel"]["flop"]
    assert tot["flop"] == expect


def test_pair_terms_counts():
    """The pair kernels' counts: every pair runs the direct term; a pair in a
    fold band runs no image term; a far pair's direct term takes the 12 x 12
    rule (a fixed count), and the image Q-family costs in proportion to its
    order's points."""
    import ctypes
    import numpy as np
    from mhs_b200 import flops
    lib = flops._load()
    tri = np.ascontiguousarray([[0.0, 0.0, -0.02], [1.0, 0.0, -0.6], [0.0, 1.0, -0.4]])

    def terms(x):
        od, orr, oq = flops._ops(), flops._ops(), flops._ops()
        qo, band = ctypes.c_int(), ctypes.c_int()
        x = np.ascontiguousarray(x, dtype=np.float64)
        lib.oc_pair_terms(0, 1, tri.ctypes.data_as(ctypes.c_void_p), flops._D(0.05),
                          flops._D(30.0), flops._D(30.0), x.ctypes.data_as(ctypes.c_void_p),
                          od, orr, oq, ctypes.byref(qo), ctypes.byref(band))
        return flops._as(od), flops._as(orr), flops._as(oq), qo.value, band.value

    d, r, q, n, band = terms([0.3, 0.3, -0.01])          # in the band of a straddler
    assert band == 1 and d["flop"] > 0 and r["flop"] == 0 and q["flop"] == 0
    far_a = terms([25.0, 3.0, -4.0])
    far_b = terms([-20.0, 14.0, -9.0])
    assert far_a[4] == 0 and far_a[0]["flop"] == far_b[0]["flop"] > 0
    assert far_a[3] == far_b[3] == 8 and far_a[2]["flop"] == far_b[2]["flop"]
    near = terms([0.4, 0.2, -0.8])
    assert near[4] == 0 and near[3] > 8 and near[2]["flop"] > far_a[2]["flop"] * (near[3] / 8) ** 2 * 0.9


def test_imageq_flops_from_its_census():
    """The image Q-family's work is a fixed part per pair plus a part per rule
    point: doubling the points of a census adds the per-point part."""
    from mhs_b200 import flops
    a = flops.imageq_flops({"q_pairs": 10, "q_points": 640}, 0, True)
    b = flops.imageq_flops({"q_pairs": 10, "q_points": 1280}, 0, True)
    assert a["per_point_flop"] > 100
    assert abs((b["flop"] - a["flop"]) - 640 * a["per_point_flop"]) < 1e-6 * b["flop"]


@pytest.mark.gpu
def test_gpu_census_counts_image_q_pairs(cuda):
    """k_imageq counts every pair outside a fold band (here, a buried fault:
    all of them), each with at least the floor order's 64 points."""
    import mhs_b200 as m
    from mhs_b200 import _native, synthetic
    tris = synthetic.planar_fault(10.0, 60.0, 6.0, 3.0, -2.0, 6, 3)
    n = tris.shape[0]
    _native.census(True)
    m.interaction_matrix(tris, m.Material(30.0, 30.0), 0.1)
    cen = _native.census_read()
    _native.census(False)
    assert cen["pairs"] == 0 and cen["q_pairs"] == n * n
    assert cen["q_points"] >= 64 * n * n
