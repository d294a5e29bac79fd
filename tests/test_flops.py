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
    # the 12 x 12 and 8 x 8 rules differ only in their 144 vs 64 points
    for P, u in units.items():
        per_point = (u["far12"]["flop"] - u["far8"]["flop"]) / 80.0
        assert u["far12"]["sqrt"] - u["far8"]["sqrt"] == 80
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
