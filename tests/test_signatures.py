"""The drop-in contract: every public function keeps mhs's signature --
parameter names, order, kinds and defaults -- as recorded from mhs itself in
``tests/golden/signatures.json`` (``make_golden.py signatures``).  The matrix
functions add exactly one keyword-only parameter at the end,
``precision="fp64"``; nothing else may differ."""
from __future__ import annotations

import inspect
import json

import pytest

from conftest import GOLDEN

SIGS = json.loads((GOLDEN / "signatures.json").read_text())
EXTRA = ["precision", "KEYWORD_ONLY", repr("fp64")]
WITH_PRECISION = {"disp_matrix", "stress_matrix", "total_stress_matrix", "eigenstress_matrix",
                  "elastic_strain_matrix", "traction_matrix", "interaction_matrix"}


def _params(fn):
    return [[p.name, p.kind.name, None if p.default is inspect.Parameter.empty else repr(p.default)]
            for p in inspect.signature(fn).parameters.values()]


@pytest.mark.parametrize("name", sorted(SIGS))
def test_signature_matches_mhs(name):
    import mhs_b200
    got = _params(getattr(mhs_b200, name))
    want = [list(p) for p in SIGS[name]]
    if name in WITH_PRECISION:
        assert got[-1] == EXTRA, f"{name}: last parameter {got[-1]}"
        got = got[:-1]
    assert got == want


def test_no_bare_strain_matrix():
    """mhs has no strain_matrix (a cutde-style one would return total
    stress); neither does the drop-in."""
    import mhs_b200
    assert not hasattr(mhs_b200, "strain_matrix")
