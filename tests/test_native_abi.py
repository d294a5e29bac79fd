"""The C-ABI library loads on a CPU-only host and exports every entry point
include/mhs_b200.h declares (no compute calls without a GPU)."""
from __future__ import annotations

import ctypes
import re

import numpy as np

from conftest import ROOT


def _declared():
    text = (ROOT / "include" / "mhs_b200.h").read_text()
    return sorted(set(re.findall(r"\b(mhs_[a-z_]+)\s*\(", text)))


def test_library_builds_and_exports_every_declared_symbol():
    from mhs_b200 import _native, build
    build.build()
    lib = ctypes.CDLL(str(_native.LIB_PATH))
    names = _declared()
    assert "mhs_assemble" in names and "mhs_workspace_bytes" in names
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/mhs_b200.h but not exported"
    assert set(_native.EXPORTS) <= set(names)


def test_version_and_column_plan_host_helpers():
    from mhs_b200 import _native
    lib = _native.load()
    assert lib.mhs_version().startswith(b"mhs_b200")
    ids = np.array([[0, 1, 2, 5, 6, 7], [2, 1, 3, 6, 8, 9]], dtype=np.int64)
    cp = np.zeros(11, np.int32)
    ce = np.zeros(12, np.int32)
    assert lib.mhs_column_plan(ids.ctypes.data, 2, 10, cp.ctypes.data, ce.ctypes.data) == 0
    # column 6 is written by (s=0, k=4) then (s=1, k=3): entries in source order
    assert list(ce[cp[6]:cp[7]]) == [4, 9]
    assert cp[-1] == 12
    bad = ids.copy()
    bad[0, 0] = 99
    assert lib.mhs_column_plan(bad.ctypes.data, 2, 10, cp.ctypes.data, ce.ctypes.data) != 0
    assert b"out of range" in lib.mhs_last_error()


def test_request_struct_matches_header_field_order():
    from mhs_b200 import _native
    text = (ROOT / "include" / "mhs_b200.h").read_text()
    body = text[text.index("typedef struct mhs_request"):text.index("} mhs_request;")]
    flat = []
    for line in body.splitlines():
        m = re.match(r"\s*(?:const\s+)?[a-z_0-9]+\*?\s+([^;]+);", line.strip() and line or "")
        if m:
            flat += [f.strip().lstrip("*") for f in m.group(1).split(",")]
    assert [f[0] for f in _native.Request._fields_] == flat


def test_fullspace_struct_matches_header_field_order():
    from mhs_b200 import _native
    text = (ROOT / "include" / "mhs_b200.h").read_text()
    body = text[text.index("typedef struct mhs_fullspace_request"):
                text.index("} mhs_fullspace_request;")]
    flat = []
    for line in body.splitlines():
        m = re.match(r"\s*(?:const\s+)?[a-z_0-9]+\*?\s+([^;]+);", line.strip() and line or "")
        if m:
            flat += [f.strip().lstrip("*").split("[")[0] for f in m.group(1).split(",")]
    assert [f[0] for f in _native.FullspaceRequest._fields_] == flat
    assert ctypes.sizeof(_native.FullspaceRequest) == 168


def test_fullspace_refusals_before_any_launch():
    """The full-space API refuses what mhs's refuses, with its messages,
    before touching a device."""
    import pytest
    from mhs_b200 import fullspace as fs
    tri = np.array([[0.0, 0.0, -1.0], [1.0, 0.0, -1.0], [0.0, 1.0, -1.0]])
    with pytest.raises(ValueError, match="mu must be > 0"):
        fs.influence(np.zeros((1, 3)), tri, 0.0, 0.25, 0.1)
    with pytest.raises(ValueError, match="nu must be in"):
        fs.influence(np.zeros((1, 3)), tri, 1.0, 0.5, 0.1)
    with pytest.raises(ValueError, match="eps must be >= 0"):
        fs.influence(np.zeros((1, 3)), tri, 1.0, 0.25, -0.1)
    with pytest.raises(ValueError, match="tri must have shape"):
        fs.influence(np.zeros((1, 3)), tri[:2], 1.0, 0.25, 0.1)
    with pytest.raises(ValueError, match="degenerate triangle"):
        fs.influence(np.zeros((1, 3)), np.zeros((3, 3)), 1.0, 0.25, 0.1)
    with pytest.raises(ValueError, match="slip: 2 nodal values"):
        fs.displacement(np.zeros((1, 3)), tri, np.zeros((2, 3)), 1.0, 0.25, 0.1)
    with pytest.raises(ValueError, match="order=1 disagrees"):
        fs.force_stress(np.zeros((1, 3)), tri, np.zeros((1, 3)), 1.0, 0.25, 0.1, order=1)
    with pytest.raises(ValueError, match="far_field must be"):
        fs.influence(np.zeros((1, 3)), tri, 1.0, 0.25, 0.1, far_field="exact")
    assert np.allclose(fs.nodes(tri, 2)[3], [0.5, 0.0, -1.0])
    assert np.allclose(fs.traction(np.eye(3), tri), [0.0, 0.0, 1.0])
