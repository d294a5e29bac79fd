"""Shared fixtures: the gpu marker, golden loading, relmax."""
from __future__ import annotations

import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def relmax(a, b) -> float:
    """max|a - b| / max|b| -- the norm-wise relative error mhs's gates use."""
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    ref = np.max(np.abs(b))
    diff = np.max(np.abs(a - b))
    return diff / ref if ref > 1e-300 else diff


def golden(name: str) -> dict:
    d = np.load(GOLDEN / f"{name}.npz")
    return {k: d[k] for k in d.files}


HOSTCHECK_DIR = ROOT / "tests" / "engine_host"
HOSTCHECK_LIB = HOSTCHECK_DIR / "libmhs_hostcheck.so"


def build_hostcheck() -> pathlib.Path:
    """CPU build of the device engine's arithmetic (tests only)."""
    srcs = [HOSTCHECK_DIR / "hostcheck.cpp", *sorted((ROOT / "mhs_b200" / "csrc").glob("*.cuh")),
            *sorted((ROOT / "mhs_b200" / "csrc").glob("*.h")),
            *sorted((ROOT / "mhs_b200" / "csrc").glob("*.inc"))]
    if HOSTCHECK_LIB.exists() and all(s.stat().st_mtime <= HOSTCHECK_LIB.stat().st_mtime for s in srcs):
        return HOSTCHECK_LIB
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o",
                    str(HOSTCHECK_LIB), str(HOSTCHECK_DIR / "hostcheck.cpp")], check=True)
    return HOSTCHECK_LIB


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from mhs_b200 import build
    build.build()
    return torch.device("cuda", 0)
