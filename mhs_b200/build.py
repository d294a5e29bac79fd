"""Build ``libmhs_b200.so`` in-tree with nvcc for sm_100a.

The library is one host unit (``csrc/mhs_b200.cu``: the C ABI) plus kernel
units: ``csrc/unit.cu`` compiled once per (order, readout class, far-field
precision) and once per order for the per-term diagnostics.  The units are
compiled in parallel into ``_build/`` and linked into one shared object; a
unit is recompiled when any source is newer than its object."""
from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libmhs_b200.so"
OBJ = HERE.parent / "_build"
INCLUDE = HERE.parent / "include"

NVCC_FLAGS = [
    "-std=c++17", "-O3", "--expt-relaxed-constexpr",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-Xcompiler", "-fPIC",
    "-diag-suppress", "550",
]

# (object name, extra defines, source): the host unit, 18 kernel units, 3 diagnostic units.
UNITS = [("host", [], "mhs_b200.cu")]
UNITS += [(f"unit_{p}_{kc}_{rf}",
           [f"-DMHS_UNIT_P={p}", f"-DMHS_UNIT_KC={kc}", f"-DMHS_UNIT_RF={rf}"], "unit.cu")
          for p in range(3) for kc in range(3) for rf in range(2)]
UNITS += [(f"terms_{p}", [f"-DMHS_UNIT_TERMS={p}"], "unit.cu") for p in range(3)]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + \
        sorted(CSRC.glob("*.inc")) + sorted(INCLUDE.glob("*.h"))


def _newest_source(unit_src: str | None = None) -> float:
    """Newest modification time of the headers, plus one unit's own source
    (every source when unit_src is None)."""
    files = [s for s in sources() if s.suffix != ".cu" or unit_src is None or s.name == unit_src]
    return max(s.stat().st_mtime for s in files)


def stale() -> bool:
    if not LIB.exists():
        return True
    return _newest_source() > LIB.stat().st_mtime


def _compile(name, defs, src, extra, force):
    obj = OBJ / f"{name}.o"
    if not force and obj.exists() and obj.stat().st_mtime >= _newest_source(src):
        return name, None
    cmd = [_nvcc(), *NVCC_FLAGS, *extra, *defs]
    if name != "host":
        cmd += ["-Xcompiler", "-fvisibility=hidden"]
    cmd += ["-c", "-o", str(obj), str(CSRC / src)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {name} ({r.returncode}):\n{r.stderr[-4000:]}")
    return name, r.stderr


def build(force: bool = False, verbose: bool = False, extra=(), jobs: int | None = None) -> pathlib.Path:
    if not force and not stale():
        return LIB
    OBJ.mkdir(exist_ok=True)
    jobs = jobs or os.cpu_count() or 4
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_compile, n, d, s, list(extra), force) for n, d, s in UNITS]
        for f in cf.as_completed(futs):
            name, log = f.result()
            if verbose and log:
                print(f"== {name}\n{log}", file=sys.stderr)
    objs = [str(OBJ / f"{n}.o") for n, _, _ in UNITS]
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp), *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({r.returncode}):\n{r.stderr[-4000:]}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
    print(LIB)
