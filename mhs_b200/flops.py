"""Algorithmic flops of the fold stage and of the pair kernels, for the
roofline.

Two measurements multiply:

* per work unit, the operations of the engine's own arithmetic, counted by
  the op-counting host build ``csrc/opcount.cpp`` (the engine headers
  compiled with a counting scalar: add, subtract and multiply one flop each,
  a fused multiply-add two; divisions, square roots and library functions
  counted apart as special operations);
* per run, how many of each unit the fold kernel executed, from the device
  census (``_native.census``): band pairs, radial panels, polar-grid nodes
  per surface-load form (closed form, 12 x 12 rule, 8 x 8 rule) and
  near-field edge integrals per form (closed, small-|u| series, large-|u|
  series).

The per-unit counts are taken on representative inputs of each unit; every
unit except the per-pair breakpoint sort is branch-free straight-line
arithmetic in its form, so the counts do not depend on the inputs.

The pair kernels' work depends on each pair's geometry (closed form or
quadrature, edge forms, the image Q order), so ``pair_flops`` counts a
seeded uniform sample of (observer, source) pairs exactly and scales the
sample mean to all pairs.
"""
from __future__ import annotations

import ctypes
import pathlib
import shutil
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
SRC = HERE / "csrc" / "opcount.cpp"
LIB = HERE / "libmhs_opcount.so"
GL_MAX = 192

_lib = None


def build(force: bool = False) -> pathlib.Path:
    """Compile the op-counting build with the host C++ compiler."""
    deps = [SRC, *sorted((HERE / "csrc").glob("*.cuh")), *sorted((HERE / "csrc").glob("*.inc"))]
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in deps):
        return LIB
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        raise RuntimeError("no host C++ compiler for the op-counting build")
    subprocess.run([cxx, "-O1", "-std=c++17", "-fPIC", "-shared", "-o", str(LIB), str(SRC)],
                   check=True, capture_output=True, text=True)
    return LIB


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(str(build()))
        x = np.concatenate([np.polynomial.legendre.leggauss(n)[0] for n in range(1, GL_MAX + 1)])
        w = np.concatenate([np.polynomial.legendre.leggauss(n)[1] for n in range(1, GL_MAX + 1)])
        x, w = np.ascontiguousarray(x), np.ascontiguousarray(w)
        if lib.oc_set_gauss(x.ctypes.data_as(ctypes.c_void_p), w.ctypes.data_as(ctypes.c_void_p),
                            ctypes.c_int(x.size)) != 0:
            raise RuntimeError("op-count build: Gauss table size mismatch")
        _lib = lib
    return _lib


_TRI = np.array([[0.37, -0.81, -1.44], [1.92, 0.11, -2.63], [-0.25, 1.57, 0.0]])
_D = ctypes.c_double


def _ops():
    return (ctypes.c_longlong * 4)()


def _as(o):
    return {"flop": int(o[0]), "div": int(o[1]), "sqrt": int(o[2]), "special": int(o[3])}


def per_unit(order: int, want_h: bool, mu: float = 30.0, lam: float = 30.0,
             eps: float = 0.35) -> dict:
    """Operation counts of each fold work unit at this order and readout."""
    lib = _load()
    tri = np.ascontiguousarray(_TRI)
    tp = tri.ctypes.data_as(ctypes.c_void_p)
    out = {}
    for name, form, (ua, ub, rho2) in (("edge_closed", 0, (-0.5, 1.0, 0.3)),
                                       ("edge_small", 1, (0.1, 0.3, 1.0)),
                                       ("edge_large", 2, (3.0, 4.0, 1.0))):
        o = _ops()
        lib.oc_edge(order, form, _D(ua), _D(ub), _D(rho2), o)
        out[name] = _as(o)
    o = _ops()
    lib.oc_near_rest(order, tp, _D(eps), _D(mu), _D(lam), _D(0.8), _D(0.9), o)
    out["near"] = _as(o)
    for name, n, (px, py) in (("far12", 12, (30.0, 5.0)), ("far8", 8, (90.0, 10.0))):
        o = _ops()
        lib.oc_far(order, n, tp, _D(eps), _D(mu), _D(lam), _D(px), _D(py), o)
        out[name] = _as(o)
    o = _ops()
    lib.oc_node(order, 1 if want_h else 0, _D(0.05), o)
    out["node"] = _as(o)
    x = np.ascontiguousarray([0.6, 0.2, -0.05])
    po, pa = _ops(), _ops()
    lib.oc_pair(order, 1 if want_h else 0, tp, _D(eps), _D(mu), _D(lam),
                x.ctypes.data_as(ctypes.c_void_p), po, pa)
    out["pair"] = _as(po)
    out["panel"] = _as(pa)
    return out


def fold_flops(census: dict, order: int, want_h: bool, **kw) -> dict:
    """Algorithmic flops (and special operations) of the fold work a census
    counted.  Every band pair also evaluates the load at its receiver's foot,
    taken as one near node with three closed-form edges."""
    u = per_unit(order, want_h, **kw)
    nodes = census["near"] + census["far12"] + census["far8"]
    mult = {
        "edge_closed": census["edge_closed"] + 3 * census["pairs"],
        "edge_small": census["edge_small"],
        "edge_large": census["edge_large"],
        "near": census["near"] + census["pairs"],
        "far12": census["far12"],
        "far8": census["far8"],
        "node": nodes,
        "pair": census["pairs"],
        "panel": census["panels"],
    }
    tot = {k: 0 for k in ("flop", "div", "sqrt", "special")}
    for unit, n in mult.items():
        for k in tot:
            tot[k] += n * u[unit][k]
    tot["per_unit"] = u
    tot["nodes"] = nodes
    return tot


def pair_flops(obs, tris, eps, mu: float, lam: float, order: int, want_h: bool,
               samples: int = 4096, seed: int = 0) -> dict:
    """Algorithmic flops of the pair kernels over all (observer, source)
    pairs, from a seeded uniform sample counted exactly: the direct term
    (``k_pair``, every pair), the image R-family (``k_image_r``, pairs
    outside a fold band) and the image Q-family (``k_imageq``, likewise).
    Returns totals per kernel and the sample's share of fold-band pairs."""
    lib = _load()
    obs = np.ascontiguousarray(obs, dtype=np.float64)
    tris = np.ascontiguousarray(tris, dtype=np.float64)
    eps = np.broadcast_to(np.asarray(eps, dtype=np.float64), (tris.shape[0],))
    n_obs, n_src = obs.shape[0], tris.shape[0]
    rng = np.random.default_rng(seed)
    oi = rng.integers(0, n_obs, samples)
    si = rng.integers(0, n_src, samples)
    keys = ("flop", "div", "sqrt", "special")
    acc = {k: {q: 0 for q in keys} for k in ("direct", "image_r", "image_q")}
    n_band = 0
    qo = ctypes.c_int()
    band = ctypes.c_int()
    for o, s_ in zip(oi, si):
        t = np.ascontiguousarray(tris[s_])
        x = np.ascontiguousarray(obs[o])
        od, orr, oq = _ops(), _ops(), _ops()
        lib.oc_pair_terms(order, 1 if want_h else 0, t.ctypes.data_as(ctypes.c_void_p),
                          _D(float(eps[s_])), _D(mu), _D(lam), x.ctypes.data_as(ctypes.c_void_p),
                          od, orr, oq, ctypes.byref(qo), ctypes.byref(band))
        n_band += band.value
        for name, o_ in (("direct", od), ("image_r", orr), ("image_q", oq)):
            for i, q in enumerate(keys):
                acc[name][q] += int(o_[i])
    scale = n_obs * n_src / samples
    out = {name: {q: v * scale for q, v in d.items()} for name, d in acc.items()}
    out["k_pair"] = {q: out["direct"][q] + out["image_r"][q] for q in keys}
    out["k_imageq"] = out["image_q"]
    out["samples"] = samples
    out["band_share"] = n_band / samples
    return out


def imageq_flops(census: dict, order: int, want_h: bool, mu: float = 30.0,
                 lam: float = 30.0, eps: float = 0.35) -> dict:
    """Algorithmic flops of the image Q-family kernel from its census: its
    work per pair is a fixed part plus a part per rule point, taken from the
    op-counting build at two Gauss orders, times the pairs and the rule
    points (sum of n^2) the kernel counted."""
    lib = _load()
    tri = np.ascontiguousarray(_TRI)
    x = np.ascontiguousarray([4.0, -3.0, -2.0])
    per = {}
    for n in (8, 16):
        o = _ops()
        lib.oc_image_q_n(order, 1 if want_h else 0, tri.ctypes.data_as(ctypes.c_void_p), _D(eps),
                         _D(mu), _D(lam), x.ctypes.data_as(ctypes.c_void_p), n, o)
        per[n] = _as(o)
    out = {}
    for k in ("flop", "div", "sqrt", "special"):
        b = (per[16][k] - per[8][k]) / (256 - 64)   # per point
        a = per[8][k] - 64 * b                       # per pair
        out[k] = a * census["q_pairs"] + b * census["q_points"]
    out["per_point_flop"] = (per[16]["flop"] - per[8]["flop"]) / (256 - 64)
    return out

