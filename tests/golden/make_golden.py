"""Generate the golden fixtures: inputs and mhs's own outputs, as .npz.

Run where the reference package is importable, with its ``src/`` directory
in ``MHS_REFERENCE_SRC``::

    python tests/golden/make_golden.py [case ...]

Each case stores its inputs (``obs``, ``tris``, ``eps``, material, options)
and the arrays mhs returns for them.  Sizes are small so the whole set runs
in a few minutes on one core and the fixtures stay small; the GPU tests
compare the CUDA path against these arrays and the CPU tests pin the numpy
oracle against them.
"""
from __future__ import annotations

import os
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
if not os.environ.get("MHS_REFERENCE_SRC"):
    sys.exit("set MHS_REFERENCE_SRC to the reference's src/ directory (the tree that holds mhs/)")
sys.path.insert(0, os.environ["MHS_REFERENCE_SRC"])

import mhs  # noqa: E402  (the reference)

from mhs_b200 import synthetic  # noqa: E402


def _save(name: str, **arrays) -> None:
    np.savez_compressed(HERE / f"{name}.npz", **arrays)


def case_c1_subset():
    """Config-1 geometry, 60 of its 600 observers, disp + stress P0."""
    c = synthetic.config1(seed=0)
    obs = c["obs"][::10].copy()
    mat = mhs.Material(c["mu"], c["lam"])
    U = mhs.disp_matrix(obs, c["tris"], mat, c["eps"])
    S = mhs.stress_matrix(obs, c["tris"], mat, c["eps"])
    T = mhs.total_stress_matrix(obs, c["tris"], mat, c["eps"])
    _save("c1_subset", obs=obs, tris=c["tris"], mu=c["mu"], lam=c["lam"], eps=c["eps"],
          disp=U, stress=S, total_stress=T)


def _patch(seed=1, top=-0.6, dip=55.0, strike=20.0, nu=3, nv=2):
    tris = synthetic.planar_fault(strike, dip, 3.0, 2.0, top, nu, nv)
    rng = np.random.default_rng(seed)
    obs = np.concatenate([
        rng.uniform([-3, -3, -3], [3, 3, 0], (16, 3)),        # near the patch
        rng.uniform([-25, -25, -15], [25, 25, 0], (8, 3)),     # far field
    ])
    return tris, obs


def case_orders():
    """A 12-triangle patch, 24 observers, orders 0/1/2: disp, stress,
    total stress and traction (random unit normals), scalar eps."""
    tris, obs = _patch()
    rng = np.random.default_rng(7)
    nrm = rng.standard_normal((obs.shape[0], 3))
    mat = mhs.Material(30.0, 20.0)
    out = dict(obs=obs, tris=tris, mu=30.0, lam=20.0, eps=0.15, normals=nrm)
    for p in (0, 1, 2):
        out[f"disp_p{p}"] = mhs.disp_matrix(obs, tris, mat, 0.15, order=p)
        out[f"stress_p{p}"] = mhs.stress_matrix(obs, tris, mat, 0.15, order=p)
        out[f"total_p{p}"] = mhs.total_stress_matrix(obs, tris, mat, 0.15, order=p)
        out[f"traction_p{p}"] = mhs.traction_matrix(obs, nrm, tris, mat, 0.15, order=p)
    _save("orders", **out)


def case_eps_per_tri():
    """Per-triangle eps and a lam < mu material, P0 and P1."""
    tris, obs = _patch(seed=3, top=-1.2, dip=75.0, strike=-35.0)
    eps = np.linspace(0.08, 0.3, tris.shape[0])
    mat = mhs.Material(25.0, 12.0)
    out = dict(obs=obs, tris=tris, mu=25.0, lam=12.0, eps=eps)
    for p in (0, 1):
        out[f"disp_p{p}"] = mhs.disp_matrix(obs, tris, mat, eps, order=p)
        out[f"stress_p{p}"] = mhs.stress_matrix(obs, tris, mat, eps, order=p)
    _save("eps_per_tri", **out)


def case_interaction():
    """Self-interaction on a 24-triangle buried fault, P0 full 3x3, P1
    (strike, dip) x all, P2 strike x strike; plus a rectangular block with
    rows=."""
    tris = synthetic.planar_fault(10.0, 50.0, 6.0, 3.0, -1.0, 4, 3)
    mat = mhs.Material(30.0, 30.0)
    out = dict(tris=tris, mu=30.0, lam=30.0, eps=0.1)
    out["int_p0"] = mhs.interaction_matrix(tris, mat, 0.1)
    out["int_p1"] = mhs.interaction_matrix(tris, mat, 0.1, order=1, receiver=("strike", "dip"))
    out["int_p2"] = mhs.interaction_matrix(tris, mat, 0.1, order=2, receiver="strike",
                                           source="strike")
    out["int_p0_rows"] = mhs.interaction_matrix(tris, mat, 0.1, rows=(5, 17))
    out["int_p0_noeig"] = mhs.interaction_matrix(tris, mat, 0.1, subtract_eigenstress=False)
    _save("interaction", **out)


def case_fold():
    """Surface-reaching fault (top at z = 0): the top row folds.  Interaction
    P0 (3x3), stress and disp at near-surface observers, with and without
    the fold, and the P1 interaction."""
    tris = synthetic.planar_fault(0.0, 60.0, 3.0, 1.6, 0.0, 3, 2)
    rng = np.random.default_rng(11)
    obs = np.column_stack([rng.uniform(-2.0, 2.0, 6), rng.uniform(-1.0, 2.0, 6),
                           -rng.uniform(0.0, 0.9, 6)])
    mat = mhs.Material(30.0, 25.0)
    eps = 0.12
    out = dict(tris=tris, obs=obs, mu=30.0, lam=25.0, eps=eps)
    out["int_p0"] = mhs.interaction_matrix(tris, mat, eps)
    out["stress_p0"] = mhs.stress_matrix(obs, tris, mat, eps)
    out["stress_p0_nofold"] = mhs.stress_matrix(obs, tris, mat, eps, fold=False)
    out["disp_p0"] = mhs.disp_matrix(obs, tris, mat, eps)
    out["int_p1"] = mhs.interaction_matrix(tris, mat, eps, order=1, receiver=("strike",),
                                           source=("strike", "dip"))
    _save("fold", **out)


def case_continuous():
    """Continuous P2 interaction on a two-group network (buried) and its
    traction matrix at a few observers."""
    a = synthetic.planar_fault(0.0, 90.0, 2.0, 1.0, -1.0, 2, 1)
    b = synthetic.planar_fault(30.0, 60.0, 1.5, 1.0, -1.2, 2, 1, centre=(2.5, 0.5))
    tris = np.concatenate([a, b])
    groups = np.array([0] * a.shape[0] + [1] * b.shape[0])
    mat = mhs.Material(30.0, 30.0)
    sn = mhs.shared_nodes(tris, groups=groups)
    out = dict(tris=tris, groups=groups, mu=30.0, lam=30.0, eps=0.1, ids=sn.ids,
               coords=sn.coords, normals=sn.normals)
    out["int_cont"] = mhs.interaction_matrix(tris, mat, 0.1, order=2, layout="continuous",
                                             shared=sn, source=("strike", "dip"))
    rng = np.random.default_rng(5)
    obs = rng.uniform([-2, -2, -3], [4, 2, 0], (10, 3))
    nrm = rng.standard_normal((10, 3))
    out["obs"] = obs
    out["obs_normals"] = nrm
    out["trac_cont"] = mhs.traction_matrix(obs, nrm, tris, mat, 0.1, order=2,
                                           layout="continuous", shared=sn)
    _save("continuous", **out)


def case_rough_surface():
    """Scaled-down config 2: rough surface-reaching fault, per-triangle eps,
    full 3x3 interaction with the fold."""
    c = synthetic.config2(seed=3, nu=4, nv=3)
    mat = mhs.Material(c["mu"], c["lam"])
    K = mhs.interaction_matrix(c["tris"], mat, c["eps"])
    _save("rough_surface", tris=c["tris"], eps=c["eps"], mu=c["mu"], lam=c["lam"], int_p0=K)


def case_signatures():
    """The public functions' signatures as mhs declares them (parameter
    names, kinds and defaults), for the CPU test that pins the drop-in's."""
    import inspect
    import json
    names = ["disp_matrix", "stress_matrix", "total_stress_matrix", "eigenstress_matrix",
             "elastic_strain_matrix", "traction_matrix", "interaction_matrix",
             "collocation_points", "shared_nodes"]
    sig = {}
    for n in names:
        sig[n] = [[p.name, p.kind.name, None if p.default is inspect.Parameter.empty
                   else repr(p.default)] for p in inspect.signature(getattr(mhs, n)).parameters.values()]
    (HERE / "signatures.json").write_text(json.dumps(sig, indent=1) + "\n")


def case_c1_full():
    """Config 1 in full: 600 observers x 100 triangles, disp and stress P0."""
    c = synthetic.config1(seed=0)
    mat = mhs.Material(c["mu"], c["lam"])
    U = mhs.disp_matrix(c["obs"], c["tris"], mat, c["eps"])
    S = mhs.stress_matrix(c["obs"], c["tris"], mat, c["eps"])
    _save("c1_full", obs=c["obs"], tris=c["tris"], mu=c["mu"], lam=c["lam"], eps=c["eps"],
          disp=U, stress=S)


def _band_rows(pts, tris, eps):
    """Receivers that take the folded image of at least one source."""
    from mhs.kernels import fold
    eps = np.broadcast_to(np.asarray(eps, float), (tris.shape[0],))
    hit = np.zeros(pts.shape[0], bool)
    for s in range(tris.shape[0]):
        if fold.straddles(tris[s], eps[s]):
            hit[fold.band(pts, tris[s], eps[s])] = True
    return np.flatnonzero(hit)


def _one_row(args):
    """Worker: one receiver row of an interaction matrix through rows=."""
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    r, tris, mu, lam, eps, kw = args
    import mhs as m
    kw = dict(kw)
    if kw.get("layout") == "continuous":
        kw["shared"] = m.shared_nodes(tris, groups=kw.pop("groups"))
    return m.interaction_matrix(tris, m.Material(mu, lam), eps, rows=(r, r + 1), **kw)[0]


def _rows(tris, mu, lam, eps, rows, kw, workers=8):
    import concurrent.futures as cf
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with cf.ProcessPoolExecutor(workers, mp_context=ctx) as ex:
        return np.stack(list(ex.map(_one_row, [(int(r), tris, mu, lam, eps, kw) for r in rows])))


def case_c2_rows():
    """Config 2 at its full size (2,400 triangles, per-triangle eps, fold on):
    8 seeded fold-band receiver rows and 8 other rows of the full 3x3
    interaction matrix, each through rows=(r, r + 1)."""
    c = synthetic.config2(seed=0)
    tris, eps = c["tris"], c["eps"]
    pts = mhs.collocation_points(tris)
    band = _band_rows(pts, tris, eps)
    other = np.setdiff1d(np.arange(pts.shape[0]), band)
    rng = np.random.default_rng(2)
    rows = np.concatenate([np.sort(rng.choice(band, 8, replace=False)),
                           np.sort(rng.choice(other, 8, replace=False))])
    K = _rows(tris, c["mu"], c["lam"], eps, rows, {})
    _save("c2_rows", tris=tris, eps=eps, mu=c["mu"], lam=c["lam"], rows=rows, n_band=8, K=K)


def case_c4_rows():
    """Config 4 at its full size (3-fault network, continuous P2, source =
    (strike, dip), fold on at the trace): 4 seeded fold-band rows and 4
    other rows, each through rows=(r, r + 1)."""
    c = synthetic.config4()
    tris, groups = c["tris"], c["groups"]
    sn = mhs.shared_nodes(tris, groups=groups)
    band = _band_rows(sn.coords, tris, c["eps"])
    other = np.setdiff1d(np.arange(sn.n), band)
    rng = np.random.default_rng(4)
    rows = np.concatenate([np.sort(rng.choice(band, 4, replace=False)),
                           np.sort(rng.choice(other, 4, replace=False))])
    kw = dict(order=2, layout="continuous", groups=groups, source=("strike", "dip"))
    K = _rows(tris, c["mu"], c["lam"], c["eps"], rows, kw)
    _save("c4_rows", tris=tris, groups=groups, eps=c["eps"], mu=c["mu"], lam=c["lam"],
          rows=rows, n_band=4, n_cols=sn.n, K=K)


def case_fullspace():
    """The full-space single-triangle API (mhs.fullspace.api): nodal influence
    tensors U, H, E (slip source) and G, S (force source) of two triangles at
    near and far observers, orders 0-2, hybrid and quadrature far fields, and
    the contracted calls (displacement, stress, eigenstress,
    force_displacement, force_stress) for seeded nodal slip and force."""
    from mhs.fullspace import api
    rng = np.random.default_rng(21)
    tris = np.array([[[0.0, 0.0, -1.0], [1.2, 0.2, -1.4], [0.3, 1.1, -0.8]],
                     [[2.0, -1.0, 0.5], [3.5, -0.6, 1.2], [2.4, 0.8, 0.9]]])
    obs = np.concatenate([rng.uniform(-1.0, 2.0, (24, 3)), rng.uniform(-40.0, 40.0, (8, 3)),
                          rng.uniform(-400.0, 400.0, (4, 3))])
    mu, nu = 30.0, 0.27
    out = {"tris": tris, "obs": obs, "mu": np.array(mu), "nu": np.array(nu),
           "eps": np.array([0.1, 0.35])}
    for t in range(2):
        for P in (0, 1, 2):
            K = (P + 1) * (P + 2) // 2
            for ff in ("hybrid", "quadrature"):
                inf = api.influence(obs, tris[t], mu, nu, out["eps"][t], order=P,
                                    want=("U", "H", "E", "G", "S"), far_field=ff)
                for k in ("U", "H", "E", "G", "S"):
                    out[f"{k}_{t}_{P}_{ff}"] = getattr(inf, k)
            slip = rng.standard_normal((K, 3))
            force = rng.standard_normal((K, 3))
            e = out["eps"][t]
            out[f"slip_{t}_{P}"] = slip
            out[f"force_{t}_{P}"] = force
            out[f"disp_{t}_{P}"] = api.displacement(obs, tris[t], slip, mu, nu, e)
            out[f"stress_{t}_{P}"] = api.stress(obs, tris[t], slip, mu, nu, e)
            out[f"total_{t}_{P}"] = api.stress(obs, tris[t], slip, mu, nu, e,
                                               subtract_eigenstress=False)
            out[f"eigen_{t}_{P}"] = api.eigenstress(obs, tris[t], slip, mu, nu, e)
            out[f"fdisp_{t}_{P}"] = api.force_displacement(obs, tris[t], force, mu, nu, e)
            out[f"fstress_{t}_{P}"] = api.force_stress(obs, tris[t], force, mu, nu, e)
    _save("fullspace", **out)


CASES = {f.__name__[5:]: f for f in (case_c1_subset, case_orders, case_eps_per_tri,
                                     case_interaction, case_fold, case_continuous,
                                     case_rough_surface, case_signatures, case_c1_full,
                                     case_c2_rows, case_c4_rows, case_fullspace)}

if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for n in names:
        t = time.time()
        CASES[n]()
        print(f"{n}: {time.time() - t:.1f} s", flush=True)
