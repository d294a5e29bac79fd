"""Seeded synthetic meshes and observers for the benchmark workloads.

No public dataset exists for these Green's-function assemblies, so every
workload is generated from a seed:

* ``planar_fault`` -- a rectangular fault meshed into rectangles, each split
  into two triangles with one consistent winding;
* ``rough_fault`` -- the same plane perturbed along its normal by a seeded
  Gaussian random field (sum of random Fourier modes with a Gaussian
  spectrum), tapered to zero over the top row so a surface-reaching edge
  stays exactly on z = 0;
* ``fault_network`` -- a vertical strike-slip plane with two 45-degree
  splays rooted along its bottom edge, sharing those vertices bit for bit;
* the workload builders for the five benchmark configurations.

Strike is measured clockwise from +y; the dip direction is strike rotated by
+90 degrees, pointing down into the body (z <= 0).
"""
from __future__ import annotations

import math

import numpy as np


def _strike_dip_vectors(strike_deg: float, dip_deg: float):
    th = math.radians(strike_deg)
    de = math.radians(dip_deg)
    s = np.array([math.sin(th), math.cos(th), 0.0])
    d = np.array([math.cos(de) * math.cos(th), -math.cos(de) * math.sin(th), -math.sin(de)])
    return s, d


def _grid_tris(P: np.ndarray) -> np.ndarray:
    """Triangles of a vertex grid ``P (nu+1, nv+1, 3)``: each cell split along
    its diagonal, wound so the vertex-order normal points up (n_z >= 0; a
    vertical plane keeps the grid's own consistent winding)."""
    nu, nv = P.shape[0] - 1, P.shape[1] - 1
    a = P[:-1, :-1]
    b = P[1:, :-1]
    c = P[1:, 1:]
    d = P[:-1, 1:]
    t1 = np.stack([a, b, c], axis=2)
    t2 = np.stack([a, c, d], axis=2)
    t = np.stack([t1, t2], axis=2).reshape(nu * nv * 2, 3, 3)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    if np.median(n[:, 2]) < 0.0:
        t = t[:, [0, 2, 1], :]
    return np.ascontiguousarray(t)


def planar_vertices(strike_deg, dip_deg, length, width, top_z, nu, nv, centre=(0.0, 0.0)):
    """Vertex grid (nu+1, nv+1, 3) of a plane: ``u`` along strike centred on
    ``centre``, ``v`` down dip from the top edge at ``top_z``."""
    s, d = _strike_dip_vectors(strike_deg, dip_deg)
    u = np.linspace(-0.5 * length, 0.5 * length, nu + 1)
    v = np.linspace(0.0, width, nv + 1)
    o = np.array([centre[0], centre[1], top_z])
    P = o + u[:, None, None] * s + v[None, :, None] * d
    P[:, 0, 2] = top_z            # the top edge exactly at its depth
    return P


def planar_fault(strike_deg, dip_deg, length, width, top_z, nu, nv, centre=(0.0, 0.0)):
    return _grid_tris(planar_vertices(strike_deg, dip_deg, length, width, top_z, nu, nv, centre))


def gaussian_field(pts2: np.ndarray, amplitude: float, corr_len: float, seed: int,
                   n_modes: int = 256) -> np.ndarray:
    """Stationary Gaussian random field with covariance
    ``amplitude^2 exp(-r^2 / (2 corr_len^2))`` at 2-D points, by random
    Fourier features (seeded)."""
    rng = np.random.default_rng(seed)
    k = rng.standard_normal((n_modes, 2)) / corr_len
    phase = rng.uniform(0.0, 2.0 * math.pi, n_modes)
    arg = pts2 @ k.T + phase
    return amplitude * math.sqrt(2.0 / n_modes) * np.cos(arg).sum(axis=1)


def rough_fault(strike_deg, dip_deg, length, width, top_z, nu, nv, amplitude, corr_len, seed,
                taper=2.0):
    """Planar fault perturbed along its normal at the vertices (shared
    vertices move together), tapered to zero within ``taper`` of the top."""
    P = planar_vertices(strike_deg, dip_deg, length, width, top_z, nu, nv)
    s, d = _strike_dip_vectors(strike_deg, dip_deg)
    n = np.cross(s, d)
    u = np.linspace(-0.5 * length, 0.5 * length, nu + 1)
    v = np.linspace(0.0, width, nv + 1)
    U, V = np.meshgrid(u, v, indexing="ij")
    f = gaussian_field(np.stack([U.ravel(), V.ravel()], axis=1), amplitude, corr_len, seed)
    f = f.reshape(U.shape) * np.minimum(1.0, V / taper)
    P = P + f[:, :, None] * n
    P[:, 0, 2] = top_z
    return _grid_tris(P)


def mean_edge(tris: np.ndarray) -> np.ndarray:
    e = np.linalg.norm(tris - np.roll(tris, 1, axis=1), axis=2)
    return e.mean(axis=1)


def fault_network(length=80.0, depth=15.0, splay_len=40.0, splay_width=15.0, nu=100, nv=15,
                  nv_splay=15):
    """Vertical strike-slip plane (x along strike, y = 0, z in [-depth, 0])
    and two 45-degree splays, one each side, rooted on its bottom edge
    (x in [0, splay_len] and [-splay_len, 0]) and sharing those vertices.
    Returns ``(tris, fault_id)``."""
    x = np.linspace(-0.5 * length, 0.5 * length, nu + 1)
    z = np.linspace(0.0, -depth, nv + 1)
    X, Z = np.meshgrid(x, z, indexing="ij")
    main = np.stack([X, np.zeros_like(X), Z], axis=-1)
    tris = [_grid_tris(main)]
    ids = [np.zeros(tris[0].shape[0], dtype=np.int64)]
    c = math.cos(math.radians(45.0))
    half = nu // 2
    for side, (lo, hi) in ((1.0, (half, nu)), (-1.0, (0, half))):
        xs = x[lo:hi + 1]
        w = np.linspace(0.0, splay_width, nv_splay + 1)
        # root row w = 0 on the main fault's bottom edge, rising away from it
        Y = side * c * w
        Zs = -depth + c * w
        P = np.stack(np.broadcast_arrays(xs[:, None], Y[None, :], Zs[None, :]), axis=-1).copy()
        P[:, 0, 1] = 0.0
        P[:, 0, 2] = -depth
        t = _grid_tris(P)
        tris.append(t)
        ids.append(np.full(t.shape[0], len(ids), dtype=np.int64))
    return np.concatenate(tris), np.concatenate(ids)


# ------------------------------------------------------------ workloads
def config1(seed: int = 0):
    """Planar fault, strike 0, dip 60, 20 x 10, top z = -1, 10 x 5 rectangles
    (100 triangles); 400 surface observers on a 20 x 20 grid over +-30 and
    200 uniform in [-30, 30]^2 x [-20, 0].  mu = lam = 30, eps = 0.1."""
    tris = planar_fault(0.0, 60.0, 20.0, 10.0, -1.0, 10, 5)
    g = np.linspace(-30.0, 30.0, 20)
    GX, GY = np.meshgrid(g, g, indexing="ij")
    surf = np.stack([GX.ravel(), GY.ravel(), np.zeros(GX.size)], axis=1)
    rng = np.random.default_rng(seed)
    box = np.column_stack([rng.uniform(-30, 30, 200), rng.uniform(-30, 30, 200),
                           rng.uniform(-20, 0, 200)])
    return dict(obs=np.concatenate([surf, box]), tris=tris, mu=30.0, lam=30.0, eps=0.1)


def config2(seed: int = 0, nu: int = 60, nv: int = 20):
    """Rough surface-reaching fault: 60 x 20 plane dipping 45, top at z = 0,
    normal roughness amplitude 0.5 and correlation length 5; 2 nu nv
    triangles (2,400 by default); eps per triangle 0.3 x its mean edge."""
    tris = rough_fault(0.0, 45.0, 60.0, 20.0, 0.0, nu, nv, 0.5, 5.0, seed)
    return dict(tris=tris, mu=30.0, lam=30.0, eps=0.3 * mean_edge(tris))


def config4():
    """Fault network for the continuous P2 interaction (about 6,000
    triangles, V + E about 12,000); top at z = 0."""
    tris, fid = fault_network()
    return dict(tris=tris, groups=fid, mu=30.0, lam=30.0, eps=0.1)


def batched_requests(n: int = 64, seed: int = 0, tri_range=(50, 5000), obs_range=(100, 20000),
                     kinds=("disp", "stress", "traction")):
    """Uneven requests: per request (seeded) a planar rectangular fault with a
    log-uniform triangle count, log-uniform observer count in a box 3x the
    fault extent (z <= 0), order in {0, 1, 2}, dip in [15, 90], top depth in
    [0, 5], kind uniform, traction normals uniform on the sphere, mu = 30,
    lam in [20, 40], eps = 0.1."""
    reqs = []
    for i in range(n):
        rng = np.random.default_rng([seed, i])
        n_tri = int(round(math.exp(rng.uniform(math.log(tri_range[0]), math.log(tri_range[1])))))
        n_obs = int(round(math.exp(rng.uniform(math.log(obs_range[0]), math.log(obs_range[1])))))
        order = int(rng.integers(0, 3))
        dip = float(rng.uniform(15.0, 90.0))
        top = -float(rng.uniform(0.0, 5.0))
        kind = kinds[int(rng.integers(0, len(kinds)))]
        cells = max(1, n_tri // 2)
        nv = max(1, int(round(math.sqrt(cells / 2.0))))
        nu = max(1, int(round(cells / nv)))
        length, width = float(nu), float(nv)
        tris = planar_fault(0.0, dip, length, width, top, nu, nv)
        ext = 3.0 * max(length, width)
        obs = np.column_stack([rng.uniform(-ext / 2, ext / 2, n_obs),
                               rng.uniform(-ext / 2, ext / 2, n_obs),
                               -rng.uniform(0.0, ext / 2, n_obs)])
        nrm = rng.standard_normal((n_obs, 3))
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        reqs.append(dict(kind=kind, order=order, obs=obs, tris=tris, normals=nrm, mu=30.0,
                         lam=float(rng.uniform(20.0, 40.0)), eps=0.1))
    return reqs


def serving_requests(n: int, seed: int = 0, rate_per_s: float = 20.0, tri_range=(100, 20000),
                     obs_range=(100, 50000), strike_strike=(10000, 20000)):
    """The serving stream: Poisson arrivals at `rate_per_s`; per request
    (seeded) kind uniform in {disp, stress, traction, interaction}, triangle
    count log-uniform in `tri_range`, observer count log-uniform in
    `obs_range`, order in {0, 1, 2}, a planar rectangular fault as in
    batched_requests, eps per triangle 0.3 x its mean edge.  The stream also
    carries scalar strike/strike interaction requests at each size of
    `strike_strike` (placed at evenly spaced positions in the stream).
    Returns a list of dicts with 'arrival_s' (seconds after the first)."""
    rng0 = np.random.default_rng([seed, 10 ** 6])
    gaps = rng0.exponential(1.0 / rate_per_s, n)
    arrival = np.concatenate([[0.0], np.cumsum(gaps[1:])])
    big_at = {int(round((k + 1) * n / (len(strike_strike) + 1))): sz
              for k, sz in enumerate(strike_strike)}
    kinds = ("disp", "stress", "traction", "interaction")
    reqs = []
    for i in range(n):
        rng = np.random.default_rng([seed, i])
        if i in big_at:
            n_tri, kind, order = big_at[i], "interaction", 0
        else:
            n_tri = int(round(math.exp(rng.uniform(math.log(tri_range[0]), math.log(tri_range[1])))))
            kind = kinds[int(rng.integers(0, len(kinds)))]
            order = int(rng.integers(0, 3))
        n_obs = int(round(math.exp(rng.uniform(math.log(obs_range[0]), math.log(obs_range[1])))))
        dip = float(rng.uniform(15.0, 90.0))
        top = -float(rng.uniform(0.0, 5.0))
        cells = max(1, n_tri // 2)
        nv = max(1, int(round(math.sqrt(cells / 2.0))))
        nu = max(1, int(round(cells / nv)))
        tris = planar_fault(0.0, dip, float(nu), float(nv), top, nu, nv)
        ext = 3.0 * max(nu, nv)
        obs = np.column_stack([rng.uniform(-ext / 2, ext / 2, n_obs),
                               rng.uniform(-ext / 2, ext / 2, n_obs),
                               -rng.uniform(0.0, ext / 2, n_obs)])
        nrm = rng.standard_normal((n_obs, 3))
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        r = dict(kind=kind, order=order, obs=obs, tris=tris, normals=nrm, mu=30.0,
                 lam=float(rng.uniform(20.0, 40.0)), eps=0.3 * mean_edge(tris),
                 arrival_s=float(arrival[i]))
        if i in big_at:
            r.update(receiver=("strike",), source=("strike",))
        reqs.append(r)
    return reqs
