"""CPU restatement of mhs's Green's-function assembly in numpy.

TEST INFRASTRUCTURE ONLY.  This module is the oracle the CUDA path is
checked against: ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline of ``bench.py`` may import it; the ``mhs_b200`` package never does.
It restates mhs's algorithm (mhs @ the mounted revision, pure numpy) term by
term -- edge primitives, moment recursion, far-field quadrature, the
Kelvin-Cortez kernels, the image R- and Q-families, the fold and the
assembly loop -- and is pinned against outputs of mhs itself
(``tests/golden``, generated by ``tests/golden/make_golden.py``).

The image coefficients come from ``oracle/image_table.npz``, extracted from
mhs's generated table by ``oracle/make_table.py``.

Layout conventions follow mhs: per source, ``U (N, K, 3, 3)`` [obs, node,
component, slip] and ``H (N, K, 3, 3, 3)`` [obs, node, a, b, slip].
"""
from __future__ import annotations

import functools
import itertools
import math
import pathlib
from fractions import Fraction

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent

# constants (mhs/defaults.py:60-143, mhs/fullspace/defaults.py:20-35)
D_STAR, D_STAR_DISTANT = 10.0, 40.0
FAR_N, FAR_N_DISTANT = 12, 8
SERIES_U_OVER_RHO, SMALL_U_OVER_RHO, SERIES_TERMS = 2.0, 0.5, 32
Q_BUDGET_C, Q_MIN, Q_MAX = 10.0, 8, 192
FOLD_SRC_EPS, FOLD_BAND_EPS, FOLD_REACH_EPS = 3.0, 10.0, 60.0
FOLD_NR, FOLD_NA = 6, 4
FOLD_MARGIN_EPS, FOLD_FINE_EPS, FOLD_MED_EPS, FOLD_COARSE = 5.0, 0.25, 2.0, 24
FOLD_FINE_SUB_EPS, FOLD_MED_SUB_EPS, FOLD_R1_DIAM = 6.0, 16.0, 8.0
MIRROR_SLIP_SIGN = np.array([-1.0, -1.0, 1.0])


# ------------------------------------------------------------ quadrature
@functools.lru_cache(maxsize=None)
def _gl01(n):
    """Gauss-Legendre on [0, 1] (numpy's nodes)."""
    x, w = np.polynomial.legendre.leggauss(n)
    return 0.5 * (x + 1.0), 0.5 * w


@functools.lru_cache(maxsize=None)
def _tri_rule(n):
    """Collapsed product rule on the reference triangle (moments.py:401-424)."""
    g, w = _gl01(n)
    gi, gj = np.meshgrid(g, g, indexing="ij")
    wi, wj = np.meshgrid(w, w, indexing="ij")
    return gi.ravel(), (gj * (1.0 - gi)).ravel(), (wi * wj * (1.0 - gi)).ravel()


# -------------------------------------------------------------- geometry
class Frame:
    """Triangle frame: e1 along v2 - v1, nhat from the vertex order,
    centroid origin, L the longest edge (fullspace/frame.py:282-302)."""

    def __init__(self, tri):
        v = np.asarray(tri, float).reshape(3, 3)
        e1v, e2v = v[1] - v[0], v[2] - v[0]
        nn = np.cross(e1v, e2v)
        a2 = np.linalg.norm(nn)
        self.v = v
        self.n = nn / a2
        self.e1 = e1v / np.linalg.norm(e1v)
        self.e2 = np.cross(self.n, self.e1)
        self.c = v.mean(axis=0)
        d = v - self.c
        self.p = np.stack([d @ self.e1, d @ self.e2], axis=1)
        self.area = 0.5 * a2
        self.L = max(np.linalg.norm(v[1] - v[0]), np.linalg.norm(v[2] - v[1]),
                     np.linalg.norm(v[0] - v[2]))
        self.abc = np.linalg.inv(np.vstack([np.ones(3), self.p.T]))
        self.basis = (self.e1, self.e2, self.n)

    def to_plane(self, x):
        d = x - self.c
        return d @ self.n, d @ self.e1, d @ self.e2


def _lattice(P):
    if P == 0:
        return [(0, 0, 0)]
    out = [(P, 0, 0), (0, P, 0), (0, 0, P)]
    for i, j in ((0, 1), (1, 2), (2, 0)):
        for s in range(1, P):
            a = [0, 0, 0]
            a[i], a[j] = P - s, s
            out.append(tuple(a))
    return out


def _pmul(A, B, deg):
    out = {}
    for (a, b), x in A.items():
        for (c, d), y in B.items():
            if a + b + c + d <= deg:
                out[(a + c, b + d)] = out.get((a + c, b + d), 0.0) + x * y
    return out


def shape_poly(f, P, X0, X1):
    """Coefficients {(a, b): (N, K)} of the order-P shape functions in
    xi = eta - X (fullspace/shape.py:114-147)."""
    N = np.shape(X0)[0]
    if P == 0:
        return {(0, 0): np.ones((N, 1))}
    A, B, C = f.abc[:, 0], f.abc[:, 1], f.abc[:, 2]
    lam0 = A[None, :] + X0[:, None] * B[None, :] + X1[:, None] * C[None, :]
    polys = []
    for alpha in _lattice(P):
        poly = {(0, 0): np.ones(N)}
        for i in range(3):
            for j in range(alpha[i]):
                fac = {(0, 0): P * lam0[:, i] / (j + 1) - j / (j + 1),
                       (1, 0): np.full(N, P * B[i] / (j + 1)),
                       (0, 1): np.full(N, P * C[i] / (j + 1))}
                poly = _pmul(poly, fac, P)
        polys.append(poly)
    keys = [(a, b) for a in range(P + 1) for b in range(P + 1 - a)]
    return {k: np.stack([np.broadcast_to(pl.get(k, 0.0), (N,)) for pl in polys], axis=1)
            for k in keys}


# ------------------------------------------------------- degree bookkeeping
def close_degrees(need):
    """Degrees the recursion consumes (fullspace/moments.py:94-116)."""
    deg = dict(need)
    n = max(deg)
    while True:
        d = deg.get(n, -1)
        if d >= 2:
            deg[n - 2] = max(deg.get(n - 2, -1), d - 2)
        if n - 2 < min(deg):
            break
        n -= 2
    deg[3] = max(deg.get(3, -1), 0)
    for n in list(deg):
        if n >= 5:
            for m in range(3, n, 2):
                deg[m] = max(deg.get(m, -1), 0)
        if n <= 1:
            for m in range(n, 4, 2):
                deg[m] = max(deg.get(m, -1), 0)
    return {n: d for n, d in deg.items() if d >= 0}


def edge_degrees(deg):
    e = {}
    for n, d in deg.items():
        if d >= 1:
            e[n - 2] = max(e.get(n - 2, -1), d - 1)
    for n in deg:
        if n >= 5:
            e[n - 2] = max(e.get(n - 2, -1), 0)
        if n <= 1:
            e[n] = max(e.get(n, -1), 0)
    return e


NEED_U = {3: 1, 5: 3}
NEED_H = {3: 0, 5: 2, 7: 4}
NEED_E = {7: 0}
NEED_G = {1: 0, 3: 2}
NEED_S = {3: 1, 5: 3}
NEED_IMG = {3: 1, 5: 3, 7: 4, 9: 5}


# ------------------------------------------------------- edge primitives
@functools.lru_cache(maxsize=None)
def _binom_half(m, j):
    a, out = Fraction(-m, 2), Fraction(1)
    for i in range(j):
        out *= (a - i) / (i + 1)
    return float(out)


def _edge_closed(ua, ub, rho2, spec):
    Ra = np.sqrt(ua * ua + rho2)
    Rb = np.sqrt(ub * ub + rho2)
    dR = (ub - ua) * (ub + ua) / (Ra + Rb)
    J, K, P = {}, {}, {}

    def dJ(m):
        if m in J:
            return J[m]
        if m == 1:
            out = np.empty_like(ua)
            pos = ua >= 0.0
            neg = (ub <= 0.0) & ~pos
            mix = ~(pos | neg)
            with np.errstate(divide="ignore", invalid="ignore"):
                out[pos] = np.log1p(((ub - ua) + dR)[pos] / (ua + Ra)[pos])
                out[neg] = np.log1p(((ub - ua) - dR)[neg] / (Rb - ub)[neg])
                out[mix] = np.log(((ub + Rb) * (Ra - ua))[mix] / rho2[mix])
        elif m == 3:
            same = ua * ub > 0.0
            out = np.empty_like(ua)
            with np.errstate(divide="ignore", invalid="ignore"):
                den = Ra * Rb * (ub * Ra + ua * Rb)
                out[same] = ((ub - ua) * (ub + ua))[same] / den[same]
                out[~same] = (ub / Rb - ua / Ra)[~same] / rho2[~same]
        elif m >= 5:
            mm = m - 2
            out = (ub * Rb ** (-mm) - ua * Ra ** (-mm) + (mm - 1) * dJ(mm)) / (mm * rho2)
        elif m == -1:
            duR = 0.5 * (ub - ua) * (Ra + Rb) + 0.5 * (ua + ub) * dR
            out = 0.5 * (duR + rho2 * dJ(1))
        else:
            raise ValueError(m)
        J[m] = out
        return out

    def dK(m):
        if m not in K:
            q = 2 - m
            if q > 0:
                K[m] = dR * sum(Ra ** i * Rb ** (q - 1 - i) for i in range(q)) / q
            else:
                p = -q
                K[m] = dR * sum(Ra ** i * Rb ** (p - 1 - i) for i in range(p)) / (p * (Ra * Rb) ** p)
        return K[m]

    def dP(k, m):
        if (k, m) not in P:
            P[(k, m)] = dJ(m) if k == 0 else dK(m) if k == 1 else dP(k - 2, m - 2) - rho2 * dP(k - 2, m)
        return P[(k, m)]

    return {(m, k): dP(k, m) for m, km in spec.items() for k in range(km + 1)}


def _edge_small(ua, ub, rho2, spec):
    """Small-|u| series (primitives.py:351-399): P[m][k] = rho^(k+1-m)
    sum_j C(-m/2, j) (yb^pw - ya^pw) / pw, pw = k + 2j + 1, y = u / rho; each
    power difference is formed once and shared by every (m, k)."""
    rho = np.sqrt(rho2)
    ya, yb = ua / rho, ub / rho
    same = ua * ub > 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        log_r = np.where(same, np.log1p((ub - ua) / ua), 0.0)
        ratio = np.where(same, ub / ua, np.inf)
    close = same & (np.abs(ratio) < 2.0) & (np.abs(ratio) > 0.5)
    pwmax = max(km for km in spec.values()) + 2 * (SERIES_TERMS - 1) + 1
    diff = {}
    for pw in range(1, pwmax + 1):
        with np.errstate(over="ignore", invalid="ignore"):
            diff[pw] = np.where(close, ya ** pw * np.expm1(pw * log_r), yb ** pw - ya ** pw)
    out = {}
    for m, km in spec.items():
        for k in range(km + 1):
            acc = np.zeros_like(ua)
            for j in range(SERIES_TERMS):
                pw = k + 2 * j + 1
                acc = acc + _binom_half(m, j) * diff[pw] / pw
            out[(m, k)] = rho ** (k + 1 - m) * acc
    return out


def _edge_large(ua, ub, rho2, spec):
    """Large-|u| series (primitives.py:293-349) on one side of the foot:
    P[m][k] = +-a^s sum_j C(-m/2, j) x^j [t^q / q]_1^(b/a), q = s - 2j; each
    bracket is formed once per exponent q."""
    neg = ua < 0.0
    a = np.where(neg, -ub, ua)
    b = np.where(neg, -ua, ub)
    r = b / a
    log_r = np.log1p((b - a) / a)
    close = r < 2.0
    x = rho2 / (a * a)
    xp = [np.ones_like(a)]
    for _ in range(1, SERIES_TERMS):
        xp.append(xp[-1] * x)
    brk = {}

    def bracket(q):
        if q not in brk:
            if q == 0:
                brk[q] = log_r
            else:
                with np.errstate(over="ignore", invalid="ignore", divide="ignore"):
                    brk[q] = np.where(close, np.expm1(q * log_r), r ** q - 1.0) / q
        return brk[q]

    out = {}
    for m, km in spec.items():
        for k in range(km + 1):
            s_ = k - m + 1
            acc = np.zeros_like(a)
            for j in range(SERIES_TERMS):
                acc = acc + _binom_half(m, j) * xp[j] * bracket(s_ - 2 * j)
            val = a ** s_ * acc
            out[(m, k)] = np.where(neg, -val, val) if k % 2 else val
    return out


def edge_integrals(ua, ub, rho2, spec):
    """{(m, k): int_ua^ub u^k / (u^2 + rho^2)^(m/2) du} (primitives.py:431-504)."""
    rho = np.sqrt(rho2)
    umax = np.maximum(np.abs(ua), np.abs(ub))
    umin = np.minimum(np.abs(ua), np.abs(ub))
    small = umax <= SMALL_U_OVER_RHO * rho
    ser = (ua * ub > 0.0) & (umin >= SERIES_U_OVER_RHO * rho) & ~small
    closed = ~small & ~ser
    out = {(m, k): np.empty_like(ua) for m, km in spec.items() for k in range(km + 1)}
    for sel, fn in ((closed, _edge_closed), (small, _edge_small), (ser, _edge_large)):
        if np.any(sel):
            vals = fn(ua[sel], ub[sel], rho2[sel], spec)
            for key, v in vals.items():
                out[key][sel] = v
    return out


def solid_angle(v, x):
    r = v[None, :, :] - x[:, None, :]
    R = np.linalg.norm(r, axis=2)
    numer = np.einsum("ni,ni->n", r[:, 0], np.cross(r[:, 1], r[:, 2]))
    denom = (R[:, 0] * R[:, 1] * R[:, 2] + R[:, 2] * np.einsum("ni,ni->n", r[:, 0], r[:, 1])
             + R[:, 0] * np.einsum("ni,ni->n", r[:, 1], r[:, 2])
             + R[:, 1] * np.einsum("ni,ni->n", r[:, 0], r[:, 2]))
    return 2.0 * np.arctan2(numer, denom)


# ------------------------------------------------------ moment tables
def closed_moments(f, X0, X1, h2, need):
    """{(n, a, b): (N,)} by the divergence-theorem recursion
    (fullspace/moments.py:171-355)."""
    deg = close_degrees(need)
    edeg = edge_degrees(deg)
    N = X0.shape[0]
    p = f.p[None, :, :] - np.stack([X0, X1], axis=1)[:, None, :]
    BN1, BN2, BD = {}, {}, {}
    for e in range(3):
        pa, pb = p[:, e], p[:, (e + 1) % 3]
        ev = pb - pa
        L = np.linalg.norm(ev, axis=1)
        t = ev / L[:, None]
        nout = np.stack([t[:, 1], -t[:, 0]], axis=1)
        dp = np.einsum("ni,ni->n", pa, nout)
        ua = np.einsum("ni,ni->n", pa, t)
        ub = np.einsum("ni,ni->n", pb, t)
        rho2 = dp * dp + h2
        tab = edge_integrals(ua, ub, rho2, edeg)
        c1, c2, s1, s2 = nout[:, 0], nout[:, 1], t[:, 0], t[:, 1]
        for m, km in edeg.items():
            BD[m] = BD.get(m, 0.0) + dp * tab[(m, 0)]
            for a in range(km + 1):
                for b in range(km + 1 - a):
                    val = np.zeros(N)
                    for i in range(a + 1):
                        for j in range(b + 1):
                            pw = a + b - i - j
                            coeff = (math.comb(a, i) * math.comb(b, j) * dp ** pw
                                     * c1 ** (a - i) * s1 ** i * c2 ** (b - j) * s2 ** j)
                            val += coeff * tab[(m, i + j)]
                    BN1[(a, b, m)] = BN1.get((a, b, m), 0.0) + c1 * val
                    BN2[(a, b, m)] = BN2.get((a, b, m), 0.0) + c2 * val
    h = np.sqrt(h2)
    x_eff = (f.c[None, :] + X0[:, None] * f.e1 + X1[:, None] * f.e2 + h[:, None] * f.n[None, :])
    M = {(3, 0, 0): -solid_angle(f.v, x_eff) / h}
    n = 3
    while n + 2 in deg:
        M[(n + 2, 0, 0)] = (BD[n] + (n - 2) * M[(n, 0, 0)]) / (n * h2)
        n += 2
    n = 1
    while n in deg:
        M[(n, 0, 0)] = (BD[n] - n * h2 * M[(n + 2, 0, 0)]) / (2.0 - n)
        n -= 2
    for n in sorted(deg):
        m = n - 2
        for q in range(1, deg[n] + 1):
            for a in range(q, -1, -1):
                b = q - a
                if a >= 1:
                    val = -BN1[(a - 1, b, m)]
                    if a >= 2:
                        val = val + (a - 1) * M[(m, a - 2, b)]
                else:
                    val = -BN2[(0, b - 1, m)]
                    if b >= 2:
                        val = val + (b - 1) * M[(m, 0, b - 2)]
                M[(n, a, b)] = val / (n - 2)
    return M


def weighted_tables(f, x, eps, P, need0):
    """{(n, a, b): (N, K)} per-node weighted moments with the near/far split
    (fullspace/moments.py:515-606).  Returns (W, z)."""
    N = x.shape[0]
    K = (P + 1) * (P + 2) // 2
    z, X0, X1 = f.to_plane(x)
    h2 = z * z + eps * eps
    D = np.sqrt(np.sum((x - f.c) ** 2, axis=1) + eps * eps)
    near = D <= D_STAR * f.L
    W = {(n, a, b): np.empty((N, K)) for n, d in need0.items()
         for a in range(d + 1) for b in range(d + 1 - a)}
    if np.any(near):
        sel = near
        M = closed_moments(f, X0[sel], X1[sel], h2[sel], {n: d + P for n, d in need0.items()})
        c = shape_poly(f, P, X0[sel], X1[sel])
        for (n, a, b) in W:
            acc = 0.0
            for (ap, bp), cv in c.items():
                acc = acc + cv * M[(n, a + ap, b + bp)][:, None]
            W[(n, a, b)][sel] = acc
    far = ~near
    if np.any(far):
        ng = np.where(D > D_STAR_DISTANT * f.L, FAR_N_DISTANT, FAR_N)
        for g in np.unique(ng[far]):
            sel = far & (ng == g)
            x1, x2, w = _tri_rule(int(g))
            lam = np.stack([1.0 - x1 - x2, x1, x2], axis=1)
            eta = lam @ f.p
            wq = w * (2.0 * f.area)
            c0 = shape_poly(f, P, np.zeros(1), np.zeros(1))
            Nq = sum(c0[(a, b)][0][None, :] * (eta[:, 0] ** a * eta[:, 1] ** b)[:, None]
                     for (a, b) in c0)
            xi0 = eta[None, :, 0] - X0[sel][:, None]
            xi1 = eta[None, :, 1] - X1[sel][:, None]
            R2 = xi0 * xi0 + xi1 * xi1 + h2[sel][:, None]
            # in-plane monomials (weights folded in) from power tables, and
            # R^-n from one reciprocal square root and a ladder in R^-2, in
            # the order of mhs/fullspace/moments.py:456-498
            dmax = max(need0.values())
            p0, p1 = _pow_table(xi0, max(dmax, 1)), _pow_table(xi1, max(dmax, 1))
            inv = 1.0 / np.sqrt(R2)
            inv2 = inv * inv
            rn, cur = {}, inv
            for n in range(1, max(need0) + 1, 2):
                rn[n] = cur
                cur = cur * inv2
            for (n, a, b) in W:
                if a and b:
                    mono = wq[None, :] * p0[a] * p1[b]
                elif a:
                    mono = wq[None, :] * p0[a]
                elif b:
                    mono = wq[None, :] * p1[b]
                else:
                    mono = np.broadcast_to(wq[None, :], R2.shape)
                W[(n, a, b)][sel] = (mono * rn[n]) @ Nq
    return W, z


# --------------------------------------------------------------- lift
@functools.lru_cache(maxsize=64)
def _assignments(rank):
    return list(itertools.product(range(3), repeat=rank))


def lift(W, z, f, rank, n):
    """Rank-r tensor moment (N, K, 3^r flattened) (fullspace/kernels.py:90-123)."""
    basis = np.stack(f.basis)                                 # (3 basis, 3 xyz)
    N, K = next(iter(W.values())).shape
    out = np.zeros((N, K) + (3,) * rank)
    geo = {}
    for asg in _assignments(rank):
        a, b = asg.count(0), asg.count(1)
        g = np.array(1.0)
        for s in asg:
            g = np.multiply.outer(g, basis[s])
        geo[(a, b)] = geo.get((a, b), 0.0) + g
    for (a, b), g in geo.items():
        scal = ((-1.0) ** (a + b)) * (z ** (rank - a - b))[:, None] * W[(n, a, b)]
        out += scal.reshape((N, K) + (1,) * rank) * g
    return out


def _material(mu, lam):
    nu = 0.5 * lam / (lam + mu)
    lam_d = 2.0 * mu * nu / (1.0 - 2.0 * nu)
    return nu, lam_d


def direct(x, tri, P, mu, lam, eps, want):
    """Full-space Kelvin-Cortez U / H / E of one triangle, and the force
    (Kelvin single-layer) kernels G / S (fullspace/kernels.py:126-215;
    (mu, lam) -> nu at assemble.py:58-66)."""
    f = Frame(tri)
    nu, lam_d = _material(mu, lam)
    need0 = {}
    for w in want:
        for n, d in {"U": NEED_U, "H": NEED_H, "E": NEED_E, "G": NEED_G, "S": NEED_S}[w].items():
            need0[n] = max(need0.get(n, -1), d)
    W, z = weighted_tables(f, x, eps, P, need0)
    C1 = 1.0 / (16.0 * np.pi * mu * (1.0 - nu))
    c34 = 3.0 - 4.0 * nu
    e2 = eps * eps
    n = f.n
    eye = np.eye(3)
    out = {}
    if "U" in want or "S" in want:
        V3 = lift(W, z, f, 1, 3)
        V5 = lift(W, z, f, 1, 5)
        T35 = lift(W, z, f, 3, 5)
        G1 = (-c34 * np.einsum("ij,nkm->nkijm", eye, V3) + np.einsum("im,nkj->nkijm", eye, V3)
              + np.einsum("jm,nki->nkijm", eye, V3) - 3.0 * T35
              - 6.0 * (1.0 - nu) * e2 * np.einsum("ij,nkm->nkijm", eye, V5)) * C1
    if "U" in want:
        out["U"] = -(mu * np.einsum("m,nkijm->nkij", n, G1)
                     + lam_d * np.einsum("j,nkimm->nkij", n, G1)
                     + mu * np.einsum("m,nkimj->nkij", n, G1))
    if "G" in want:
        # force density -> displacement: C1 [(3 - 4 nu) I1 delta + T23
        # + 2 (1 - nu) eps^2 I3 delta]
        G = (c34 * np.einsum("ij,nk->nkij", eye, W[(1, 0, 0)]) + lift(W, z, f, 2, 3)
             + 2.0 * (1.0 - nu) * e2 * np.einsum("ij,nk->nkij", eye, W[(3, 0, 0)]))
        out["G"] = C1 * G
    if "S" in want:
        # force density -> stress: S[i, j, c] = C_ijab G1[a, c, b]
        trG1 = np.einsum("nkaca->nkc", G1)
        out["S"] = (lam_d * np.einsum("ij,nkc->nkijc", eye, trG1)
                    + mu * np.einsum("nkicj->nkijc", G1) + mu * np.einsum("nkjci->nkijc", G1))
    if "H" in want:
        I3 = W[(3, 0, 0)]
        I5 = W[(5, 0, 0)]
        T25 = lift(W, z, f, 2, 5)
        T27 = lift(W, z, f, 2, 7)
        T47 = lift(W, z, f, 4, 7)
        D2 = (-c34 * (np.einsum("rp,sq,nk->nkrpsq", eye, eye, I3) - 3.0 * np.einsum("rp,nksq->nkrpsq", eye, T25))
              + np.einsum("rs,pq,nk->nkrpsq", eye, eye, I3) - 3.0 * np.einsum("rs,nkpq->nkrpsq", eye, T25)
              + np.einsum("ps,rq,nk->nkrpsq", eye, eye, I3) - 3.0 * np.einsum("ps,nkrq->nkrpsq", eye, T25)
              - 3.0 * (np.einsum("rq,nkps->nkrpsq", eye, T25) + np.einsum("pq,nkrs->nkrpsq", eye, T25)
                       + np.einsum("sq,nkrp->nkrpsq", eye, T25))
              + 15.0 * T47
              + 2.0 * (1.0 - nu) * e2 * (-3.0 * np.einsum("rp,sq,nk->nkrpsq", eye, eye, I5)
                                        + 15.0 * np.einsum("rp,nksq->nkrpsq", eye, T27))) * C1
        trD = np.einsum("nkrpsp->nkrs", D2)
        B = (lam_d * np.einsum("j,nkrs->nkrsj", n, trD) + mu * np.einsum("q,nkrjsq->nkrsj", n, D2)
             + mu * np.einsum("p,nkrpsj->nkrsj", n, D2))
        trB = np.einsum("nkrrj->nkj", B)
        out["H"] = -(lam_d * np.einsum("ml,nkj->nkmlj", eye, trB) + mu * (B + np.swapaxes(B, 2, 3)))
    if "E" in want:
        out["E"] = (15.0 * eps ** 4 / (8.0 * np.pi)) * W[(7, 0, 0)]
    return out


# ----------------------------------------------------------- the image
@functools.lru_cache(maxsize=1)
def _table():
    d = np.load(HERE / "image_table.npz")
    return {k: d[k] for k in d.files}


def _coef_by_record(terms, n_rec, z, nu, with_z):
    """Per record (N,) or scalar coefficient sum num/den z^pz nu^pnu."""
    out = [0.0] * n_rec
    for r, pz, pnu, num, den in terms:
        v = (num / den) * (nu ** pnu)
        if with_z:
            v = v * (z ** pz)
        out[r] = out[r] + v
    return out


def _contract(DG, DDG, nrm, mu, lam):
    out = {}
    # indices: n observer, q node, i/p/a/b components, k slip, l/m summed
    if DG is not None:
        tr = np.einsum("nqimm->nqi", DG)
        out["U"] = (mu * np.einsum("l,nqikl->nqik", nrm, DG) + mu * np.einsum("l,nqilk->nqik", nrm, DG)
                    + lam * np.einsum("k,nqi->nqik", nrm, tr))
    if DDG is not None:
        trm = np.einsum("nqimpm->nqip", DDG)
        S = (mu * np.einsum("l,nqikpl->nqipk", nrm, DDG) + mu * np.einsum("l,nqilpk->nqipk", nrm, DDG)
             + lam * np.einsum("k,nqip->nqipk", nrm, trm))
        e = 0.5 * (S + np.swapaxes(S, 2, 3))
        tr = e[:, :, 0, 0] + e[:, :, 1, 1] + e[:, :, 2, 2]
        out["H"] = 2.0 * mu * e + lam * np.einsum("ab,nqk->nqabk", np.eye(3), tr)
    return out


def image_r(x, tri, P, mu, lam, eps, want):
    """Closed-form R-family on the reflected element (kernels/image.py:435-497)."""
    t = _table()
    nu = lam / (2.0 * (lam + mu))
    scale = 2.0 * (lam + mu) / (np.pi * mu * (lam + 2.0 * mu))
    tri_img = np.asarray(tri, float) * np.array([1.0, 1.0, -1.0])
    fi = Frame(tri_img)
    W, zp = weighted_tables(fi, x, eps, P, NEED_IMG)
    N = x.shape[0]
    K = (P + 1) * (P + 2) // 2
    zo = x[:, 2]
    cache = {}

    def moment(a, b, c, n):
        r = a + b + c
        if r == 0:
            return W[(n, 0, 0)]
        if (r, n) not in cache:
            cache[(r, n)] = lift(W, zp, fi, r, n)
        return cache[(r, n)][(slice(None), slice(None)) + (0,) * a + (1,) * b + (2,) * c]

    DG = DDG = None
    if "U" in want:
        DG = np.zeros((N, K, 3, 3, 3))
        coefs = _coef_by_record(t["dg_terms"], len(t["dg_idx"]), zo, nu, True)
        for r, (ix, ex) in enumerate(zip(t["dg_idx"], t["dg_exp"])):
            DG[:, :, ix[0], ix[1], ix[2]] += (coefs[r] * scale)[:, None] * moment(*ex)
    if "H" in want:
        DDG = np.zeros((N, K, 3, 3, 3, 3))
        coefs = _coef_by_record(t["ddg_terms"], len(t["ddg_idx"]), zo, nu, True)
        for r, (ix, ex) in enumerate(zip(t["ddg_idx"], t["ddg_exp"])):
            DDG[:, :, ix[0], ix[1], ix[2], ix[3]] += (coefs[r] * scale)[:, None] * moment(*ex)
    return _contract(DG, DDG, Frame(tri).n, mu, lam)


def _tri_distance(x, t):
    a, b, c = t
    ab, ac = b - a, c - a
    nr = np.cross(ab, ac)
    ap = x - a
    d20, d21 = ap @ ab, ap @ ac
    d00, d01, d11 = ab @ ab, ab @ ac, ac @ ac
    den = d00 * d11 - d01 * d01
    v = (d11 * d20 - d01 * d21) / den
    w = (d00 * d21 - d01 * d20) / den
    u = 1.0 - v - w
    inside = (u >= 0) & (v >= 0) & (w >= 0)
    out = np.empty(x.shape[0])
    out[inside] = np.abs(ap[inside] @ nr) / np.linalg.norm(nr)
    best = np.full(x.shape[0], np.inf)
    for p0, p1 in ((a, b), (b, c), (c, a)):
        e = p1 - p0
        tt = np.clip(((x - p0) @ e) / (e @ e), 0.0, 1.0)
        best = np.minimum(best, np.linalg.norm(x - (p0[None, :] + tt[:, None] * e[None, :]), axis=1))
    out[~inside] = best[~inside]
    return out


@functools.lru_cache(maxsize=8)
def _q_dense(nu):
    """Monomial keys (a, b, c, n, q) of the Q-family records and, per
    readout, the (slots, monomials) matrix of record coefficients summed by
    (slot, monomial) -- each record adds one number to one output slot
    (kernels/image.py:257-297)."""
    t = _table()
    monos = sorted({tuple(e) for e in t["q_dg_exp"]} | {tuple(e) for e in t["q_ddg_exp"]})
    midx = {m: i for i, m in enumerate(monos)}
    mats = {}
    for key, nix in (("q_dg", 3), ("q_ddg", 4)):
        coefs = _coef_by_record(t[f"{key}_terms"], len(t[f"{key}_idx"]), 0.0, nu, False)
        C = np.zeros((3 ** nix, len(monos)))
        for r, (ix, ex) in enumerate(zip(t[f"{key}_idx"], t[f"{key}_exp"])):
            slot = 0
            for i in ix:
                slot = slot * 3 + int(i)
            C[slot, midx[tuple(ex)]] += coefs[r]
        mats[key] = C
    return monos, mats


def _pow_table(v, kmax):
    """[1, v, v^2, ..., v^kmax] by repeated multiplication."""
    out = [None, v]
    for _ in range(2, kmax + 1):
        out.append(out[-1] * v)
    return out


def image_q(x, tri, P, mu, lam, eps, want):
    """Q-family by per-observer Gauss quadrature (kernels/image.py:211-432):
    observers grouped by their Gauss order, monomials formed from power
    tables, one dense contraction of the records per group."""
    tri = np.asarray(tri, float)
    nu = lam / (2.0 * (lam + mu))
    scale = 2.0 * (lam + mu) / (np.pi * mu * (lam + 2.0 * mu))
    f = Frame(tri)
    N = x.shape[0]
    K = (P + 1) * (P + 2) // 2
    delta = _tri_distance(x, tri * np.array([1.0, 1.0, -1.0]))
    orders = np.clip(np.ceil(Q_BUDGET_C * f.L / np.sqrt(delta * delta + eps * eps)) + P,
                     Q_MIN, Q_MAX).astype(int)
    monos, mats = _q_dense(nu)
    emax = [max(m[i] for m in monos) for i in range(5)]
    DG = np.zeros((N, K, 27)) if "U" in want else None
    DDG = np.zeros((N, K, 81)) if "H" in want else None
    c0 = shape_poly(f, P, np.zeros(1), np.zeros(1))
    for nq in np.unique(orders):
        sel = orders == nq
        x1, x2, w = _tri_rule(int(nq))
        bary = np.stack([1.0 - x1 - x2, x1, x2], axis=1)
        y = bary @ tri
        eta = bary @ f.p
        Nq = sum(c0[(a, b)][0][None, :] * (eta[:, 0] ** a * eta[:, 1] ** b)[:, None] for (a, b) in c0)
        wN = (w * 2.0 * f.area)[:, None] * Nq
        xs = x[sel]
        d1 = xs[:, 0:1] - y[None, :, 0]
        d2 = xs[:, 1:2] - y[None, :, 1]
        d3 = xs[:, 2:3] + y[None, :, 2]
        r2 = np.sqrt(d1 * d1 + d2 * d2 + d3 * d3 + eps ** 2)
        pw = [_pow_table(v, e) for v, e in zip((d1, d2, d3, 1.0 / r2, 1.0 / (r2 - d3)), emax)]
        basis = np.empty((len(monos), xs.shape[0], K))
        for k, mono in enumerate(monos):
            term = None
            for table, e in zip(pw, mono):
                if e:
                    term = table[e] if term is None else term * table[e]
            basis[k] = (np.ones_like(r2) if term is None else term) @ wN
        for key, arr in (("q_dg", DG), ("q_ddg", DDG)):
            if arr is not None:
                flat = np.tensordot(mats[key], basis, axes=([1], [0]))     # (slots, n, K)
                arr[sel] = np.moveaxis(flat, 0, -1) * scale
    return _contract(None if DG is None else DG.reshape(N, K, 3, 3, 3),
                     None if DDG is None else DDG.reshape(N, K, 3, 3, 3, 3), f.n, mu, lam)


# ------------------------------------------------------------- the fold
def straddles(tri, eps):
    return float(-np.asarray(tri)[:, 2].max()) < FOLD_SRC_EPS * eps


def crease(tri, eps):
    tri = np.asarray(tri, float)
    depth = -tri[:, 2]
    top = tri[depth < FOLD_SRC_EPS * eps]
    if top.shape[0] == 0:
        top = tri[depth == depth.min()]
    centre = top[:, :2].mean(axis=0)
    spread = float(np.linalg.norm(top[:, :2] - centre, axis=1).max())
    return centre, spread + FOLD_MARGIN_EPS * eps + float((-top[:, 2]).max())


def band(x, tri, eps):
    centre, _ = crease(tri, eps)
    reach = np.hypot(x[:, 0] - centre[0], x[:, 1] - centre[1])
    return np.flatnonzero((-x[:, 2] < FOLD_BAND_EPS * eps) & (reach < FOLD_REACH_EPS * eps))


def _composite(breaks, n):
    u, wu = _gl01(n)
    a = np.asarray(breaks[:-1], float)
    b = np.asarray(breaks[1:], float)
    return (a[:, None] + (b - a)[:, None] * u[None, :]).ravel(), ((b - a)[:, None] * wu[None, :]).ravel()


def _halfwidth(ra, rb, rho_s, radius):
    if rb < rho_s - radius or ra > rho_s + radius:
        return 0.0
    if rho_s <= radius:
        return np.pi
    return float(np.arcsin(min(1.0, radius / rho_s)))


def _angular(theta_c, w_fine, w_med, rb, eps):
    n = FOLD_NA
    if w_fine >= np.pi or w_med >= np.pi:
        sp = FOLD_FINE_EPS if w_fine >= np.pi else FOLD_MED_EPS
        m = max(8, int(np.ceil(2 * np.pi * rb / (n * sp * eps))))
        return _composite(np.linspace(0, 2 * np.pi, m + 1), n)
    pieces = []
    if w_fine > 0:
        m = max(1, int(np.ceil(2 * w_fine * rb / (n * FOLD_FINE_EPS * eps))))
        pieces.append(np.linspace(theta_c - w_fine, theta_c + w_fine, m + 1))
    if w_med > w_fine:
        m = max(1, int(np.ceil((w_med - w_fine) * rb / (n * FOLD_MED_EPS * eps))))
        pieces.insert(0, np.linspace(theta_c - w_med, theta_c - w_fine, m + 1))
        pieces.append(np.linspace(theta_c + w_fine, theta_c + w_med, m + 1))
    start = theta_c + w_med if w_med > 0 else 0.0
    pieces.append(np.linspace(start, start + 2 * np.pi - 2 * w_med, max(1, FOLD_COARSE // n) + 1))
    nodes, weights = [], []
    for br in pieces:
        if br.size >= 2 and br[-1] > br[0]:
            t_, w_ = _composite(br, n)
            nodes.append(t_)
            weights.append(w_)
    return np.concatenate(nodes), np.concatenate(weights)


def polar_grid(xh, zeta, centre, r_f, eps, diam):
    """Surface quadrature about the receiver's foot (kernels/fold.py:290-330)."""
    rho_s = float(np.hypot(*(centre - xh)))
    theta_c = float(np.arctan2(centre[1] - xh[1], centre[0] - xh[0]))
    r1_target = rho_s + 4 * r_f + FOLD_R1_DIAM * diam
    geo = [0.0]
    if 0 < zeta < 0.5 * eps:
        geo += [z for z in (0.5 * zeta, zeta, 2 * zeta, 4 * zeta) if z < 0.5 * eps]
    r = 0.5 * eps
    while True:
        geo.append(r)
        if r >= r1_target:
            break
        r *= 2.0
    R1 = geo[-1]
    lo_m, hi_m, lo_f, hi_f = rho_s - 4 * r_f, rho_s + 4 * r_f, rho_s - r_f, rho_s + r_f
    breaks = [g for g in geo if g < lo_m or g > hi_m]
    ann = []
    for a0, b0, width in ((max(0.0, lo_m), max(0.0, lo_f), FOLD_MED_SUB_EPS),
                          (max(0.0, lo_f), min(R1, hi_f), FOLD_FINE_SUB_EPS),
                          (min(R1, hi_f), min(R1, hi_m), FOLD_MED_SUB_EPS)):
        if b0 > a0:
            ann += list(np.linspace(a0, b0, max(1, int(np.ceil((b0 - a0) / (width * eps)))) + 1))
    breaks = np.unique(np.concatenate([np.asarray(breaks, float), np.asarray(ann, float)]))
    breaks = breaks[breaks <= R1 + 1e-12 * R1]
    pts, wts = [], []
    for ra, rb in zip(breaks[:-1], breaks[1:]):
        if rb - ra < 1e-9 * eps:
            continue
        rq, wr = _composite([ra, rb], FOLD_NR)
        tq, wt = _angular(theta_c, _halfwidth(ra, rb, rho_s, r_f), _halfwidth(ra, rb, rho_s, 4 * r_f), rb, eps)
        R, T = np.meshgrid(rq, tq, indexing="ij")
        pts.append(np.stack([xh[0] + R * np.cos(T), xh[1] + R * np.sin(T)], axis=-1).reshape(-1, 2))
        wts.append((wr[:, None] * wt[None, :] * R).ravel())
    return np.concatenate(pts), np.concatenate(wts), R1


def _point_stress(dx, dy, zeta, nu):
    r2 = dx * dx + dy * dy
    rho = np.sqrt(r2 + zeta * zeta)
    rho3 = rho ** 3
    rho5 = rho3 * rho * rho
    a = 1.0 / (rho * (rho + zeta))
    c = 1.0 - 2.0 * nu
    s_th = c * (-a + zeta / rho3)
    s_r_th = 2.0 * c * a - 3.0 * zeta * r2 / rho5 - c * zeta / rho3
    r = np.sqrt(r2)
    ex = np.where(r > 0, dx / np.where(r > 0, r, 1.0), 0.0)
    ey = np.where(r > 0, dy / np.where(r > 0, r, 1.0), 0.0)
    pref = 1.0 / (2.0 * np.pi)
    S = np.empty(dx.shape + (3, 3))
    S[..., 0, 0] = pref * (s_th + s_r_th * ex * ex)
    S[..., 1, 1] = pref * (s_th + s_r_th * ey * ey)
    S[..., 0, 1] = S[..., 1, 0] = pref * s_r_th * ex * ey
    t_rz = pref * 3.0 * r * zeta * zeta / rho5
    S[..., 0, 2] = S[..., 2, 0] = t_rz * ex
    S[..., 1, 2] = S[..., 2, 1] = t_rz * ey
    S[..., 2, 2] = -pref * 3.0 * zeta ** 3 / rho5
    return S


def _point_disp(dx, dy, zeta, mu, nu):
    rho = np.sqrt(dx * dx + dy * dy + zeta * zeta)
    pref = 1.0 / (4.0 * np.pi * mu)
    ur = pref * (zeta / rho ** 3 - (1.0 - 2.0 * nu) / (rho * (rho + zeta)))
    return np.stack([ur * dx, ur * dy, -pref * (2.0 * (1.0 - nu) / rho + zeta * zeta / rho ** 3)], axis=-1)


def _surface_load(pts, tri, mu, lam, eps, P):
    x = np.column_stack([pts, np.zeros(pts.shape[0])])
    blk = direct(x, tri, P, mu, lam, eps, ("H", "E"))
    nrm = Frame(tri).n
    e_zz = lam * nrm + 2.0 * mu * nrm[2] * np.array([0.0, 0.0, 1.0])
    return 2.0 * (blk["H"][:, :, 2, 2, :] - blk["E"][:, :, None] * e_zz[None, None, :])


def fold_image(x, tri, P, mu, lam, eps, want):
    """Mirror element + Boussinesq at band receivers (kernels/fold.py:334-380)."""
    tri = np.asarray(tri, float)
    nu = 0.5 * lam / (lam + mu)
    centre, r_f = crease(tri, eps)
    diam = max(float(np.linalg.norm(tri[i] - tri[j])) for i in range(3) for j in range(3))
    K = (P + 1) * (P + 2) // 2
    blk = direct(x, tri * np.array([1.0, 1.0, -1.0]), P, mu, lam, eps, want)
    s_h = _surface_load(x[:, :2], tri, mu, lam, eps, P)
    out = {k: blk[k] * MIRROR_SLIP_SIGN for k in want}
    for o in range(x.shape[0]):
        xh = x[o, :2]
        zeta = max(0.0, float(-x[o, 2]))
        pts, wts, R1 = polar_grid(xh, zeta, centre, r_f, eps, diam)
        s = _surface_load(pts, tri, mu, lam, eps, P) - s_h[o][None]
        dx, dy = xh[0] - pts[:, 0], xh[1] - pts[:, 1]
        rho = math.sqrt(R1 * R1 + zeta * zeta)
        if "H" in want:
            SB = _point_stress(dx, dy, zeta, nu)
            szz = -(1.0 - zeta ** 3 / rho ** 3)
            srr = -0.5 * ((1.0 + 2.0 * nu) - 2.0 * (1.0 + nu) * zeta / rho + zeta ** 3 / rho ** 3)
            disk = np.diag([srr, srr, szz])
            out["H"][o] += (np.einsum("n,nab,nkm->kabm", wts, SB, s)
                            + s_h[o][:, None, None, :] * disk[None, :, :, None])
        if "U" in want:
            UB = _point_disp(dx, dy, zeta, mu, nu)
            uz = -(0.5 / mu) * (2.0 * (1.0 - nu) * (rho - zeta) + zeta - zeta * zeta / rho)
            out["U"][o] += (np.einsum("n,ni,nkm->kim", wts, UB, s)
                            + s_h[o][:, None, :] * np.array([0.0, 0.0, uz])[None, :, None])
    return out


# ---------------------------------------------------------- assembly
def _hooke(n, mu, lam):
    eye = np.eye(3)
    return lam * np.einsum("mn,k->mnk", eye, n) + mu * (np.einsum("mk,n->mnk", eye, n)
                                                        + np.einsum("nk,m->mnk", eye, n))


def source_block(x, tri, P, mu, lam, eps, want, fold=True):
    """One source at every observer: direct + image (fold in the band) and
    the eigenstress terms [(phi (N, K), C (3, 3, 3))] (kernels/assemble.py:96-262)."""
    tri = np.asarray(tri, float)
    dwant = tuple(w for w in want if w in ("U", "H")) + (("E",) if "E" in want else ())
    blk = direct(x, tri, P, mu, lam, eps, dwant) if dwant else {}
    iw = tuple(w for w in want if w in ("U", "H"))
    sel = band(x, tri, eps) if (fold and straddles(tri, eps)) else np.zeros(0, int)
    if iw:
        img = image_r(x, tri, P, mu, lam, eps, iw)
        q = image_q(x, tri, P, mu, lam, eps, iw)
        img = {k: img[k] + q[k] for k in iw}
        if sel.size:
            fb = fold_image(x[sel], tri, P, mu, lam, eps, iw)
            for k in iw:
                img[k][sel] = fb[k]
        for k in iw:
            blk[k] = blk[k] + img[k]
    terms = None
    if "E" in want:
        terms = [(blk["E"], _hooke(Frame(tri).n, mu, lam))]
        if sel.size:
            trim = tri * np.array([1.0, 1.0, -1.0])
            phi_m = np.zeros_like(blk["E"])
            phi_m[sel] = direct(x[sel], trim, P, mu, lam, eps, ("E",))["E"]
            terms.append((phi_m, _hooke(Frame(trim).n, mu, lam) * MIRROR_SLIP_SIGN[None, None, :]))
    return blk, terms


def _put(out, s, K, block, ids, axis):
    sl = [slice(None)] * out.ndim
    if ids is None:
        sl[axis] = slice(s * K, (s + 1) * K)
        out[tuple(sl)] = block
    else:
        sl[axis] = ids[s]
        out[tuple(sl)] += block


def _eps_arr(eps, n):
    return np.broadcast_to(np.asarray(eps, float), (n,))


def disp_matrix(obs, tris, mu, lam, eps, order=0, fold=True, ids=None, n_dof=None):
    obs, tris = np.asarray(obs, float), np.asarray(tris, float)
    K = (order + 1) * (order + 2) // 2
    n_dof = tris.shape[0] * K if n_dof is None else n_dof
    out = np.zeros((obs.shape[0], 3, n_dof, 3))
    e = _eps_arr(eps, tris.shape[0])
    for s in range(tris.shape[0]):
        blk, _ = source_block(obs, tris[s], order, mu, lam, e[s], ("U",), fold)
        _put(out, s, K, np.moveaxis(blk["U"], 1, 2), ids, 2)
    return out


def _stress_like(obs, tris, mu, lam, eps, order, fold, ids, n_dof, total, eigen):
    obs, tris = np.asarray(obs, float), np.asarray(tris, float)
    K = (order + 1) * (order + 2) // 2
    n_dof = tris.shape[0] * K if n_dof is None else n_dof
    sig = np.zeros((obs.shape[0], 3, 3, n_dof, 3))
    star = np.zeros_like(sig)
    e = _eps_arr(eps, tris.shape[0])
    for s in range(tris.shape[0]):
        blk, terms = source_block(obs, tris[s], order, mu, lam, e[s], ("H", "E"), fold)
        _put(sig, s, K, np.moveaxis(blk["H"], 1, 3), ids, 3)
        eb = sum(phi[:, None, None, :, None] * C[None, :, :, None, :] for phi, C in terms)
        _put(star, s, K, eb, ids, 3)
    return sig, star


def stress_matrix(obs, tris, mu, lam, eps, order=0, fold=True, ids=None, n_dof=None,
                  subtract_eigenstress=True):
    sig, star = _stress_like(obs, tris, mu, lam, eps, order, fold, ids, n_dof, True, True)
    return sig - star if subtract_eigenstress else sig


def total_stress_matrix(obs, tris, mu, lam, eps, order=0, fold=True, ids=None, n_dof=None):
    return _stress_like(obs, tris, mu, lam, eps, order, fold, ids, n_dof, True, False)[0]


def eigenstress_matrix(obs, tris, mu, lam, eps, order=0, fold=True, ids=None, n_dof=None):
    return _stress_like(obs, tris, mu, lam, eps, order, fold, ids, n_dof, False, True)[1]


def elastic_strain_matrix(obs, tris, mu, lam, eps, order=0, fold=True, ids=None, n_dof=None,
                          subtract_eigenstress=True):
    buf = stress_matrix(obs, tris, mu, lam, eps, order, fold, ids, n_dof, subtract_eigenstress)
    tr = buf[:, 0, 0] + buf[:, 1, 1] + buf[:, 2, 2]
    tre = tr / (3.0 * lam + 2.0 * mu)
    for a in range(3):
        buf[:, a, a] -= lam * tre
    return buf / (2.0 * mu)


def _traction_blocks(obs, nrm, tri, P, mu, lam, eps, fold, subtract):
    want = ("H", "E") if subtract else ("H",)
    blk, terms = source_block(obs, tri, P, mu, lam, eps, want, fold)
    t = np.einsum("okijm,oj->okim", blk["H"], nrm)
    if subtract:
        for phi, C in terms:
            t = t - phi[:, :, None, None] * np.einsum("ijk,oj->oik", C, nrm)[:, None, :, :]
    return t


def traction_matrix(obs, normals, tris, mu, lam, eps, order=0, fold=True, ids=None, n_dof=None,
                    subtract_eigenstress=True):
    obs, tris = np.asarray(obs, float), np.asarray(tris, float)
    nrm = np.asarray(normals, float)
    nrm = nrm / np.linalg.norm(nrm, axis=1, keepdims=True)
    K = (order + 1) * (order + 2) // 2
    n_dof = tris.shape[0] * K if n_dof is None else n_dof
    out = np.zeros((obs.shape[0], 3, n_dof, 3))
    e = _eps_arr(eps, tris.shape[0])
    for s in range(tris.shape[0]):
        t = _traction_blocks(obs, nrm, tris[s], order, mu, lam, e[s], fold, subtract_eigenstress)
        _put(out, s, K, np.moveaxis(t, 1, 2), ids, 2)
    return out


def interaction_matrix(obs, nrm, rec_basis, tris, src_basis, mu, lam, eps, order=0, fold=True,
                       ids=None, n_dof=None, subtract_eigenstress=True):
    """``einsum('oai,okim,bm->okab')`` per source (kernels/assemble.py:295-331);
    with ``ids`` the source basis is per column."""
    obs, tris = np.asarray(obs, float), np.asarray(tris, float)
    K = (order + 1) * (order + 2) // 2
    n_dof = tris.shape[0] * K if n_dof is None else n_dof
    out = np.zeros((obs.shape[0], n_dof, rec_basis.shape[1], src_basis.shape[1]))
    e = _eps_arr(eps, tris.shape[0])
    for s in range(tris.shape[0]):
        t = _traction_blocks(obs, nrm, tris[s], order, mu, lam, e[s], fold, subtract_eigenstress)
        if ids is None:
            out[:, s * K:(s + 1) * K] = np.einsum("oai,okim,bm->okab", rec_basis, t, src_basis[s])
        else:
            out[:, ids[s]] += np.einsum("oai,okim,kbm->okab", rec_basis, t, src_basis[ids[s]])
    return out


# ------------------------------------------------- frames and collocation
def slip_frame(tris):
    """Rows [strike, dip, tensile] on upward normals (mhs/tdcs.py:49-98)."""
    t = np.asarray(tris, float).reshape(-1, 3, 3)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    n = n / np.linalg.norm(n, axis=1, keepdims=True)
    n = np.where(n[:, 2:3] < 0.0, -n, n)
    return frame_from_normals(n)


def frame_from_normals(n):
    n = np.asarray(n, float).reshape(-1, 3)
    strike = np.stack([-n[:, 1], n[:, 0], np.zeros(len(n))], axis=1)
    mag = np.linalg.norm(strike, axis=1, keepdims=True)
    flat = mag[:, 0] <= 1e-12
    strike = np.where(flat[:, None], np.array([1.0, 0.0, 0.0]), strike / np.where(mag > 0, mag, 1.0))
    return np.stack([strike, np.cross(n, strike), n], axis=1)


def collocation_points(tris, order=0, shrink=0.5):
    tri = np.asarray(tris, float).reshape(-1, 3, 3)
    bary = np.full((1, 3), 1.0 / 3.0) if order == 0 else np.array(_lattice(order), float) / order
    bary = bary + shrink * (1.0 / 3.0 - bary)
    return (bary[None, :, :] @ tri).reshape(-1, 3)


def self_interaction(tris, mu, lam, eps, order=0, receiver=(0, 1, 2), source=(0, 1, 2), fold=True,
                     subtract_eigenstress=True):
    """Square interaction at the shrunk collocation points (matrices.py:378-480)."""
    K = (order + 1) * (order + 2) // 2
    pts = collocation_points(tris, order)
    fr = slip_frame(tris)
    rec = np.repeat(fr, K, axis=0)
    return interaction_matrix(pts, rec[:, 2, :], rec[:, list(receiver), :], tris,
                              fr[:, list(source), :], mu, lam, eps, order, fold,
                              subtract_eigenstress=subtract_eigenstress)
