"""The full-space single-triangle API, on the device: mhs.fullspace.api's calls
(mhs/fullspace/api.py:90-180) with the same signatures, conventions and
refusals, evaluated by the engine's kernels (``mhs_fullspace_influence``).

    displacement(obs, tri, slip, mu, nu, eps)        -> (N, 3)
    stress(obs, tri, slip, mu, nu, eps)              -> (N, 3, 3)  elastic (default)
    eigenstress(obs, tri, slip, mu, nu, eps)         -> (N, 3, 3)  C:eps*
    force_displacement(obs, tri, force, mu, nu, eps) -> (N, 3)
    force_stress(obs, tri, force, mu, nu, eps)       -> (N, 3, 3)
    influence(obs, tri, mu, nu, eps, order=p)        -> nodal tensors
    traction(sigma, tri)                             -> sigma . nhat

``slip`` / ``force`` are (K, 3) nodal values (K = 1, 3, 6 for constant,
linear, quadratic; a (3,) vector is constant), nodes as ``influence(...).nodes``.
Observers are numpy arrays (results come back as numpy arrays) or CUDA
tensors (results stay on the device).  One difference from mhs: with
``eps = 0`` every observer must lie off the triangle's plane (this engine
has no on-plane limit; mhs evaluates the single layer G on the element).
"""
from __future__ import annotations

import ctypes
from typing import NamedTuple

import numpy as np

from . import _native
from .matrices import _is_torch, _lattice, _torch, n_nodes

WANT_BITS = {"U": 1, "H": 2, "E": 4, "G": 8, "S": 16}
FAR_FIELD = {"hybrid": 0, "analytic": 1, "quadrature": 2}


class Influence(NamedTuple):
    U: object | None      # (N, K, 3, 3)     slip -> displacement
    H: object | None      # (N, K, 3, 3, 3)  slip -> TOTAL stress
    E: object | None      # (N, K)           eigenstress weight
    nodes: np.ndarray     # (K, 3)
    order: int
    G: object | None = None   # (N, K, 3, 3)     force density -> displacement
    S: object | None = None   # (N, K, 3, 3, 3)  force density -> stress


def _triangle(tri) -> np.ndarray:
    tri = np.asarray(tri.detach().cpu() if _is_torch(tri) else tri, dtype=float)
    if tri.shape != (3, 3):
        raise ValueError(f"tri must have shape (3, 3), got {tri.shape}")
    return tri


def _normal(tri: np.ndarray) -> np.ndarray:
    n = np.cross(tri[1] - tri[0], tri[2] - tri[0])
    nn = np.linalg.norm(n)
    if nn == 0.0:
        raise ValueError("degenerate triangle (zero area)")
    return n / nn


def _check_material(mu, nu, eps) -> float:
    if not (mu > 0.0):
        raise ValueError("mu must be > 0")
    if not (-1.0 < nu < 0.5):
        raise ValueError("nu must be in (-1, 1/2)")
    eps = float(np.asarray(eps))
    if eps < 0.0:
        raise ValueError("eps must be >= 0")
    return eps


def _order_of(k: int) -> int:
    p = 0
    while n_nodes(p) < k:
        p += 1
    if n_nodes(p) != k:
        raise ValueError(f"{k} nodal values do not correspond to a Lagrange "
                         "order on a triangle (need 1, 3, 6, 10, ...)")
    return p


def _nodal(values, order, name="slip"):
    values = np.asarray(values.detach().cpu() if _is_torch(values) else values, float)
    if values.ndim == 1:
        if values.shape != (3,):
            raise ValueError(f"a 1-D {name} must have 3 components")
        values = values[None, :]
    if values.ndim != 2 or values.shape[1] != 3:
        raise ValueError(f"{name} must have shape (K, 3), got {values.shape}")
    try:
        p = _order_of(values.shape[0])
    except ValueError as exc:
        raise ValueError(f"{name}: {exc}") from None
    if order is not None and int(order) != p:
        raise ValueError(f"order={order} disagrees with {values.shape[0]} nodal "
                         f"{name} values (order {p})")
    return values, p


def nodes(tri, order: int) -> np.ndarray:
    """Node coordinates (K, 3) of order ``order`` on ``tri``."""
    tri = _triangle(tri)
    if order == 0:
        return tri.mean(axis=0, keepdims=True)
    return (_lattice(order) / order) @ tri


def influence(obs, tri, mu, nu, eps, *, order=0, want=("U", "H", "E"),
              far_field="hybrid") -> Influence:
    """Nodal influence tensors of one triangle at the observation points:
    ``U[n, k, i, j]`` displacement i per unit slip j at node k; ``H[n, k, m,
    l, j]`` TOTAL stress ml; ``E[n, k]`` eigenstress weight; ``G`` and ``S``
    the same for a force density per unit area (Kelvin single layer)."""
    eps = _check_material(mu, nu, eps)
    tri = _triangle(tri)
    _normal(tri)
    order = int(order)
    if order not in (0, 1, 2):
        raise ValueError(f"order must be 0, 1 or 2, got {order}")
    if far_field not in FAR_FIELD:
        raise ValueError("far_field must be 'hybrid', 'analytic' or 'quadrature'")
    bits = 0
    for w in want:
        if w not in WANT_BITS:
            raise ValueError(f"unknown kernel {w!r}; choose from U, H, E, G, S")
        bits |= WANT_BITS[w]
    torch = _torch()
    on_device = _is_torch(obs) and obs.is_cuda
    if on_device:
        dev = obs.device
        o = obs.detach().to(torch.float64).reshape(-1, 3).contiguous()
    else:
        if not torch.cuda.is_available():
            raise RuntimeError("mhs_b200 evaluates on a CUDA device and none is available "
                               "(there is no CPU path)")
        dev = torch.device("cuda", torch.cuda.current_device())
        o = torch.as_tensor(np.ascontiguousarray(np.asarray(obs, float).reshape(-1, 3)),
                            device=dev)
    if eps == 0.0:
        # the engine's closed form needs h = sqrt(z^2 + eps^2) > 0
        z = (o - torch.as_tensor(tri.mean(axis=0), device=dev)) @ \
            torch.as_tensor(_normal(tri), device=dev)
        L = max(np.linalg.norm(tri[1] - tri[0]), np.linalg.norm(tri[2] - tri[1]),
                np.linalg.norm(tri[0] - tri[2]))
        if bool((z.abs() <= 1e-12 * L).any()):
            raise ValueError("eps = 0 needs every observation point off the triangle's plane")
    n, K = o.shape[0], n_nodes(order)
    shapes = {"U": (n, K, 3, 3), "H": (n, K, 3, 3, 3), "E": (n, K), "G": (n, K, 3, 3),
              "S": (n, K, 3, 3, 3)}
    outs = {w: torch.empty(shapes[w], dtype=torch.float64, device=dev) for w in WANT_BITS
            if bits & WANT_BITS[w]}
    req = _native.FullspaceRequest()
    req.order, req.want, req.far_field = order, bits, FAR_FIELD[far_field]
    req.n_obs = n
    req.obs = ctypes.c_void_p(o.data_ptr())
    for i, v in enumerate(tri.reshape(-1)):
        req.tri[i] = float(v)
    req.mu, req.nu, req.eps = float(mu), float(nu), eps
    for w, t in outs.items():
        setattr(req, w, ctypes.c_void_p(t.data_ptr()))
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev)
        _native.check(_native.load().mhs_fullspace_influence(
            ctypes.byref(req), ctypes.c_void_p(stream.cuda_stream)))
    if not on_device:
        outs = {w: t.cpu().numpy() for w, t in outs.items()}
    return Influence(U=outs.get("U"), H=outs.get("H"), E=outs.get("E"),
                     nodes=nodes(tri, order), order=order, G=outs.get("G"), S=outs.get("S"))


def _squeeze(out, obs):
    """A single observation point (a (3,) array) gives unbatched results."""
    ndim = obs.dim() if _is_torch(obs) else np.ndim(obs)
    return out[0] if ndim == 1 else out


def _einsum(spec, a, b):
    if _is_torch(a):
        torch = _torch()
        return torch.einsum(spec, a, torch.as_tensor(b, device=a.device))
    return np.einsum(spec, a, b)


def displacement(obs, tri, slip, mu, nu, eps, *, order=None, far_field="hybrid"):
    """Displacement (N, 3) at ``obs`` from the nodal slip on ``tri``."""
    slip, p = _nodal(slip, order)
    inf = influence(obs, tri, mu, nu, eps, order=p, want=("U",), far_field=far_field)
    return _squeeze(_einsum("nkij,kj->ni", inf.U, slip), obs)


def _eigen_sigma(slip, tri, mu, nu):
    """Per node, C : sym(slip_k (x) nhat) (K, 3, 3)."""
    lam = 2.0 * mu * nu / (1.0 - 2.0 * nu)
    n = _normal(_triangle(tri))
    sym = 0.5 * (slip[:, :, None] * n[None, None, :] + n[None, :, None] * slip[:, None, :])
    tr = np.trace(sym, axis1=1, axis2=2)
    return lam * tr[:, None, None] * np.eye(3)[None] + 2.0 * mu * sym


def eigenstress(obs, tri, slip, mu, nu, eps, *, order=None, far_field="hybrid"):
    """Eigenstress ``C:eps*`` (N, 3, 3) of the smeared slip (the anelastic term)."""
    slip, p = _nodal(slip, order)
    inf = influence(obs, tri, mu, nu, eps, order=p, want=("E",), far_field=far_field)
    return _squeeze(_einsum("nk,kij->nij", inf.E, _eigen_sigma(slip, tri, mu, nu)), obs)


def stress(obs, tri, slip, mu, nu, eps, *, order=None, subtract_eigenstress=True,
           far_field="hybrid"):
    """Stress (N, 3, 3) at ``obs``: elastic (default) or total."""
    slip, p = _nodal(slip, order)
    want = ("H", "E") if subtract_eigenstress else ("H",)
    inf = influence(obs, tri, mu, nu, eps, order=p, want=want, far_field=far_field)
    sig = _einsum("nkmlj,kj->nml", inf.H, slip)
    if subtract_eigenstress:
        sig = sig - _einsum("nk,kij->nij", inf.E, _eigen_sigma(slip, tri, mu, nu))
    return _squeeze(sig, obs)


def force_displacement(obs, tri, force, mu, nu, eps, *, order=None, far_field="hybrid"):
    """Displacement (N, 3) at ``obs`` from a nodal FORCE density per unit area
    on ``tri`` (Kelvin convention, ``div sigma + f phi_eps = 0``)."""
    force, p = _nodal(force, order, name="force")
    inf = influence(obs, tri, mu, nu, eps, order=p, want=("G",), far_field=far_field)
    return _squeeze(_einsum("nkij,kj->ni", inf.G, force), obs)


def force_stress(obs, tri, force, mu, nu, eps, *, order=None, far_field="hybrid"):
    """Stress (N, 3, 3) at ``obs`` from a nodal FORCE density on ``tri``: a
    mollified body force is a genuine body force, so there is no eigenstress
    to subtract."""
    force, p = _nodal(force, order, name="force")
    inf = influence(obs, tri, mu, nu, eps, order=p, want=("S",), far_field=far_field)
    return _squeeze(_einsum("nkijc,kc->nij", inf.S, force), obs)


def traction(sigma, tri):
    """Traction vector(s) ``sigma . nhat`` on the triangle's plane."""
    n = _normal(_triangle(tri))
    if _is_torch(sigma):
        return sigma @ _torch().as_tensor(n, device=sigma.device, dtype=sigma.dtype)
    return np.asarray(sigma, float) @ n
