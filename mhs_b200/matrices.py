"""The public surface: mhs's matrix functions, assembled on a B200.

Same names, arguments, index order, validation and error messages as
mhs/matrices.py:75-580, so a call site switches by changing the import:

* ``disp_matrix``          (n_obs, 3, n_dof, 3)
* ``stress_matrix``        (n_obs, 3, 3, n_dof, 3), eigenstress removed
* ``total_stress_matrix``  (n_obs, 3, 3, n_dof, 3)
* ``eigenstress_matrix``   (n_obs, 3, 3, n_dof, 3)
* ``elastic_strain_matrix``(n_obs, 3, 3, n_dof, 3)
* ``traction_matrix``      (n_obs, 3, n_dof, 3)
* ``interaction_matrix``   (n_rec_dof, n_src_dof, n_a, n_b)

Inputs may be numpy arrays (the result is then a numpy array, as from mhs)
or torch tensors (the result stays on the device as a torch tensor).
``out=`` may be a numpy array (filled from the device) or a CUDA torch
tensor (written in place), float64 or float32.

One extra keyword, ``precision="fp64"`` (default, every term in float64) or
``"mixed"`` (far-field quadrature in float32), selects the arithmetic.
"""
from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _native, chunking, defaults, tdcs
from .materials import Material
from .shared import CONTINUOUS_ORDER, SharedNodes, check_layout, shared_nodes

__all__ = [
    "disp_matrix",
    "stress_matrix",
    "total_stress_matrix",
    "eigenstress_matrix",
    "elastic_strain_matrix",
    "traction_matrix",
    "interaction_matrix",
    "collocation_points",
    "interaction_matvec",
    "disp_matvec",
    "stress_matvec",
    "traction_matvec",
]

COLLOCATION_SHRINK = 0.5


def _torch():
    import torch
    return torch


def n_nodes(p: int) -> int:
    return (p + 1) * (p + 2) // 2


def _lattice(p: int) -> np.ndarray:
    """Node multi-indices in the kernels' order (mhs/fullspace/shape.py:55-78)."""
    if p == 0:
        return np.array([[0, 0, 0]])
    out = [[p, 0, 0], [0, p, 0], [0, 0, p]]
    for i, j in ((0, 1), (1, 2), (2, 0)):
        for s in range(1, p):
            a = [0, 0, 0]
            a[i] = p - s
            a[j] = s
            out.append(a)
    for a1 in range(1, p):
        for a2 in range(1, p - a1):
            if p - a1 - a2 >= 1:
                out.append([a1, a2, p - a1 - a2])
    return np.array(out, dtype=int)


def _is_torch(x) -> bool:
    try:
        import torch
    except ImportError:  # pragma: no cover
        return False
    return isinstance(x, torch.Tensor)


# --------------------------------------------------------------- coercion
def _coerce(obs_pts, tris, material, eps):
    """Validate the four arguments every entry point takes; numpy float64
    views for the checks (mhs/matrices.py:75-128)."""
    if not isinstance(material, Material):
        raise TypeError(
            f"material must be an mhs_b200.Material(mu, lam), got {type(material).__name__}. "
            f"(mu, lam) and never nu -- use Material.from_mu_nu(mu, nu) to convert someone "
            f"else's parameters once, at the boundary.")
    obs = _as_np(obs_pts)
    tri = _as_np(tris)
    if obs.ndim != 2 or obs.shape[1] != 3:
        raise ValueError(f"obs_pts must have shape (n_obs, 3), got {obs.shape}")
    if tri.ndim != 3 or tri.shape[1:] != (3, 3):
        raise ValueError(f"tris must have shape (n_src, 3, 3) = (triangle, vertex, xyz), "
                         f"got {tri.shape}")
    if obs.shape[0] == 0 or tri.shape[0] == 0:
        raise ValueError(f"nothing to assemble: {obs.shape[0]} obs points, "
                         f"{tri.shape[0]} source triangles")
    if not np.all(np.isfinite(obs)) or not np.all(np.isfinite(tri)):
        raise ValueError("obs_pts and tris must be finite")
    if np.any(obs[:, 2] > 0.0):
        bad = int(np.argmax(obs[:, 2]))
        raise ValueError(f"the half space is z <= 0 with the free surface at z = 0, but "
                         f"obs_pts[{bad}] has z = {obs[bad, 2]:+.6g} > 0")
    if np.any(tri[:, :, 2] > 0.0):
        s, v = np.unravel_index(int(np.argmax(tri[:, :, 2])), tri.shape[:2])
        raise ValueError(f"the half space is z <= 0, but tris[{s}] vertex {v} has "
                         f"z = {tri[s, v, 2]:+.6g} > 0")
    n_src = tri.shape[0]
    eps_arr = np.ascontiguousarray(np.broadcast_to(_as_np(eps), (n_src,)))
    if not np.all(np.isfinite(eps_arr)) or np.any(eps_arr <= 0.0):
        raise ValueError("eps must be finite and strictly positive -- one value, or one per "
                         "source triangle. eps = 0 is the classical singular kernel, which "
                         "is cutde's job, not this package's.")
    return obs, tri, float(material.mu), float(material.lam), eps_arr


def _as_np(x) -> np.ndarray:
    if _is_torch(x):
        return np.ascontiguousarray(x.detach().to("cpu", dtype=_torch().float64).numpy())
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def _order(order) -> int:
    p = int(order)
    if p not in (0, 1, 2):
        raise ValueError(f"order must be 0, 1 or 2 (P0, P1, P2); got {order!r}. The nodal "
                         f"layout and the generated moment degrees exist for those three.")
    return p


def _coerce_normals(normals, n_obs):
    arr = np.atleast_2d(_as_np(normals))
    if arr.shape == (1, 3) and n_obs != 1:
        arr = np.repeat(arr, n_obs, axis=0)
    if arr.shape != (n_obs, 3):
        raise ValueError(f"obs_normals has shape {np.shape(normals)}; expected ({n_obs}, 3) "
                         f"to match obs_pts, or (3,) for one shared normal")
    mag = np.linalg.norm(arr, axis=1)
    if not np.all(mag > 1e-13):
        raise ValueError(f"obs_normals[{int(np.argmin(mag))}] has length "
                         f"{float(mag.min()):.3e} and so names no plane")
    return arr / mag[:, None]


def _columns(tri, p, layout, shared):
    check_layout(layout)
    if layout == "discontinuous":
        if shared is not None:
            raise ValueError("shared= is the continuous layout's table; pass "
                             "layout='continuous' with it")
        return None, tri.shape[0] * n_nodes(p), None
    if p != CONTINUOUS_ORDER:
        raise ValueError(f"layout='continuous' is quadratic only (order={CONTINUOUS_ORDER}), "
                         f"got order={p}. Continuous P1 is 15-22 % too stiff on the penny "
                         f"crack and P0 has no shared nodes.")
    sn = shared_nodes(tri) if shared is None else shared
    if not isinstance(sn, SharedNodes):
        raise TypeError(f"shared must be a SharedNodes from shared_nodes, got {type(sn).__name__}")
    if sn.n_tri != tri.shape[0]:
        raise ValueError(f"shared describes {sn.n_tri} triangles, tris has {tri.shape[0]}")
    return sn.ids, sn.n, sn


def _precision(precision) -> int:
    if precision in ("fp64", None):
        return _native.FP64
    if precision == "mixed":
        return _native.MIXED
    raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}")


# ------------------------------------------------------------ the device
class _Workspace:
    """Per-device scratch buffer, grown on demand and reused across calls.

    A call holds its device's lock from taking the buffer until its stream
    has synchronised (``lock(device)``), so threads that assemble on the same
    device take turns: none writes the buffer, or frees it by growing it,
    while another's kernels still use it."""

    def __init__(self):
        self.buf = {}
        self.locks = {}
        self.guard = threading.Lock()

    @staticmethod
    def _key(device):
        return device.index if device.index is not None else _torch().cuda.current_device()

    def lock(self, device) -> threading.Lock:
        key = self._key(device)
        with self.guard:
            return self.locks.setdefault(key, threading.Lock())

    def get(self, device, nbytes: int):
        """The device's buffer, at least `nbytes` long; call with lock(device) held."""
        torch = _torch()
        key = self._key(device)
        b = self.buf.get(key)
        if b is None or b.numel() < nbytes:
            b = None
            self.buf.pop(key, None)
            b = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
            self.buf[key] = b
        return b


_WS = _Workspace()

#: Largest device staging buffer of a host (numpy / memmap) ``out=``: the
#: output is assembled in observer-row blocks of at most this many bytes
#: (and at most a quarter of the free device memory), each copied into its
#: rows of ``out`` through pinned memory, so an output larger than the
#: device's memory streams instead of failing.
STREAM_BYTES = 1 << 30


def _device(*xs):
    torch = _torch()
    for x in xs:
        if _is_torch(x) and x.is_cuda:
            return x.device
    if not torch.cuda.is_available():
        raise RuntimeError("mhs_b200 assembles on a CUDA device and none is available "
                           "(there is no CPU path)")
    return torch.device("cuda", torch.cuda.current_device())


def _dev_tensor(a, device):
    torch = _torch()
    if _is_torch(a):
        return a.detach().to(device=device, dtype=torch.float64).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=device)


# Deferred mode (used by mhs_b200.serve): inside ``deferred()`` the public
# functions validate and stage their inputs on the device but return a
# Pending request instead of running it.
_defer = threading.local()


class deferred:
    """Context manager: public matrix functions return :class:`Pending`."""

    def __enter__(self):
        _defer.on = True
        return self

    def __exit__(self, *exc):
        _defer.on = False


class Pending:
    """A validated request, staged on its device and not yet run.  The
    caller supplies the stream and workspace; the result stays on the
    device."""

    def __init__(self, req, keep, out_shape, out_dtype, device, ws_bytes, entries):
        self.req, self.keep = req, keep
        self.out_shape, self.out_dtype, self.device = out_shape, out_dtype, device
        self.ws_bytes = int(ws_bytes)
        self.entries = int(entries)
        self.out = None
        self.ws = None
        self.ready = None   # event after which the staged inputs are on the device
        self.consumer = None  # stream the result is handed to (set by the server)

    @property
    def out_bytes(self) -> int:
        n = 1
        for d in self.out_shape:
            n *= int(d)
        return n * (4 if self.out_dtype == _torch().float32 else 8)

    @property
    def device_bytes(self) -> int:
        """Bytes the run holds on the device: output, workspace, inputs."""
        return self.out_bytes + self.ws_bytes + sum(t.numel() * t.element_size() for t in self.keep)

    def launch(self, stream) -> None:
        """Allocate the output and workspace and queue the assembly on `stream`."""
        torch = _torch()
        if self.ready is not None:
            stream.wait_event(self.ready)
        with torch.cuda.device(self.device), torch.cuda.stream(stream):
            self.out = torch.empty(self.out_shape, dtype=self.out_dtype, device=self.device)
            self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.device)
        self.req.out = ctypes.c_void_p(self.out.data_ptr())
        self.req.workspace = ctypes.c_void_p(self.ws.data_ptr())
        self.req.workspace_bytes = self.ws_bytes
        _native.check(_native.load().mhs_assemble(ctypes.byref(self.req),
                                                  ctypes.c_void_p(stream.cuda_stream)))

    def finish(self, stream):
        """After the stream's work completed: check the device status and
        return the device tensor (workspace and inputs are released)."""
        bits = ctypes.c_int(0)
        _native.check(_native.load().mhs_read_status(ctypes.c_void_p(self.ws.data_ptr()),
                                                     ctypes.c_void_p(stream.cuda_stream),
                                                     ctypes.byref(bits)))
        self.ws, self.keep = None, []
        if bits.value & _native.DEV_FOLD_GRID_OVERFLOW:
            raise RuntimeError("a fold polar grid exceeded its capacity (FOLD_MAX_BREAKS); "
                               "the source is far larger than its eps")
        out, self.out = self.out, None      # the caller's reference is the only one
        return out


def _launch(kind, obs, tri, mu, lam, eps_arr, p, ids, n_dof, out_shape, out, fold,
            subtract=True, normals=None, rec_basis=None, src_basis=None, precision="fp64",
            like=None, slip=None):
    """Run one request; returns the output (numpy or torch per the inputs)."""
    torch = _torch()
    lib = _native.load()
    device = _device(*(like or ()), out)
    return_torch = any(_is_torch(x) for x in (like or ()))
    defer = getattr(_defer, "on", False)
    if defer and out is not None:
        raise ValueError("a served request returns its own device tensor: out= does not apply")
    if out is not None and not _is_torch(out) and slip is None:
        return _launch_streamed(kind, obs, tri, mu, lam, eps_arr, p, ids, n_dof, out_shape, out,
                                fold, subtract, normals, rec_basis, src_basis, precision, device)
    # output buffer
    dev_out = None
    if out is not None and _is_torch(out) and out.is_cuda:
        dev_out = out
    want_f32 = out is not None and (
        (_is_torch(out) and out.dtype == torch.float32) or
        (not _is_torch(out) and np.asarray(out).dtype == np.float32))
    if dev_out is None and not defer:
        dev_out = torch.empty(out_shape, dtype=torch.float32 if want_f32 else torch.float64,
                              device=device)
    keep = []

    def ptr(a):
        if a is None:
            return None
        t = _dev_tensor(a, device)
        keep.append(t)
        return ctypes.c_void_p(t.data_ptr())

    req = _native.Request()
    req.kind = kind
    req.order = p
    req.fold = 1 if fold else 0
    req.subtract_eigenstress = 1 if subtract else 0
    req.precision = _precision(precision)
    req.out_f32 = 1 if want_f32 else 0
    req.n_obs = obs.shape[0]
    req.n_src = tri.shape[0]
    req.obs = ptr(obs)
    req.tris = ptr(tri)
    req.eps = ptr(eps_arr)
    req.mu = mu
    req.lam = lam
    req.normals = ptr(normals)
    req.rec_basis = ptr(rec_basis)
    req.src_basis = ptr(src_basis)
    req.n_a = 0 if rec_basis is None else int(np.shape(rec_basis)[1])
    req.n_b = 0 if src_basis is None else int(np.shape(src_basis)[1])
    req.slip = ptr(slip)
    if ids is not None:
        ids64 = np.ascontiguousarray(ids, dtype=np.int64)
        col_ptr = np.empty(n_dof + 1, dtype=np.int32)
        col_ent = np.empty(ids64.size, dtype=np.int32)
        _native.check(lib.mhs_column_plan(ids64.ctypes.data, ids64.shape[0], n_dof,
                                          col_ptr.ctypes.data, col_ent.ctypes.data))
        for name, arr in (("ids", ids64), ("col_ptr", col_ptr), ("col_ent", col_ent)):
            t = torch.as_tensor(arr, device=device)
            keep.append(t)
            setattr(req, name, ctypes.c_void_p(t.data_ptr()))
        req.n_cols = n_dof
    # (deferred: the output is allocated at launch; the size query only needs
    # a non-null pointer, so it is given the observers' buffer meanwhile)
    req.out = req.obs if dev_out is None else ctypes.c_void_p(dev_out.data_ptr())
    mn, good = ctypes.c_size_t(), ctypes.c_size_t()
    _native.check(lib.mhs_workspace_bytes(ctypes.byref(req), ctypes.byref(mn), ctypes.byref(good)))
    if defer:
        entries = 1
        for d in out_shape:
            entries *= int(d)
        pend = Pending(req, keep, tuple(out_shape), torch.float64, device, good.value, entries)
        # whether any source reaches the fold depth (host copies: the batch
        # sets fold = 0 for requests where it changes nothing)
        depth = -np.asarray(tri, float)[:, :, 2].max(axis=1)
        pend.straddles = bool(fold) and bool(np.any(depth < defaults.FOLD_SOURCE_DEPTH_EPS *
                                                    np.asarray(eps_arr, float)))
        return pend
    with _WS.lock(device):
        ws = _WS.get(device, good.value)
        req.workspace = ctypes.c_void_p(ws.data_ptr())
        req.workspace_bytes = ws.numel()
        with torch.cuda.device(device):
            stream = torch.cuda.current_stream(device)
            _native.check(lib.mhs_assemble(ctypes.byref(req), ctypes.c_void_p(stream.cuda_stream)))
            bits = ctypes.c_int(0)
            _native.check(lib.mhs_read_status(ctypes.c_void_p(ws.data_ptr()),
                                              ctypes.c_void_p(stream.cuda_stream),
                                              ctypes.byref(bits)))
    if bits.value & _native.DEV_FOLD_GRID_OVERFLOW:
        raise RuntimeError("a fold polar grid exceeded its capacity (FOLD_MAX_BREAKS); "
                           "the source is far larger than its eps")
    del keep
    if out is not None:
        if dev_out is not out:
            out.copy_(dev_out)
        return out
    return dev_out if return_torch else dev_out.cpu().numpy()


def _launch_streamed(kind, obs, tri, mu, lam, eps_arr, p, ids, n_dof, out_shape, out, fold,
                     subtract, normals, rec_basis, src_basis, precision, device):
    """A host ``out=`` (numpy array or memmap, possibly larger than the
    device): assemble blocks of observer rows into a device staging buffer
    and copy each into its rows of ``out`` through pinned memory.  Every
    layout's first axis is the observer (receiver) row, so a block of rows
    is a contiguous slab of ``out``; the columns (sources) are whole in each
    block, so the result equals the one-pass assembly (mhs/chunking.py:85-106
    plans the same observer-axis slabs for its own ``out=``)."""
    torch = _torch()
    n_obs = out_shape[0]
    dt = torch.float32 if out.dtype == np.float32 else torch.float64
    row_bytes = int(np.prod(out_shape[1:])) * (4 if dt == torch.float32 else 8)
    free, _ = torch.cuda.mem_get_info(device)
    rows = chunking.stream_rows(n_obs, row_bytes, free, STREAM_BYTES)
    stage = torch.empty((rows,) + tuple(out_shape[1:]), dtype=dt, device=device)
    pinned = torch.empty(stage.shape, dtype=dt, pin_memory=True)

    def part(a, lo, hi):
        return None if a is None else a[lo:hi]

    for lo in range(0, n_obs, rows):
        hi = min(n_obs, lo + rows)
        dev = stage[: hi - lo]
        _launch(kind, obs[lo:hi], tri, mu, lam, eps_arr, p, ids, n_dof,
                (hi - lo,) + tuple(out_shape[1:]), dev, fold, subtract=subtract,
                normals=part(normals, lo, hi), rec_basis=part(rec_basis, lo, hi),
                src_basis=src_basis, precision=precision, like=None)
        host = pinned[: hi - lo]
        host.copy_(dev)
        np.copyto(out[lo:hi], host.numpy())
    return out


def _check_out(out, shape, n_obs, n_src, kind, parts):
    if out is None:
        # a served request's output stays on the device: the serving loop
        # admits it against its device-memory budget instead of the host ceiling
        if not getattr(_defer, "on", False):
            chunking.refuse_if_too_large(n_obs, n_src, kind, np.float64, parts)
        return
    if _is_torch(out):
        torch = _torch()
        if tuple(out.shape) != tuple(shape):
            raise ValueError(f"out has shape {tuple(out.shape)}, expected {shape}")
        if out.dtype not in (torch.float64, torch.float32):
            raise ValueError(f"out must be float64 or float32, got {out.dtype}.")
        if not out.is_contiguous():
            raise ValueError("out must be contiguous")
        return
    if not isinstance(out, np.ndarray):
        raise TypeError(f"out must be a numpy array or torch tensor, got {type(out).__name__}")
    if out.shape != tuple(shape):
        raise ValueError(f"out has shape {out.shape}, expected {shape}")
    if out.dtype not in (np.float64, np.float32):
        raise ValueError(f"out must be float64 or float32, got {out.dtype}. The kernels "
                         f"compute in float64 registers either way; a float32 out is a "
                         f"storage choice that halves the footprint.")


# ----------------------------------------------------------------- public
def disp_matrix(obs_pts, tris, material, eps, *, order=0, layout="discontinuous", shared=None,
                out=None, fold=True, precision="fp64"):
    """Displacement Green's function matrix ``(n_obs, 3, n_dof, 3)``:
    ``[o, i, s, k]`` is displacement ``i`` at ``obs_pts[o]`` from unit
    Cartesian slip ``k`` on source dof ``s`` (mhs/matrices.py:231-248)."""
    obs, tri, mu, lam, eps_arr = _coerce(obs_pts, tris, material, eps)
    p = _order(order)
    ids, n_dof, _ = _columns(tri, p, layout, shared)
    shape = (obs.shape[0], 3, n_dof, 3)
    _check_out(out, shape, obs.shape[0], n_dof, "disp", False)
    return _launch(_native.DISP, obs, tri, mu, lam, eps_arr, p, ids, n_dof, shape, out, fold,
                   precision=precision, like=(obs_pts, tris))


def stress_matrix(obs_pts, tris, material, eps, *, subtract_eigenstress=True, parts=False,
                  order=0, layout="discontinuous", shared=None, out=None, fold=True,
                  precision="fp64"):
    """ELASTIC stress matrix ``(n_obs, 3, 3, n_dof, 3)``, eigenstress removed
    by default; ``parts=True`` returns ``(stress, eigenstress)``
    (mhs/matrices.py:251-295)."""
    obs, tri, mu, lam, eps_arr = _coerce(obs_pts, tris, material, eps)
    p = _order(order)
    ids, n_dof, _ = _columns(tri, p, layout, shared)
    shape = (obs.shape[0], 3, 3, n_dof, 3)
    _check_out(out, shape, obs.shape[0], n_dof, "stress", parts)
    if parts and out is not None:
        raise ValueError("parts=True returns two arrays, so out= cannot name the destination "
                         "of both; call twice with out=, or drop out=.")
    if parts and getattr(_defer, "on", False):
        raise ValueError("a served request returns one matrix: submit stress and "
                         "eigenstress separately")
    sig = _launch(_native.STRESS, obs, tri, mu, lam, eps_arr, p, ids, n_dof, shape, out, fold,
                  subtract=subtract_eigenstress, precision=precision, like=(obs_pts, tris))
    if not parts:
        return sig
    eig = _launch(_native.EIGENSTRESS, obs, tri, mu, lam, eps_arr, p, ids, n_dof, shape, None,
                  fold, precision=precision, like=(obs_pts, tris))
    return sig, eig


def total_stress_matrix(obs_pts, tris, material, eps, *, order=0, layout="discontinuous",
                        shared=None, out=None, fold=True, precision="fp64"):
    """RAW mollified stress, eigenstress included (mhs/matrices.py:494-515)."""
    obs, tri, mu, lam, eps_arr = _coerce(obs_pts, tris, material, eps)
    p = _order(order)
    ids, n_dof, _ = _columns(tri, p, layout, shared)
    shape = (obs.shape[0], 3, 3, n_dof, 3)
    _check_out(out, shape, obs.shape[0], n_dof, "stress", False)
    return _launch(_native.TOTAL_STRESS, obs, tri, mu, lam, eps_arr, p, ids, n_dof, shape, out,
                   fold, precision=precision, like=(obs_pts, tris))


def eigenstress_matrix(obs_pts, tris, material, eps, *, order=0, layout="discontinuous",
                       shared=None, out=None, fold=True, precision="fp64"):
    """The eigenstress ``C:eps*`` alone (mhs/matrices.py:518-543)."""
    obs, tri, mu, lam, eps_arr = _coerce(obs_pts, tris, material, eps)
    p = _order(order)
    ids, n_dof, _ = _columns(tri, p, layout, shared)
    shape = (obs.shape[0], 3, 3, n_dof, 3)
    _check_out(out, shape, obs.shape[0], n_dof, "eigenstress", False)
    return _launch(_native.EIGENSTRESS, obs, tri, mu, lam, eps_arr, p, ids, n_dof, shape, out,
                   fold, precision=precision, like=(obs_pts, tris))


def elastic_strain_matrix(obs_pts, tris, material, eps, *, subtract_eigenstress=True, order=0,
                          layout="discontinuous", shared=None, out=None, fold=True,
                          precision="fp64"):
    """ELASTIC strain ``(n_obs, 3, 3, n_dof, 3)`` by inverting Hooke in
    ``(mu, lam)`` (mhs/matrices.py:546-580)."""
    obs, tri, mu, lam, eps_arr = _coerce(obs_pts, tris, material, eps)
    p = _order(order)
    ids, n_dof, _ = _columns(tri, p, layout, shared)
    shape = (obs.shape[0], 3, 3, n_dof, 3)
    _check_out(out, shape, obs.shape[0], n_dof, "strain", False)
    return _launch(_native.STRAIN, obs, tri, mu, lam, eps_arr, p, ids, n_dof, shape, out, fold,
                   subtract=subtract_eigenstress, precision=precision, like=(obs_pts, tris))


def traction_matrix(obs_pts, obs_normals, tris, material, eps, *, subtract_eigenstress=True,
                    order=0, layout="discontinuous", shared=None, out=None, fold=True,
                    precision="fp64"):
    """ELASTIC traction ``(n_obs, 3, n_dof, 3)`` on the plane through each
    observer with normal ``obs_normals[o]`` (mhs/matrices.py:298-329)."""
    obs, tri, mu, lam, eps_arr = _coerce(obs_pts, tris, material, eps)
    p = _order(order)
    ids, n_dof, _ = _columns(tri, p, layout, shared)
    nrm = _coerce_normals(obs_normals, obs.shape[0])
    shape = (obs.shape[0], 3, n_dof, 3)
    _check_out(out, shape, obs.shape[0], n_dof, "traction", False)
    return _launch(_native.TRACTION, obs, tri, mu, lam, eps_arr, p, ids, n_dof, shape, out, fold,
                   subtract=subtract_eigenstress, normals=nrm, precision=precision,
                   like=(obs_pts, tris))


def collocation_points(tris, order: int = 0, shrink: float = COLLOCATION_SHRINK,
                       layout: str = "discontinuous", shared=None) -> np.ndarray:
    """``(n_dof, 3)`` collocation points in source-dof order: nodes shrunk
    toward the centroid, or the shared nodes themselves
    (mhs/matrices.py:348-375)."""
    tri = _as_np(tris).reshape(-1, 3, 3)
    p = _order(order)
    ids, _, sn = _columns(tri, p, layout, shared)
    if sn is not None:
        if shrink != COLLOCATION_SHRINK:
            raise ValueError("shrink does not apply to the continuous layout: its collocation "
                             "points are the shared nodes")
        return sn.coords.copy()
    bary = np.full((1, 3), 1.0 / 3.0) if p == 0 else _lattice(p) / p
    bary = bary + float(shrink) * (1.0 / 3.0 - bary)
    return (bary[None, :, :] @ tri).reshape(-1, 3)


def _rows(rows, n_rec: int):
    if rows is None:
        return 0, n_rec
    lo, hi = int(rows[0]), int(rows[1])
    if not (0 <= lo < hi <= n_rec):
        raise ValueError(f"rows={rows!r} is not a block of the {n_rec} receiver rows")
    return lo, hi


def _interaction_setup(tris, material, eps, receiver, source, obs_tris, obs_pts, order, shrink,
                       layout, shared, rows):
    tri = _as_np(tris).reshape(-1, 3, 3)
    p = _order(order)
    K = n_nodes(p)
    ids, n_src_dof, sn = _columns(tri, p, layout, shared)
    if sn is not None:
        if obs_tris is not None or obs_pts is not None:
            raise ValueError("layout='continuous' collocates at the shared nodes of tris: "
                             "obs_tris and obs_pts cannot be given. For traction at other "
                             "points use traction_matrix(..., layout='continuous').")
        if shrink != COLLOCATION_SHRINK:
            raise ValueError("shrink does not apply to the continuous layout: its collocation "
                             "points are the shared nodes")
        pts = sn.coords
        rec_frame = sn.frames
        src_frame = sn.frames
        n_rec_dof = sn.n
    else:
        rec_tri = tri if obs_tris is None else _as_np(obs_tris).reshape(-1, 3, 3)
        pts = collocation_points(rec_tri, p, shrink) if obs_pts is None else _as_np(obs_pts)
        n_rec_dof = rec_tri.shape[0] * K
        if np.asarray(pts).shape[0] != n_rec_dof:
            raise ValueError(
                f"interaction_matrix pairs observers with RECEIVER slip DOFs row by row, so at "
                f"order {p} it needs {K} per receiver element: got {np.asarray(pts).shape[0]} "
                f"observers for {rec_tri.shape[0]} receiver triangles ({n_rec_dof} DOFs). For "
                f"traction at unrelated points use traction_matrix(obs_pts, obs_normals, ...).")
        rec_frame = np.repeat(tdcs.slip_frame(rec_tri), K, axis=0)
        src_frame = tdcs.slip_frame(tri)
    lo, hi = _rows(rows, n_rec_dof)
    obs, tri, mu, lam, eps_arr = _coerce(np.asarray(pts, float)[lo:hi], tri, material, eps)
    rec = tdcs.component_index(receiver)
    src = tdcs.component_index(source)
    rec_basis = np.ascontiguousarray(rec_frame[lo:hi][:, rec, :])
    src_basis = np.ascontiguousarray(src_frame[:, src, :])
    normals = np.ascontiguousarray(rec_frame[lo:hi, 2, :])
    return dict(obs=obs, tri=tri, mu=mu, lam=lam, eps_arr=eps_arr, p=p, ids=ids,
                n_src_dof=n_src_dof, lo=lo, hi=hi, rec=rec, src=src, rec_basis=rec_basis,
                src_basis=src_basis, normals=normals)


def interaction_matrix(tris, material, eps, *, receiver=("strike", "dip", "normal"),
                       source=("strike", "dip", "tensile"), obs_tris=None, obs_pts=None, order=0,
                       shrink=COLLOCATION_SHRINK, subtract_eigenstress=True,
                       layout="discontinuous", shared=None, rows=None, out=None, fold=True,
                       precision="fp64"):
    """On-fault interaction ``(n_rec_dof, n_src_dof, n_a, n_b)``: traction on
    each receiver dof's own plane resolved on its (strike, dip, tensile)
    frame from unit slip along each source frame direction
    (mhs/matrices.py:378-480)."""
    g = _interaction_setup(tris, material, eps, receiver, source, obs_tris, obs_pts, order,
                           shrink, layout, shared, rows)
    shape = (g["hi"] - g["lo"], g["n_src_dof"], len(g["rec"]), len(g["src"]))
    _check_out(out, shape, g["hi"] - g["lo"], g["n_src_dof"], (len(g["rec"]), len(g["src"])), False)
    return _launch(_native.INTERACTION, g["obs"], g["tri"], g["mu"], g["lam"], g["eps_arr"], g["p"],
                   g["ids"], g["n_src_dof"], shape, out, fold, subtract=subtract_eigenstress,
                   normals=g["normals"], rec_basis=g["rec_basis"], src_basis=g["src_basis"],
                   precision=precision, like=(tris,))


# ------------------------------------------------------------ apply mode
def _slip_arg(slip, n_dof, n_s, name):
    a = slip.detach().cpu().numpy() if _is_torch(slip) else np.asarray(slip, float)
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.shape != (n_dof, n_s):
        raise ValueError(f"{name}: slip must have shape ({n_dof}, {n_s}), got {a.shape}")
    return a


def interaction_matvec(tris, material, eps, slip, *, receiver=("strike", "dip", "normal"),
                       source=("strike", "dip", "tensile"), obs_tris=None, obs_pts=None, order=0,
                       shrink=COLLOCATION_SHRINK, subtract_eigenstress=True,
                       layout="discontinuous", shared=None, rows=None, fold=True,
                       precision="fp64"):
    """``interaction_matrix(...)`` contracted with a slip vector without
    storing the matrix: ``y[r, a] = sum_{c, b} K[r, c, a, b] slip[c, b]``,
    slip ``(n_src_dof, n_b)``, result ``(n_rec_dof, n_a)`` -- the traction a
    slip distribution puts on every receiver dof (the product a cycle or
    cascade model reads; studies/active_fractal/kernel.py:1-30 stores K
    for it)."""
    g = _interaction_setup(tris, material, eps, receiver, source, obs_tris, obs_pts, order,
                           shrink, layout, shared, rows)
    s = _slip_arg(slip, g["n_src_dof"], len(g["src"]), "interaction_matvec")
    shape = (g["hi"] - g["lo"], len(g["rec"]))
    return _launch(_native.INTERACTION, g["obs"], g["tri"], g["mu"], g["lam"], g["eps_arr"], g["p"],
                   g["ids"], g["n_src_dof"], shape, None, fold, subtract=subtract_eigenstress,
                   normals=g["normals"], rec_basis=g["rec_basis"], src_basis=g["src_basis"],
                   precision=precision, like=(tris, slip), slip=s)


def _field_matvec(kind, comps, name, obs_pts, tris, material, eps, slip, order, layout, shared,
                  fold, precision, subtract=True, normals=None):
    obs, tri, mu, lam, eps_arr = _coerce(obs_pts, tris, material, eps)
    p = _order(order)
    ids, n_dof, _ = _columns(tri, p, layout, shared)
    s = _slip_arg(slip, n_dof, 3, name)
    nrm = None if normals is None else _coerce_normals(normals, obs.shape[0])
    shape = (obs.shape[0],) + comps
    return _launch(kind, obs, tri, mu, lam, eps_arr, p, ids, n_dof, shape, None, fold,
                   subtract=subtract, normals=nrm, precision=precision,
                   like=(obs_pts, tris, slip), slip=s)


def disp_matvec(obs_pts, tris, material, eps, slip, *, order=0, layout="discontinuous",
                shared=None, fold=True, precision="fp64"):
    """``disp_matrix(...)`` contracted with Cartesian slip ``(n_dof, 3)``:
    the displacement ``(n_obs, 3)`` of that slip distribution."""
    return _field_matvec(_native.DISP, (3,), "disp_matvec", obs_pts, tris, material, eps, slip,
                         order, layout, shared, fold, precision)


def stress_matvec(obs_pts, tris, material, eps, slip, *, subtract_eigenstress=True, order=0,
                  layout="discontinuous", shared=None, fold=True, precision="fp64"):
    """``stress_matrix(...)`` contracted with Cartesian slip ``(n_dof, 3)``:
    the stress ``(n_obs, 3, 3)`` of that slip distribution."""
    return _field_matvec(_native.STRESS, (3, 3), "stress_matvec", obs_pts, tris, material, eps,
                         slip, order, layout, shared, fold, precision,
                         subtract=subtract_eigenstress)


def traction_matvec(obs_pts, obs_normals, tris, material, eps, slip, *, subtract_eigenstress=True,
                    order=0, layout="discontinuous", shared=None, fold=True, precision="fp64"):
    """``traction_matrix(...)`` contracted with Cartesian slip
    ``(n_dof, 3)``: the traction ``(n_obs, 3)`` of that slip distribution."""
    return _field_matvec(_native.TRACTION, (3,), "traction_matvec", obs_pts, tris, material, eps,
                         slip, order, layout, shared, fold, precision,
                         subtract=subtract_eigenstress, normals=obs_normals)
