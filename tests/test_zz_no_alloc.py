"""The allocation-free entry point, through the C ABI.

``mhs_assemble_noalloc`` serves callers that must not allocate device
memory while they run (a solver whose pool owns the device, a framework
that pre-reserved nearly all of HBM, real-time code that cannot take an
allocation's implicit synchronisation).  It runs the same pipeline on one
fixed scratch array inside the library, so its output must equal the
workspace entry point's -- checked on two calls in a row, because the
array keeps the previous call's contents.  This file is collected last.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import golden, relmax

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _lib():
    from mhs_b200 import _native
    lib = _native.load()
    lib.mhs_assemble_noalloc.argtypes = [ctypes.POINTER(_native.Request), ctypes.c_void_p,
                                         ctypes.POINTER(ctypes.c_int)]
    lib.mhs_assemble_noalloc.restype = ctypes.c_int
    return lib


def _device_memory():
    """Free device bytes and the count of torch allocations made so far."""
    import torch
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    return free, torch.cuda.memory_stats().get("allocation.all.allocated", 0)


def _request(kind, obs, tris, eps, mu, lam, out, keep, normals=None, rec=None, src=None):
    import torch
    from mhs_b200 import _native
    dev = out.device

    def ptr(a):
        t = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
        keep.append(t)
        return ctypes.c_void_p(t.data_ptr())

    r = _native.Request()
    r.kind, r.order, r.fold, r.subtract_eigenstress = kind, 0, 1, 1
    r.precision, r.out_f32 = _native.FP64, 0
    r.n_obs, r.n_src = obs.shape[0], tris.shape[0]
    r.obs, r.tris = ptr(obs), ptr(tris)
    r.eps = ptr(np.broadcast_to(np.asarray(eps, float), (tris.shape[0],)))
    r.mu, r.lam = mu, lam
    if normals is not None:
        r.normals, r.rec_basis, r.src_basis = ptr(normals), ptr(rec), ptr(src)
        r.n_a, r.n_b = rec.shape[1], src.shape[1]
    r.out = ctypes.c_void_p(out.data_ptr())
    return r


def _run_twice(lib, req, out):
    """A set-up call, then two calls in a row.  The first call on a device
    looks up the scratch array's device address, and the kernels' modules
    load on their first launch; after it, a call must leave the device's
    free memory and torch's allocation count exactly as they were.  The
    second of the measured calls reads its status word through
    mhs_read_status(NULL, ...), the array's own status."""
    import torch
    bits = ctypes.c_int(-1)
    assert lib.mhs_assemble_noalloc(ctypes.byref(req), None, ctypes.byref(bits)) == 0, \
        lib.mhs_last_error()
    assert bits.value == 0
    got = [out.cpu().numpy().copy()]
    for i in range(2):
        out.fill_(float("nan"))
        before = _device_memory()
        bits = ctypes.c_int(-1)
        if i == 0:
            rc = lib.mhs_assemble_noalloc(ctypes.byref(req), None, ctypes.byref(bits))
        else:
            rc = lib.mhs_assemble_noalloc(ctypes.byref(req), None, None)
            assert rc == 0, lib.mhs_last_error()
            rc = lib.mhs_read_status(None, None, ctypes.byref(bits))
        assert rc == 0, lib.mhs_last_error()
        assert bits.value == 0
        after = _device_memory()
        assert after == before, f"device memory changed across the call: {before} -> {after}"
        torch.cuda.synchronize()
        got.append(out.cpu().numpy().copy())
    return got


def test_noalloc_matches_workspace_entry_disp(cuda):
    import torch
    import mhs_b200 as m
    from mhs_b200 import _native
    lib = _lib()
    d = golden("c1_subset")
    mu, lam, eps = float(d["mu"]), float(d["lam"]), float(d["eps"])
    ref = m.disp_matrix(d["obs"], d["tris"], m.Material(mu, lam), eps)
    out = torch.empty(ref.shape, dtype=torch.float64, device=cuda)
    keep = []
    req = _request(_native.DISP, d["obs"], d["tris"], eps, mu, lam, out, keep)
    for got in _run_twice(lib, req, out):
        assert relmax(got, ref) < TOL


def test_noalloc_matches_workspace_entry_fold_interaction(cuda):
    import torch
    import mhs_b200 as m
    from mhs_b200 import _native, tdcs
    lib = _lib()
    d = golden("fold")
    mu, lam, eps = float(d["mu"]), float(d["lam"]), float(d["eps"])
    tris = d["tris"]
    ref = m.interaction_matrix(tris, m.Material(mu, lam), eps)
    fr = tdcs.slip_frame(tris)
    pts = m.collocation_points(tris)
    out = torch.empty(ref.shape, dtype=torch.float64, device=cuda)
    keep = []
    req = _request(_native.INTERACTION, pts, tris, eps, mu, lam, out, keep,
                   normals=fr[:, 2, :], rec=fr, src=fr)
    for got in _run_twice(lib, req, out):
        assert relmax(got, ref) < TOL
    assert relmax(got, d["int_p0"]) < TOL


def test_noalloc_refuses_what_does_not_fit(cuda):
    import torch
    from mhs_b200 import _native
    lib = _lib()
    n_src = 20000           # one observer row of P2 tensors exceeds the array
    tris = np.tile(np.array([[[0.0, 0.0, -1.0], [1.0, 0.0, -1.0], [0.0, 1.0, -1.5]]]), (n_src, 1, 1))
    obs = np.array([[0.2, 0.3, -2.0]])
    out = torch.empty((1, 3, n_src * 6, 3), dtype=torch.float64, device=cuda)
    keep = []
    req = _request(_native.DISP, obs, tris, 0.1, 30.0, 30.0, out, keep)
    req.order = 2
    rc = lib.mhs_assemble_noalloc(ctypes.byref(req), None, None)
    assert rc == 2      # MHS_ERR_WORKSPACE
    assert b"allocation-free entry point" in lib.mhs_last_error()
