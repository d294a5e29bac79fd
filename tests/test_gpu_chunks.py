"""Chunked assembly through the C ABI.  A workspace that holds only a few
observer rows at a time (so the last chunk is ragged) must give the same
matrix, bit for bit, as the good-size workspace's single chunk: the pair
table, the image R-family's table buffer (observer-innermost, strided by the
chunk's rows) and the fold's region are all laid out per chunk, and no sum
depends on how rows fall into chunks or panels into waves."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(a, dev, keep):
    import torch
    t = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    keep.append(t)
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("order", [0, 1, 2])
def test_small_workspace_chunks_equal_one_chunk(cuda, order):
    import torch
    import mhs_b200 as m
    from mhs_b200 import _native, synthetic
    lib = _native.load()
    c = synthetic.config2(seed=3, nu=6, nv=3)            # 36 triangles reaching z = 0
    tris, eps = c["tris"], np.asarray(c["eps"], float)      # eps per triangle
    mat = m.Material(c["mu"], c["lam"])
    cen = tris.mean(axis=1)
    obs = np.concatenate([cen - [0.0, 0.0, 0.05], cen[:17] * [1.0, 1.0, 0.02] - [0.3, 0.1, 0.01]])
    ref = m.stress_matrix(obs, tris, mat, eps, order=order)   # one chunk (good size)
    ref = ref.cpu().numpy() if hasattr(ref, "cpu") else np.asarray(ref)

    keep = []
    out = torch.full(ref.shape, float("nan"), dtype=torch.float64, device=cuda)
    r = _native.Request()
    r.kind, r.order, r.fold, r.subtract_eigenstress = _native.STRESS, order, 1, 1
    r.precision, r.out_f32 = _native.FP64, 0
    r.n_obs, r.n_src = obs.shape[0], tris.shape[0]
    r.obs, r.tris, r.eps = _ptr(obs, cuda, keep), _ptr(tris, cuda, keep), _ptr(eps, cuda, keep)
    r.mu, r.lam = float(c["mu"]), float(c["lam"])
    r.out = ctypes.c_void_p(out.data_ptr())
    mn, good = ctypes.c_size_t(), ctypes.c_size_t()
    assert lib.mhs_workspace_bytes(ctypes.byref(r), ctypes.byref(mn), ctypes.byref(good)) == 0
    # The minimum holds one observer row beside the smallest fold region; a
    # few rows more (per row and source: its band-list entry, and per node
    # the 27 + 2 doubles of the pair table and the 49 of the image tables)
    # make chunks of about four rows, the last one ragged.
    K = (order + 1) * (order + 2) // 2
    row = tris.shape[0] * (4 + K * (29 + 49) * 8)
    nbytes = int(mn.value + 3.5 * row)
    assert nbytes < good.value
    ws = torch.empty(nbytes, dtype=torch.uint8, device=cuda)
    r.workspace, r.workspace_bytes = ctypes.c_void_p(ws.data_ptr()), nbytes
    _native.kernel_count()                                   # the count resets on reading
    assert lib.mhs_assemble(ctypes.byref(r), None) == 0, lib.mhs_last_error()
    n_small = _native.kernel_count()
    m.stress_matrix(obs, tris, mat, eps, order=order)
    n_one = _native.kernel_count()
    assert n_small > 2 * n_one, (n_small, n_one)              # several chunks ran
    bits = ctypes.c_int(-1)
    assert lib.mhs_read_status(ctypes.c_void_p(ws.data_ptr()), None, ctypes.byref(bits)) == 0
    assert bits.value == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.isfinite(got).all()
    assert np.array_equal(got, ref)
