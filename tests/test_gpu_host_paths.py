"""Host-side paths around the kernels, on the device:

* more than 65,535 sources in one call (sources ride on the grid's x axis);
* a host ``out=`` (numpy array or memmap) filled in observer-row slabs
  equals the one-pass result, for a discontinuous and a continuous layout;
* two threads assembling on the same device at once get exactly what each
  gets alone (the shared workspace is taken in turns);
* served results freed by the caller while later requests run stay intact
  until freed (the consumer's stream is recorded on them).
"""
from __future__ import annotations

import threading

import numpy as np
import pytest

from conftest import golden, relmax
from mhs_b200 import synthetic

pytestmark = pytest.mark.gpu


def test_more_sources_than_one_grid_row(cuda):
    import mhs_b200 as m
    n = 70_003
    base = np.array([[0.0, 0.0, -2.0], [0.3, 0.0, -2.0], [0.0, 0.3, -2.2]])
    shift = np.zeros((n, 1, 3))
    shift[:, 0, 0] = 0.5 * np.arange(n)
    tris = base[None] + shift
    obs = np.array([[10.0, 5.0, -1.0], [35_000.0, -3.0, -4.0], [1e5, 2.0, 0.0]])
    mat = m.Material(30.0, 30.0)
    U = m.disp_matrix(obs, tris, mat, 0.1, fold=False)
    assert U.shape == (3, 3, n, 3)
    for lo, hi in ((0, 50), (65_530, 65_545), (n - 40, n)):
        part = m.disp_matrix(obs, tris[lo:hi], mat, 0.1, fold=False)
        assert np.array_equal(U[:, :, lo:hi], part)


@pytest.mark.parametrize("layout", ["discontinuous", "continuous"])
def test_host_out_streams_in_row_slabs(cuda, monkeypatch, tmp_path, layout):
    import mhs_b200 as m
    from mhs_b200 import matrices
    d = golden("continuous")
    mat = m.Material(float(d["mu"]), float(d["lam"]))
    kw = dict(order=2, layout=layout) if layout == "continuous" else dict(order=1)
    whole = m.traction_matrix(d["obs"], d["obs_normals"], d["tris"], mat, 0.1, **kw)
    row_bytes = whole[0].nbytes
    monkeypatch.setattr(matrices, "STREAM_BYTES", 3 * row_bytes)      # slabs of 3 rows
    out = np.full(whole.shape, np.nan)
    res = m.traction_matrix(d["obs"], d["obs_normals"], d["tris"], mat, 0.1, out=out, **kw)
    assert res is out and np.array_equal(out, whole)
    mm = np.lib.format.open_memmap(tmp_path / "t.npy", mode="w+", dtype=np.float64,
                                   shape=whole.shape)
    m.traction_matrix(d["obs"], d["obs_normals"], d["tris"], mat, 0.1, out=mm, **kw)
    assert np.array_equal(np.asarray(mm), whole)
    out32 = np.zeros(whole.shape, dtype=np.float32)
    m.traction_matrix(d["obs"], d["obs_normals"], d["tris"], mat, 0.1, out=out32, **kw)
    assert relmax(out32, whole) < 1e-6


def test_interaction_rows_stream_into_host_out(cuda, monkeypatch):
    import mhs_b200 as m
    from mhs_b200 import matrices
    d = golden("interaction")
    mat = m.Material(float(d["mu"]), float(d["lam"]))
    ref = d["int_p0"]
    monkeypatch.setattr(matrices, "STREAM_BYTES", 5 * ref[0].nbytes)
    out = np.empty_like(ref)
    m.interaction_matrix(d["tris"], mat, float(d["eps"]), out=out)
    assert relmax(out, ref) < 1e-12


def test_two_threads_on_one_device(cuda):
    import torch
    import mhs_b200 as m
    c = synthetic.config2(seed=5, nu=6, nv=3)
    mat = m.Material(c["mu"], c["lam"])
    d = golden("orders")
    jobs = [lambda: m.interaction_matrix(c["tris"], mat, c["eps"]),
            lambda: m.stress_matrix(d["obs"], d["tris"], m.Material(30.0, 20.0), 0.15, order=2)]
    alone = [j() for j in jobs]
    got = [None] * len(jobs)
    errors = []

    def worker(i):
        try:
            s = torch.cuda.Stream(cuda)
            with torch.cuda.stream(s):
                for _ in range(3):
                    got[i] = jobs[i]()
        except Exception as e:  # noqa: BLE001
            errors.append(e)

    th = [threading.Thread(target=worker, args=(i,)) for i in range(len(jobs))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
    for a, b in zip(alone, got):
        assert np.array_equal(a, b)


def test_served_results_freed_while_later_requests_run(cuda):
    import torch
    import mhs_b200 as m
    from mhs_b200 import serve
    d = golden("orders")
    mat = m.Material(30.0, 20.0)
    obs = torch.as_tensor(d["obs"], device=cuda)
    tris = torch.as_tensor(d["tris"], device=cuda)
    ref = m.stress_matrix(obs, tris, mat, 0.15, order=1)
    ref_sum = float(ref.double().abs().sum())
    sums = []
    with serve.Server(cuda, slots=2) as srv:
        futs = [srv.submit(m.stress_matrix, obs, tris, mat, 0.15, order=1) for _ in range(12)]
        for f in futs:
            r = f.result(timeout=300)
            # read the result on the caller's stream, then drop it while the
            # server keeps launching requests on its own streams
            sums.append(r.abs().sum())
            del r
        srv.drain()
    torch.cuda.synchronize()
    assert all(abs(float(s) - ref_sum) == 0.0 for s in sums)
