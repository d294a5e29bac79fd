"""The serving loop (mhs_b200.serve): requests of different kinds, sizes,
orders and precisions submitted together run overlapped on the device, and
each result equals the same request run alone through the public API."""
from __future__ import annotations

import numpy as np
import pytest

from mhs_b200 import synthetic

pytestmark = pytest.mark.gpu


def _requests(torch, dev):
    import mhs_b200 as m
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(10):
        n_u, n_v = int(rng.integers(2, 7)), int(rng.integers(2, 5))
        tris = synthetic.planar_fault(rng.uniform(0, 90), rng.uniform(20, 90), 6.0, 4.0,
                                      -rng.uniform(0, 2), n_u, n_v)
        obs = np.column_stack([rng.uniform(-15, 15, 60), rng.uniform(-15, 15, 60),
                               -rng.uniform(0, 8, 60)])
        t = torch.as_tensor(tris, device=dev)
        o = torch.as_tensor(obs, device=dev)
        mat = m.Material(30.0, float(rng.uniform(20, 40)))
        order = int(rng.integers(0, 3))
        prec = "mixed" if i % 3 == 2 else "fp64"
        kind = i % 4
        if kind == 0:
            reqs.append((m.disp_matrix, (o, t, mat, 0.1), dict(order=order, precision=prec)))
        elif kind == 1:
            reqs.append((m.stress_matrix, (o, t, mat, 0.1), dict(order=order, precision=prec)))
        elif kind == 2:
            nrm = torch.as_tensor(rng.standard_normal((60, 3)), device=dev)
            reqs.append((m.traction_matrix, (o, nrm, t, mat, 0.1), dict(order=order, precision=prec)))
        else:
            reqs.append((m.interaction_matrix, (t, mat, 0.1), dict(order=order, precision=prec)))
    return reqs


@pytest.mark.parametrize("slots", [4, 1])
def test_each_result_is_the_same_alone_and_in_the_mix(cuda, slots):
    import torch
    from mhs_b200 import serve
    reqs = _requests(torch, cuda)
    alone = [fn(*a, **k) for fn, a, k in reqs]
    torch.cuda.synchronize()
    with serve.Server(cuda, slots=slots) as srv:
        futs = [srv.submit(fn, *a, **k) for fn, a, k in reqs]
        mixed = [f.result(timeout=300) for f in futs]
        st = srv.stats()
        peak = srv.peak_in_flight
    for r_alone, r_mix in zip(alone, mixed):
        assert r_mix.is_cuda and r_mix.shape == r_alone.shape
        assert torch.equal(r_alone, r_mix)
    assert st["requests"] == len(reqs) and st["p50_ms"] > 0 and st["p99_ms"] >= st["p50_ms"]
    assert 1 <= peak <= slots
    if slots > 1:
        assert peak > 1, "requests were never in flight together"


def test_byte_budget_admission_and_refusal(cuda):
    import torch
    from mhs_b200 import matrices, serve
    reqs = _requests(torch, cuda)[:6]
    alone = [fn(*a, **k) for fn, a, k in reqs]
    with matrices.deferred():
        sizes = [fn(*a, **k).device_bytes for fn, a, k in reqs]
    budget = max(sizes) + min(sizes)          # never all six at once
    with serve.Server(cuda, budget_bytes=budget, slots=8) as srv:
        res = [f.result(timeout=300) for f in [srv.submit(fn, *a, **k) for fn, a, k in reqs]]
        assert srv.peak_bytes <= budget
    for a, b in zip(alone, res):
        assert torch.equal(a, b)
    big = int(np.argmax(sizes))
    with serve.Server(cuda, budget_bytes=sizes[big] - 1, slots=2) as srv:
        with pytest.raises(MemoryError, match="serving budget"):
            srv.submit(reqs[big][0], *reqs[big][1], **reqs[big][2])


def test_held_results_count_until_dropped(cuda):
    import torch
    from mhs_b200 import matrices, serve
    reqs = _requests(torch, cuda)[:3]
    with matrices.deferred():
        outs = [fn(*a, **k).out_bytes for fn, a, k in reqs]
    with serve.Server(cuda, slots=4) as srv:
        r0 = srv.submit(reqs[0][0], *reqs[0][1], **reqs[0][2]).result(timeout=300)
        srv.drain()
        assert srv.held_bytes == outs[0]
        futs = [srv.submit(fn, *a, **k) for fn, a, k in reqs[1:]]
        res = [f.result(timeout=300) for f in futs]
        srv.drain()
        assert srv.held_bytes == sum(outs)
        del futs, res
        assert _settles(srv, outs[0])
        del r0
        assert _settles(srv, 0)


def _settles(srv, want, seconds=5.0):
    import gc
    import time
    t = time.perf_counter()
    while time.perf_counter() - t < seconds:
        gc.collect()
        if srv.held_bytes == want:
            return True
        time.sleep(0.01)
    return False


@pytest.mark.parametrize("fails", [1, 10**9])
def test_allocator_out_of_memory(cuda, monkeypatch, fails):
    """A launch that the byte budget admitted but the caching allocator
    cannot place (its free blocks fragmented across sizes and streams) is
    retried once after the cache is returned to the device, and requeued
    while other requests are in flight; a request that never fits is
    reported through its future once nothing else is in flight, and every
    other request completes unchanged.  The failures are made on the host:
    the first `fails` launches of the second request to start raise the
    allocator's out-of-memory error."""
    import torch
    from mhs_b200 import matrices, serve
    reqs = _requests(torch, cuda)
    alone = [fn(*a, **k) for fn, a, k in reqs]
    torch.cuda.synchronize()
    real = matrices.Pending.launch
    calls = {}       # launch attempts per request, by order of first launch

    def flaky(self, st):
        # tagged on the object: finished requests are freed, so ids recur
        if not hasattr(self, "_first_launch"):
            self._first_launch = len(calls)
        calls[self._first_launch] = calls.get(self._first_launch, 0) + 1
        if self._first_launch == 1 and calls[1] <= fails:
            raise torch.OutOfMemoryError("CUDA out of memory (made by the test)")
        return real(self, st)

    monkeypatch.setattr(matrices.Pending, "launch", flaky)
    got = []
    with serve.Server(cuda, slots=4) as srv:
        futs = [srv.submit(fn, *a, **k) for fn, a, k in reqs]
        for f in futs:
            try:
                got.append(f.result(timeout=300))
            except torch.OutOfMemoryError:
                got.append(None)
        st = srv.stats()
    failed = [i for i, g in enumerate(got) if g is None]
    assert len(calls) == len(reqs)
    if fails == 1:
        assert not failed and calls[1] == 2                # the retry after emptying the cache
    else:
        assert len(failed) == 1                            # only the request that never fits
    assert all(n == 1 for k, n in calls.items() if k != 1)
    for i, (r_alone, r_mix) in enumerate(zip(alone, got)):
        if i not in failed:
            assert torch.equal(r_alone, r_mix)
    assert st["requests"] == len(reqs) - len(failed)
