"""Batched assembly (mhs_b200.batch): uneven requests of every kind, order
and precision queued as one group of launches per class give exactly the
matrices the same calls give alone; a batch without fold work captured
into a CUDA graph replays to the same matrices; the autotuner's launch
shapes change no result."""
from __future__ import annotations

import numpy as np
import pytest

from mhs_b200 import synthetic

pytestmark = pytest.mark.gpu


def _calls(torch, dev, seed, surface=True, n=12):
    import mhs_b200 as m
    rng = np.random.default_rng(seed)
    calls = []
    for i in range(n):
        n_u, n_v = int(rng.integers(2, 6)), int(rng.integers(1, 4))
        top = -rng.uniform(0.0, 0.3) if (surface and i % 3 == 0) else -rng.uniform(1.0, 3.0)
        tris = synthetic.planar_fault(rng.uniform(0, 90), rng.uniform(25, 90), 5.0, 3.0, top,
                                      n_u, n_v)
        no = int(rng.integers(20, 90))
        obs = np.column_stack([rng.uniform(-9, 9, no), rng.uniform(-9, 9, no),
                               -rng.uniform(0, 5, no)])
        t = torch.as_tensor(tris, device=dev)
        o = torch.as_tensor(obs, device=dev)
        mat = m.Material(30.0, float(rng.uniform(20, 40)))
        kw = dict(order=int(rng.integers(0, 3)), precision="mixed" if i % 4 == 3 else "fp64")
        eps = 0.1 + 0.05 * (i % 2)
        k = i % 4
        if k == 0:
            calls.append((m.disp_matrix, (o, t, mat, eps), kw))
        elif k == 1:
            calls.append((m.stress_matrix, (o, t, mat, eps), kw))
        elif k == 2:
            nrm = torch.as_tensor(rng.standard_normal((no, 3)), device=dev)
            calls.append((m.traction_matrix, (o, nrm, t, mat, eps), kw))
        else:
            calls.append((m.interaction_matrix, (t, mat, eps), kw))
    return calls


def test_batch_equals_each_call_alone(cuda):
    import torch
    from mhs_b200 import batch
    calls = _calls(torch, cuda, 3)
    alone = [fn(*a, **k) for fn, a, k in calls]
    b = batch.Batch(calls, cuda)
    assert not b.capturable            # some requests reach the surface
    outs = b.run()
    b.wait()
    for x, y in zip(alone, outs):
        assert x.shape == y.shape and torch.equal(x, y)
    # a second submission over the same arena gives the same matrices
    for y in outs:
        y.fill_(float("nan"))
    b.run()
    b.wait()
    for x, y in zip(alone, outs):
        assert torch.equal(x, y)


def test_captured_batch_replays(cuda):
    import torch
    from mhs_b200 import batch
    calls = _calls(torch, cuda, 5, surface=False)
    alone = [fn(*a, **k) for fn, a, k in calls]
    b = batch.Batch(calls, cuda)
    assert b.capturable
    b.graph()
    for _ in range(2):
        for y in b.outputs:
            y.fill_(float("nan"))
        outs = b.replay()
        torch.cuda.synchronize()
        for x, y in zip(alone, outs):
            assert torch.equal(x, y)


def test_autotuned_shapes_change_no_result(cuda):
    import torch
    import mhs_b200 as m
    from mhs_b200 import batch
    c = synthetic.config2(seed=7, nu=8, nv=3)
    t = torch.as_tensor(c["tris"], device=cuda)
    e = torch.as_tensor(c["eps"], device=cuda)
    mat = m.Material(c["mu"], c["lam"])
    before = m.interaction_matrix(t, mat, e)
    shape, ms = batch.autotune(m.interaction_matrix, t, mat, e)
    assert shape["pair_tb"] in (64, 128) and shape["far_mult"] in (2, 4, 8) and ms > 0
    after = m.interaction_matrix(t, mat, e)
    assert torch.equal(before, after)


def test_split_respects_budget_and_covers_all(cuda):
    import torch
    from mhs_b200 import batch, matrices
    calls = _calls(torch, cuda, 9, n=10)
    with matrices.deferred():
        pend = [fn(*a, **k) for fn, a, k in calls]
    budget = 3 * max(p.out_bytes + p.ws_bytes for p in pend)
    groups, alone = batch.split(calls, budget)
    assert not alone
    assert sorted(i for g in groups for i in g) == list(range(len(calls)))
    assert len(groups) > 1
