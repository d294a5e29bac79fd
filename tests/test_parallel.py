"""Row sharding across GPUs: cost-balanced contiguous blocks, the band
weighting, and the gather of blocks (world size 2 over gloo on the CPU)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

from mhs_b200 import parallel, synthetic


def test_blocks_cover_the_rows_contiguously_and_balance_cost():
    rng = np.random.default_rng(0)
    costs = rng.uniform(1, 3, 1000)
    costs[100:140] *= 400          # a fold band
    for world in (1, 2, 3, 8):
        b = parallel.row_blocks(costs, world)
        assert b[0][0] == 0 and b[-1][1] == 1000
        assert all(lo < hi for lo, hi in b)
        assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
        tot = [costs[lo:hi].sum() for lo, hi in b]
        assert max(tot) - min(tot) <= 2 * costs.max()
    with pytest.raises(ValueError):
        parallel.row_blocks(np.ones(3), 4)


def test_band_rows_cost_more():
    c = synthetic.config2(seed=1, nu=6, nv=3)
    tris, eps = c["tris"], c["eps"]
    n = tris.shape[0]
    top = tris[np.argmax(tris[:, :, 2].max(axis=1))].mean(axis=0)
    obs = np.array([[top[0], top[1], -0.01], [top[0], top[1], -1e4]])
    cost = parallel.row_costs(obs, tris, eps)
    assert cost[1] == n                                   # no band: one unit per source
    assert cost[0] >= n + parallel.FOLD_PAIR_COST         # inside at least one band
    buried = tris.copy()
    buried[:, :, 2] -= 1e3
    assert np.all(parallel.row_costs(obs, buried, eps) == n)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gather_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 11
        full = torch.arange(n * 4, dtype=torch.float64).reshape(n, 2, 2)
        lo, hi = parallel.row_blocks(np.linspace(1, 5, n), world)[rank]
        got = parallel.gather_rows(full[lo:hi].clone(), lo, hi, n)
        q.put((rank, bool(torch.equal(got, full))))
    finally:
        dist.destroy_process_group()


def test_gather_rows_over_gloo():
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: True, 1: True}
