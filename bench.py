#!/usr/bin/env python
"""Benchmark: Green's-function entries/s of mhs's interaction matrix on B200.

Workload (one step): the full (3, 3) on-fault interaction matrix of a rough
surface-reaching fault -- a 60 x 20 plane dipping 45 degrees, top edge on
z = 0 (so the fold runs), seeded Gaussian roughness (amplitude 0.5,
correlation length 5), 2,400 triangles, eps per triangle 0.3 x its mean
edge, receivers at the centroids with cutde frames, mu = lam = 30: output
(2400, 2400, 3, 3) float64.  Synthetic, seeded inputs (there is no dataset).

  value      entries/s with inputs resident on the device (CUDA events)
  e2e        entries/s through the public API from pinned host inputs, with
             the host->device copies and the full device->host read of the
             matrix inside the timed region
  roofline   the dominant kernel (a part of the fold): its algorithmic flops
             -- per-unit operation counts of the op-counting host build times
             the device census of its work units in an untimed step -- over
             its time per launch, against the measured FP64 FMA ceiling
  cpu_baseline  the numpy oracle (a restatement of mhs's CPU path, timed
             within 20 % of mhs itself on the same inputs) on a stratified
             sample of the same workload, extrapolated

Further legs (``--legs``): ``mixed`` (the mixed-precision form and its
error against this run's FP64 matrix), ``e2e``, ``c4`` (the continuous P2
interaction of the 3-fault network, ~6,000 triangles, FP64 and mixed),
``serving`` (a seeded Poisson stream through the serving loop at scaled-down
sizes), ``batch`` (the 64 uneven requests of the batched configuration at
their stated sizes), ``serve_full`` (the serving stream at its stated sizes,
bounded by ``--serve-requests``).

``--impl reference`` times the CPU implementation alone on the host cores.
``--gpus N`` (under torchrun): the rows of ONE matrix are split across the
ranks by cost-balanced receiver blocks (mhs_b200.parallel), timed as the
max over ranks; no collective on the data path (strong scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Green's-fn entries/s"
UNIT = "entries/s"
WORKLOAD = "interaction_matrix (3,3), rough surface-reaching fault, 2400 tris, per-tri eps, fold on"
LEGS = ("main", "mixed", "e2e", "c4", "serving", "batch")

#: Wall time of the numpy oracle over mhs itself on the same inputs, timed in
#: the build container (one core each, BLAS at one thread): config-1
#: disp_matrix 7.94 s vs 9.62 s; a config-2 block of 10 ordinary sources x 40
#: receivers 0.31 s vs 0.26 s; one config-2 fold pair 0.26 s vs 0.28 s.
PORT_OVER_MHS = {"c1_disp_matrix": 0.83, "c2_ordinary_block": 1.20, "c2_fold_pair": 0.92}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--nu", type=int, default=60, help="rectangles along strike")
    ap.add_argument("--nv", type=int, default=20, help="rectangles down dip")
    ap.add_argument("--legs", default=",".join(LEGS),
                    help=f"comma list of {LEGS + ('serve_full',)}")
    ap.add_argument("--serve-requests", type=int, default=24)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    return ap.parse_args()


def workload(seed: int, nu: int, nv: int):
    from mhs_b200 import synthetic
    c = synthetic.config2(seed=seed, nu=nu, nv=nv)
    return c["tris"], c["eps"], c["mu"], c["lam"]


# ------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.p = None
        self.out = ""

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                self.out = ""

    def summary(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------- CPU baseline
def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _oracle_rows(args):
    """Oracle interaction of sources `srcs` at receivers `recs` (worker)."""
    import numpy as _np
    sys.path.insert(0, ROOT)
    from oracle import mhs_oracle as O
    tris, eps, mu, lam, recs, srcs = args
    pts = O.collocation_points(tris)
    fr = O.slip_frame(tris)
    t = time.perf_counter()
    O.interaction_matrix(pts[recs], fr[recs, 2, :], fr[recs], tris[srcs], fr[srcs], mu, lam,
                         _np.asarray(eps)[srcs])
    return time.perf_counter() - t


def _one_thread_blas():
    os.environ.update({k: "1" for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS",
                                        "MKL_NUM_THREADS", "NUMEXPR_NUM_THREADS")})
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(1)
    except ImportError:
        pass


def cpu_baseline(tris, eps, mu, lam, seconds: float, seed: int = 1, fold_pairs: int = 256):
    """Stratified sample of the workload through the numpy oracle on all
    host cores (spawned pool, BLAS at one thread per worker): ordinary pairs
    and fold pairs (straddling source, band receiver) timed separately,
    extrapolated to the full matrix."""
    import multiprocessing as mp
    sys.path.insert(0, ROOT)
    from oracle import mhs_oracle as O
    n = tris.shape[0]
    pts = O.collocation_points(tris)
    strad = [s for s in range(n) if O.straddles(tris[s], eps[s])]
    band_of = {s: O.band(pts, tris[s], eps[s]) for s in strad}
    all_fold = [(s, int(r)) for s in strad for r in band_of[s]]
    n_fold = len(all_fold)
    n_reg = n * n - n_fold
    rng = np.random.default_rng(seed)
    cores = max(1, min(os.cpu_count() or 1, 64))
    saved = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS",
                                            "MKL_NUM_THREADS", "NUMEXPR_NUM_THREADS")}
    _one_thread_blas()   # inherited by the spawned workers
    ctx = mp.get_context("spawn")
    jobs_reg = []
    for s in rng.choice(n, size=min(n, 4 * cores), replace=False):
        excl = set(band_of.get(int(s), []))
        recs = [r for r in rng.choice(n, size=min(n, 48), replace=False) if r not in excl]
        if recs:
            jobs_reg.append((tris, eps, mu, lam, np.array(recs, dtype=np.int64),
                             np.array([s], dtype=np.int64)))
    pick = rng.choice(n_fold, size=min(n_fold, fold_pairs), replace=False) if n_fold else []
    jobs_fold = [(tris, eps, mu, lam, np.array([all_fold[i][1]]), np.array([all_fold[i][0]]))
                 for i in pick]
    t_start = time.perf_counter()
    try:
        with ctx.Pool(cores, initializer=_one_thread_blas) as pool:
            pool.map(_oracle_rows, jobs_reg[:cores])  # warm the workers
            t0 = time.perf_counter()
            pool.map(_oracle_rows, jobs_reg)
            t_reg = (time.perf_counter() - t0) / sum(len(j[4]) for j in jobs_reg)
            t0 = time.perf_counter()
            if jobs_fold:
                pool.map(_oracle_rows, jobs_fold, chunksize=1)
            t_fold = (time.perf_counter() - t0) / max(1, len(jobs_fold))
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    total = n_reg * t_reg + n_fold * t_fold
    entries = n * n * 9
    return {"value": entries / total, "unit": UNIT, "cores": cores, "kind": "port",
            "cpu_model": _cpu_model(), "blas_threads_per_worker": 1,
            "port_time_over_mhs": PORT_OVER_MHS,
            "sample": (f"numpy oracle, {sum(len(j[4]) for j in jobs_reg)} ordinary pairs and "
                       f"{len(jobs_fold)} fold pairs (stratified, seeded) timed on a "
                       f"{cores}-process pool, extrapolated to {n_reg} ordinary + {n_fold} fold "
                       f"pairs"),
            "seconds": time.perf_counter() - t_start}


# ------------------------------------------------------------ our arm
def _sync_max(torch, dev, world, x):
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def timed(torch, dev, world, fn, steps, flush):
    """Device time of `steps` calls (CUDA events on the current stream, L2
    flushed before each), max over ranks."""
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(steps)]
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    for i in range(steps):
        flush.fill_(i & 0xFF)
        ev[i][0].record()
        fn()
        ev[i][1].record()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    return _sync_max(torch, dev, world, sum(a.elapsed_time(b) for a, b in ev))


# Algorithmic flops per fold part, from the census and the op-counting build.
def _fold_parts_flops(census, u):
    near_units = (census["near"] * u["near"]["flop"] +
                  census["edge_closed"] * u["edge_closed"]["flop"] +
                  census["edge_small"] * u["edge_small"]["flop"] +
                  census["edge_large"] * u["edge_large"]["flop"])
    far_units = census["far12"] * u["far12"]["flop"] + census["far8"] * u["far8"]["flop"]
    return {"fold_near": near_units, "fold_far": far_units}


def run_ours(a, rank, world, legs):
    import torch
    import mhs_b200 as mhs
    from mhs_b200 import _native, parallel

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    tris, eps, mu, lam = workload(0, a.nu, a.nv)
    n = tris.shape[0]
    mat = mhs.Material(mu, lam)
    t_dev = torch.as_tensor(tris, device=dev)
    e_dev = torch.as_tensor(eps, device=dev)
    # rows of this rank (all of them at N = 1)
    if world > 1:
        costs = parallel.row_costs(mhs.collocation_points(tris), tris, eps)
        lo, hi = parallel.row_blocks(costs, world)[rank]
    else:
        lo, hi = 0, n
    rows = None if world == 1 else (lo, hi)
    out = torch.empty((hi - lo, n, 3, 3), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step(precision=a.precision):
        return mhs.interaction_matrix(t_dev, mat, e_dev, out=out, precision=precision, rows=rows)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    # untimed census of the fold's work units (algorithmic flops, below)
    _native.census(True)
    step()
    census = _native.census_read()
    _native.census(False)
    _native.profile(True)
    _native.profile_read()
    _native.kernel_count()
    with Clocks(dev.index) as clk:
        ms = timed(torch, dev, world, step, a.steps, flush)
    launches = _native.kernel_count() // max(1, a.steps)
    stages = _native.profile_read()
    _native.profile(False)
    entries = n * n * 9
    value = entries * a.steps / (ms * 1e-3)
    stage_ms = {k: v[0] / a.steps for k, v in stages.items()}

    # roofline of the dominant kernel: the fold's near or far loads (or a
    # whole stage when the fold is absent), algorithmic flops over its time
    from mhs_b200 import flops as _flops
    peak = _native.fp_peak(fp64=True)
    fl = _flops.fold_flops(census, order=0, want_h=True, mu=mu, lam=lam,
                           eps=float(np.mean(eps)))
    parts = _fold_parts_flops(census, fl["per_unit"])
    # the pair kernels: a seeded sample of this rank's pairs counted exactly
    pts = mhs.collocation_points(tris)[lo:hi]
    pf = _flops.pair_flops(pts, tris, eps, mu, lam, order=0, want_h=True, samples=4096)
    parts["pair_direct"] = pf["direct"]["flop"]
    parts["pair_image_r"] = pf["image_r"]["flop"]
    # the image Q-family from its census (pairs and rule points counted)
    qf = _flops.imageq_flops(census, order=0, want_h=True, mu=mu, lam=lam)
    parts["imageq"] = qf["flop"]
    per_kernel = {}
    for k, f in parts.items():
        t = stage_ms.get(k, 0.0)
        if t > 0:
            per_kernel[k] = {"ms_per_step": t, "flop_per_step": f,
                             "achieved_tflops": f / (t * 1e-3) / 1e12,
                             "frac_of_measured_fp64": f / (t * 1e-3) / 1e12 / peak}
    top = max(per_kernel, key=lambda k: per_kernel[k]["ms_per_step"]) if per_kernel else None
    fold_ms = stage_ms.get("fold", 0.0)
    roof = {"bound": "fp64", "kernel": top, "unit": "TFLOP/s", "peak": peak,
            "achieved": per_kernel[top]["achieved_tflops"] if top else None,
            "frac": per_kernel[top]["frac_of_measured_fp64"] if top else None,
            "traffic": None,
            "peak_source": "measured FP64 FMA ceiling of this device (mhs_fp_peak, this run); "
                           "of measured",
            "fold_stage": {"ms_per_step": fold_ms, "flop_per_step": fl["flop"],
                           "achieved_tflops": fl["flop"] / (fold_ms * 1e-3) / 1e12 if fold_ms else None,
                           "frac": fl["flop"] / (fold_ms * 1e-3) / 1e12 / peak if fold_ms else None},
            "kernels": per_kernel,
            "pair_kernels": {"samples": pf["samples"], "band_share": pf["band_share"],
                             "k_pair (direct)": pf["direct"], "k_image_r": pf["image_r"],
                             "k_imageq": qf,
                             "counting": "k_pair and k_image_r: a seeded uniform sample of "
                                         "(observer, source) pairs, each counted exactly by the "
                                         "op-counting build, scaled to all pairs; k_imageq: its "
                                         "device census of pairs and rule points times the "
                                         "op-counting build's per-pair and per-point counts"},
            "algorithmic": {"flop_fold": fl["flop"], "div": fl["div"], "sqrt": fl["sqrt"],
                            "special": fl["special"], "census": census,
                            "counting": "op-counting host build of the engine "
                                        "(mhs_b200/csrc/opcount.cpp): add/sub/mul 1 flop, fma 2; "
                                        "div, sqrt, library calls apart"},
            "stage_ms_per_step": stage_ms}

    line = {"metric": METRIC, "value": value,
            "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "weak" if world == 1 else "strong", "vs_baseline": None,
            "dtype": "f64" if a.precision == "fp64" else "f64+f32",
            "data": "synthetic (seeded rough fault mesh)",
            "config": {"workload": WORKLOAD, "n_tri": n, "entries_per_step": entries,
                       "precision": a.precision, "global_batch": 1,
                       "l2": "L2 flushed between steps (256 MiB write); output 415 MB per step",
                       "parallelism": f"row blocks x{world}" if world > 1 else "single GPU"},
            "roofline": roof, "clocks": clk.summary(), "gpu_launches": launches}
    if world > 1:
        # every rank assembled its own row block of the one matrix; value is
        # the whole matrix over the slowest rank's time
        line["config"]["rows_of_rank0"] = [lo, hi]

    if "mixed" in legs and a.precision == "fp64":
        ref = out.clone()
        for _ in range(max(1, a.warmup)):
            step("mixed")
        _native.profile(True)
        _native.profile_read()
        ms_m = timed(torch, dev, world, lambda: step("mixed"), a.steps, flush)
        stages_m = _native.profile_read()
        _native.profile(False)
        err = _sync_max(torch, dev, world,
                        float(((out - ref).abs().max() / ref.abs().max()).item()))
        vm = entries * a.steps / (ms_m * 1e-3)
        line["mixed"] = {"value": vm, "unit": UNIT, "ms_per_step": ms_m / a.steps,
                         "speedup_vs_fp64": vm / line["value"],
                         "relmax_vs_fp64": err,
                         "dtype": "f64+f32 (far-field quadrature bulk in f32)",
                         "stage_ms_per_step": {k: v[0] / a.steps for k, v in stages_m.items()}}
        del ref

    if "e2e" in legs:
        # pinned host inputs, H2D inside, this rank's rows read back
        h_tris = torch.as_tensor(tris).pin_memory()
        h_eps = torch.as_tensor(eps).pin_memory()
        h_out = torch.empty(tuple(out.shape), dtype=torch.float64).pin_memory()
        e2e_steps = max(1, min(a.steps, 3))
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(e2e_steps):
            td = h_tris.to(dev, non_blocking=True)
            ed = h_eps.to(dev, non_blocking=True)
            r = mhs.interaction_matrix(td, mat, ed, out=out, precision=a.precision, rows=rows)
            h_out.copy_(r, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        e2e_ms = _sync_max(torch, dev, world, e0.elapsed_time(e1))
        line["e2e"] = {"value": entries * e2e_steps / (e2e_ms * 1e-3), "unit": UNIT,
                       "h2d_bytes_per_step": int(tris.nbytes + eps.nbytes),
                       "d2h_bytes_per_step": int(out.numel() * 8)}
    del out
    torch.cuda.empty_cache()

    if world == 1:
        if "c4" in legs:
            line["c4"] = c4_leg(torch, dev, flush)
        if "serving" in legs:
            line["serving"] = {"stream": dict(SERVE, note="sizes scaled down from the serving "
                                              "config; arrivals Poisson, seeded; latency = submit "
                                              "to result ready on the device, host clock"),
                               "fp64": serve_stream(dev, "fp64", 100),
                               "mixed": serve_stream(dev, "mixed", 100)}
        if "batch" in legs:
            line["batch"] = {"config": {"requests": 64, "tris": [50, 5000], "obs": [100, 20000],
                                        "note": "the batched configuration at its stated sizes "
                                                "(synthetic.batched_requests) through "
                                                "mhs_b200.batch: one group of launches per class "
                                                "and sub-batch"},
                             "fp64": batch_run(dev, "fp64", 0),
                             "mixed": batch_run(dev, "mixed", 0)}
        if "serve_full" in legs:
            line["serve_full"] = serve_full(dev, a.serve_requests)
    return line, tris, eps, mu, lam


# ------------------------------------------------------------ config 4
def c4_leg(torch, dev, flush):
    """Continuous P2 interaction of the 3-fault network, source = (strike,
    dip), FP64 and mixed: one untimed and one timed step each."""
    import mhs_b200 as mhs
    from mhs_b200 import _native, synthetic
    c = synthetic.config4()
    sn = mhs.shared_nodes(c["tris"], groups=c["groups"])
    mat = mhs.Material(c["mu"], c["lam"])
    t = torch.as_tensor(c["tris"], device=dev)
    out = torch.empty((sn.n, sn.n, 3, 2), dtype=torch.float64, device=dev)
    res = {"workload": "interaction_matrix order=2 continuous, 3-fault network, source=(strike,dip)",
           "n_tri": int(c["tris"].shape[0]), "n_nodes": int(sn.n),
           "entries_per_step": int(out.numel())}
    ref = None
    for prec in ("fp64", "mixed"):
        def step():
            return mhs.interaction_matrix(t, mat, c["eps"], order=2, layout="continuous", shared=sn,
                                          source=("strike", "dip"), out=out, precision=prec)
        step()
        _native.profile(True)
        _native.profile_read()
        ms = timed(torch, dev, 1, step, 1, flush)
        st = _native.profile_read()
        _native.profile(False)
        res[prec] = {"value": out.numel() / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                     "stage_ms_per_step": {k: v[0] for k, v in st.items() if v[1]}}
        if prec == "fp64":
            ref = out.clone()
        else:
            res[prec]["relmax_vs_fp64"] = float(((out - ref).abs().max() / ref.abs().max()).item())
            res[prec]["speedup_vs_fp64"] = res["fp64"]["ms_per_step"] / ms
    del out, ref
    torch.cuda.empty_cache()
    return res


# ------------------------------------------------------------ serving
# Scaled-down serving stream: seeded Poisson arrivals of uneven requests
# (the serving configuration's distributions with the sizes scaled down so
# the stream takes seconds): kind uniform in {disp, stress, traction,
# interaction}, triangles log-uniform in [100, 2000], observers log-uniform
# in [100, 5000], order uniform in {0, 1, 2}, eps per triangle 0.3 x edge.
SERVE = {"requests": 48, "rate_per_s": 20.0, "tris": (100, 2000), "obs": (100, 5000)}


def _submit_args(torch, dev, r, precision):
    import mhs_b200 as mhs
    t = torch.as_tensor(r["tris"], device=dev)
    mat = mhs.Material(r["mu"], r["lam"])
    eps = torch.as_tensor(np.broadcast_to(np.asarray(r["eps"], float), (t.shape[0],)).copy(),
                          device=dev)
    kw = {"order": r["order"], "precision": precision}
    if r["kind"] == "interaction":
        if "receiver" in r:
            kw.update(receiver=r["receiver"], source=r["source"])
        return mhs.interaction_matrix, (t, mat, eps), kw
    o = torch.as_tensor(r["obs"], device=dev)
    if r["kind"] == "disp":
        return mhs.disp_matrix, (o, t, mat, eps), kw
    if r["kind"] == "stress":
        return mhs.stress_matrix, (o, t, mat, eps), kw
    nrm = torch.as_tensor(r["normals"], device=dev)
    return mhs.traction_matrix, (o, nrm, t, mat, eps), kw


def _stream(dev, precision, reqs, slots, budget=None):
    import torch
    from mhs_b200 import serve
    torch.cuda.synchronize()
    refused = 0
    errors = []

    def consume(fut):
        # the client takes each result as it completes and drops it (the
        # server counts a result against its budget while it is referenced)
        e = fut.exception()
        if e is not None:
            errors.append(e)

    with serve.Server(dev, slots=slots, budget_bytes=budget) as srv:
        t0 = time.perf_counter()
        for r in reqs:
            delay = t0 + r["arrival_s"] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            fn, args, kw = _submit_args(torch, dev, r, precision)
            try:
                srv.submit(fn, *args, **kw).add_done_callback(consume)
            except MemoryError:
                refused += 1
        srv.drain()
        t1 = time.perf_counter()
        if errors:
            raise errors[0]
        st = srv.stats()
        st["peak_in_flight"] = srv.peak_in_flight
    st["refused"] = refused
    st["wall_s"] = t1 - t0
    return st


def serve_stream(dev, precision, seed):
    """Latency percentiles and throughput of the scaled-down stream."""
    from mhs_b200 import synthetic
    reqs = synthetic.serving_requests(SERVE["requests"], seed=seed, rate_per_s=SERVE["rate_per_s"],
                                      tri_range=SERVE["tris"], obs_range=SERVE["obs"],
                                      strike_strike=())
    return _stream(dev, precision, reqs, slots=8)


def serve_full(dev, n_requests):
    """The serving stream at its stated sizes (100-20k triangles, 100-50k
    observers, strike/strike interactions at n = 10k and 20k), bounded to
    `n_requests` arrivals at 20/s; admission by device bytes against a
    140 GB budget (requests above it are refused and counted)."""
    from mhs_b200 import synthetic
    reqs = synthetic.serving_requests(n_requests, seed=5)
    out = {"requests_offered": n_requests, "rate_per_s": 20.0, "budget_bytes": 140e9,
           "sizes": {"tris": [100, 20000], "obs": [100, 50000], "strike_strike": [10000, 20000]}}
    for prec in ("fp64", "mixed"):
        out[prec] = _stream(dev, prec, reqs, slots=8, budget=int(140e9))
    return out


def batch_run(dev, precision, seed, budget=50e9):
    """The batched configuration's 64 requests at their stated sizes through
    mhs_b200.batch: packed into sub-batches of at most `budget` output and
    scratch bytes (batch.split), each queued as one group of launches per class; a request
    whose one-pass scratch is above the batch limit runs alone through its
    public function.  Device time from the first submission to the last
    completion (staging and planning apart), and the wall time of it all."""
    import torch
    from mhs_b200 import batch, synthetic
    reqs = synthetic.batched_requests(64, seed=seed)
    calls = [_submit_args(torch, dev, r, precision) for r in reqs]
    groups, big = batch.split(calls, budget)
    rest = [i for g in groups for i in g]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dev_ms, entries = 0.0, 0
    for g in groups:
        bt = batch.Batch([calls[i] for i in g], dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        bt.run()
        e1.record()
        bt.wait()
        dev_ms += e0.elapsed_time(e1)
        entries += bt.entries
        bt.close()
        del bt
    from mhs_b200 import matrices
    for i in big:
        # above the batch limit: through its public function, into a
        # preallocated device output (mhs's own escape from its byte ceiling)
        fn, args, kw = calls[i]
        with matrices.deferred():
            p = fn(*args, **kw)
        out = torch.empty(p.out_shape, dtype=p.out_dtype, device=dev)
        del p
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn(*args, out=out, **kw)
        e1.record()
        torch.cuda.synchronize()
        dev_ms += e0.elapsed_time(e1)
        entries += out.numel()
        del out
    torch.cuda.empty_cache()
    wall = time.perf_counter() - t0
    return {"device_s": dev_ms * 1e-3, "wall_s": wall, "entries": int(entries),
            "entries_per_s": entries / (dev_ms * 1e-3), "sub_batches": len(groups),
            "requests_batched": len(rest), "requests_alone": len(big)}


def main():
    a = parse()
    legs = set(x.strip() for x in a.legs.split(",") if x.strip())
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if a.impl == "reference":
        if rank != 0:
            return 0
        tris, eps, mu, lam = workload(0, a.nu, a.nv)
        vals = []
        for i in range(a.warmup + a.steps):
            r = cpu_baseline(tris, eps, mu, lam, a.cpu_seconds, seed=100 + i,
                             fold_pairs=64 if i < a.warmup else 256)
            if i >= a.warmup:
                vals.append(r)
        v = statistics.median(x["value"] for x in vals)
        cb = dict(vals[-1])
        cb["value"] = v
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
                          "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f64", "data": "synthetic (seeded rough fault mesh)",
                          "config": {"workload": WORKLOAD, "n_tri": tris.shape[0]},
                          "cpu_baseline": cb,
                          "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return 0
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line, tris, eps, mu, lam = run_ours(a, rank, world, legs)
    if rank == 0:
        if world == 1 and not a.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(tris, eps, mu, lam, a.cpu_seconds)
        print(json.dumps(line))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
