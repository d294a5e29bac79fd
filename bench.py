#!/usr/bin/env python
"""Benchmark: Green's-function entries/s of mhs's interaction matrix on B200.

Workload (one step): the full (3, 3) on-fault interaction matrix of a rough
surface-reaching fault -- a 60 x 20 plane dipping 45 degrees, top edge on
z = 0 (so the fold runs), seeded Gaussian roughness (amplitude 0.5,
correlation length 5), 2,400 triangles, eps per triangle 0.3 x its mean
edge, receivers at the centroids with cutde frames, mu = lam = 30: output
(2400, 2400, 3, 3) float64.  Synthetic, seeded inputs (there is no dataset).

  value  entries/s with inputs resident on the device (CUDA events)
  e2e    entries/s through the public API from pinned host inputs, with the
         host->device copies and the full device->host read of the matrix
         inside the timed region
  roofline   the dominant stage (the fold): its algorithmic flops -- per-unit
         operation counts of the op-counting host build times the device
         census of its work units in an untimed step -- over its time per
         launch, against the measured FP64 FMA ceiling
  cpu_baseline   the numpy oracle (a restatement of mhs's CPU path) on a
         stratified sample of the same workload, extrapolated

``--impl reference`` times that CPU implementation alone on the host cores.
``--gpus N`` (under torchrun) runs N independent replicas, one seeded mesh
per rank (weak scaling, no collective on the data path).
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

# DRAM bytes (read + write) of one k_fold launch on this workload, from
# profiles/fold_c2_traffic.md; keyed by (nu, nv, precision).
FOLD_TRAFFIC_PER_LAUNCH = {(60, 20, "fp64"): 120.4e6 + 1.78e9}
# Kernels each profiled stage launches (csrc/mhs_b200.cu: run()).
KERNELS_PER_STAGE = {"prep": 2, "pair": 1, "imageq": 1, "fold": 3, "final": 1}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--nu", type=int, default=60, help="rectangles along strike")
    ap.add_argument("--nv", type=int, default=20, help="rectangles down dip")
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
def _oracle_rows(args):
    """Oracle interaction of sources `srcs` at receivers `recs` (worker)."""
    import numpy as _np
    sys.path.insert(0, ROOT)
    from oracle import mhs_oracle as O
    tris, eps, mu, lam, recs, srcs = args
    K = O.self_interaction  # noqa: F841  (module warm-up)
    pts = O.collocation_points(tris)
    fr = O.slip_frame(tris)
    t = time.perf_counter()
    O.interaction_matrix(pts[recs], fr[recs, 2, :], fr[recs], tris[srcs], fr[srcs], mu, lam,
                         _np.asarray(eps)[srcs])
    return time.perf_counter() - t


def cpu_baseline(tris, eps, mu, lam, seconds: float, seed: int = 1):
    """Stratified sample of the workload through the numpy oracle on all
    host cores (spawned pool): fold pairs (straddling source, band receiver)
    and ordinary pairs timed separately, extrapolated to the full matrix."""
    import multiprocessing as mp
    sys.path.insert(0, ROOT)
    from oracle import mhs_oracle as O
    n = tris.shape[0]
    pts = O.collocation_points(tris)
    strad = [s for s in range(n) if O.straddles(tris[s], eps[s])]
    band_of = {s: O.band(pts, tris[s], eps[s]) for s in strad}
    n_fold = sum(len(b) for b in band_of.values())
    n_reg = n * n - n_fold
    rng = np.random.default_rng(seed)
    cores = max(1, min(os.cpu_count() or 1, 64))
    ctx = mp.get_context("spawn")
    jobs_reg, jobs_fold = [], []
    # ordinary pairs: sources paired with receivers outside their band
    for s in rng.choice(n, size=min(n, 4 * cores), replace=False):
        excl = set(band_of.get(int(s), []))
        recs = [r for r in rng.choice(n, size=min(n, 48), replace=False) if r not in excl]
        if recs:
            jobs_reg.append((tris, eps, mu, lam, np.array(recs, dtype=np.int64),
                             np.array([s], dtype=np.int64)))
    for s in rng.choice(strad, size=min(len(strad), 2 * cores), replace=False):
        b = band_of[int(s)]
        if len(b):
            jobs_fold.append((tris, eps, mu, lam, rng.choice(b, size=1), np.array([s])))
    t_start = time.perf_counter()
    with ctx.Pool(cores) as pool:
        pool.map(_oracle_rows, jobs_reg[:cores])  # warm the workers
        t0 = time.perf_counter()
        pool.map(_oracle_rows, jobs_reg)
        t_reg = (time.perf_counter() - t0) / sum(len(j[4]) for j in jobs_reg)
        t0 = time.perf_counter()
        pool.map(_oracle_rows, jobs_fold)
        t_fold = (time.perf_counter() - t0) / max(1, len(jobs_fold))
    total = n_reg * t_reg + n_fold * t_fold
    entries = n * n * 9
    return {"value": entries / total, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": (f"numpy oracle, {sum(len(j[4]) for j in jobs_reg)} ordinary pairs and "
                       f"{len(jobs_fold)} fold pairs timed on a {cores}-process pool, "
                       f"extrapolated to {n_reg} ordinary + {n_fold} fold pairs"),
            "seconds": time.perf_counter() - t_start}


# ----------------------------------------------------------- our arm
# Serving stream: seeded Poisson arrivals of uneven requests (the BASELINE
# serving config's distributions with the sizes scaled down so the stream
# takes seconds): kind uniform in {disp, stress, traction, interaction},
# triangles log-uniform in [100, 2000], observers log-uniform in [100, 5000],
# order uniform in {0, 1, 2}, eps per triangle 0.3 x its mean edge.
SERVE = {"requests": 48, "rate_per_s": 20.0, "tris": (100, 2000), "obs": (100, 5000)}


def _serve_requests(torch, dev, seed):
    import mhs_b200 as mhs
    from mhs_b200 import synthetic
    rng = np.random.default_rng(seed)
    out = []
    for i in range(SERVE["requests"]):
        nt = int(np.exp(rng.uniform(*np.log(SERVE["tris"]))))
        no = int(np.exp(rng.uniform(*np.log(SERVE["obs"]))))
        nv = max(1, int(round(np.sqrt(nt / 6.0))))
        nu = max(1, int(round(nt / (2 * nv))))
        L, W = 2.0 * nu, 2.0 * nv
        tris = synthetic.planar_fault(rng.uniform(0, 180), rng.uniform(15, 90), L, W,
                                      -rng.uniform(0, 5), nu, nv)
        edges = np.linalg.norm(tris - np.roll(tris, 1, axis=1), axis=2).mean(axis=1)
        eps = torch.as_tensor(0.3 * edges, device=dev)
        ext = 1.5 * max(L, W)
        obs = np.column_stack([rng.uniform(-ext, ext, no), rng.uniform(-ext, ext, no),
                               -rng.uniform(0, ext, no)])
        t = torch.as_tensor(tris, device=dev)
        o = torch.as_tensor(obs, device=dev)
        mat = mhs.Material(30.0, float(rng.uniform(20, 40)))
        order = int(rng.integers(0, 3))
        kind = int(rng.integers(0, 4))
        if kind == 0:
            r = (mhs.disp_matrix, (o, t, mat, eps), {"order": order})
        elif kind == 1:
            r = (mhs.stress_matrix, (o, t, mat, eps), {"order": order})
        elif kind == 2:
            nrm = torch.as_tensor(rng.standard_normal((no, 3)), device=dev)
            r = (mhs.traction_matrix, (o, nrm, t, mat, eps), {"order": order})
        else:
            r = (mhs.interaction_matrix, (t, mat, eps), {"order": order})
        out.append((r, float(rng.exponential(1.0 / SERVE["rate_per_s"]))))
    return out


def serve_stream(dev, precision, seed):
    """Latency percentiles and throughput of the seeded stream through the
    serving loop (requests overlap on the device)."""
    import torch
    from mhs_b200 import serve
    reqs = _serve_requests(torch, dev, seed)
    torch.cuda.synchronize()
    with serve.Server(dev, slots=8) as srv:
        futs = []
        t_next = time.perf_counter()
        for (fn, args, kw), gap in reqs:
            t_next += gap
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            futs.append(srv.submit(fn, *args, precision=precision, **kw))
        for f in futs:
            f.result()
        st = srv.stats()
        st["peak_in_flight"] = srv.peak_in_flight
    return st


# Batched uneven assembly: 64 seeded requests (the batched config's
# distributions: kind uniform in {disp, stress, traction}, order uniform in
# {0, 1, 2}, dip in [15, 90] degrees, top depth in [0, 5], lam in [20, 40],
# eps 0.1; sizes scaled down -- triangles log-uniform in [50, 1000],
# observers in [100, 4000] -- so the batch takes seconds), all submitted at
# once to the serving loop, which overlaps them on the device.
BATCH = {"requests": 64, "tris": (50, 1000), "obs": (100, 4000)}


def _batch_requests(torch, dev, seed):
    import mhs_b200 as mhs
    from mhs_b200 import synthetic
    rng = np.random.default_rng(seed)
    out = []
    for i in range(BATCH["requests"]):
        nt = int(np.exp(rng.uniform(*np.log(BATCH["tris"]))))
        no = int(np.exp(rng.uniform(*np.log(BATCH["obs"]))))
        nv = max(1, int(round(np.sqrt(nt / 6.0))))
        nu = max(1, int(round(nt / (2 * nv))))
        L, W = 2.0 * nu, 2.0 * nv
        tris = synthetic.planar_fault(0.0, rng.uniform(15, 90), L, W, -rng.uniform(0, 5), nu, nv)
        ext = 1.5 * max(L, W)
        obs = np.column_stack([rng.uniform(-ext, ext, no), rng.uniform(-ext, ext, no),
                               -rng.uniform(0, ext, no)])
        t = torch.as_tensor(tris, device=dev)
        o = torch.as_tensor(obs, device=dev)
        mat = mhs.Material(30.0, float(rng.uniform(20, 40)))
        order = int(rng.integers(0, 3))
        kind = int(rng.integers(0, 3))
        if kind == 0:
            out.append((mhs.disp_matrix, (o, t, mat, 0.1), {"order": order}))
        elif kind == 1:
            out.append((mhs.stress_matrix, (o, t, mat, 0.1), {"order": order}))
        else:
            v = rng.standard_normal((no, 3))
            nrm = torch.as_tensor(v / np.linalg.norm(v, axis=1, keepdims=True), device=dev)
            out.append((mhs.traction_matrix, (o, nrm, t, mat, 0.1), {"order": order}))
    return out


def batch_run(dev, precision, seed):
    """Makespan and entries/s of the seeded batch, all requests submitted at
    once (device time from the first submit to the last result)."""
    import torch
    from mhs_b200 import serve
    reqs = _batch_requests(torch, dev, seed)
    torch.cuda.synchronize()
    with serve.Server(dev, slots=16) as srv:
        t0 = time.perf_counter()
        futs = [srv.submit(fn, *args, precision=precision, **kw) for fn, args, kw in reqs]
        for f in futs:
            f.result()
        t1 = time.perf_counter()
        st = srv.stats()
    return {"makespan_s": t1 - t0, "entries": st["entries"],
            "entries_per_s": st["entries"] / (t1 - t0), "p50_ms": st["p50_ms"],
            "p99_ms": st["p99_ms"], "peak_in_flight": srv.peak_in_flight}


def run_ours(a, rank, world):
    import torch
    import mhs_b200 as mhs
    from mhs_b200 import _native

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    tris, eps, mu, lam = workload(rank, a.nu, a.nv)
    n = tris.shape[0]
    mat = mhs.Material(mu, lam)
    t_dev = torch.as_tensor(tris, device=dev)
    e_dev = torch.as_tensor(eps, device=dev)
    out = torch.empty((n, n, 3, 3), dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        return mhs.interaction_matrix(t_dev, mat, e_dev, out=out, precision=a.precision)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    # untimed census of the fold's work units (algorithmic flops, below)
    _native.census(True)
    step()
    census = _native.census_read()
    _native.census(False)
    if world > 1:
        torch.distributed.barrier()
    _native.profile(True)
    _native.profile_read()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(a.steps)]
    torch.cuda.synchronize()
    with Clocks(dev.index) as clk:
        for i in range(a.steps):
            flush.fill_(i & 0xFF)          # evict L2 between steps (untimed)
            ev[i][0].record()
            step()
            ev[i][1].record()
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    stages = _native.profile_read()
    _native.profile(False)
    ms = sum(s.elapsed_time(e) for s, e in ev)
    ms_t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(ms_t, op=torch.distributed.ReduceOp.MAX)
    ms = float(ms_t.item())
    entries = n * n * 9
    value = world * entries * a.steps / (ms * 1e-3)

    # the mixed form beside the FP64 one, same protocol; its error is the
    # relmax of its matrix against this run's FP64 matrix
    mixed = None
    if a.precision == "fp64":
        ref = out.clone()

        def step_mixed():
            return mhs.interaction_matrix(t_dev, mat, e_dev, out=out, precision="mixed")

        for _ in range(max(1, a.warmup)):
            step_mixed()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        _native.profile(True)
        _native.profile_read()
        evm = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(a.steps)]
        for i in range(a.steps):
            flush.fill_(i & 0xFF)
            evm[i][0].record()
            step_mixed()
            evm[i][1].record()
        torch.cuda.synchronize()
        stages_m = _native.profile_read()
        _native.profile(False)
        ms_m = sum(x.elapsed_time(y) for x, y in evm)
        ms_mt = torch.tensor([ms_m], dtype=torch.float64, device=dev)
        err = float(((out - ref).abs().max() / ref.abs().max()).item())
        err_t = torch.tensor([err], dtype=torch.float64, device=dev)
        if world > 1:
            torch.distributed.all_reduce(ms_mt, op=torch.distributed.ReduceOp.MAX)
            torch.distributed.all_reduce(err_t, op=torch.distributed.ReduceOp.MAX)
        ms_m = float(ms_mt.item())
        vm = world * entries * a.steps / (ms_m * 1e-3)
        mixed = {"value": vm, "unit": UNIT, "ms_per_step": ms_m / a.steps,
                 "speedup_vs_fp64": vm / value, "relmax_vs_fp64": float(err_t.item()),
                 "dtype": "f64+f32 (far-field quadrature bulk in f32)",
                 "stage_ms_per_step": {k: v[0] / a.steps for k, v in stages_m.items()}}
        del ref

    # end to end: pinned host inputs, H2D inside, full matrix read back
    h_tris = torch.as_tensor(tris).pin_memory()
    h_eps = torch.as_tensor(eps).pin_memory()
    h_out = torch.empty((n, n, 3, 3), dtype=torch.float64).pin_memory()
    e2e_steps = max(1, min(a.steps, 3))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(e2e_steps):
        td = h_tris.to(dev, non_blocking=True)
        ed = h_eps.to(dev, non_blocking=True)
        r = mhs.interaction_matrix(td, mat, ed, out=out, precision=a.precision)
        h_out.copy_(r, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_t = torch.tensor([e2e_ms], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
    e2e_ms = float(e2e_t.item())
    e2e_val = world * entries * e2e_steps / (e2e_ms * 1e-3)

    # serving: the seeded Poisson stream through the request loop, FP64 and mixed
    serving = {"stream": dict(SERVE, note="sizes scaled down from the serving config; "
                                        "arrivals Poisson, seeded; latency = submit to "
                                        "result ready on the device, host clock"),
               "fp64": serve_stream(dev, "fp64", 100 + rank),
               "mixed": serve_stream(dev, "mixed", 100 + rank)}

    batch = {"config": dict(BATCH, note="sizes scaled down from the batched config; all "
                                        "submitted at once to the serving loop (stream overlap)"),
             "fp64": batch_run(dev, "fp64", 200 + rank),
             "mixed": batch_run(dev, "mixed", 200 + rank)}

    # roofline of the dominant stage (the fold): algorithmic flops of the
    # census'd work units over the stage's time per launch
    top = max(stages, key=lambda s: stages[s][0])
    top_ms, top_n = stages[top]
    peak = _native.fp_peak(fp64=True)
    achieved, fl = None, None
    if top == "fold":
        from mhs_b200 import flops as _flops
        fl = _flops.fold_flops(census, order=0, want_h=True, mu=mu, lam=lam,
                               eps=float(np.mean(eps)))
        achieved = fl["flop"] / (top_ms / max(top_n, 1) * 1e-3) / 1e12
    roof = {"bound": "fp64", "kernel": top, "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": (achieved / peak) if achieved else None,
            "traffic": FOLD_TRAFFIC_PER_LAUNCH.get((a.nu, a.nv, a.precision)) if top == "fold" else None,
            "peak_source": "measured FP64 FMA ceiling (mhs_fp_peak, this run)",
            "algorithmic": None if fl is None else {
                "flop_per_launch": fl["flop"], "div": fl["div"], "sqrt": fl["sqrt"],
                "special": fl["special"], "census": census,
                "counting": "op-counting host build of the engine (mhs_b200/csrc/opcount.cpp): "
                            "add/sub/mul 1 flop, fma 2; div, sqrt, library calls apart"},
            "stage_ms_per_step": {k: v[0] / a.steps for k, v in stages.items()},
            "stage_launches_per_step": {k: v[1] / a.steps for k, v in stages.items()}}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if a.precision == "fp64" else "f64+f32",
            "data": "synthetic (seeded rough fault mesh per rank)",
            "config": {"workload": WORKLOAD, "n_tri": n, "entries_per_step": entries,
                       "precision": a.precision, "global_batch": world,
                       "l2": "L2 flushed between steps (256 MiB write); output 415 MB per step",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_val, "unit": UNIT,
                    "h2d_bytes_per_step": int(tris.nbytes + eps.nbytes),
                    "d2h_bytes_per_step": int(entries * 8)},
            "roofline": roof, "mixed": mixed, "serving": serving, "batch": batch,
            "clocks": clk.summary(),
            "gpu_launches": int(sum(v[1] * KERNELS_PER_STAGE[k] for k, v in stages.items()))}
    return line, tris, eps, mu, lam


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if a.impl == "reference":
        if rank != 0:
            return 0
        tris, eps, mu, lam = workload(0, a.nu, a.nv)
        vals = []
        for i in range(a.warmup + a.steps):
            r = cpu_baseline(tris, eps, mu, lam, a.cpu_seconds, seed=100 + i)
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
    line, tris, eps, mu, lam = run_ours(a, rank, world)
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
