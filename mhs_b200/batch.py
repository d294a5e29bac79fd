"""Batched assembly: uneven requests as one group of launches per (order,
readout, precision), optionally captured into a CUDA graph and replayed.

``Batch(calls)`` takes a list of ``(fn, args, kwargs)`` -- the public matrix
functions with their usual arguments, as for ``mhs_b200.serve`` -- validates
and stages every request on the device, allocates the outputs and one device
arena, and plans the launches (``mhs_batch_create`` / ``mhs_batch_bind``):
each stage of the pipeline (image coefficients, per-source data, the two
pair kernels, the output stage) then runs once over all requests of a
group, its blocks finding their request by a prefix of block counts.  A
request with sources that reach the fold depth runs its fold between the
pair kernels and the output stage, per request; a request whose sources
all lie deeper is given ``fold = 0`` (the same result), so a batch with no
surface-reaching source queues kernels only.

``run()`` queues the batch (``mhs_submit_batch``) on the current stream and
returns the outputs (CUDA tensors).  ``graph()`` captures one submission
into a CUDA graph, so later ``replay()`` calls launch it as one graph --
the batch must have no fold work (``capturable``).  ``poll()`` asks whether
the last submission completed (``mhs_poll``) without blocking.
"""
from __future__ import annotations

import ctypes

from . import _native, matrices


class Batch:
    def __init__(self, calls, device=None):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None \
            else torch.device(device)
        self.pending = []
        with torch.cuda.device(self.device), matrices.deferred():
            for fn, args, kw in calls:
                p = fn(*args, **kw)
                if not isinstance(p, matrices.Pending):
                    raise TypeError(f"{getattr(fn, '__name__', fn)} is not a batchable function")
                self.pending.append(p)
        torch.cuda.current_stream(self.device).synchronize()   # staged inputs
        n = len(self.pending)
        self.reqs = (_native.Request * n)()
        self.outputs = []
        with torch.cuda.device(self.device):
            for i, p in enumerate(self.pending):
                out = torch.empty(p.out_shape, dtype=p.out_dtype, device=self.device)
                self.outputs.append(out)
                r = p.req
                r.out = ctypes.c_void_p(out.data_ptr())
                if not p.straddles:
                    r.fold = 0
                ctypes.memmove(ctypes.byref(self.reqs, i * ctypes.sizeof(_native.Request)),
                               ctypes.byref(r), ctypes.sizeof(_native.Request))
        self.capturable = not any(self.reqs[i].fold for i in range(n))
        lib = _native.load()
        self.handle = ctypes.c_void_p()
        _native.check(lib.mhs_batch_create(self.reqs, n, ctypes.byref(self.handle)))
        nbytes = ctypes.c_size_t()
        _native.check(lib.mhs_batch_workspace_bytes(self.handle, ctypes.byref(nbytes)))
        self.arena = torch.empty(max(1, nbytes.value), dtype=torch.uint8, device=self.device)
        stream = torch.cuda.current_stream(self.device)
        _native.check(lib.mhs_batch_bind(self.handle, ctypes.c_void_p(self.arena.data_ptr()),
                                         nbytes.value, ctypes.c_void_p(stream.cuda_stream)))
        self.cuda_graph = None
        self.entries = sum(p.entries for p in self.pending)

    def _submit(self, stream):
        _native.check(_native.load().mhs_submit_batch(self.handle,
                                                      ctypes.c_void_p(stream.cuda_stream)))

    def run(self):
        """Queue the batch on the current stream; returns the outputs."""
        self._submit(self.torch.cuda.current_stream(self.device))
        return self.outputs

    def poll(self):
        """(done, device status bits) of the last submission, without waiting."""
        done, bits = ctypes.c_int(0), ctypes.c_int(0)
        _native.check(_native.load().mhs_poll(self.handle, ctypes.byref(done), ctypes.byref(bits)))
        return bool(done.value), int(bits.value)

    def wait(self):
        """Block until the last run() completed; raise on a device status."""
        self.torch.cuda.current_stream(self.device).synchronize()
        done, bits = self.poll()
        if bits & _native.DEV_FOLD_GRID_OVERFLOW:
            raise RuntimeError("a fold polar grid exceeded its capacity (FOLD_MAX_BREAKS)")
        return self.outputs

    def graph(self):
        """Capture one submission into a CUDA graph (a batch without fold
        work); replay() then launches it as one graph."""
        torch = self.torch
        if not self.capturable:
            raise RuntimeError("a batch with fold work synchronises its stream and cannot be "
                               "captured; assemble it with run()")
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self._submit(s)          # warm the modules outside capture
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self._submit(torch.cuda.current_stream(self.device))
        self.cuda_graph = g
        return g

    def replay(self):
        """Launch the captured graph on the current stream; returns the outputs."""
        if self.cuda_graph is None:
            self.graph()
        self.cuda_graph.replay()
        return self.outputs

    def close(self):
        if getattr(self, "handle", None):
            _native.load().mhs_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


def split(calls, budget_bytes):
    """Partition calls for batching: (groups, alone) -- lists of indices.
    A call whose one-pass scratch (``mhs_batch_pass_bytes``) is above the
    batch limit goes to ``alone`` (assemble it through its own function,
    which chunks its observers); the rest are packed in order into groups
    whose output plus scratch bytes stay within ``budget_bytes``."""
    lib = _native.load()
    groups, alone, cur, cur_b = [], [], [], 0
    with matrices.deferred():
        pend = [fn(*args, **kw) for fn, args, kw in calls]
    for i, p in enumerate(pend):
        nb, lim = ctypes.c_size_t(), ctypes.c_size_t()
        _native.check(lib.mhs_batch_pass_bytes(ctypes.byref(p.req), ctypes.byref(nb),
                                               ctypes.byref(lim)))
        if nb.value > lim.value:
            alone.append(i)
            continue
        b = nb.value + p.out_bytes
        if cur and cur_b + b > budget_bytes:
            groups.append(cur)
            cur, cur_b = [], 0
        cur.append(i)
        cur_b += b
    if cur:
        groups.append(cur)
    return groups, alone


def autotune(fn, *args, **kwargs):
    """Pick the launch shapes for the class of this call (its order, readout
    and precision) on the current device by timing it under each candidate
    shape (``mhs_autotune``); returns (shape dict, best ms).  Results do not
    depend on the shape."""
    import torch
    with matrices.deferred():
        p = fn(*args, **kwargs)
    stream = torch.cuda.current_stream()
    with torch.cuda.stream(stream):
        p.launch(stream)
    t = _native.Tune()
    ms = ctypes.c_double()
    _native.check(_native.load().mhs_autotune(ctypes.byref(p.req), ctypes.c_void_p(stream.cuda_stream),
                                              ctypes.byref(t), ctypes.byref(ms)))
    stream.synchronize()
    return {"pair_tb": t.pair_tb, "final_tb": t.final_tb, "far_mult": t.far_mult,
            "near_mult": t.near_mult}, ms.value
