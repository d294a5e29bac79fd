"""A request loop that keeps the GPU busy with several assemblies at once.

``Server.submit(fn, *args, **kwargs)`` takes one of the public matrix
functions (``mhs_b200.disp_matrix``, ``stress_matrix``, ``traction_matrix``,
``interaction_matrix``, ...) with its usual arguments and returns a
``concurrent.futures.Future`` whose result is the matrix as a CUDA tensor
(results stay on the device).  The arguments are validated and the inputs
staged on the device in the caller's thread, exactly as a direct call does.

A dispatcher thread admits queued requests in arrival order as slots and
device memory free up: a request is admitted while fewer than ``slots``
requests are in flight and the device bytes it holds (output, workspace,
inputs) fit, with those of the requests in flight, in ``budget_bytes``.
Each admitted request runs on its own CUDA stream with its own workspace,
so the kernels of requests in flight overlap on the device (continuous
batching: a request that arrives while others run starts as soon as it is
admitted, not when the current group ends).  Every request computes exactly
what a direct call computes -- the kernels are deterministic and requests
share no scratch -- so a result is the same alone and in the mix.

A result keeps counting against the budget, with its output bytes, until
the caller drops the last reference to it (the device memory is in use
until then), so a client that holds results slows admission instead of
running the device out of memory.  When nothing is in flight and only held
results keep the next request out, it is admitted if the device's free
memory holds it, and otherwise fails with MemoryError (the caller's results
fill the device).  A request larger than the whole budget is refused with
MemoryError, the way mhs refuses a matrix above its byte ceiling.  ``stats()`` returns the
latency percentiles (submit to result ready, host clock) and throughput.
"""
from __future__ import annotations

import collections
import threading
import time
import weakref
from concurrent.futures import Future

from . import matrices


def admissible(need: int, in_flight_bytes: int, n_in_flight: int, budget: int, slots: int) -> bool:
    """Admission rule: a free slot and room in the byte budget."""
    return n_in_flight < slots and in_flight_bytes + need <= budget


class Server:
    def __init__(self, device=None, budget_bytes: int | None = None, slots: int = 8,
                 poll_s: float = 2e-4):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None \
            else torch.device(device)
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget_bytes = int(0.8 * free)
        self.budget = int(budget_bytes)
        self.slots = int(slots)
        self.poll_s = poll_s
        with torch.cuda.device(self.device):
            self.streams = [torch.cuda.Stream(self.device) for _ in range(self.slots)]
        self.free_streams = list(range(self.slots))
        self.queue = collections.deque()
        self.in_flight = []          # (pending, future, stream index, event, t_submit)
        self.in_flight_bytes = 0
        self.held_bytes = 0          # outputs handed out and still referenced
        self.peak_bytes = 0          # most device bytes ever in flight at once
        self.peak_in_flight = 0      # most requests ever in flight at once
        self.lat = []
        self.entries = 0
        self.t_first = None
        self.t_last = None
        self.cv = threading.Condition(threading.RLock())
        self.outstanding = 0         # submitted requests whose futures are not settled
        self.oom_wait = False        # admissions wait for a completion (allocator out of memory)
        self.oom_retries = 0
        self.running = True
        self.error = None
        self.thread = threading.Thread(target=self._loop, name="mhs-serve", daemon=True)
        self.thread.start()

    # ------------------------------------------------------------ client
    def submit(self, fn, *args, **kwargs) -> Future:
        fut = Future()
        t0 = time.perf_counter()
        with self.torch.cuda.device(self.device), matrices.deferred():
            pend = fn(*args, **kwargs)
            if not isinstance(pend, matrices.Pending):
                raise TypeError(f"{getattr(fn, '__name__', fn)} is not a servable matrix function")
            # the inputs were staged on this thread's current stream, which is
            # also the stream the result is handed to
            pend.ready = self.torch.cuda.Event()
            pend.ready.record()
            pend.consumer = self.torch.cuda.current_stream(self.device)
        if pend.device_bytes > self.budget:
            raise MemoryError(f"request needs {pend.device_bytes / 2**30:.2f} GiB on the device, "
                              f"above the serving budget of {self.budget / 2**30:.2f} GiB; "
                              f"split it by rows")
        with self.cv:
            if self.t_first is None:
                self.t_first = t0
            self.outstanding += 1
            self.queue.append((pend, fut, t0))
            self.cv.notify()
        fut.add_done_callback(self._settled)
        return fut

    def _settled(self, fut) -> None:
        with self.cv:
            self.outstanding -= 1
            self.cv.notify_all()

    def close(self) -> None:
        with self.cv:
            self.running = False
            self.cv.notify()
        self.thread.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def drain(self) -> None:
        """Wait until every submitted request's future is settled (its
        result or error set, its statistics recorded)."""
        with self.cv:
            while self.outstanding:
                self.cv.wait(0.01)

    def stats(self) -> dict:
        lat = sorted(self.lat)
        n = len(lat)

        def pct(q):
            if not n:
                return None
            i = min(n - 1, max(0, int(round(q * (n - 1)))))
            return 1e3 * lat[i]

        span = (self.t_last - self.t_first) if (self.t_last and self.t_first) else None
        return {"requests": n, "p50_ms": pct(0.50), "p99_ms": pct(0.99),
                "mean_ms": (1e3 * sum(lat) / n) if n else None,
                "entries": self.entries, "span_s": span,
                "entries_per_s": (self.entries / span) if span else None,
                "req_per_s": (n / span) if span else None, "oom_retries": self.oom_retries}

    def _device_room(self) -> int:
        torch = self.torch
        free, _ = torch.cuda.mem_get_info(self.device)
        return int(free + torch.cuda.memory_reserved(self.device)
                   - torch.cuda.memory_allocated(self.device))

    def _release(self, nbytes: int) -> None:
        with self.cv:
            self.held_bytes -= nbytes
            self.cv.notify_all()

    # -------------------------------------------------------- dispatcher
    def _launch(self, pend, st):
        """Launch one request; on an allocator out-of-memory, return the
        cached free blocks to the device and try once more."""
        torch = self.torch
        try:
            pend.launch(st)
        except torch.OutOfMemoryError:
            torch.cuda.empty_cache()
            pend.launch(st)

    def _loop(self):
        torch = self.torch
        torch.cuda.set_device(self.device)
        while True:
            with self.cv:
                if not self.running and not self.queue and not self.in_flight:
                    return
                admit = []
                while self.queue and self.free_streams and not self.oom_wait:
                    pend, fut, t0 = self.queue[0]
                    need = pend.device_bytes
                    n_now = len(self.in_flight) + len(admit)
                    ok = admissible(need, self.in_flight_bytes + self.held_bytes, n_now,
                                    self.budget, self.slots)
                    if not ok and n_now == 0 and self.held_bytes > 0:
                        # only results the caller still holds keep it out
                        ok = need <= self._device_room()
                        if not ok:
                            self.queue.popleft()
                            fut.set_exception(MemoryError(
                                f"request needs {need / 2**30:.2f} GiB on the device; results "
                                f"still held by the caller ({self.held_bytes / 2**30:.2f} GiB) "
                                f"leave no room"))
                            continue
                    if not ok:
                        break
                    self.queue.popleft()
                    self.in_flight_bytes += need
                    admit.append((pend, fut, t0, self.free_streams.pop()))
                    self.peak_bytes = max(self.peak_bytes, self.in_flight_bytes)
                    self.peak_in_flight = max(self.peak_in_flight, len(self.in_flight) + len(admit))
            requeue = []
            for pend, fut, t0, si in admit:
                st = self.streams[si]
                try:
                    self._launch(pend, st)
                    ev = torch.cuda.Event()
                    ev.record(st)
                    with self.cv:
                        self.in_flight.append((pend, fut, si, ev, t0))
                except torch.OutOfMemoryError as e:
                    # the byte budget admitted it, but the allocator's free
                    # blocks (fragmented across sizes and streams) do not
                    # hold it: with work in flight, wait for a completion
                    # and try again; with none, report it
                    with self.cv:
                        self.in_flight_bytes -= pend.device_bytes
                        self.free_streams.append(si)
                        if self.in_flight:
                            requeue.append((pend, fut, t0))
                            self.oom_wait = True
                            self.oom_retries += 1
                            continue
                    fut.set_exception(e)
                except Exception as e:  # noqa: BLE001 - reported through the future
                    with self.cv:
                        self.in_flight_bytes -= pend.device_bytes
                        self.free_streams.append(si)
                    fut.set_exception(e)
            if requeue:
                with self.cv:
                    self.queue.extendleft(reversed(requeue))
            done = []
            with self.cv:
                for item in list(self.in_flight):
                    if item[3].query():
                        self.in_flight.remove(item)
                        done.append(item)
            for pend, fut, si, ev, t0 in done:
                need = pend.device_bytes
                try:
                    res = pend.finish(self.streams[si])
                    # the result was allocated on a serving stream: record the
                    # consumer's stream so that, when the caller frees it, the
                    # allocator waits for the caller's work before a later
                    # request on that serving stream reuses the memory
                    if res is not None and getattr(pend, "consumer", None) is not None:
                        res.record_stream(pend.consumer)
                    t1 = time.perf_counter()
                    with self.cv:
                        if res is not None:
                            self.held_bytes += pend.out_bytes
                            weakref.finalize(res, self._release, pend.out_bytes)
                        self.lat.append(t1 - t0)
                        self.entries += pend.entries
                        self.t_last = t1
                    fut.set_result(res)
                except Exception as e:  # noqa: BLE001
                    fut.set_exception(e)
                with self.cv:
                    self.in_flight_bytes -= need
                    self.free_streams.append(si)
                    self.oom_wait = False
                    self.cv.notify_all()
            idle = not admit and not done
            # drop this pass's references, so that a result lives only as long
            # as the caller keeps it
            admit = done = item = pend = fut = res = None
            if idle:
                with self.cv:
                    self.cv.wait(self.poll_s)
