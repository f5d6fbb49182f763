"""A fit server on one GPU with continuous batching.

Requests (DtiJob, DkiJob, MfodJob from larmor_b200.batch) arrive at any time through submit(),
which returns a future. A dispatcher admits them in arrival order whenever a slot (a CUDA
stream with its worker thread) is free and the request fits in the HBM budget next to the
requests already running; a request that arrives while others are on the GPU starts as soon as
one of them releases its slot and memory, and its kernels run beside theirs on its own stream.
Each worker uploads its request's inputs, enqueues the fit (the mFOD fit without host waits:
lar_fit_multi_tissue_async), copies the results to the host once the stream finishes and then
frees its slot; every slot has a thread of its own, and its waits release the GIL.

Design handles (log-fit designs, deconvolution kernels and solvers) are built once per
(model, gradient table, responses) and slot and kept resident; a handle's scratch belongs to
its slot, so requests running at the same time never share one. The budget counts each running
request's inputs, outputs and per-voxel state (larmor_b200.batch.job_device_bytes) plus an
estimate of the resident handles' scratch.

A request's result does not depend on what else is running: every voxel is fitted by the same
arithmetic on its own, whatever the stream, slot or neighbours.
"""

from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future, ThreadPoolExecutor

# Estimated device scratch of one slot's handles for a table (the constrained DKI re-fit's warp
# slots; the mFOD solvers' per-warp NNLS and fraction workspaces).
HANDLE_SCRATCH_BYTES = {"dti": 8 << 20, "dki": 512 << 20, "mfod": 1280 << 20}


class _Request:
    __slots__ = ("job", "future", "arrival", "need", "admitted", "finished")

    def __init__(self, job, need: int) -> None:
        self.job = job
        self.future: Future = Future()
        self.arrival = time.perf_counter()
        self.need = need
        self.admitted = None
        self.finished = None


class FitServer:
    """See the module docstring. `slots` requests run at once at most; `budget_bytes` bounds
    their device memory."""

    def __init__(self, budget_bytes: int = 80 << 30, slots: int = 8, device=None) -> None:
        self.budget = int(budget_bytes)
        self.slots = int(slots)
        if self.slots < 1:
            raise ValueError("slots must be at least 1")
        self.device = device
        self._cv = threading.Condition()
        self._pending: collections.deque[_Request] = collections.deque()
        self._free = list(range(self.slots))
        self._used = 0
        self._resident: dict = {}   # (job key, slot) -> handles
        self._resident_bytes = 0
        self._closed = False
        self._pool = ThreadPoolExecutor(max_workers=self.slots, thread_name_prefix="larmor-fit")
        self._streams = None
        self.completed: list[_Request] = []
        self.peak_running = 0
        self.peak_bytes = 0
        self._running = 0
        self._dispatcher = threading.Thread(target=self._dispatch, name="larmor-dispatch", daemon=True)
        self._dispatcher.start()

    # ---- public -----------------------------------------------------------------------------

    def submit(self, job) -> Future:
        """Queues a fit; the future's result is the dict of host numpy outputs."""
        need = self.request_bytes(job)
        if need > self.budget:
            raise ValueError(f"the request needs {need} bytes of device memory, above the {self.budget}-byte budget")
        req = _Request(job, need)
        with self._cv:
            if self._closed:
                raise RuntimeError("the server is closed")
            self._pending.append(req)
            self._cv.notify_all()
        return req.future

    def close(self) -> None:
        """Waits for every queued request, then stops the workers."""
        with self._cv:
            while self._pending or self._running:
                self._cv.wait()
            self._closed = True
            self._cv.notify_all()
        self._dispatcher.join()
        self._pool.shutdown(wait=True)

    def latencies_ms(self) -> list[float]:
        """Arrival-to-result times of the completed requests, in completion order."""
        return [1e3 * (r.finished - r.arrival) for r in self.completed]

    def request_bytes(self, job) -> int:
        from larmor_b200.batch import job_device_bytes

        return int(job_device_bytes(job))

    # ---- dispatching ------------------------------------------------------------------------

    def _dispatch(self) -> None:
        while True:
            with self._cv:
                while not self._closed and not self._admissible():
                    self._cv.wait()
                if self._closed and not self._pending:
                    return
                req = self._pending.popleft()
                slot = self._free.pop()
                self._used += req.need
                self._running += 1
                self.peak_running = max(self.peak_running, self._running)
                self.peak_bytes = max(self.peak_bytes, self._used + self._resident_bytes)
                req.admitted = time.perf_counter()
            self._pool.submit(self._work, slot, req)

    def _admissible(self) -> bool:
        """The head of the queue may start: a free slot and room in the budget (arrival order:
        a large request at the head waits for memory rather than being overtaken)."""
        if not self._pending or not self._free:
            return False
        return self._used + self._resident_bytes + self._pending[0].need <= self.budget

    def _work(self, slot: int, req: _Request) -> None:
        try:
            result = self._run(slot, req.job)
            req.finished = time.perf_counter()
            req.future.set_result(result)
        except BaseException as exc:  # noqa: BLE001 - handed to the caller through the future
            req.finished = time.perf_counter()
            req.future.set_exception(exc)
        finally:
            with self._cv:
                self._free.append(slot)
                self._used -= req.need
                self._running -= 1
                self.completed.append(req)
                self._cv.notify_all()

    # ---- the GPU work of one request (replaceable in tests) -------------------------------------

    def _handles(self, slot: int, job):
        from larmor_b200.batch import job_handles, job_key

        key = (job_key(job), slot)
        with self._cv:
            handles = self._resident.get(key)
        if handles is None:
            handles = job_handles(job)
            with self._cv:
                self._resident[key] = handles
                self._resident_bytes += HANDLE_SCRATCH_BYTES[job.kind]
        return handles

    def _run(self, slot: int, job) -> dict:
        import torch

        from larmor_b200.batch import job_inputs_host, job_outputs, launch_job

        dev = torch.device("cuda", torch.cuda.current_device() if self.device is None else self.device)
        torch.cuda.set_device(dev)
        with self._cv:
            if self._streams is None:
                self._streams = [torch.cuda.Stream(dev) for _ in range(self.slots)]
            stream = self._streams[slot]
        handles = self._handles(slot, job)
        with torch.cuda.stream(stream):
            d_in = tuple(torch.from_numpy(a).to(dev, non_blocking=True) for a in job_inputs_host(job))
            out = job_outputs(job, handles, dev)
            launch_job(job, handles, d_in, out, asynchronous=True)
            host = {k: t.to("cpu", non_blocking=True) for k, t in out.items()}
        stream.synchronize()
        return {k: t.numpy() for k, t in host.items()}
