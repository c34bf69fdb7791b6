"""Tracking-job server for one GPU: continuous batching of strack/strackw +
cullst jobs.

A job is one image pair tracked with `strack` (Strack/speckleTrack.c) or
`strackw` (Strackw/corrTrackFast.c), optionally followed by the cullst passes
(Cullst/cullst.c:71-101) on its offsets grid.  The server owns `slots` library
contexts; each has its own CUDA stream and reusable device buffers and is
driven by its own host thread, so jobs on different slots overlap on the GPU
(the C calls release the GIL).  A job starts when a slot is free and the
device memory the slots hold or need stays within the HBM budget (see
JobServer); admission is first come, first
served (the head of the queue is never bypassed, so a large job cannot
starve).  Images may be torch CUDA tensors (device-resident, nothing copied)
or host arrays (copied inside the call).  Results are the same whether a job
runs alone or beside others: every kernel is deterministic and contexts share
no buffers.
"""
import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Any, Callable, Optional

import numpy as np

from . import abi

# per-point device buffers of one strack call (plan, record, lists, fit job,
# five output grids), bytes
_STRACK_POINT_BYTES = 20 + 80 + 16 + 160 + 17 + 64
# complex-peak hand-off (PeakJob, csrc/strack_kernels.h), allocated for at
# most one list chunk (kPeakChunk in csrc/capi.cu)
_PEAK_JOB_BYTES = 960
_PEAK_CHUNK = 1 << 19
# per-CTA workspaces (float2 elements), sized like the kernels' own
_AMP_SCRATCH = {16: 3 * 16 * 16 + 32 * 32 * 3 // 2, 24: 3 * 24 * 24 + 48 * 48 * 3 // 2,
                32: 3 * 32 * 32 + 64 * 64 * 3 // 2, 48: 3 * 48 * 48 + 96 * 96 * 3 // 2,
                64: 3 * 64 * 64 + 128 * 128 * 3 // 2, 96: 3 * 96 * 96 + 192 * 192 * 3 // 2,
                128: 3 * 128 * 128 + 256 * 256 * 3 // 2}


@dataclass
class Job:
    """One tracking job.  kind: "strack", "strackw" or "cull" (culling only:
    img1 = (offR, offA, corr, type)); cull: CullParams or None; inject:
    optional callable(offR, offA, corr, type) run on the host copies of the
    offsets before culling (used to plant outliers)."""
    kind: str
    params: Any
    img1: Any
    img2: Any
    cull: Any = None
    inject: Optional[Callable] = None
    tag: Any = None
    arrival: float = field(default=0.0)


def _image_bytes(img):
    try:
        import torch
        if isinstance(img, torch.Tensor):
            return 0 if img.is_cuda else img.numel() * img.element_size()
    except ImportError:
        pass
    return int(np.asarray(img).nbytes)


def job_device_bytes(job, num_sm=148):
    """Upper estimate of the device memory a job holds while it runs."""
    if job.kind == "cull":
        return int(job.cull.nR) * int(job.cull.nA) * 64
    p = job.params
    n = int(p.nR) * int(p.nA)
    b = _image_bytes(job.img1) + _image_bytes(job.img2)
    ctas = 2 * num_sm
    if job.kind == "strack":
        b += n * _STRACK_POINT_BYTES
        if not getattr(p, "gaussFlag", 0):
            b += min(n, _PEAK_CHUNK) * _PEAK_JOB_BYTES
        if p.maxTries > 0:
            wa = int(p.wRa)
            b += ctas * 8 * _AMP_SCRATCH.get(wa, _AMP_SCRATCH[128])
            if p.maxTries > 1 and 2 * wa in _AMP_SCRATCH:
                b += ctas * 8 * _AMP_SCRATCH[2 * wa]
    else:
        W = int(p.wRa)
        N = 2 * W
        L = 4 * (int(p.edgePadR) + 5) + 1
        b += n * 40 + ctas * 8 * (3 * W * W + 3 * N * N + 2 * N * L + 3 * L * L)
    if job.cull is not None:
        b += n * 64
    return int(b)


class JobServer:
    """Continuous-batching server.  context_factory(device) -> an object with
    the runtime.Context methods strack/strackw/cull/close, and optionally
    device_bytes/release (a fake one in the CPU tests).

    Device-memory budget: a context keeps the buffers its calls grew (reused
    by its next job), so the budget counts, per slot, the larger of what its
    context holds (measured after each job with device_bytes) and the
    estimate of the job it runs.  A job is admitted on a free slot when that
    sum over all slots stays within the budget; when the head of the queue
    does not fit, idle slots release their buffers first.  Images passed as
    CUDA tensors belong to the caller and are not counted."""

    def __init__(self, device=0, slots=4, hbm_budget=120e9, context_factory=None, num_sm=148, max_batch=1):
        if context_factory is None:
            from . import runtime
            context_factory = runtime.Context
        self.budget = float(hbm_budget)
        self.num_sm = num_sm
        self.max_batch = int(max_batch)  # > 1: strack jobs queued together share one sb_strack_batch call
        self.batches = []                # sizes of the batches run
        self._ctx = [context_factory(device) for _ in range(slots)]
        self._cv = threading.Condition()
        self._queue = collections.deque()
        self._held = [self._measure(c) for c in self._ctx]   # bytes each context holds
        self._running = [0.0] * slots                          # estimate of the job on each slot
        self._peak = 0.0
        self._closed = False
        self.releases = 0
        self.started = []  # (tag, start time) in admission order
        self._threads = [threading.Thread(target=self._worker, args=(k,), daemon=True) for k in range(slots)]
        for t in self._threads:
            t.start()

    @staticmethod
    def _measure(ctx):
        f = getattr(ctx, "device_bytes", None)
        return float(f()) if f else 0.0

    @property
    def peak_bytes(self):
        """Largest device memory reserved at once (sum over slots of the held
        or estimated bytes), bytes."""
        return self._peak

    def reserved_bytes(self):
        with self._cv:
            return self._reserved()

    def _reserved(self, skip=None):
        return sum(max(h, r) for k, (h, r) in enumerate(zip(self._held, self._running)) if k != skip)

    def submit(self, job):
        """Queues a job; returns a Future resolving to a dict with the track
        result, the cull result (or None) and the job's start/end times."""
        fut = Future()
        need = job_device_bytes(job, self.num_sm)
        if need > self.budget:
            fut.set_exception(ValueError(f"job needs ~{need / 1e9:.1f} GB, above the {self.budget / 1e9:.1f} GB "
                                         "HBM budget"))
            return fut
        job.arrival = job.arrival or time.perf_counter()
        with self._cv:
            if self._closed:
                raise RuntimeError("server closed")
            self._queue.append((job, need, fut))
            self._cv.notify_all()
        return fut

    def _take(self, k):
        """Next work for slot k: a list of (job, need, future); more than one
        when queued strack jobs can share one batched call."""
        ctx = self._ctx[k]
        with self._cv:
            while True:
                if self._closed and not self._queue:
                    return None
                if self._queue:
                    job, need, fut = self._queue[0]
                    if self._reserved(skip=k) + max(self._held[k], need) <= self.budget:
                        self._queue.popleft()
                        items = [(job, need, fut)]
                        total = float(need)
                        key = _batch_key(job)
                        # continuous batching: later queued jobs that can share the call
                        while (key is not None and len(items) < self.max_batch and self._queue and
                               _batch_key(self._queue[0][0]) == key and
                               self._reserved(skip=k) + max(self._held[k], total + self._queue[0][1]) <= self.budget):
                            nxt = self._queue.popleft()
                            items.append(nxt)
                            total += nxt[1]
                        self._running[k] = total
                        self._peak = max(self._peak, self._reserved())
                        now = time.perf_counter()
                        self.started += [(j.tag, now) for j, _, _ in items]
                        self.batches.append(len(items))
                        self._cv.notify_all()
                        return items
                    if self._held[k] > 0 and getattr(ctx, "release", None):
                        # the head does not fit: this idle slot gives its buffers back
                        self._cv.release()
                        try:
                            ctx.release()
                        finally:
                            self._cv.acquire()
                        self._held[k] = self._measure(ctx)
                        self.releases += 1
                        self._cv.notify_all()
                        continue
                self._cv.wait()

    def _finish(self, k):
        held = self._measure(self._ctx[k])
        with self._cv:
            self._held[k] = held
            self._running[k] = 0.0
            self._peak = max(self._peak, self._reserved())
            self._cv.notify_all()

    def _worker(self, k):
        ctx = self._ctx[k]
        while True:
            items = self._take(k)
            if items is None:
                return
            try:
                t0 = time.perf_counter()
                if len(items) == 1:
                    results = [run_job(ctx, items[0][0])]
                else:
                    results = run_batch(ctx, [j for j, _, _ in items])
                t1 = time.perf_counter()
                held = self._measure(ctx)
                for (job, _, fut), res in zip(items, results):
                    res.update(start=t0, end=t1, arrival=job.arrival, slot=k, held_bytes=held, batch=len(items))
                    fut.set_result(res)
            except Exception as e:  # reported through the futures
                for _, _, fut in items:
                    if not fut.done():
                        fut.set_exception(e)
            finally:
                self._finish(k)

    def close(self):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        for c in self._ctx:
            c.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def run_job(ctx, job):
    """Runs one job on a context (also how a job runs alone).  kind "cull":
    culling only, job.img1 = (offR, offA, corr, type) grids."""
    if job.kind == "cull":
        offR, offA, corr, mt = (np.array(x, copy=True) for x in job.img1)
        if job.inject is not None:
            job.inject(offR, offA, corr, mt)
        return {"track": None, "cull": ctx.cull(job.cull, offR, offA, corr, mt)}
    if job.kind == "strack":
        tr = ctx.strack(job.params, job.img1, job.img2)
    elif job.kind == "strackw":
        tr = ctx.strackw(job.params, job.img1, job.img2)
    else:
        raise ValueError(f"unknown job kind {job.kind!r}")
    cu = None
    if job.cull is not None:
        offR = np.array(tr["offR"], np.float32, copy=True)
        offA = np.array(tr["offA"], np.float32, copy=True)
        corr = np.array(tr["corr"], np.float32, copy=True)
        mt = np.array(tr["type"], np.uint8, copy=True)
        if job.inject is not None:
            job.inject(offR, offA, corr, mt)
        cu = ctx.cull(job.cull, offR, offA, corr, mt)
    return {"track": tr, "cull": cu}


def _batch_key(job):
    """Jobs with equal keys can share one sb_strack_batch call (strack jobs
    with the same flags and image sample type); None: the job runs alone."""
    if job.kind != "strack" or not hasattr(job.params, "hanningFlag"):
        return None
    p = job.params
    if getattr(p, "baseline", None) is not None or getattr(p, "intf", None) is not None:
        return None
    dt = getattr(job.img1, "dtype", None)
    return (str(dt), p.noComplex, p.hanningFlag, p.maxTries, p.checkAzFocus, p.gaussFlag,
            float(p.azDefocusThresh), p.scaleFactor)


def run_batch(ctx, jobs):
    """Runs strack jobs with one batched call (sb_strack_batch), then each
    job's culling; per job the same result as run_job."""
    tracks = ctx.strack_batch([j.params for j in jobs], [j.img1 for j in jobs], [j.img2 for j in jobs])
    out = []
    for job, tr in zip(jobs, tracks):
        cu = None
        if job.cull is not None:
            offR = np.array(tr["offR"], np.float32, copy=True)
            offA = np.array(tr["offA"], np.float32, copy=True)
            corr = np.array(tr["corr"], np.float32, copy=True)
            mt = np.array(tr["type"], np.uint8, copy=True)
            if job.inject is not None:
                job.inject(offR, offA, corr, mt)
            cu = ctx.cull(job.cull, offR, offA, corr, mt)
        out.append({"track": tr, "cull": cu})
    return out


def latency_stats(results):
    """p50/p99 of arrival-to-completion latency (ms) over result dicts, split
    into the queue wait (arrival to start) and the service time (start to
    end) of the same jobs."""
    lat = np.array([1e3 * (r["end"] - r["arrival"]) for r in results])
    wait = np.array([1e3 * (r["start"] - r["arrival"]) for r in results])
    svc = lat - wait
    return {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
            "max": float(lat.max()), "mean": float(lat.mean()),
            "wait_p50": float(np.percentile(wait, 50)), "wait_p99": float(np.percentile(wait, 99)),
            "service_p50": float(np.percentile(svc, 50)), "service_p99": float(np.percentile(svc, 99))}
