"""Request serving with continuous batching over the batched C ABI.

A request is one encode or recover of one codeword whose shards are resident
in device memory (the serving system keeps shard buffers on the GPU).
``BatchServer`` accepts requests as they arrive and, whenever one of its
streams is free, packs every waiting request that fits the device-memory
admission cap into the next persistent batched launch (``afrs_batch_dev``);
batches on different streams overlap on the GPU, so requests that arrive
while others run are admitted as slots and memory free up.  ``PlainServer``
serves the same requests one call at a time (the per-call path).

Both record, per request, the latency from arrival to completion (host
clock, completion observed through CUDA events).

Stream order: ``submit`` records an event on the caller's current stream, and
the stream that runs the request waits on it, so work the caller enqueued on
the request's buffers before submitting (a fill, a copy) is finished first.
The buffers are also recorded on the running stream, so that torch's caching
allocator does not hand their memory to another tensor while the request is
still on the GPU.
"""
from __future__ import annotations

import collections
import ctypes
import time

from . import _lib
from .codec import Codec, Context, Job, _check, _dev_ptr

__all__ = ["Request", "BatchServer", "PlainServer", "percentiles", "make_job_array"]


class Request(Job):
    """A Job plus its arrival and completion times (seconds, perf_counter)."""

    def __init__(self, job: Job, arrival: float = 0.0):
        super().__init__(job.op, job.n, job.t, job.src, job.dst, job.shard_len, job.positions)
        self.arrival = arrival
        self.done = None
        self.ready = None  # event on the submitter's stream (mark_submitted)

    def mark_submitted(self) -> None:
        """Records, on the caller's current stream, the point after which the
        request's buffers may be used."""
        import torch

        self.ready = torch.cuda.Event()
        self.ready.record()

    def enter_stream(self, s) -> None:
        """Orders stream ``s`` after the submitter's work on the buffers and
        keeps the buffers' memory from being reused before ``s`` is done."""
        if self.ready is not None:
            s.wait_event(self.ready)
        for buf in (self.src, self.dst):
            if buf is not None and hasattr(buf, "record_stream"):
                buf.record_stream(s)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def make_job_array(jobs):
    """ctypes array of struct afrs_job for ``jobs`` (see include/afrs.h)."""
    arr = (_lib.AfrsJob * max(len(jobs), 1))()
    for i, j in enumerate(jobs):
        a = arr[i]
        a.op, a.n, a.t, a.shard_len = j.op, j.n, j.t, j.shard_len
        a.e = len(j.positions)
        for q, p in enumerate(j.positions[:256]):
            a.positions[q] = p
        a.src = _dev_ptr(j.src) if j.src is not None else None
        a.dst = _dev_ptr(j.dst) if j.dst is not None else None
    return arr


def percentiles(values, ps=(50, 99, 99.9)):
    xs = sorted(values)
    if not xs:
        return {p: None for p in ps}
    out = {}
    for p in ps:
        k = min(len(xs) - 1, max(0, int(round(p / 100.0 * (len(xs) - 1)))))
        out[p] = xs[k]
    return out


class BatchServer:
    """Continuous batching: up to ``streams`` batches in flight, each holding
    at most ``max_batch_bytes`` of codewords, all in flight together at most
    ``hbm_cap`` bytes (the admission cap on device memory).

    Requests of at least ``large_bytes`` are not batched: one such codeword
    already fills the GPU, and the per-shape kernels of the per-call path run
    it faster than the batched kernel's shape-generic code, so they go one at
    a time to a stream of their own, under the same admission cap, and never
    hold back the small requests' batches."""

    def __init__(self, device: int = 0, streams: int = 3, max_batch_bytes: int = 512 << 20,
                 hbm_cap: int = 32 << 30, large_bytes: int = 16 << 20):
        import torch

        self.device = device
        self.ctx = Context.get(device)
        self.streams = [torch.cuda.Stream(device) for _ in range(streams)]
        self.busy = [None] * streams  # (event, requests, bytes) per stream
        self.queue = collections.deque()
        self.max_batch_bytes = max_batch_bytes
        self.hbm_cap = hbm_cap
        self.inflight_bytes = 0
        self.batches = 0
        self.large_bytes = large_bytes
        self.large = PlainServer(device, window=4)

    def submit(self, req: Request) -> None:
        req.mark_submitted()
        if req.nbytes >= self.large_bytes:
            self.large.submit(req)
        else:
            self.queue.append(req)

    def pending(self) -> int:
        return len(self.queue) + sum(len(b[1]) for b in self.busy if b is not None) + self.large.pending()

    def _poll_large(self) -> list:
        # admission: a large request enters the per-call stream only while the cap allows
        admit = []
        while self.large.queue and (self.inflight_bytes + self.large.queue[0].nbytes <= self.hbm_cap
                                    or self.inflight_bytes == 0):
            r = self.large.queue.popleft()
            self.inflight_bytes += r.nbytes
            admit.append(r)
        held = list(self.large.queue)
        self.large.queue = collections.deque(admit)
        finished = self.large.poll()
        self.large.queue.extend(held)
        for r in finished:
            self.inflight_bytes -= r.nbytes
        return finished

    def poll(self) -> list:
        """Retire finished batches, launch new ones; returns finished requests."""
        import torch

        finished = self._poll_large()
        now = time.perf_counter()
        for i, b in enumerate(self.busy):
            if b is not None and b[0].query():
                for r in b[1]:
                    r.done = now
                finished.extend(b[1])
                self.inflight_bytes -= b[2]
                self.busy[i] = None
        for i in range(len(self.streams)):
            if self.busy[i] is not None or not self.queue:
                continue
            take, nbytes = [], 0
            while self.queue:
                r = self.queue[0]
                if take and nbytes + r.nbytes > self.max_batch_bytes:
                    break
                if self.inflight_bytes + nbytes + r.nbytes > self.hbm_cap and (take or self.inflight_bytes):
                    break
                take.append(self.queue.popleft())
                nbytes += r.nbytes
            if not take:
                break
            arr = make_job_array(take)
            s = self.streams[i]
            for r in take:
                r.enter_stream(s)
            _check(_lib.lib().afrs_batch_dev(self.ctx.handle, arr, len(take), s.cuda_stream), "afrs_batch_dev")
            for q, r in enumerate(take):
                r.status = int(arr[q].status)
            ev = torch.cuda.Event()
            ev.record(s)
            self.busy[i] = (ev, take, nbytes)
            self.inflight_bytes += nbytes
            self.batches += 1
        return finished


class PlainServer:
    """One request per call, in arrival order, on one stream."""

    def __init__(self, device: int = 0, window: int = 64):
        import torch

        self.device = device
        self.stream = torch.cuda.Stream(device)
        self.queue = collections.deque()
        self.inflight = collections.deque()  # (event, request)
        self.window = window
        self.codecs = {}

    def submit(self, req: Request) -> None:
        if req.ready is None:
            req.mark_submitted()
        self.queue.append(req)

    def pending(self) -> int:
        return len(self.queue) + len(self.inflight)

    def _codec(self, n, t):
        c = self.codecs.get((n, t))
        if c is None:
            c = self.codecs[(n, t)] = Codec(n, t, self.device)
        return c

    def poll(self) -> list:
        import torch

        finished = []
        now = time.perf_counter()
        while self.inflight and self.inflight[0][0].query():
            _, r = self.inflight.popleft()
            r.done = now
            finished.append(r)
        with torch.cuda.stream(self.stream):
            while self.queue and len(self.inflight) < self.window:
                r = self.queue.popleft()
                r.enter_stream(self.stream)
                c = self._codec(r.n, r.t)
                if r.op == _lib.AFRS_OP_ENCODE:
                    c.encode_parity(r.src, r.dst, r.shard_len)
                    r.status = 0
                else:
                    r.status = int(c.recover_erasure_shards(r.dst, None, r.shard_len, r.positions))
                ev = torch.cuda.Event()
                ev.record(self.stream)
                self.inflight.append((ev, r))
        return finished


def serve_open_loop(server, requests, arrivals, timeout_s: float = 60.0):
    """Feed ``requests`` at the given arrival offsets (seconds from start,
    increasing) and run the server until all finish.  Returns (finished
    requests, wall seconds)."""
    t0 = time.perf_counter()
    i, done = 0, []
    n = len(requests)
    while len(done) < n:
        now = time.perf_counter()
        if now - t0 > timeout_s:
            raise TimeoutError(f"serving did not finish in {timeout_s} s ({len(done)}/{n} done)")
        while i < n and t0 + arrivals[i] <= now:
            requests[i].arrival = t0 + arrivals[i]
            server.submit(requests[i])
            i += 1
        done.extend(server.poll())
        if i < n and not server.pending():
            time.sleep(max(0.0, min(1e-4, t0 + arrivals[i] - time.perf_counter())))
    return done, time.perf_counter() - t0
