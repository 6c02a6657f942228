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

Stream order: ``submit`` / ``submit_many`` record one event on the caller's
current stream for the requests they accept, and the stream that runs a
request waits on it, so work the caller enqueued on the request's buffers
before submitting (a fill, a copy) is finished first.  The buffers are also
recorded on the running stream, so that torch's caching allocator does not
hand their memory to another tensor while the request is still on the GPU.

Host cost per request is what bounds a server of small requests, so events
are reused (creating a CUDA event costs several microseconds, recording a
reused one about one), requests that arrive together share one submission
event, and a batch's stream waits once per distinct submission event.
"""
from __future__ import annotations

import collections
import time

from . import _lib
from .codec import Codec, Context, Job, _check, _job_array, _job_statuses

__all__ = ["Request", "BatchServer", "PlainServer", "percentiles", "make_job_array"]


class Request(Job):
    """A Job plus its arrival and completion times (seconds, perf_counter)."""

    def __init__(self, job: Job, arrival: float = 0.0):
        super().__init__(job.op, job.n, job.t, job.src, job.dst, job.shard_len, job.positions)
        self.arrival = arrival
        self.done = None
        self.ready = None  # event on the submitter's stream (mark_submitted)

    def mark_submitted(self, event=None) -> None:
        """Records, on the caller's current stream, the point after which the
        request's buffers may be used (or takes ``event``, recorded there
        already, which requests submitted together share)."""
        import torch

        if event is None:
            event = torch.cuda.Event()
            event.record()
        self.ready = event

    def enter_stream(self, s, events=None, waited=None) -> None:
        """Orders stream ``s`` after the submitter's work on the buffers and
        keeps the buffers' memory from being reused before ``s`` is done.
        ``waited`` (a set) holds the ids of submission events ``s`` already
        waits on; ``events`` (an _EventPool) takes the event back once every
        request sharing it has entered its stream."""
        ev = self.ready
        if ev is not None:
            if waited is None or id(ev) not in waited:
                s.wait_event(ev)
                if waited is not None:
                    waited.add(id(ev))
            if events is not None:
                events.release(ev)
        for buf in (self.src, self.dst):
            if buf is not None and hasattr(buf, "record_stream"):
                buf.record_stream(s)

    @property
    def latency(self) -> float:
        return self.done - self.arrival


class _EventPool:
    """CUDA events for reuse.  ``record`` hands out a recorded event that
    ``uses`` holders will ``release``; after the last release it is recorded
    again for a later holder.  Re-recording is safe once the holders are done
    with it: a stream wait enqueued on an event keeps the work the event
    captured when the wait was enqueued, and completion events are released
    only after ``query()`` returned True."""

    def __init__(self):
        self.free = []
        self.uses = {}

    def record(self, stream=None, uses: int = 1):
        import torch

        ev = self.free.pop() if self.free else torch.cuda.Event()
        ev.record(stream)
        self.uses[id(ev)] = (ev, uses)
        return ev

    def release(self, ev) -> None:
        k = id(ev)
        held = self.uses.get(k)
        if held is None:
            return
        if held[1] <= 1:
            del self.uses[k]
            self.free.append(ev)
        else:
            self.uses[k] = (ev, held[1] - 1)


def make_job_array(jobs):
    """ctypes array of struct afrs_job for ``jobs`` (see include/afrs.h)."""
    return _job_array(jobs)


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
        self.events = _EventPool()
        # Large requests queue on the GPU up to 16 deep, so that their stream
        # keeps running while the host packs the next batch of small ones.
        self.large = PlainServer(device, window=16, events=self.events)

    def submit(self, req: Request) -> None:
        self.submit_many((req,))

    def submit_many(self, reqs) -> None:
        """Accepts requests that arrived together (one submission event)."""
        if not reqs:
            return
        ev = self.events.record(uses=len(reqs))
        for r in reqs:
            r.mark_submitted(ev)
            if r.nbytes >= self.large_bytes:
                self.large.queue.append(r)
            else:
                self.queue.append(r)

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
        finished = self._poll_large()
        now = time.perf_counter()
        for i, b in enumerate(self.busy):
            if b is not None and b[0].query():
                for r in b[1]:
                    r.done = now
                finished.extend(b[1])
                self.inflight_bytes -= b[2]
                self.events.release(b[0])
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
            waited = set()
            for r in take:
                r.enter_stream(s, self.events, waited)
            _check(_lib.lib().afrs_batch_dev(self.ctx.handle, arr, len(take), s.cuda_stream), "afrs_batch_dev")
            for r, st in zip(take, _job_statuses(arr, len(take))):
                r.status = st
            self.busy[i] = (self.events.record(s), take, nbytes)
            self.inflight_bytes += nbytes
            self.batches += 1
        return finished


class PlainServer:
    """One request per call, in arrival order, on one stream."""

    def __init__(self, device: int = 0, window: int = 64, events: "_EventPool | None" = None):
        import torch

        self.device = device
        self.stream = torch.cuda.Stream(device)
        self.queue = collections.deque()
        self.inflight = collections.deque()  # (event, request)
        self.window = window
        self.codecs = {}
        self.events = events if events is not None else _EventPool()

    def submit(self, req: Request) -> None:
        self.submit_many((req,))

    def submit_many(self, reqs) -> None:
        """Accepts requests that arrived together (one submission event)."""
        if not reqs:
            return
        ev = self.events.record(uses=len(reqs))
        for r in reqs:
            r.mark_submitted(ev)
            self.queue.append(r)

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
            ev, r = self.inflight.popleft()
            r.done = now
            self.events.release(ev)
            finished.append(r)
        if not self.queue or len(self.inflight) >= self.window:
            return finished
        waited = set()
        with torch.cuda.stream(self.stream):
            while self.queue and len(self.inflight) < self.window:
                r = self.queue.popleft()
                r.enter_stream(self.stream, self.events, waited)
                c = self._codec(r.n, r.t)
                if r.op == _lib.AFRS_OP_ENCODE:
                    c.encode_parity(r.src, r.dst, r.shard_len)
                    r.status = 0
                else:
                    r.status = int(c.recover_erasure_shards(r.dst, None, r.shard_len, r.positions))
                self.inflight.append((self.events.record(self.stream), r))
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
        due = []
        while i < n and t0 + arrivals[i] <= now:
            requests[i].arrival = t0 + arrivals[i]
            due.append(requests[i])
            i += 1
        if due:
            server.submit_many(due)
        done.extend(server.poll())
        if i < n and not server.pending():
            time.sleep(max(0.0, min(1e-4, t0 + arrivals[i] - time.perf_counter())))
    return done, time.perf_counter() - t0
