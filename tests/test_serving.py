"""Serving loop: continuous batching gives every request the same bytes as
serving it alone, respects the device-memory admission cap, and reports
latency percentiles."""
import numpy as np
import pytest

from oracle import oracle

torch = pytest.importorskip("torch")


def test_percentiles(afrs):
    p = afrs.serving.percentiles(list(range(1, 1001)))
    assert p[50] == 501 and p[99] == 990 and p[99.9] == 999
    assert afrs.serving.percentiles([])[50] is None


def _requests(afrs, count, seed):
    """Seeded jobs of config-3 shapes and, per job, the bytes the oracle says
    its dst must hold afterwards: the parity (encode) or the whole original
    codeword (recover)."""
    rng = np.random.default_rng(seed)
    out, expect = [], []
    for i in range(count):
        n = int(rng.choice([32, 64, 128, 256]))
        t = int(rng.choice([4, 8, n // 4, n // 2]))
        L = 64 * int(rng.integers(1, 40))
        msg = oracle.random_bytes((n - t) * L, seed * 7919 + i)
        par = np.zeros(t * L, np.uint8)
        oracle.encode_systematic_sharded(n, t, msg, par, L)
        if i % 2 == 0:
            job = afrs.Job.encode(n, t, torch.from_numpy(msg).cuda(), torch.zeros(t * L, dtype=torch.uint8,
                                                                                   device="cuda"), L)
            expect.append(par)
        else:
            cw = np.concatenate([par, msg])
            expect.append(cw.copy())
            pos = rng.choice(n, int(rng.integers(1, t + 1)), replace=False).tolist()
            for p in pos:
                cw[p * L:(p + 1) * L] = 0
            job = afrs.Job.recover(n, t, torch.from_numpy(cw).cuda(), L, pos)
        out.append(job)
    return out, expect


def _clone(afrs, j):
    src = j.src.clone() if j.src is not None else None
    return afrs.Job(j.op, j.n, j.t, src, j.dst.clone(), j.shard_len, j.positions)


@pytest.mark.gpu
def test_result_alone_equals_result_in_the_mix(afrs):
    S = afrs.serving
    jobs, expect = _requests(afrs, 60, seed=4)
    alone = [_clone(afrs, j) for j in jobs]
    reqs = [S.Request(j) for j in jobs]
    arrivals = [i * 2e-5 for i in range(len(reqs))]  # arrivals overlap running batches
    # requests of 200 KB and more take the per-call path inside the server
    server = S.BatchServer(streams=3, max_batch_bytes=1 << 20, large_bytes=200_000)
    done, _ = S.serve_open_loop(server, reqs, arrivals)
    torch.cuda.synchronize()
    assert len(done) == len(reqs) and server.batches > 1
    assert any(r.nbytes >= 200_000 for r in reqs) and any(r.nbytes < 200_000 for r in reqs)
    for j in alone:  # each request served alone, as a batch of one
        afrs.run_batch([j])
    torch.cuda.synchronize()
    for r, a, want in zip(reqs, alone, expect):
        assert r.status == a.status
        # exact: integer arithmetic, no tolerance; the oracle's bytes, served
        # in the mix and served alone
        got = r.dst.cpu().numpy()
        assert (got == want).all()
        assert torch.equal(r.dst, a.dst)
        assert r.latency >= 0


@pytest.mark.gpu
def test_admission_cap_and_plain_server(afrs):
    S = afrs.serving
    jobs, expect = _requests(afrs, 30, seed=8)
    plain_jobs = [_clone(afrs, j) for j in jobs]
    reqs = [S.Request(j) for j in jobs]
    cap = 3 * max(r.nbytes for r in reqs)
    server = S.BatchServer(streams=4, hbm_cap=cap)
    peak = 0
    for r in reqs:
        server.submit(r)
    done = []
    while len(done) < len(reqs):
        done.extend(server.poll())
        peak = max(peak, server.inflight_bytes)
    assert peak <= cap
    preqs = [S.Request(j) for j in plain_jobs]
    pdone, _ = S.serve_open_loop(S.PlainServer(), preqs, [0.0] * len(preqs))
    torch.cuda.synchronize()
    for r, p, want in zip(reqs, preqs, expect):
        assert (r.dst.cpu().numpy() == want).all()
        assert torch.equal(r.dst, p.dst)


class _FakeEvent:
    def __init__(self):
        self.records = 0

    def record(self, stream=None):
        self.records += 1


def test_event_pool_reuses_an_event_after_its_last_holder(afrs):
    pool = afrs.serving._EventPool()
    a, b = _FakeEvent(), _FakeEvent()
    pool.free = [b, a]
    ev = pool.record(uses=3)
    assert ev is a and a.records == 1
    pool.release(ev)
    pool.release(ev)
    assert pool.free == [b]  # two of three holders released it
    pool.release(ev)
    assert pool.free == [b, a]
    pool.release(ev)  # not held any more: ignored
    assert pool.free == [b, a]
    assert pool.record() is a and a.records == 2
    pool.release(_FakeEvent())  # an event the pool never handed out
    assert pool.free == [b]


def test_a_batch_stream_waits_once_per_submission_event(afrs):
    S = afrs.serving

    class Stream:
        def __init__(self):
            self.waits = []

        def wait_event(self, ev):
            self.waits.append(ev)

    pool = S._EventPool()
    e1, e2 = _FakeEvent(), _FakeEvent()
    pool.free = [e2, e1]
    reqs = [S.Request(afrs.Job(1, 32, 8, None, None, 64, [1])) for _ in range(5)]
    first = pool.record(uses=3)
    second = pool.record(uses=2)
    for r in reqs[:3]:
        r.mark_submitted(first)
    for r in reqs[3:]:
        r.mark_submitted(second)
    s, waited = Stream(), set()
    for r in reqs:
        r.enter_stream(s, pool, waited)
    assert s.waits == [first, second]
    assert sorted(map(id, pool.free)) == sorted([id(e1), id(e2)]) and not pool.uses


def test_job_array_layout(afrs):
    """The packed records match struct afrs_job field by field."""
    jobs = [afrs.Job(1, 128, 32, None, None, 1024, [3, 5, 200]), afrs.Job(0, 64, 8, None, None, 64)]
    arr = afrs.codec._job_array(jobs)
    a, b = arr[0], arr[1]
    assert (a.op, a.n, a.t, a.e, a.shard_len, a.status) == (1, 128, 32, 3, 1024, 0)
    assert list(a.positions[:4]) == [3, 5, 200, 0] and not a.src and not a.dst
    assert (b.op, b.n, b.t, b.e, b.shard_len) == (0, 64, 8, 0, 64) and not any(b.positions)
    a.status, b.status = 7, -3
    assert afrs.codec._job_statuses(arr, 2) == [7, -3]
    with pytest.raises(afrs.AfrsError):
        afrs.codec._job_array([afrs.Job(1, 128, 32, None, None, 1024, [300])])
    assert len(afrs.codec._job_array([])) == 1
