"""The few-erasure recover (n >= 32, 1 <= e <= 8: one pass over the surviving
shards and an e x e solve) gives the oracle's bytes (rs/src/codec.rs:479-569)
on codewords and on words that are not codewords, for every chunk size it
uses (T = 1, 2, 4, 8), on the device, host-buffer and graph-captured paths,
and equals the Leopard-form kernels it replaces on long shards."""
import numpy as np
import pytest

from oracle import oracle

torch = pytest.importorskip("torch")


def _codeword(n, t, L, seed):
    msg = oracle.random_bytes((n - t) * L, seed)
    par = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, par, L)
    return np.concatenate([par, msg])


def _erase(cw, L, pos):
    rx = cw.copy()
    for p in pos:
        rx[p * L:(p + 1) * L] = 0
    return rx


def _recover_dev(afrs, n, t, rx, L, pos, route=None):
    ctx = afrs.Context(0)
    if route is not None:
        ctx.set_route(getattr(afrs._lib, route))
    d = torch.from_numpy(rx.copy()).cuda()
    ok = afrs.Codec(n, t, context=ctx).recover_erasure_shards(d, None, L, pos)
    out = d.cpu().numpy()
    ctx.close()
    return ok, out


@pytest.mark.gpu
@pytest.mark.parametrize("n", [32, 64, 128, 256])
@pytest.mark.parametrize("e", [1, 2, 3, 4, 5, 7, 8])
@pytest.mark.parametrize("L", [64, 1000, 4096 + 37])
def test_few_matches_oracle_on_codewords_and_other_words(afrs, n, e, L):
    t = max(8, e)
    rng = np.random.default_rng(n * 131 + e * 7 + L)
    cw = _codeword(n, t, L, seed=n + e + L)
    for word in (cw, rng.integers(0, 256, n * L, dtype=np.uint8)):
        pos = rng.choice(n, e, replace=False).tolist()
        rx = _erase(word, L, pos)
        ref = rx.copy()
        assert oracle.recover_erasure_shards(n, t, ref, L, pos)
        for route in ("AFRS_ROUTE_TABLE", "AFRS_ROUTE_FEW"):
            ok, out = _recover_dev(afrs, n, t, rx, L, pos, route)
            assert ok and (out == ref).all(), (n, e, L, route)
        if word is cw:
            assert (ref == cw).all()


# Patterns at the edges of the chunk structure: all erasures in the parity
# chunk, in one message chunk, across a chunk boundary, first and last rows,
# and unsorted positions.
PATTERNS = [
    (256, 8, [0, 1, 2, 3, 4, 5, 6, 7]),
    (256, 8, [8, 9, 10, 11, 12, 13, 14, 15]),
    (256, 8, [6, 7, 8, 9, 10]),
    (256, 8, [0, 255]),
    (256, 8, [255, 3, 128, 64, 17, 200]),
    (32, 4, [28, 29, 30, 31]),
    (64, 16, [63]),
    (128, 64, [5, 69, 70]),
]


@pytest.mark.gpu
@pytest.mark.parametrize("n,t,pos", PATTERNS)
def test_few_edge_patterns(afrs, n, t, pos):
    L = 777
    cw = _codeword(n, t, L, seed=n * 3 + len(pos))
    rx = _erase(cw, L, pos)
    ok, out = _recover_dev(afrs, n, t, rx, L, pos)
    assert ok and (out == cw).all()
    other = _erase(np.random.default_rng(len(pos)).integers(0, 256, n * L, dtype=np.uint8), L, pos)
    ref = other.copy()
    oracle.recover_erasure_shards(n, t, ref, L, pos)
    ok, out = _recover_dev(afrs, n, t, other, L, pos)
    assert ok and (out == ref).all()


@pytest.mark.gpu
def test_few_is_one_launch_and_falls_back_beyond_eight(afrs):
    lib = afrs.lib()
    # Every n >= 32 takes it for e <= 8; beyond, the three Leopard-form phase
    # kernels.
    for n, e, launches in ((256, 1, 1), (256, 2, 1), (256, 8, 1), (128, 8, 1), (128, 9, 3), (256, 9, 3)):
        t, L = 32, 4096
        cw = _codeword(n, t, L, seed=5 + n)
        pos = list(range(40, 40 + e))
        d = torch.from_numpy(_erase(cw, L, pos)).cuda()
        codec = afrs.Codec(n, t)
        torch.cuda.synchronize()
        before = lib.afrs_kernel_launches()
        assert codec.recover_erasure_shards(d, None, L, pos)
        torch.cuda.synchronize()
        assert lib.afrs_kernel_launches() - before == launches, (n, e)
        assert (d.cpu().numpy() == cw).all()


@pytest.mark.gpu
@pytest.mark.parametrize("e", [1, 4, 8])
def test_few_long_shards_equal_the_leopard_kernels(afrs, e):
    # Sizes where the oracle is slow: the round trip of a GPU-encoded
    # codeword, and, on a word that is not a codeword, the Leopard-form phase
    # kernels (forced with AFRS_ROUTE_SPECIAL), which the oracle pins above.
    n, t, L = 256, 32, (1 << 20) + 5
    g = torch.Generator(device="cuda")
    g.manual_seed(e)
    cw = torch.randint(0, 256, (n * L,), dtype=torch.uint8, device="cuda", generator=g)
    codec = afrs.Codec(n, t)
    cw[: t * L].zero_()
    codec.encode_systematic_sharded(cw[t * L:], cw[: t * L], None, L)
    pos = sorted(np.random.default_rng(e).choice(n, e, replace=False).tolist())
    rx = cw.clone()
    for p in pos:
        rx[p * L:(p + 1) * L].zero_()
    assert codec.recover_erasure_shards(rx, None, L, pos)
    assert torch.equal(rx, cw)
    word = torch.randint(0, 256, (n * L,), dtype=torch.uint8, device="cuda", generator=g)
    for p in pos:
        word[p * L:(p + 1) * L].zero_()
    outs = []
    for route in ("AFRS_ROUTE_FEW", "AFRS_ROUTE_SPECIAL"):
        ctx = afrs.Context(0)
        ctx.set_route(getattr(afrs._lib, route))
        w = word.clone()
        assert afrs.Codec(n, t, context=ctx).recover_erasure_shards(w, None, L, pos)
        torch.cuda.synchronize()
        outs.append(w)
        ctx.close()
    assert torch.equal(outs[0], outs[1])


@pytest.mark.gpu
@pytest.mark.parametrize("n,t,L,pos", [(64, 16, 65536 + 77, [3, 40, 41]), (256, 8, 3 * 65536 + 1, [7, 8, 100, 255]),
                                       (32, 8, 5000, [31])])
def test_few_host_buffers(afrs, n, t, L, pos):
    cw = _codeword(n, t, L, seed=L)
    codec = afrs.Codec(n, t)
    rx = _erase(cw, L, pos)
    assert codec.recover_erasure_shards(rx, None, L, pos)  # pageable: staged windows
    assert (rx == cw).all()
    pinned = torch.from_numpy(_erase(cw, L, pos)).pin_memory()
    assert codec.recover_erasure_shards(pinned.numpy(), None, L, pos)  # page-locked: direct
    assert (pinned.numpy() == cw).all()


@pytest.mark.gpu
def test_few_in_a_cuda_graph(afrs):
    n, t, L = 128, 16, 8192 + 3
    cw = _codeword(n, t, L, seed=21)
    pos = [1, 50, 127]
    codec = afrs.Codec(n, t)
    src = torch.from_numpy(_erase(cw, L, pos)).cuda()
    d = src.clone()
    assert codec.recover_erasure_shards(d, None, L, pos)  # first call outside capture
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        d.copy_(src)
        with torch.cuda.graph(graph, stream=s):
            codec.recover_erasure_shards(d, None, L, pos)
    for _ in range(2):
        d.copy_(src)
        graph.replay()
        torch.cuda.synchronize()
        assert (d.cpu().numpy() == cw).all()


@pytest.mark.gpu
def test_few_batch_groups_match_oracle(afrs):
    """afrs_batch_dev: recovers of at most 8 erasures (n >= 32) form groups of
    one n and chunk size on the few-erasure kernel once a group holds 1 MiB;
    smaller ones and e > 8 take the other kernels.  Codewords and other words
    (erased rows hold garbage, which every path ignores), byte-exact."""
    rng = np.random.default_rng(77)
    specs = [(256, 8, 2000, 1, 4), (256, 8, 1500, 2, 4), (128, 16, 3000, 4, 6), (64, 32, 5000, 7, 6),
             (32, 16, 9000, 8, 6), (256, 64, 700, 5, 8), (32, 8, 100, 3, 3), (256, 32, 1000, 20, 3)]
    jobs, expect = [], []
    for q, (n, t, L, e, count) in enumerate(specs):
        for i in range(count):
            word = _codeword(n, t, L, seed=500 + 31 * q + i) if i % 2 == 0 else \
                rng.integers(0, 256, n * L, dtype=np.uint8)
            pos = rng.choice(n, e, replace=False).tolist()
            ref = _erase(word, L, pos)
            assert oracle.recover_erasure_shards(n, t, ref, L, pos)
            rx = word.copy()
            for p in pos:
                rx[p * L:(p + 1) * L] = 0x5A
            jobs.append(afrs.Job.recover(n, t, torch.from_numpy(rx).cuda(), L, pos))
            expect.append(ref)
    for _ in range(2):  # the second batch reuses the context's tables
        status = afrs.run_batch(jobs)
        torch.cuda.synchronize()
        for j, ex, st in zip(jobs, expect, status):
            assert st == 1
            assert (j.dst.cpu().numpy() == ex).all(), (j.n, j.t, len(j.positions), j.shard_len)


@pytest.mark.gpu
def test_few_from_concurrent_threads_with_different_patterns(afrs):
    """Host threads recovering different few-erasure patterns at once (each
    thread keeps its own cached solve; pageable and page-locked buffers,
    device buffers on its own context) give the oracle's bytes every time."""
    import threading

    n, t, L, steps = 128, 16, 6000, 5
    cw = _codeword(n, t, L, seed=77)
    rng = np.random.default_rng(12)
    patterns = [sorted(rng.choice(n, e, replace=False).tolist()) for e in (1, 3, 5, 8, 2, 7)]
    errors = []

    def work(q, pos):
        try:
            codec = afrs.Codec(n, t, context=afrs.Context(0))
            for s in range(steps):
                p = pos if s % 2 == 0 else patterns[(q + 1) % len(patterns)]
                rx = _erase(cw, L, p)
                if q % 3 == 0:
                    buf = rx
                elif q % 3 == 1:
                    buf = torch.from_numpy(rx).pin_memory().numpy()
                else:
                    buf = torch.from_numpy(rx).cuda()
                assert codec.recover_erasure_shards(buf, None, L, p)
                out = buf.cpu().numpy() if isinstance(buf, torch.Tensor) else buf
                assert (out == cw).all(), (q, s)
        except Exception as ex:  # surfaced below
            errors.append(ex)

    ths = [threading.Thread(target=work, args=(q, p)) for q, p in enumerate(patterns)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    assert not errors, errors[0]
