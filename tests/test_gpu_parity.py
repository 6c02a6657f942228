"""GPU parity: the CUDA path through the C ABI against the CPU oracle,
bit-exact, on seeded inputs.  Covers every (n, t) shape the reference's own
tests cover (rs/src/poly_11d_lut.rs:431-566), odd and misaligned shard
lengths, random and adversarial erasure patterns, and the Kernel-trait ops."""
import numpy as np
import pytest

from oracle import oracle

torch = pytest.importorskip("torch")

PAIRS_ALL = [(n, t) for n in (2, 4, 8, 16, 32, 64, 128, 256) for t in (1, 2, 4, 8, 16, 32, 64, 128) if t < n]
T = oracle.tables()


def _codeword(n, t, L, seed):
    msg = oracle.random_bytes((n - t) * L, seed)
    par = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, par, L)
    return msg, par


def _erase(cw, L, pos):
    rx = cw.copy()
    for p in pos:
        rx[p * L:(p + 1) * L] = 0
    return rx


@pytest.mark.gpu
@pytest.mark.parametrize("n,t", PAIRS_ALL)
@pytest.mark.parametrize("L", [1, 33, 256])
def test_encode_matches_oracle(afrs, n, t, L):
    msg, ref = _codeword(n, t, L, seed=n * 131 + t * 7 + L)
    d_par = torch.zeros(t * L, dtype=torch.uint8, device="cuda")
    afrs.Codec(n, t).encode_parity(torch.from_numpy(msg).cuda(), d_par, L)
    assert (d_par.cpu().numpy() == ref).all()


@pytest.mark.gpu
@pytest.mark.parametrize("n,t", [(4, 2), (32, 8), (64, 32), (256, 128), (256, 32), (128, 4)])
def test_encode_accumulates_like_reference(afrs, n, t):
    # codec.rs:259-264: parity buffer is XOR-accumulated before the final FFT.
    L = 100
    msg = oracle.random_bytes((n - t) * L, 3)
    p0 = oracle.random_bytes(t * L, 4)
    ref = p0.copy()
    oracle.encode_systematic_sharded(n, t, msg, ref, L)
    got = p0.copy()
    afrs.Codec(n, t).encode_systematic_sharded(msg, got, None, L)  # host buffers
    assert (got == ref).all()
    d = torch.from_numpy(p0.copy()).cuda()
    afrs.Codec(n, t).encode_systematic_sharded(torch.from_numpy(msg).cuda(), d, None, L)
    assert (d.cpu().numpy() == ref).all()


@pytest.mark.gpu
@pytest.mark.parametrize("n,t", PAIRS_ALL)
def test_recover_reference_pattern(afrs, n, t):
    # rs/src/poly_11d_lut.rs:536-566: L = 1, erase odd positions 1..2T-1,
    # message[i][j] = T + i + j.
    L = 1
    msg = ((t + np.arange(n - t)) % 256).astype(np.uint8)
    par = np.zeros(t, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, par, L)
    cw = np.concatenate([par, msg])
    pos = list(range(1, 2 * t, 2))
    d = torch.from_numpy(_erase(cw, L, pos)).cuda()
    assert afrs.Codec(n, t).recover_erasure_shards(d, None, L, pos)
    assert (d.cpu().numpy() == cw).all()


@pytest.mark.gpu
@pytest.mark.parametrize("n,t", PAIRS_ALL)
def test_recover_random_patterns_match_oracle(afrs, n, t):
    rng = np.random.default_rng(n * 17 + t)
    L = 77
    msg, par = _codeword(n, t, L, seed=n + t)
    cw = np.concatenate([par, msg])
    codec = afrs.Codec(n, t)
    for e in sorted({1, max(1, t // 2), t}):
        pos = rng.choice(n, e, replace=False).tolist()
        rx = _erase(cw, L, pos)
        ref = rx.copy()
        assert oracle.recover_erasure_shards(n, t, ref, L, pos)
        d = torch.from_numpy(rx).cuda()
        assert codec.recover_erasure_shards(d, None, L, pos)
        out = d.cpu().numpy()
        assert (out == ref).all() and (out == cw).all(), (n, t, e)


@pytest.mark.gpu
@pytest.mark.parametrize("n,t", [(16, 8), (64, 16), (256, 64), (256, 128)])
def test_recover_non_codeword_input_matches_reference(afrs, n, t):
    # Surviving rows that are not a codeword (e < t): the GPU decoder still
    # computes the reference's map exactly (erased rows zero).
    rng = np.random.default_rng(99 + n + t)
    L = 48
    for e in sorted({1, t // 2}):
        rx = rng.integers(0, 256, n * L, dtype=np.uint8)
        pos = rng.choice(n, e, replace=False).tolist()
        rx = _erase(rx, L, pos)
        ref = rx.copy()
        oracle.recover_erasure_shards(n, t, ref, L, pos)
        d = torch.from_numpy(rx).cuda()
        afrs.Codec(n, t).recover_erasure_shards(d, None, L, pos)
        assert (d.cpu().numpy() == ref).all()


@pytest.mark.gpu
def test_host_buffer_api_and_adversarial_patterns(afrs):
    n, t, L = 256, 32, 4096 + 3
    msg, par = _codeword(n, t, L, seed=11)
    cw = np.concatenate([par, msg])
    codec = afrs.Codec(n, t)
    got = np.zeros(t * L, np.uint8)
    codec.encode_systematic_sharded(msg, got, None, L)
    assert (got == par).all()
    for pos in (list(range(40, 72)), list(range(200, 232)), list(range(0, 32)), list(range(224, 256))):
        rx = _erase(cw, L, pos)
        assert codec.recover_erasure_shards(rx, None, L, pos)
        assert (rx == cw).all()


@pytest.mark.gpu
def test_misaligned_and_ragged_buffers(afrs):
    n, t, L = 64, 16, 1000 + 1
    msg, par = _codeword(n, t, L, seed=5)
    cw = np.concatenate([par, msg])
    big = torch.zeros(n * L + 64, dtype=torch.uint8, device="cuda")
    for off in (1, 3, 8):
        view = big[off:off + n * L]
        view.copy_(torch.from_numpy(cw))
        view[: t * L].zero_()
        afrs.Codec(n, t).encode_parity(view[t * L:], view[: t * L], L)
        assert (view.cpu().numpy() == cw).all()
        pos = [0, 5, 17, 33, 40, 41, 62, 63]
        for p in pos:
            view[p * L:(p + 1) * L].zero_()
        assert afrs.Codec(n, t).recover_erasure_shards(view, None, L, pos)
        assert (view.cpu().numpy() == cw).all()


@pytest.mark.gpu
def test_recover_edge_cases(afrs):
    n, t, L = 32, 8, 64
    msg, par = _codeword(n, t, L, seed=2)
    cw = np.concatenate([par, msg])
    codec = afrs.Codec(n, t)
    d = torch.from_numpy(cw.copy()).cuda()
    assert codec.recover_erasure_shards(d, None, L, [])  # e == 0 -> true, no-op
    assert not codec.recover_erasure_shards(d, None, L, list(range(9)))  # e > t -> false
    assert (d.cpu().numpy() == cw).all()
    with pytest.raises(afrs.AfrsError):
        codec.recover_erasure_shards(d, None, L, [1, 1])
    with pytest.raises(afrs.AfrsError):
        codec.recover_erasure_shards(d, None, L, [40])
    with pytest.raises(afrs.AfrsError):
        afrs.Codec(24, 8)
        afrs.Codec(24, 8).encode_parity(torch.zeros(16 * L, dtype=torch.uint8, device="cuda"),
                                        torch.zeros(8 * L, dtype=torch.uint8, device="cuda"), L)
    z = torch.zeros(0, dtype=torch.uint8, device="cuda")
    afrs.Codec(4, 2).encode_parity(z, z, 0)  # empty shards


@pytest.mark.gpu
@pytest.mark.parametrize("L", [1, 63, 64, 65, 128, 1000])
def test_kernel_trait_transforms_and_scale(afrs, L):
    # rs/src/kernel/gfni_kernel.rs:324-387: input i*37 + j*13 + 1, beta = omega_n
    for k in range(0, 9):
        n = 1 << k
        i = np.arange(n)[:, None]
        j = np.arange(L)[None, :]
        base = ((i * 37 + j * 13 + 1) % 256).astype(np.uint8).reshape(-1)
        for beta in (0, int(T.subspace[n & 255]), 0x5A):
            for inv in (False, True):
                ref = base.copy()
                (oracle.ifft_sharded if inv else oracle.fft_sharded)(ref, L, k, beta)
                d = torch.from_numpy(base.copy()).cuda()
                (afrs.ifft_sharded if inv else afrs.fft_sharded)(d, L, k, beta)
                assert (d.cpu().numpy() == ref).all(), (k, beta, inv)
    src = oracle.random_bytes(L, 1)
    for c in (0, 1, 2, 0x53, 0xFF):
        ref = np.zeros(L, np.uint8)
        oracle.lib().orc_scale(src.ctypes.data_as(oracle._u8p), ref.ctypes.data_as(oracle._u8p), L, c)
        d_src = torch.from_numpy(src).cuda()
        d_dst = torch.empty_like(d_src)
        afrs.scale(d_src, d_dst, c)
        assert (d_dst.cpu().numpy() == ref).all()


@pytest.mark.gpu
@pytest.mark.parametrize("t", [1, 2, 8, 32, 128])
def test_recompute_data_from_parity(afrs, t):
    # rs/src/poly_11d_lut.rs:471-494
    n, L = 2 * t, 16
    msg, par = _codeword(n, t, L, seed=t)
    cw = np.concatenate([par, msg])
    rx = cw.copy()
    rx[t * L:] = 0
    d = torch.from_numpy(rx).cuda()
    afrs.Codec(n, t).recompute_data_from_parity_sharded(d, None, L)
    assert (d.cpu().numpy() == cw).all()


def _batch_mix(afrs, count, seed, max_len=4096):
    """A config-3-like mix: n in {32..256}, t in {4, 8, n/4, n/2}, shard
    lengths log-uniform (multiples of 64 B and ragged ones), e in 1..t."""
    rng = np.random.default_rng(seed)
    jobs, expect = [], []
    for i in range(count):
        n = int(rng.choice([2, 4, 16, 32, 64, 128, 256]))
        t = int(rng.choice([c for c in (1, 2, 4, 8, n // 4, n // 2) if 1 <= c < n]))
        L = int(np.exp(rng.uniform(np.log(1), np.log(max_len))))
        msg = oracle.random_bytes((n - t) * L, seed * 10007 + i)
        par = np.zeros(t * L, np.uint8)
        oracle.encode_systematic_sharded(n, t, msg, par, L)
        if i % 2 == 0:
            d_par = torch.full((t * L,), 0xA5, dtype=torch.uint8, device="cuda")
            jobs.append(afrs.Job.encode(n, t, torch.from_numpy(msg).cuda(), d_par, L))
            expect.append(par)
        else:
            cw = np.concatenate([par, msg])
            e = int(rng.integers(1, t + 1))
            pos = rng.choice(n, e, replace=False).tolist()
            rx = cw.copy()
            for p in pos:
                rx[p * L:(p + 1) * L] = 0x5A  # erased rows need not be zero here
            jobs.append(afrs.Job.recover(n, t, torch.from_numpy(rx).cuda(), L, pos))
            expect.append(cw)
    return jobs, expect


@pytest.mark.gpu
def test_batch_matches_oracle_on_mixed_shapes(afrs):
    jobs, expect = _batch_mix(afrs, 120, seed=3)
    status = afrs.run_batch(jobs)
    torch.cuda.synchronize()
    for j, ex, st in zip(jobs, expect, status):
        assert st == (0 if j.op == 0 else 1)
        assert (j.dst.cpu().numpy() == ex).all(), (j.op, j.n, j.t, j.shard_len)


@pytest.mark.gpu
def test_batch_equals_per_call_path_and_reports_status(afrs):
    jobs, expect = _batch_mix(afrs, 40, seed=9, max_len=700)
    bad = afrs.Job.recover(64, 8, torch.zeros(64 * 10, dtype=torch.uint8, device="cuda"), 10, [3, 3])
    too_many = afrs.Job.recover(64, 8, torch.zeros(64 * 10, dtype=torch.uint8, device="cuda"), 10, list(range(9)))
    status = afrs.run_batch(jobs + [bad, too_many])
    torch.cuda.synchronize()
    assert status[-2] == afrs._lib.AFRS_EINVAL and status[-1] == 0
    for j, ex in zip(jobs, expect):
        if j.op == 0:
            ref = torch.zeros_like(j.dst)
            afrs.Codec(j.n, j.t).encode_parity(j.src, ref, j.shard_len)
        else:
            ref = torch.from_numpy(ex.copy()).cuda()
            for p in j.positions:
                ref[p * j.shard_len:(p + 1) * j.shard_len] = 0
            afrs.Codec(j.n, j.t).recover_erasure_shards(ref, None, j.shard_len, j.positions)
        assert torch.equal(ref, j.dst)


@pytest.mark.gpu
@pytest.mark.parametrize("n,t", PAIRS_ALL)
@pytest.mark.parametrize("L", [1, 33, 1029])
def test_syndrome_matches_oracle(afrs, n, t, L):
    """Sharded syndrome (codec.rs:269-301): zero on codewords, equal to the
    oracle's on a word with corrupted bytes in parity and message shards."""
    msg, par = _codeword(n, t, L, seed=n * 17 + t + L)
    cw = np.concatenate([par, msg])
    codec = afrs.Codec(n, t)
    syn, nz = codec.syndrome_sharded(torch.from_numpy(cw).cuda(), L)
    assert not syn.cpu().numpy().any() and int(nz.item()) == 0
    bad = cw.copy()
    rng = np.random.default_rng(n + t + L)
    for i in rng.choice(n * L, min(5, n * L), replace=False):
        bad[i] ^= int(rng.integers(1, 256))
    ref = oracle.syndrome_sharded(n, t, bad, L)
    syn, nz = codec.syndrome_sharded(torch.from_numpy(bad).cuda(), L)
    assert (syn.cpu().numpy() == ref).all()
    assert int(nz.item()) == int(np.count_nonzero(ref))


def _pinned(a):
    return torch.from_numpy(a).pin_memory().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("n,t,L", [(256, 128, 3 * 16384 + 1000), (64, 16, 2 * 65536 + 77), (16, 8, 300000),
                                   (256, 32, 16384), (32, 16, 3 * 131072 + 333), (64, 32, 200000)])
@pytest.mark.parametrize("pinned", [True, False])
def test_staged_host_path_windows_and_runs(afrs, n, t, L, pinned):
    """The host-buffer entry points stage column windows (4 MiB per window:
    16 KiB columns at n = 256) through two device slots and copy only the
    rows an operation reads or writes, as merged runs.  Shards spanning
    several windows with a ragged last one, page-locked and pageable buffers,
    accumulate, and erasure patterns with long runs, isolated rows and gaps.
    The windows take the routed kernels: at n = 32 (128 KiB windows) recovers
    and at n = 64, t = 32 (64 KiB windows) encodes run the one-launch form."""
    msg, par = _codeword(n, t, L, seed=n + L)
    cw = np.concatenate([par, msg])
    codec = afrs.Codec(n, t)
    h_msg = _pinned(msg) if pinned else msg.copy()
    got = _pinned(np.zeros(t * L, np.uint8)) if pinned else np.zeros(t * L, np.uint8)
    codec.encode_systematic_sharded(h_msg, got, None, L)
    assert (got == par).all()
    p0 = oracle.random_bytes(t * L, 9)
    ref = p0.copy()
    oracle.encode_systematic_sharded(n, t, msg, ref, L)
    acc = _pinned(p0) if pinned else p0.copy()
    codec.encode_systematic_sharded(h_msg, acc, None, L)
    assert (acc == ref).all()
    rng = np.random.default_rng(n * 3 + t)
    patterns = [sorted(rng.choice(n, t, replace=False).tolist()), list(range(n - t, n)), list(range(0, n, n // t))[:t],
                [0, n - 1], [n // 2]]
    for pos in patterns:
        rx = _erase(cw, L, pos)
        if pinned:
            rx = _pinned(rx)
        assert codec.recover_erasure_shards(rx, None, L, pos)
        assert (rx == cw).all(), pos


@pytest.mark.gpu
@pytest.mark.parametrize("n,t,L", [(256, 128, 65536), (64, 32, 1024), (16, 8, 5000)])
def test_cuda_graph_capture_and_replay(afrs, n, t, L):
    """Device entry points inside stream capture: one eager call grows the
    scratch, then encode and recover are captured into CUDA graphs and
    replayed; results equal the oracle's."""
    msg, par = _codeword(n, t, L, seed=n + 7 * t)
    cw = np.concatenate([par, msg])
    pos = sorted(np.random.default_rng(n).choice(n, t, replace=False).tolist())
    codec = afrs.Codec(n, t, context=afrs.Context(0))
    d_msg = torch.from_numpy(msg).cuda()
    d_par = torch.zeros(t * L, dtype=torch.uint8, device="cuda")
    d_rx = torch.from_numpy(_erase(cw, L, pos)).cuda()
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        codec.encode_parity(d_msg, d_par, L)
        assert codec.recover_erasure_shards(d_rx.clone(), None, L, pos)
    torch.cuda.synchronize()
    d_par.zero_()
    ge, gr = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
    with torch.cuda.graph(ge, stream=side):
        codec.encode_parity(d_msg, d_par, L)
    with torch.cuda.graph(gr, stream=side):
        codec.recover_erasure_shards(d_rx, None, L, pos)
    torch.cuda.synchronize()
    assert not d_par.any()  # capture does not run the kernels
    for _ in range(3):
        ge.replay()
        gr.replay()
    torch.cuda.synchronize()
    assert (d_par.cpu().numpy() == par).all()
    assert (d_rx.cpu().numpy() == cw).all()


def _staged_bytes(afrs):
    import ctypes

    a, b = ctypes.c_uint64(), ctypes.c_uint64()
    afrs.lib().afrs_staged_bytes(ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


@pytest.mark.gpu
@pytest.mark.parametrize("n,t,L", [(256, 128, 65536), (64, 32, 1000), (16, 4, 4097)])
def test_direct_path_for_page_locked_buffers(afrs, n, t, L):
    """Page-locked host buffers are read and written by the kernels directly:
    recover moves exactly the surviving shards in and the erased shards out,
    encode the message in and the parity out; results equal the oracle's."""
    msg, par = _codeword(n, t, L, seed=3 * n + t)
    cw = np.concatenate([par, msg])
    codec = afrs.Codec(n, t)
    h_msg, h_par = _pinned(msg), _pinned(np.zeros(t * L, np.uint8))
    b0 = _staged_bytes(afrs)
    codec.encode_parity(h_msg, h_par, L)
    b1 = _staged_bytes(afrs)
    assert (h_par == par).all()
    assert (b1[0] - b0[0], b1[1] - b0[1]) == ((n - t) * L, t * L)
    pos = sorted(np.random.default_rng(L).choice(n, t, replace=False).tolist())
    h_rx = _pinned(_erase(cw, L, pos))
    assert codec.recover_erasure_shards(h_rx, None, L, pos)
    b2 = _staged_bytes(afrs)
    assert (h_rx == cw).all()
    assert (b2[0] - b1[0], b2[1] - b1[1]) == ((n - len(pos)) * L, len(pos) * L)


@pytest.mark.gpu
def test_direct_path_from_a_fresh_host_thread(afrs):
    """The first call of a host thread that has made no CUDA call yet still
    takes the direct path: exactly the surviving shards in, the erased out."""
    import threading

    n, t, L = 256, 128, 65536
    msg, par = _codeword(n, t, L, seed=5)
    cw = np.concatenate([par, msg])
    pos = sorted(np.random.default_rng(9).choice(n, t, replace=False).tolist())
    h_rx = _pinned(_erase(cw, L, pos))
    codec = afrs.Codec(n, t)
    out = {}

    def run():
        b0 = _staged_bytes(afrs)
        out["ok"] = codec.recover_erasure_shards(h_rx, None, L, pos)
        out["moved"] = tuple(b - a for a, b in zip(b0, _staged_bytes(afrs)))

    th = threading.Thread(target=run)
    th.start()
    th.join()
    assert out["ok"] and (h_rx == cw).all()
    assert out["moved"] == ((n - t) * L, t * L)


@pytest.mark.gpu
def test_host_api_from_concurrent_threads(afrs):
    """Pairs of host threads (one encoding, one recovering, own contexts and
    buffers) running back to back at once give the oracle's results."""
    import threading

    n, t, L, P, steps = 64, 16, 4096, 3, 6
    msg, par = _codeword(n, t, L, seed=41)
    cw = np.concatenate([par, msg])
    pos = sorted(np.random.default_rng(4).choice(n, t, replace=False).tolist())
    h_msg = _pinned(msg)
    pars = [_pinned(np.zeros(t * L, np.uint8)) for _ in range(P)]
    rxs = [_pinned(_erase(cw, L, pos)) for _ in range(P)]
    encs = [afrs.Codec(n, t, context=afrs.Context(0)) for _ in range(P)]
    recs = [afrs.Codec(n, t, context=afrs.Context(0)) for _ in range(P)]
    errors = []

    def work(i, enc):
        try:
            for _ in range(steps):
                if enc:
                    encs[i].encode_parity(h_msg, pars[i], L)
                else:
                    assert recs[i].recover_erasure_shards(rxs[i], None, L, pos)
        except Exception as ex:  # surfaced below
            errors.append(ex)

    ths = [threading.Thread(target=work, args=(i, e)) for i in range(P) for e in (True, False)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    assert not errors
    for i in range(P):
        assert (pars[i] == par).all() and (rxs[i] == cw).all()


@pytest.mark.gpu
def test_host_registered_buffers(afrs):
    """Memory page-locked with cudaHostRegister (whose device alias may differ
    from its host address) and a sub-range of a page-locked buffer."""
    n, t, L = 128, 32, 3000
    msg, par = _codeword(n, t, L, seed=77)
    cw = np.concatenate([par, msg])
    pos = list(range(10, 10 + t))
    size = (n * L + 8192 + 4095) // 4096 * 4096
    raw = np.zeros(size + 4096, np.uint8)
    off = (-raw.ctypes.data) % 4096
    big = raw[off:off + size]  # page-aligned start and size
    view = big[4096:4096 + n * L]
    view[:] = _erase(cw, L, pos)
    rt = torch.cuda.cudart()
    assert int(rt.cudaHostRegister(big.ctypes.data, big.nbytes, 0)) == 0
    try:
        assert afrs.Codec(n, t).recover_erasure_shards(view, None, L, pos)
        assert (view == cw).all()
    finally:
        rt.cudaHostUnregister(big.ctypes.data)
    sub = _pinned(np.zeros(n * L + 100, np.uint8))[37:37 + n * L]
    sub[:] = _erase(cw, L, pos)
    assert afrs.Codec(n, t).recover_erasure_shards(sub, None, L, pos)
    assert (sub == cw).all()


@pytest.mark.gpu
def test_batch_large_shape_groups_match_oracle(afrs):
    """Shape groups of at least 8 MiB run on the grouped specialised kernels
    (codeword per blockIdx.z): phase shapes, t <= 16 encodes, n <= 16
    recovers, ragged shard lengths, one recover group holding several t;
    small groups alongside take the generic kernel.  Byte-exact results."""
    rng = np.random.default_rng(2024)
    specs = [(0, 256, 128, 3000, 12), (1, 256, 128, 3000, 12), (1, 256, 32, 2100, 16), (0, 64, 8, 4096, 33),
             (0, 128, 16, 2048, 33), (0, 64, 32, 4099, 33), (1, 16, 4, 16384, 33), (1, 128, 64, 2048, 33),
             (0, 32, 8, 100, 5), (1, 64, 16, 77, 5)]
    jobs, expect = [], []
    for q, (op, n, t, L, count) in enumerate(specs):
        for i in range(count):
            msg = oracle.random_bytes((n - t) * L, 7000 + 97 * q + i)
            par = np.zeros(t * L, np.uint8)
            oracle.encode_systematic_sharded(n, t, msg, par, L)
            if op == 0:
                d_par = torch.full((t * L,), 0x3C, dtype=torch.uint8, device="cuda")
                jobs.append(afrs.Job.encode(n, t, torch.from_numpy(msg).cuda(), d_par, L))
                expect.append(par)
            else:
                cw = np.concatenate([par, msg])
                pos = rng.choice(n, int(rng.integers(1, t + 1)), replace=False).tolist()
                rx = cw.copy()
                for p in pos:
                    rx[p * L:(p + 1) * L] = 0xC3
                jobs.append(afrs.Job.recover(n, t, torch.from_numpy(rx).cuda(), L, pos))
                expect.append(cw)
    launches0 = afrs.lib().afrs_kernel_launches()
    status = afrs.run_batch(jobs)
    torch.cuda.synchronize()
    assert afrs.lib().afrs_kernel_launches() - launches0 > 2  # grouped launches, not only the generic kernel
    for j, ex, st in zip(jobs, expect, status):
        assert st == (0 if j.op == 0 else 1)
        assert (j.dst.cpu().numpy() == ex).all(), (j.op, j.n, j.t, j.shard_len)
