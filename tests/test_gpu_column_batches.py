"""GPU parity of the column-batched phase path: when a call needs more
scratch than its context allows (afrs_ctx_set_work_cap; by default above
1 GiB, e.g. n = 256 with 4 MiB shards), the phase kernels run over column
batches [cw0, cw0 + ncw) of the shard, with a ragged last batch.  Every
result is compared with the CPU oracle (rs/src/codec.rs:241-265 encode,
:479-569 recover)."""
import numpy as np
import pytest

from oracle import oracle

torch = pytest.importorskip("torch")

# Scratch per colword (32 byte columns): recover 2 * n * 32 bytes, encode
# (n - t) * 32 bytes (the phase kernels' bit-sliced rows).
REC_CW = lambda n: 2 * n * 32  # noqa: E731
ENC_CW = lambda n, t: (n - t) * 32  # noqa: E731


def _colwords(L):
    return (L + 1023) // 1024 * 32


def _ctx_with_cap(afrs, cap):
    ctx = afrs.Context(0)
    ctx.set_work_cap(cap)
    return ctx


def _codeword(n, t, L, seed):
    msg = oracle.random_bytes((n - t) * L, seed)
    par = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, par, L)
    return msg, par


def test_work_cap_argument_checks(afrs):
    E = afrs._lib.AFRS_EINVAL
    assert afrs.lib().afrs_ctx_set_work_cap(None, 0) == E


@pytest.mark.gpu
def test_work_cap_limits(afrs):
    ctx = afrs.Context(0)
    with pytest.raises(afrs.AfrsError):
        ctx.set_work_cap(1000)  # below one colword of an n = 256 recover
    with pytest.raises(afrs.AfrsError):
        ctx.set_work_cap((1 << 30) + 256)
    ctx.set_work_cap(0)
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("batch_cw", [600, 611])  # 611: batches not a multiple of 8 colwords
def test_recover_in_column_batches(afrs, batch_cw):
    n, t, L = 256, 128, 65536 + 77
    assert _colwords(L) > 3 * batch_cw  # >= 4 batches, the last one ragged
    msg, par = _codeword(n, t, L, seed=batch_cw)
    cw = np.concatenate([par, msg])
    rng = np.random.default_rng(batch_cw)
    pos = sorted(rng.choice(n, t, replace=False).tolist())
    rx = cw.copy()
    for p in pos:
        rx[p * L:(p + 1) * L] = 0
    ref = rx.copy()
    assert oracle.recover_erasure_shards(n, t, ref, L, pos)
    ctx = _ctx_with_cap(afrs, batch_cw * REC_CW(n))
    d = torch.from_numpy(rx).cuda()
    assert afrs.Codec(n, t, context=ctx).recover_erasure_shards(d, None, L, pos)
    got = d.cpu().numpy()
    assert (got == ref).all() and (got == cw).all()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("t,batch_cw", [(32, 700), (128, 333)])
@pytest.mark.parametrize("accumulate", [False, True])
def test_encode_in_column_batches(afrs, t, batch_cw, accumulate):
    n, L = 256, 65536 + 77
    assert _colwords(L) > 2 * batch_cw
    msg = oracle.random_bytes((n - t) * L, t + batch_cw)
    p0 = oracle.random_bytes(t * L, 5) if accumulate else np.zeros(t * L, np.uint8)
    ref = p0.copy()
    oracle.encode_systematic_sharded(n, t, msg, ref, L)
    ctx = _ctx_with_cap(afrs, batch_cw * ENC_CW(n, t))
    d = torch.from_numpy(p0.copy()).cuda()
    afrs.Codec(n, t, context=ctx).encode_systematic_sharded(torch.from_numpy(msg).cuda(), d, None, L)
    assert (d.cpu().numpy() == ref).all()
    ctx.close()


@pytest.mark.gpu
def test_large_shard_patterns_in_column_batches(afrs):
    """The large-shard stress shape (n = 256, k = 224, t = 32) with 1 MiB + 37
    byte shards, in 3+ column batches: encode against the oracle, then both
    adversarial erasure patterns, 32 erasures inside the message shards and
    one contiguous run of 32 shard indices."""
    n, t, L = 256, 32, (1 << 20) + 37
    cap = 11000 * REC_CW(n)  # 32800 colwords -> 3 batches of 11000 and a ragged 9800
    msg, par = _codeword(n, t, L, seed=55)
    ctx = _ctx_with_cap(afrs, cap)
    codec = afrs.Codec(n, t, context=ctx)
    d_par = torch.zeros(t * L, dtype=torch.uint8, device="cuda")
    codec.encode_parity(torch.from_numpy(msg).cuda(), d_par, L)
    assert (d_par.cpu().numpy() == par).all()
    cw = np.concatenate([par, msg])
    rng = np.random.default_rng(9)
    inside = sorted(rng.choice(np.arange(t, n), 32, replace=False).tolist())
    run = list(range(100, 132))
    for k, pos in enumerate((inside, run)):
        rx = cw.copy()
        for p in pos:
            rx[p * L:(p + 1) * L] = 0
        d = torch.from_numpy(rx).cuda()
        assert codec.recover_erasure_shards(d, None, L, pos)
        got = d.cpu().numpy()
        if k == 0:
            ref = rx.copy()
            assert oracle.recover_erasure_shards(n, t, ref, L, pos)
            assert (got == ref).all()
        assert (got == cw).all()  # round trip: every erased shard is back
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [64, 256])
@pytest.mark.parametrize("accumulate", [False, True])
def test_t16_encode_one_warp_per_slice(afrs, n, accumulate):
    """t = 16 with more than 128 slices of 1024 columns per launch takes the
    layout with one warp per slice and shared-memory accumulators (not the
    split layout that shorter shards take)."""
    t, L = 16, 132133  # 130 slices
    msg = oracle.random_bytes((n - t) * L, n + 16)
    p0 = oracle.random_bytes(t * L, 6) if accumulate else np.zeros(t * L, np.uint8)
    ref = p0.copy()
    oracle.encode_systematic_sharded(n, t, msg, ref, L)
    d = torch.from_numpy(p0.copy()).cuda()
    afrs.Codec(n, t).encode_systematic_sharded(torch.from_numpy(msg).cuda(), d, None, L)
    assert (d.cpu().numpy() == ref).all()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [64, 256])
def test_t16_encode_group_of_a_batch(afrs, n):
    """The same layout through afrs_batch_dev: a shape group above the 8 MiB
    grouping threshold runs the grouped one-warp-per-slice kernel."""
    t, L = 16, 132133
    jobs, refs = [], []
    for i in range(2):
        msg = oracle.random_bytes((n - t) * L, 300 + i)
        ref = np.zeros(t * L, np.uint8)
        oracle.encode_systematic_sharded(n, t, msg, ref, L)
        jobs.append(afrs.Job.encode(n, t, torch.from_numpy(msg).cuda(),
                                    torch.full((t * L,), 0xA5, dtype=torch.uint8, device="cuda"), L))
        refs.append(ref)
    assert afrs.run_batch(jobs) == [0, 0]
    for j, ref in zip(jobs, refs):
        assert (j.dst.cpu().numpy() == ref).all()


@pytest.mark.gpu
def test_t16_encode_group_of_many_short_codewords(afrs):
    """A t = 16 group of many short, ragged codewords (more than 128 slices
    in the group, at most 5 per codeword) also takes the one-warp-per-slice
    grouped kernel; each codeword's parity equals the oracle's."""
    n, t = 64, 16
    rng = np.random.default_rng(16)
    jobs, refs = [], []
    for i in range(60):
        L = int(rng.choice([1000, 3001, 4096, 5000]))
        msg = oracle.random_bytes((n - t) * L, 900 + i)
        ref = np.zeros(t * L, np.uint8)
        oracle.encode_systematic_sharded(n, t, msg, ref, L)
        jobs.append(afrs.Job.encode(n, t, torch.from_numpy(msg).cuda(),
                                    torch.full((t * L,), 0x5A, dtype=torch.uint8, device="cuda"), L))
        refs.append(ref)
    assert sum(j.nbytes for j in jobs) >= 8 << 20
    assert afrs.run_batch(jobs) == [0] * len(jobs)
    for j, ref in zip(jobs, refs):
        assert (j.dst.cpu().numpy() == ref).all()
