"""The allocation-free recover entry point (afrs_recover_dev_noalloc).

It serves callers that may not allocate device memory when they recover
shards (inside stream capture, in serving loops that must not stall on an
allocation, under a fixed memory budget).  Its output must equal the regular
entry point's, byte for byte, on consecutive calls that share its fixed
scratch array.  This file is collected last on purpose.
"""
import ctypes

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


def _noalloc(afrs, n, t, d_rx, L, pos):
    lib = afrs.lib()
    p = np.ascontiguousarray(np.asarray(pos, dtype=np.uint8))
    stream = torch.cuda.current_stream().cuda_stream
    return lib.afrs_recover_dev_noalloc(n, t, d_rx.data_ptr(), L, p.ctypes.data, p.size, stream)


@pytest.mark.gpu
@pytest.mark.parametrize("n,t,L", [(256, 128, 65536), (256, 32, 5000), (64, 32, 1024), (16, 8, 333), (128, 8, 3000)])
def test_noalloc_matches_regular_entry_point_twice(afrs, n, t, L):
    rng = np.random.default_rng(n + t + L)
    codec = afrs.Codec(n, t)
    for call in range(2):  # two calls in a row share the scratch array
        cw = _codeword(n, t, L, seed=call * 1000 + n)
        pos = sorted(rng.choice(n, t if call == 0 else max(1, t // 2), replace=False).tolist())
        rx = _erase(cw, L, pos)
        d_ref = torch.from_numpy(rx.copy()).cuda()
        assert codec.recover_erasure_shards(d_ref, None, L, pos)
        d_new = torch.from_numpy(rx.copy()).cuda()
        assert _noalloc(afrs, n, t, d_new, L, pos) == 1, afrs.lib().afrs_last_error()
        torch.cuda.synchronize()
        out_new = d_new.cpu().numpy()
        assert (out_new == d_ref.cpu().numpy()).all()  # exact: integer arithmetic
        assert (out_new == cw).all()


@pytest.mark.gpu
def test_noalloc_refuses_shards_beyond_its_scratch(afrs):
    n, t, L = 256, 128, 68 * 1024  # needs 34 MiB of scratch
    d = torch.zeros(n * L, dtype=torch.uint8, device="cuda")
    r = _noalloc(afrs, n, t, d, L, [0, 1])
    assert r == afrs._lib.AFRS_EINVAL
    assert b"scratch" in afrs.lib().afrs_last_error()
    assert _noalloc(afrs, n, t, d, L, list(range(t + 1))) == 0  # e > t: false, as the reference
