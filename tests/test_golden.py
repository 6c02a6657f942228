"""Committed golden vectors (tests/golden/vectors.json, made by
tests/golden/make_golden.py): the oracle must reproduce every fixture (CPU),
and the CUDA path through the C ABI must reproduce them byte for byte (GPU)."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "vectors.json")) as _f:
    GOLDEN = json.load(_f)["cases"]
BYTES = [c for c in GOLDEN if c["kind"] == "encode_recover_bytes"]
DIGESTS = [c for c in GOLDEN if c["kind"] == "digests"]


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _erase(cw, L, pos):
    rx = cw.copy()
    for p in pos:
        rx[p * L:(p + 1) * L] = 0
    return rx


def _inputs(c):
    n, t, L = c["n"], c["t"], c["shard_len"]
    msg = oracle.random_bytes((n - t) * L, c["seed"])
    return n, t, L, msg


# ---- CPU: the oracle reproduces the fixtures --------------------------------

@pytest.mark.parametrize("c", BYTES, ids=lambda c: f"{c['n']}-{c['t']}-{c['shard_len']}")
def test_oracle_reproduces_golden_bytes(c):
    n, t, L, msg = _inputs(c)
    assert msg.tobytes().hex() == c["message"]
    par = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, par, L)
    assert par.tobytes().hex() == c["parity"]
    cw = np.concatenate([par, msg])
    rx = _erase(cw, L, c["positions"])
    assert oracle.recover_erasure_shards(n, t, rx, L, c["positions"])
    assert (rx == cw).all()


@pytest.mark.parametrize("c", DIGESTS, ids=lambda c: f"{c['n']}-{c['t']}")
def test_oracle_reproduces_golden_digests(c):
    n, t, L, msg = _inputs(c)
    par = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, par, L)
    assert sha(par) == c["parity_sha256"]
    acc = oracle.random_bytes(t * L, c["acc_seed"])
    oracle.encode_systematic_sharded(n, t, msg, acc, L)
    assert sha(acc) == c["acc_parity_sha256"]
    junk = _erase(oracle.random_bytes(n * L, c["junk_seed"]), L, c["junk_positions"])
    assert oracle.recover_erasure_shards(n, t, junk, L, c["junk_positions"])
    assert sha(junk) == c["junk_recovered_sha256"]
    bad = np.concatenate([par, msg])
    bad[c["flip"][0]] ^= c["flip"][1]
    assert sha(oracle.syndrome_sharded(n, t, bad, L)) == c["syndrome_sha256"]


# ---- GPU: the CUDA path reproduces the fixtures ------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("c", BYTES, ids=lambda c: f"{c['n']}-{c['t']}-{c['shard_len']}")
def test_gpu_golden_bytes(afrs, c):
    import torch

    n, t, L = c["n"], c["t"], c["shard_len"]
    msg = np.frombuffer(bytes.fromhex(c["message"]), np.uint8)
    ref = np.frombuffer(bytes.fromhex(c["parity"]), np.uint8)
    codec = afrs.Codec(n, t)
    d_par = torch.zeros(t * L, dtype=torch.uint8, device="cuda")
    codec.encode_parity(torch.from_numpy(msg.copy()).cuda(), d_par, L)
    assert d_par.cpu().numpy().tobytes() == ref.tobytes()
    cw = np.concatenate([ref, msg])
    d_rx = torch.from_numpy(_erase(cw, L, c["positions"])).cuda()
    assert codec.recover_erasure_shards(d_rx, None, L, c["positions"])
    assert (d_rx.cpu().numpy() == cw).all()


@pytest.mark.gpu
@pytest.mark.parametrize("c", DIGESTS, ids=lambda c: f"{c['n']}-{c['t']}")
def test_gpu_golden_digests(afrs, c):
    import torch

    n, t, L, msg = _inputs(c)
    codec = afrs.Codec(n, t)
    d_msg = torch.from_numpy(msg).cuda()
    d_par = torch.zeros(t * L, dtype=torch.uint8, device="cuda")
    codec.encode_parity(d_msg, d_par, L)
    par = d_par.cpu().numpy()
    assert sha(par) == c["parity_sha256"]
    d_acc = torch.from_numpy(oracle.random_bytes(t * L, c["acc_seed"])).cuda()
    codec.encode_systematic_sharded(d_msg, d_acc, None, L)  # XOR-accumulating form
    assert sha(d_acc.cpu().numpy()) == c["acc_parity_sha256"]
    cw = np.concatenate([par, msg])
    d_rx = torch.from_numpy(_erase(cw, L, c["positions"])).cuda()
    assert codec.recover_erasure_shards(d_rx, None, L, c["positions"])
    assert (d_rx.cpu().numpy() == cw).all()
    d_junk = torch.from_numpy(_erase(oracle.random_bytes(n * L, c["junk_seed"]), L, c["junk_positions"])).cuda()
    assert codec.recover_erasure_shards(d_junk, None, L, c["junk_positions"])
    assert sha(d_junk.cpu().numpy()) == c["junk_recovered_sha256"]
    bad = torch.from_numpy(cw.copy()).cuda()
    bad[c["flip"][0]] ^= c["flip"][1]
    syn, nz = codec.syndrome_sharded(bad, L)
    assert sha(syn.cpu().numpy()) == c["syndrome_sha256"]
    assert int(nz.item()) == int(np.count_nonzero(syn.cpu().numpy())) > 0
    assert codec.is_codeword(torch.from_numpy(cw).cuda(), L)
    if "recompute_sha256" in c:
        d_rc = torch.from_numpy(cw.copy()).cuda()
        d_rc[t * L:] = 0
        codec.recompute_data_from_parity_sharded(d_rc, None, L)
        assert sha(d_rc.cpu().numpy()) == c["recompute_sha256"]
