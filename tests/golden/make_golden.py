"""Generates tests/golden/vectors.json: golden input/output vectors of the
sharded encoder, erasure decoder, recompute and syndrome of the reference
(rs/src/codec.rs), computed by the CPU oracle (oracle/afrs_oracle.c, itself
pinned by the reference's own tests in tests/test_oracle.py) and, for the
cases small enough, confirmed column by column by the independent pure-Python
restatement (oracle/pyref.py).

The reference ships no golden codeword bytes, so these fixtures freeze the
oracle's outputs: a later change to the oracle or to the GPU path that moves
a single byte fails tests/test_golden.py.

Inputs are splitmix64 streams (oracle.random_bytes(nbytes, seed)); small
cases store the bytes as hex, larger ones store SHA-256 digests.

    python tests/golden/make_golden.py      # rewrites vectors.json
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle, pyref  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "vectors.json")
PAIRS = [(n, t) for n in (2, 4, 8, 16, 32, 64, 128, 256) for t in (1, 2, 4, 8, 16, 32, 64, 128) if t < n]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(a.tobytes()).hexdigest()


def positions(n: int, e: int, seed: int) -> list[int]:
    return sorted(np.random.default_rng(seed).choice(n, e, replace=False).tolist())


def codeword(n: int, t: int, L: int, seed: int):
    msg = oracle.random_bytes((n - t) * L, seed)
    par = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, par, L)
    return msg, par


def check_columns_with_pyref(n, t, L, msg, par, pos, rec):
    """Every column of a small case through the pure-Python restatement."""
    for c in range(L):
        m = [int(msg[r * L + c]) for r in range(n - t)]
        p = pyref.encode_column(n, t, m)
        assert p == [int(par[r * L + c]) for r in range(t)], (n, t, L, c)
        if pos is not None:
            col = p + m
            rx = [0 if r in pos else col[r] for r in range(n)]
            assert pyref.recover_column(n, t, rx, pos) == [int(rec[r * L + c]) for r in range(n)]


def main() -> None:
    cases = []
    # Full bytes: the reference README shape (n=64, k=32, 64-byte shards) and n=256, k=128.
    for n, t, L, seed in [(64, 32, 64, 1), (256, 128, 16, 2), (16, 4, 33, 3)]:
        msg, par = codeword(n, t, L, seed)
        pos = positions(n, t, seed + 100)
        rx = np.concatenate([par, msg])
        for p in pos:
            rx[p * L:(p + 1) * L] = 0
        rec = rx.copy()
        assert oracle.recover_erasure_shards(n, t, rec, L, pos)
        assert (rec == np.concatenate([par, msg])).all()
        check_columns_with_pyref(n, t, L, msg, par, pos, rec)
        cases.append({"kind": "encode_recover_bytes", "n": n, "t": t, "shard_len": L, "seed": seed,
                      "message": msg.tobytes().hex(), "parity": par.tobytes().hex(), "positions": pos})

    # Digests over every (n, t) the reference tests cover, odd shard length.
    for n, t in PAIRS:
        L = 37
        seed = 1000 + n * 8 + t
        msg, par = codeword(n, t, L, seed)
        pos = positions(n, t, seed + 1)
        cw = np.concatenate([par, msg])
        rx = cw.copy()
        for p in pos:
            rx[p * L:(p + 1) * L] = 0
        assert oracle.recover_erasure_shards(n, t, rx, L, pos) and (rx == cw).all()
        # Accumulate semantics: parity buffer pre-filled with bytes of its own.
        acc = oracle.random_bytes(t * L, seed + 2)
        acc_out = acc.copy()
        oracle.encode_systematic_sharded(n, t, msg, acc_out, L)
        # Decoder on a word that is not a codeword (erased rows zero): the
        # reference's linear map, pinned on arbitrary survivors.
        junk = oracle.random_bytes(n * L, seed + 3)
        jpos = positions(n, max(1, t // 2), seed + 4)
        for p in jpos:
            junk[p * L:(p + 1) * L] = 0
        jout = junk.copy()
        assert oracle.recover_erasure_shards(n, t, jout, L, jpos)
        # Syndrome of the codeword with one byte flipped.
        bad = cw.copy()
        bad[(seed % n) * L + 5] ^= 0x5A
        syn = oracle.syndrome_sharded(n, t, bad, L)
        assert not oracle.syndrome_sharded(n, t, cw, L).any() and syn.any()
        case = {"kind": "digests", "n": n, "t": t, "shard_len": L, "seed": seed, "positions": pos,
                "parity_sha256": sha(par), "acc_seed": seed + 2, "acc_parity_sha256": sha(acc_out),
                "junk_seed": seed + 3, "junk_positions": jpos, "junk_recovered_sha256": sha(jout),
                "flip": [(seed % n) * L + 5, 0x5A], "syndrome_sha256": sha(syn)}
        if n == 2 * t:
            rc = cw.copy()
            rc[t * L:] = 0
            oracle.recompute_data_from_parity_sharded(n, t, rc, L)
            assert (rc == cw).all()
            case["recompute_sha256"] = sha(rc)
        cases.append(case)

    with open(OUT, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "rng": "splitmix64 (oracle.random_bytes)",
                   "cases": cases}, f, indent=1)
        f.write("\n")
    print(f"wrote {len(cases)} cases to {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
