"""Pins the CPU oracle to the reference crate's own tests.

Each test restates a reference test (file:line given) against the C oracle,
and the two CPU restatements (C and pure Python) are checked against each
other.  The reference commits no golden codeword bytes, so these known-answer
and property tests are what pins the oracle.
"""
import itertools

import numpy as np
import pytest

from oracle import oracle, pyref

T = oracle.tables()
PAIRS_2T = [(2 * t, t) for t in (2, 4, 8, 16, 32, 64, 128)]
PAIRS_ALL = [(n, t) for n in (2, 4, 8, 16, 32, 64, 128, 256) for t in (1, 2, 4, 8, 16, 32, 64, 128) if t < n]


def test_subspace_poly_trace_golden():
    # rs/src/poly_11d_lut.rs:419-429
    assert [int(T.subspace[1 << i]) for i in range(8)] == [1, 214, 152, 146, 86, 200, 88, 231]


def test_wrap_mul_basic_mul_add():
    # gf2p8/src/poly_11d.rs:62-82
    assert oracle.mul(2, 0x80) == 0x1D
    assert oracle.mul(0x57, 0) == 0 and oracle.mul(0x57, 1) == 0x57
    assert (0x57 ^ 0x83) == 0x57 ^ 0x83 and (0x57 ^ 0x57) == 0
    assert not oracle.lib().orc_trace(1)  # poly_11d.rs:57-60


def test_mul_inv_and_tables():
    # gf2p8/src/poly_11d.rs:84-97; field.rs:68-102
    for a in range(1, 256):
        assert oracle.mul(a, int(T.inv[a])) == 1
    assert T.inv[0] == 0
    for i in range(255):
        assert T.log[T.exp[i]] == i and T.exp[i + 255] == T.exp[i]


def test_mul_lut_matches_mul():
    # rs/src/poly_11d_lut.rs:58-66, exhaustively
    lib = oracle.lib()
    for a in range(256):
        for b in range(0, 256, 7):
            assert lib.orc_mul_lut(a, b) == lib.orc_mul_slow(a, b)


def test_gfni_mul_matrix_correctness():
    # rs/src/poly_11d_lut.rs:68-81 (all 256 x 256 pairs)
    lib = oracle.lib()
    for a in range(256):
        m = int(T.gfni_mul[a])
        assert m == lib.orc_mul_matrix(a)
        for b in range(256):
            assert lib.orc_bitmatrix_apply(m, b) == lib.orc_mul_slow(a, b)


def test_bit_matrix_identity_and_linearity():
    # gf2p8/src/bit_matrix.rs:91-121
    lib = oracle.lib()
    ident = int.from_bytes(bytes([1, 2, 4, 8, 16, 32, 64, 128]), "big")  # BitMatrix rows, be bytes
    assert ident == lib.orc_mul_matrix(1)
    for v in range(256):
        assert lib.orc_bitmatrix_apply(ident, v) == v
    m = lib.orc_mul_matrix(0x42)
    assert lib.orc_bitmatrix_apply(m, 0x57 ^ 0x83) == lib.orc_bitmatrix_apply(m, 0x57) ^ lib.orc_bitmatrix_apply(m, 0x83)


def test_cantor_basis_properties():
    # gf2p8/src/poly_11d.rs:99-157
    b = [int(x) for x in T.cantor_basis]
    for i in range(1, 8):
        assert oracle.mul(b[i], b[i]) ^ b[i] == b[i - 1]
    for i in range(7):
        assert not oracle.lib().orc_trace(b[i])
    assert len({T.subspace[i] for i in range(256)}) == 256  # linear independence
    assert b == pyref.BASIS


def test_subspace_points_and_luts():
    # gf2p8/src/poly_11d.rs:159-202
    for i in range(8):
        assert T.subspace[1 << i] == T.cantor_basis[i]
    for j in range(9):
        for x in range(256):
            assert T.spv[j][x] == pyref.SPV[j][x]


def test_normalization_factors_id():
    # rs/src/poly_11d_lut.rs:123-129
    out = np.zeros(256, np.uint8)
    oracle.lib().orc_normalization_factors(out.ctypes.data_as(oracle._u8p))
    assert (out == 1).all()


def test_deriv_subspace_poly_luts():
    # gf2p8/src/poly_11d.rs:204-213
    out = np.zeros(9, np.uint8)
    oracle.lib().orc_deriv_subspace_polys(out.ctypes.data_as(oracle._u8p))
    assert (out == 1).all()


def test_field_non_degeneracy():
    # rs/src/poly_11d_lut.rs:406-417
    for k in range(1, 8):
        assert T.spv[k - 1][T.subspace[1 << k]] != T.spv[k - 1][T.subspace[1 << (k - 1)]]


def test_scalar_fft_ifft_id():
    # rs/src/poly_11d_lut.rs:131-155
    d = np.zeros(256, np.uint8)
    d[:128] = np.arange(128)
    orig = d.copy()
    oracle.fft_scalar(d, 8, 0)
    assert (d != orig).any()
    oracle.ifft_scalar(d, 8, 0)
    assert (d == orig).all()


def _ref_message(n, t, L):
    # rs/src/poly_11d_lut.rs:109-113: message[i][j] = T + i + j (mod 256)
    k = n - t
    i = np.arange(k)[:, None]
    j = np.arange(L)[None, :]
    return ((t + i + j) % 256).astype(np.uint8).reshape(-1)


def _sharded_codeword(n, t, L, message=None):
    # rs/src/poly_11d_lut.rs:100-121
    msg = _ref_message(n, t, L) if message is None else message
    parity = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, parity, L)
    return np.concatenate([parity, msg])


@pytest.mark.parametrize("n,t", PAIRS_2T)
def test_encode_sharded_generalizes_scalar(n, t):
    # rs/src/poly_11d_lut.rs:453-469
    k = n - t
    msg = ((t + np.arange(k)) % 256).astype(np.uint8)
    scalar = np.concatenate([oracle.encode_systematic_scalar(n, t, msg), msg])
    assert (scalar == _sharded_codeword(n, t, 1)).all()


@pytest.mark.parametrize("n,t", PAIRS_2T)
def test_encode_sharded_writes_parity(n, t):
    # rs/src/poly_11d_lut.rs:431-451
    cw = _sharded_codeword(n, t, 32)
    assert (cw[: t * 32] != 0).any()


@pytest.mark.parametrize("n,t", PAIRS_2T)
def test_recompute_max_corrupt_data_sharded(n, t):
    # rs/src/poly_11d_lut.rs:471-494
    orig = _sharded_codeword(n, t, 16)
    rec = orig.copy()
    rec[t * 16:] = 0
    oracle.recompute_data_from_parity_sharded(n, t, rec, 16)
    assert (rec == orig).all()


@pytest.mark.parametrize("n,t", PAIRS_ALL)
def test_recover_erasure_shards_odd_pattern(n, t):
    # rs/src/poly_11d_lut.rs:496-566 (L = 1, erase positions 1, 3, ..., 2T-1)
    orig = _sharded_codeword(n, t, 1)
    rec = orig.copy()
    pos = list(range(1, 2 * t, 2))
    rec[pos] = 0
    assert oracle.recover_erasure_shards(n, t, rec, 1, pos)
    assert (rec == orig).all()


def test_recover_more_than_t_returns_false_and_e0_true():
    # rs/src/codec.rs:491-496
    n, t, L = 16, 4, 8
    cw = _sharded_codeword(n, t, L)
    rec = cw.copy()
    assert not oracle.recover_erasure_shards(n, t, rec, L, [0, 1, 2, 3, 4])
    assert (rec == cw).all()
    assert oracle.recover_erasure_shards(n, t, rec, L, [])
    assert (rec == cw).all()


def _make_shards(n, L):
    # rs/src/kernel/gfni_kernel.rs:314-322: i*37 + j*13 + 1
    i = np.arange(n)[:, None]
    j = np.arange(L)[None, :]
    return ((i * 37 + j * 13 + 1) % 256).astype(np.uint8).reshape(-1)


@pytest.mark.parametrize("L", [1, 63, 64, 65, 128])
def test_gfni_matches_lut(L):
    # rs/src/kernel/gfni_kernel.rs:324-387
    for k in range(1, 5):
        n = 1 << k
        beta = int(T.subspace[n])
        for fwd in (True, False):
            a = _make_shards(n, L)
            b = a.copy()
            if fwd:
                oracle.fft_sharded(a, L, k, beta)
                oracle.gfni_fft_sharded(b, L, k, beta)
            else:
                oracle.ifft_sharded(a, L, k, beta)
                oracle.gfni_ifft_sharded(b, L, k, beta)
            assert (a == b).all()
        d = _make_shards(n, L)
        orig = d.copy()
        oracle.gfni_ifft_sharded(d, L, k, beta)
        oracle.gfni_fft_sharded(d, L, k, beta)
        assert (d == orig).all()


def test_two_restatements_agree():
    rng = np.random.default_rng(5)
    for n, t in [(4, 2), (8, 2), (16, 4), (32, 8), (64, 32), (256, 128), (256, 32)]:
        msg = rng.integers(0, 256, n - t, dtype=np.uint8)
        par_c = oracle.encode_systematic_scalar(n, t, msg)
        par_py = pyref.encode_column(n, t, [int(x) for x in msg])
        assert list(par_c) == par_py
        cw = np.concatenate([par_c, msg])
        e = int(rng.integers(1, t + 1))
        pos = sorted(rng.choice(n, e, replace=False).tolist())
        rx = cw.copy()
        rx[pos] = 0
        got_py = pyref.recover_column(n, t, [int(x) for x in rx], pos)
        oracle.recover_erasure_shards(n, t, rx, 1, pos)
        assert list(rx) == got_py == list(cw)


@pytest.mark.parametrize("n,t", [(8, 4), (32, 8), (64, 32), (128, 32), (256, 128), (256, 64), (256, 32)])
def test_random_patterns_round_trip_and_gfni_equal(n, t):
    rng = np.random.default_rng(n * 1000 + t)
    L = 37
    msg = rng.integers(0, 256, (n - t) * L, dtype=np.uint8)
    cw = _sharded_codeword(n, t, L, msg)
    par_g = np.zeros(t * L, np.uint8)
    oracle.gfni_encode(n, t, msg, par_g, L)
    assert (par_g == cw[: t * L]).all()
    for e in sorted({1, max(1, t // 2), t}):
        pos = sorted(rng.choice(n, e, replace=False).tolist())
        rx = cw.copy()
        for p in pos:
            rx[p * L:(p + 1) * L] = 0
        a, b = rx.copy(), rx.copy()
        assert oracle.recover_erasure_shards(n, t, a, L, pos)
        assert oracle.gfni_recover(n, t, b, L, pos)
        assert (a == cw).all() and (b == cw).all()


@pytest.mark.parametrize("n,t", [(4, 2), (16, 4), (32, 16), (64, 8), (128, 64), (256, 128), (256, 16)])
def test_leopard_form_equals_reference_form_on_any_input(n, t):
    """The two decoders are the same linear map whenever erased rows are zero,
    even when the surviving rows are not a codeword (e < t)."""
    rng = np.random.default_rng(n + 7 * t)
    L = 16
    for e in sorted({1, max(1, t // 2), t}):
        rx = rng.integers(0, 256, n * L, dtype=np.uint8)
        pos = sorted(rng.choice(n, e, replace=False).tolist())
        for p in pos:
            rx[p * L:(p + 1) * L] = 0
        a, b = rx.copy(), rx.copy()
        oracle.recover_erasure_shards(n, t, a, L, pos)
        oracle.recover_leopard_form(n, t, b, L, pos)
        assert (a == b).all(), (n, t, e)


def test_encode_accumulates_into_parity():
    # codec.rs:259-264: parity is XOR-accumulated, then transformed
    n, t, L = 32, 8, 5
    rng = np.random.default_rng(1)
    msg = rng.integers(0, 256, (n - t) * L, dtype=np.uint8)
    p0 = rng.integers(0, 256, t * L, dtype=np.uint8)
    zero = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, zero, L)
    acc = p0.copy()
    oracle.encode_systematic_sharded(n, t, msg, acc, L)
    f = p0.copy()
    oracle.fft_sharded(f, L, 3, 0)
    assert (acc == (zero ^ f)).all()


@pytest.mark.parametrize("n,t", [(4, 2), (16, 4), (64, 16), (256, 128)])
def test_syndrome_restatements_agree(n, t):
    """oracle.syndrome_sharded (numpy over the C transforms) and the
    pure-Python scalar form (codec.rs:269-301) on every column; zero on a
    codeword."""
    from oracle import pyref

    L = 3
    msg = oracle.random_bytes((n - t) * L, n + t)
    par = np.zeros(t * L, np.uint8)
    oracle.encode_systematic_sharded(n, t, msg, par, L)
    cw = np.concatenate([par, msg])
    assert not oracle.syndrome_sharded(n, t, cw, L).any()
    bad = cw.copy()
    bad[::7] ^= 0x33
    syn = oracle.syndrome_sharded(n, t, bad, L)
    for c in range(L):
        col = [int(bad[r * L + c]) for r in range(n)]
        assert pyref.syndrome_column(n, t, col) == [int(syn[r * L + c]) for r in range(t)]
