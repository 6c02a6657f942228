"""Second, independent CPU restatement in pure Python (small cases only).

Test infrastructure only.  It re-derives the field, the Cantor basis and the
codec from the reference's definitions without sharing code with the C
oracle, so that the two restatements can check each other.
"""
from __future__ import annotations

POLY = 0x11D


def gf_mul(a: int, b: int) -> int:
    """gf2p8/src/field.rs:22-37."""
    r = 0
    for _ in range(8):
        if b & 1:
            r ^= a
        a <<= 1
        if a & 0x100:
            a ^= POLY
        b >>= 1
    return r


def trace(a: int) -> int:
    """gf2p8/src/field.rs:122-130."""
    t, s = a, a
    for _ in range(7):
        t = gf_mul(t, t)
        s ^= t
    return s & 1


def cantor_basis() -> list[int]:
    """gf2p8/src/field.rs:174-198."""
    basis = [1]
    cur = 1
    while len(basis) < 8:
        if trace(cur):
            break
        x = next(c for c in range(256) if gf_mul(c, c) ^ c == cur)
        cur = x ^ 1 if trace(x) else x
        basis.append(cur)
    return basis


BASIS = cantor_basis()
OMEGA = [0] * 256
for _i in range(256):
    for _b in range(8):
        if (_i >> _b) & 1:
            OMEGA[_i] ^= BASIS[_b]


def s_poly(j: int, x: int) -> int:
    """s_j(x) = prod over span(v_0..v_{j-1}) of (x + a) (gf2p8/src/poly_11d.rs:187-202)."""
    r = 1
    for m in range(1 << j):
        r = gf_mul(r, x ^ OMEGA[m])
    return r


SPV = [[s_poly(j, x) for x in range(256)] for j in range(9)]


def fft(d: list[int], k: int, beta: int) -> None:
    """rs/src/poly_arith.rs:129-162 on a list slice view."""
    _fft(d, 0, k, beta)


def _fft(d, off, k, beta):
    if k == 0:
        return
    half = 1 << (k - 1)
    tw = SPV[k - 1][beta]
    for i in range(off, off + half):
        g0 = d[i] ^ gf_mul(tw, d[i + half])
        d[i + half] = g0 ^ d[i + half]
        d[i] = g0
    _fft(d, off, k - 1, beta)
    _fft(d, off + half, k - 1, beta ^ BASIS[k - 1])


def ifft(e: list[int], k: int, beta: int) -> None:
    """rs/src/poly_arith.rs:165-189."""
    _ifft(e, 0, k, beta)


def _ifft(e, off, k, beta):
    if k == 0:
        return
    half = 1 << (k - 1)
    _ifft(e, off, k - 1, beta)
    _ifft(e, off + half, k - 1, beta ^ BASIS[k - 1])
    tw = SPV[k - 1][beta]
    for i in range(off, off + half):
        h = e[i] ^ e[i + half]
        e[i] ^= gf_mul(tw, h)
        e[i + half] = h


def encode_column(n: int, t: int, msg: list[int]) -> list[int]:
    """rs/src/codec.rs:222-239 for one byte column (k = n - t message symbols)."""
    k_log = t.bit_length() - 1
    par = [0] * t
    for i in range((n - t) // t):
        w = msg[i * t:(i + 1) * t]
        ifft(w, k_log, OMEGA[(i + 1) * t])
        par = [p ^ x for p, x in zip(par, w)]
    fft(par, k_log, 0)
    return par


def syndrome_column(n: int, t: int, received: list[int]) -> list[int]:
    """rs/src/codec.rs:269-301 (compute_syndrome_scalar): XOR over chunks i of
    IFFT_t(chunk i, omega_{it}); the t syndrome symbols."""
    k_log = t.bit_length() - 1
    syn = [0] * t
    for i in range(n // t):
        w = list(received[i * t:(i + 1) * t])
        ifft(w, k_log, OMEGA[i * t])
        syn = [s ^ x for s, x in zip(syn, w)]
    return syn


def recover_column(n: int, t: int, received: list[int], positions: list[int]) -> list[int]:
    """rs/src/codec.rs:479-569 for one byte column; returns the new column."""
    e = len(positions)
    r = list(received)
    if e > t:
        raise ValueError("e > t")
    if e == 0:
        return r
    t_log, n_log = t.bit_length() - 1, n.bit_length() - 1
    pts = [OMEGA[p] for p in positions]
    lam = [0] * (n + 1)
    lam[0] = 1
    for kk, p in enumerate(pts):
        for j in range(kk + 1, 0, -1):
            lam[j] = lam[j - 1] ^ gf_mul(p, lam[j])
        lam[0] = gf_mul(p, lam[0])
    den = []
    for j in range(e):
        acc = 1
        for i in range(e):
            if i != j:
                acc = gf_mul(acc, pts[j] ^ pts[i])
        den.append(acc)
    ws = r[:t]
    ifft(ws, t_log, 0)
    for c in range(1, n // t):
        tmp = r[c * t:(c + 1) * t]
        ifft(tmp, t_log, OMEGA[c * t])
        ws = [a ^ b for a, b in zip(ws, tmp)]
    ws = ws + [0] * (n - t)
    lev = []
    for i in range(n):
        v = lam[e]
        for j in range(e - 1, -1, -1):
            v = gf_mul(v, OMEGA[i]) ^ lam[j]
        lev.append(v)
    fft(ws, n_log, 0)
    ws = [gf_mul(a, b) for a, b in zip(ws, lev)]
    ifft(ws, n_log, 0)
    ws = ws[t:t + e] + [0] * (n - e)
    fft(ws, n_log, 0)
    for j, p in enumerate(positions):
        inv = next(x for x in range(1, 256) if gf_mul(x, den[j]) == 1)
        r[p] = gf_mul(ws[p], inv)
    return r
