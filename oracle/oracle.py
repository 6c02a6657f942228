"""ctypes binding of the C oracle (afrs_oracle.c) and the GFNI CPU baseline.

Test infrastructure only.  Functions take and return numpy uint8 arrays and
follow the reference crate's argument order (rs/src/codec.rs).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_u8p = ctypes.POINTER(ctypes.c_uint8)


def build() -> None:
    """Compile the oracle and the baseline with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load(name: str) -> ctypes.CDLL:
    path = os.path.join(_BUILD, name)
    if not os.path.exists(path):
        build()
    return ctypes.CDLL(path)


_orc = None
_gfb = None


def lib() -> ctypes.CDLL:
    global _orc
    if _orc is None:
        _orc = _load("liborc.so")
        _orc.orc_get_tables.restype = ctypes.c_void_p
        _orc.orc_mul_slow.restype = ctypes.c_uint8
        _orc.orc_mul_lut.restype = ctypes.c_uint8
        _orc.orc_trace.restype = ctypes.c_int
        _orc.orc_mul_matrix.restype = ctypes.c_uint64
        _orc.orc_mul_matrix.argtypes = [ctypes.c_uint8]
        _orc.orc_bitmatrix_apply.restype = ctypes.c_uint8
        _orc.orc_bitmatrix_apply.argtypes = [ctypes.c_uint64, ctypes.c_uint8]
        _orc.orc_recover_erasure_shards.restype = ctypes.c_int
        _orc.orc_recover_leopard_form.restype = ctypes.c_int
        _orc.orc_splitmix64.restype = ctypes.c_uint64
        for f in ("orc_fft_sharded", "orc_ifft_sharded"):
            getattr(_orc, f).argtypes = [_u8p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint8]
    return _orc


def baseline_lib() -> ctypes.CDLL:
    global _gfb
    if _gfb is None:
        _gfb = _load("libgfni_baseline.so")
        _gfb.gfb_throughput.restype = ctypes.c_double
        _gfb.gfb_throughput.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_size_t,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_uint64]
        _gfb.gfb_recover.restype = ctypes.c_int
        for f in ("gfb_fft_sharded", "gfb_ifft_sharded"):
            getattr(_gfb, f).argtypes = [_u8p, ctypes.c_size_t, ctypes.c_int, ctypes.c_uint8]
    return _gfb


def _p(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u8p)


class Tables:
    """The tables rs/build.rs:549-601 emits, read from the oracle."""

    def __init__(self):
        class _T(ctypes.Structure):
            _fields_ = [("exp", ctypes.c_uint8 * 510), ("log", ctypes.c_uint8 * 256),
                        ("inv", ctypes.c_uint8 * 256), ("cantor_basis", ctypes.c_uint8 * 8),
                        ("subspace", ctypes.c_uint8 * 256), ("spv", (ctypes.c_uint8 * 256) * 9),
                        ("spc", ctypes.c_uint8 * 9), ("gfni_mul", ctypes.c_uint64 * 256)]

        t = _T.from_address(lib().orc_get_tables())
        self.exp = np.frombuffer(bytes(t.exp), np.uint8)
        self.log = np.frombuffer(bytes(t.log), np.uint8)
        self.inv = np.frombuffer(bytes(t.inv), np.uint8)
        self.cantor_basis = np.frombuffer(bytes(t.cantor_basis), np.uint8)
        self.subspace = np.frombuffer(bytes(t.subspace), np.uint8)
        self.spv = np.array([np.frombuffer(bytes(t.spv[j]), np.uint8) for j in range(9)])
        self.spc = np.frombuffer(bytes(t.spc), np.uint8)
        self.gfni_mul = np.array(list(t.gfni_mul), dtype=np.uint64)


_tables = None


def tables() -> Tables:
    global _tables
    if _tables is None:
        _tables = Tables()
    return _tables


def mul(a: int, b: int) -> int:
    return int(lib().orc_mul_slow(a, b))


def fft_sharded(shards: np.ndarray, shard_len: int, k: int, beta: int) -> None:
    lib().orc_fft_sharded(_p(shards), shard_len, k, beta)


def ifft_sharded(shards: np.ndarray, shard_len: int, k: int, beta: int) -> None:
    lib().orc_ifft_sharded(_p(shards), shard_len, k, beta)


def fft_scalar(coeffs: np.ndarray, k: int, beta: int) -> None:
    lib().orc_fft_scalar(_p(coeffs), ctypes.c_int(k), ctypes.c_uint8(beta))


def ifft_scalar(evals: np.ndarray, k: int, beta: int) -> None:
    lib().orc_ifft_scalar(_p(evals), ctypes.c_int(k), ctypes.c_uint8(beta))


def encode_systematic_scalar(n: int, t: int, message: np.ndarray) -> np.ndarray:
    parity = np.zeros(t, np.uint8)
    lib().orc_encode_systematic_scalar(n, t, _p(message), _p(parity))
    return parity


def encode_systematic_sharded(n: int, t: int, message: np.ndarray, parity: np.ndarray,
                              shard_len: int) -> None:
    """codec.rs:241-265: XOR-accumulates into `parity` in place."""
    ws = np.zeros(t * shard_len, np.uint8)
    lib().orc_encode_systematic_sharded(n, t, _p(message), _p(parity), _p(ws),
                                        ctypes.c_size_t(shard_len))


def recover_erasure_shards(n: int, t: int, received: np.ndarray, shard_len: int,
                           positions) -> bool:
    """codec.rs:479-569: rewrites the erased rows of `received` in place."""
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.uint8))
    ws = np.zeros(n * shard_len, np.uint8)
    r = lib().orc_recover_erasure_shards(n, t, _p(received), _p(ws), ctypes.c_size_t(shard_len),
                                         _p(pos) if pos.size else None, ctypes.c_size_t(pos.size))
    return bool(r)


def recover_leopard_form(n: int, t: int, received: np.ndarray, shard_len: int, positions) -> bool:
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.uint8))
    r = lib().orc_recover_leopard_form(n, t, _p(received), ctypes.c_size_t(shard_len),
                                       _p(pos) if pos.size else None, ctypes.c_size_t(pos.size))
    if r < 0:
        raise MemoryError("oracle allocation failed")
    return bool(r)


def syndrome_sharded(n: int, t: int, received: np.ndarray, shard_len: int) -> np.ndarray:
    """Sharded form of Codec::compute_syndrome_scalar (codec.rs:269-301):
    s = XOR over chunks i < n/t of IFFT_t(received rows it..(i+1)t-1, omega_{it}),
    t shards of shard_len bytes; all zero iff `received` is a codeword."""
    k = t.bit_length() - 1
    omega = tables().subspace
    syn = np.zeros(t * shard_len, np.uint8)
    for i in range(n // t):
        w = np.ascontiguousarray(received[i * t * shard_len:(i + 1) * t * shard_len]).copy()
        ifft_sharded(w, shard_len, k, int(omega[i * t]))
        syn ^= w
    return syn


def recompute_data_from_parity_sharded(n: int, t: int, received: np.ndarray, shard_len: int) -> None:
    ws = np.zeros(t * shard_len, np.uint8)
    lib().orc_recompute_data_from_parity_sharded(n, t, _p(received), _p(ws), ctypes.c_size_t(shard_len))


def erasure_locator_and_denominators(n: int, positions):
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.uint8))
    lam = np.zeros(n + 1, np.uint8)
    den = np.zeros(n, np.uint8)
    lib().orc_erasure_locator_and_denominators(n, _p(pos), ctypes.c_size_t(pos.size), _p(lam), _p(den))
    return lam[:n], den


def random_bytes(nbytes: int, seed: int) -> np.ndarray:
    out = np.empty(nbytes, np.uint8)
    lib().orc_fill_random(_p(out), ctypes.c_size_t(nbytes), ctypes.c_uint64(seed))
    return out


def gfni_encode(n: int, t: int, message: np.ndarray, parity: np.ndarray, shard_len: int) -> None:
    ws = np.zeros(t * shard_len, np.uint8)
    baseline_lib().gfb_encode(n, t, _p(message), _p(parity), _p(ws), ctypes.c_size_t(shard_len))


def gfni_recover(n: int, t: int, received: np.ndarray, shard_len: int, positions) -> bool:
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.uint8))
    ws = np.zeros(n * shard_len, np.uint8)
    return bool(baseline_lib().gfb_recover(n, t, _p(received), _p(ws), ctypes.c_size_t(shard_len),
                                           _p(pos) if pos.size else None, ctypes.c_size_t(pos.size)))


def gfni_fft_sharded(shards, shard_len, k, beta):
    baseline_lib().gfb_fft_sharded(_p(shards), shard_len, k, beta)


def gfni_ifft_sharded(shards, shard_len, k, beta):
    baseline_lib().gfb_ifft_sharded(_p(shards), shard_len, k, beta)


def gfni_throughput(op: str, n: int, t: int, shard_len: int, iters: int, threads: int,
                    seed: int = 42) -> float:
    """Bytes/s (n*L per operation) of the GFNI baseline; raises on failure."""
    r = baseline_lib().gfb_throughput(0 if op == "encode" else 1, n, t, shard_len, iters, threads, seed)
    if r < 0:
        raise RuntimeError(f"gfni baseline failed ({r})")
    return r
