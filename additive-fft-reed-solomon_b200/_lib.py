"""Loads libafrs_b200.so (built from csrc/ for sm_100a) and declares the C ABI
of include/afrs.h for ctypes."""
from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libafrs_b200.so")

AFRS_OK = 0
AFRS_EINVAL = -1
AFRS_ECUDA = -2
AFRS_ENOMEM = -3
AFRS_ETIMEOUT = -4

_u8p = ctypes.c_void_p
_sz = ctypes.c_size_t
_u32 = ctypes.c_uint32

AFRS_HOST_AUTO = 0
AFRS_HOST_STAGED = 1
AFRS_HOST_DIRECT = 2

AFRS_ROUTE_TABLE = 0
AFRS_ROUTE_GENERIC = 1
AFRS_ROUTE_SPECIAL = 2
AFRS_ROUTE_SPECIAL_SPLIT = 3
AFRS_ROUTE_FUSED = 4
AFRS_ROUTE_FEW = 5

AFRS_OP_ENCODE = 0
AFRS_OP_RECOVER = 1


class AfrsJob(ctypes.Structure):
    """struct afrs_job of include/afrs.h."""

    _fields_ = [("op", ctypes.c_uint32), ("n", ctypes.c_uint32), ("t", ctypes.c_uint32), ("e", ctypes.c_uint32),
                ("shard_len", ctypes.c_size_t), ("src", ctypes.c_void_p), ("dst", ctypes.c_void_p),
                ("positions", ctypes.c_uint8 * 256), ("status", ctypes.c_int32), ("reserved", ctypes.c_uint32)]


# name -> (restype, argtypes); the list mirrors include/afrs.h.
SIGNATURES = {
    "afrs_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "afrs_ctx_destroy": (None, [ctypes.c_void_p]),
    "afrs_last_error": (ctypes.c_char_p, []),
    "afrs_version": (ctypes.c_char_p, []),
    "afrs_kernel_launches": (ctypes.c_uint64, []),
    "afrs_ctx_set_staging": (ctypes.c_int, [ctypes.c_void_p, _sz, _sz, ctypes.c_int]),
    "afrs_ctx_set_work_cap": (ctypes.c_int, [ctypes.c_void_p, _sz]),
    "afrs_ctx_set_route": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "afrs_staged_bytes": (None, [ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]),
    "afrs_encode": (ctypes.c_int, [ctypes.c_void_p, _u32, _u32, _u8p, _u8p, _sz, ctypes.c_int]),
    "afrs_recover": (ctypes.c_int, [ctypes.c_void_p, _u32, _u32, _u8p, _sz, _u8p, _sz]),
    "afrs_encode_dev": (ctypes.c_int, [ctypes.c_void_p, _u32, _u32, _u8p, _u8p, _sz, ctypes.c_int, ctypes.c_void_p]),
    "afrs_recover_dev": (ctypes.c_int, [ctypes.c_void_p, _u32, _u32, _u8p, _sz, _u8p, _sz, ctypes.c_void_p]),
    "afrs_recompute_data_from_parity_dev": (ctypes.c_int, [ctypes.c_void_p, _u32, _u32, _u8p, _sz, ctypes.c_void_p]),
    "afrs_syndrome_dev": (ctypes.c_int, [ctypes.c_void_p, _u32, _u32, _u8p, _sz, _u8p, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    "afrs_fft_sharded_dev": (ctypes.c_int, [ctypes.c_void_p, _u8p, _sz, _u32, ctypes.c_uint8, ctypes.c_void_p]),
    "afrs_ifft_sharded_dev": (ctypes.c_int, [ctypes.c_void_p, _u8p, _sz, _u32, ctypes.c_uint8, ctypes.c_void_p]),
    "afrs_scale_dev": (ctypes.c_int, [ctypes.c_void_p, _u8p, _u8p, _sz, ctypes.c_uint8, ctypes.c_void_p]),
    "afrs_recover_dev_noalloc": (ctypes.c_int, [_u32, _u32, _u8p, _sz, _u8p, _sz, ctypes.c_void_p]),
    "afrs_batch_dev": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AfrsJob), _sz, ctypes.c_void_p]),
    "afrs_batch_plan_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(AfrsJob), _sz,
                                              ctypes.POINTER(ctypes.c_void_p)]),
    "afrs_batch_plan_launch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "afrs_batch_plan_destroy": (None, [ctypes.c_void_p]),
}


def build(jobs: int = 8) -> str:
    """Compile csrc/ with nvcc for sm_100a (the library and the multiply
    benchmark program); returns the library path."""
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", os.path.join(HERE, "csrc"), "all", "bench_multiply"], check=True)
    return LIB_PATH


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded library.  There is no fallback: a missing library is an error."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                               "(make -C additive-fft-reed-solomon_b200/csrc)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib
