"""CPU checks of the C ABI library: it is built for sm_100a, loads, and
exports every entry point include/afrs.h declares (no compute without a GPU)."""
import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    src = open(os.path.join(ROOT, "include", "afrs.h")).read()
    return sorted(set(re.findall(r"\b(afrs_[a-z_0-9]+)\s*\(", src)))


def test_header_and_binding_agree(afrs):
    declared = _declared_functions()
    assert declared == sorted(afrs._lib.SIGNATURES)


def test_library_exports_every_declared_symbol(afrs):
    if not os.path.exists(afrs.LIB_PATH):
        afrs.build()
    out = subprocess.run(["nm", "-D", "--defined-only", afrs.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (afrs_\w+)", out))
    missing = [f for f in _declared_functions() if f not in exported]
    assert not missing, missing
    lib = afrs.lib()
    for f in _declared_functions():
        assert getattr(lib, f) is not None


def test_null_context_is_einval(afrs):
    lib = afrs.lib()
    assert lib.afrs_encode_dev(None, 4, 2, None, None, 16, 0, None) == afrs._lib.AFRS_EINVAL
    assert b"NULL" in lib.afrs_last_error()
    assert lib.afrs_recover_dev(None, 4, 2, None, 16, None, 1, None) == afrs._lib.AFRS_EINVAL
    assert lib.afrs_version().startswith(b"afrs_b200")
    assert lib.afrs_kernel_launches() >= 0


def test_no_device_context_fails_cleanly(afrs):
    import torch

    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    r = afrs.lib().afrs_ctx_create(0, ctypes.byref(h))
    assert r < 0 and not h.value


def test_newer_entry_points_validate_arguments(afrs):
    """No device needed: invalid arguments are rejected before any CUDA call."""
    import ctypes

    lib = afrs.lib()
    E = afrs._lib.AFRS_EINVAL
    assert lib.afrs_ctx_set_staging(None, 0, 0, 0) == E
    assert lib.afrs_syndrome_dev(None, 4, 2, None, 16, None, None, None) == E
    assert lib.afrs_batch_dev(None, None, 0, None) == E
    a, b = ctypes.c_uint64(7), ctypes.c_uint64(7)
    lib.afrs_staged_bytes(ctypes.byref(a), ctypes.byref(b))
    assert a.value >= 0 and b.value >= 0
    lib.afrs_staged_bytes(None, None)  # either pointer may be NULL
