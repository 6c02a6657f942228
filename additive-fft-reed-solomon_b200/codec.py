"""Host-side mirror of the reference crate's codec API over the C ABI.

`Codec(n, t)` stands for the reference's `Rs::<N, T>` / `Codec<G, B, K, N, T>`
(rs/src/lib.rs:20-45, rs/src/codec.rs:10-27) with the same method names,
argument meaning and results:

* ``encode_systematic_sharded(message, parity, workspace, shard_len)``
  (codec.rs:241-265) XOR-accumulates into ``parity`` and transforms it, as the
  reference does; ``workspace`` is accepted and not used.
* ``recover_erasure_shards(received, workspace, shard_len, erasure_positions)``
  (codec.rs:479-569) returns ``False`` iff there are more erasures than t and
  otherwise rewrites the erased shards of ``received`` and returns ``True``.
* ``recompute_data_from_parity_sharded(received, workspace, shard_len)``
  (codec.rs:321-340, n == 2t).

Buffers are numpy uint8 arrays in host memory (the call copies them to and
from the GPU) or uint8 CUDA tensors (the call enqueues on the current torch
stream and returns without waiting).  Where the reference panics (bad sizes,
``unreachable!``), these raise ``AfrsError``.
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from . import _lib

__all__ = ["AfrsError", "Context", "Codec", "Job", "run_batch", "BatchPlan", "fft_sharded", "ifft_sharded", "scale"]


class AfrsError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = _lib.lib().afrs_last_error().decode(errors="replace")
        super().__init__(f"{where} failed ({code}): {msg}")
        self.code = code


def _check(code: int, where: str) -> int:
    if code < 0:
        raise AfrsError(code, where)
    return code


class Context:
    """A device context (device tables, stream, scratch for host buffers)."""

    _by_device: dict = {}

    def __init__(self, device: int = 0):
        self._h = ctypes.c_void_p()
        _check(_lib.lib().afrs_ctx_create(device, ctypes.byref(self._h)), "afrs_ctx_create")
        self.device = device

    @classmethod
    def get(cls, device: int = 0) -> "Context":
        ctx = cls._by_device.get(device)
        if ctx is None:
            ctx = cls._by_device[device] = cls(device)
        return ctx

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def set_work_cap(self, nbytes: int) -> None:
        """Largest device scratch the context's calls use between kernels
        (afrs_ctx_set_work_cap); longer shards run in column batches.  0
        restores the default."""
        _check(_lib.lib().afrs_ctx_set_work_cap(self._h, int(nbytes)), "afrs_ctx_set_work_cap")

    def set_route(self, route: int) -> None:
        """Kernel family of the context's per-call encodes and recovers
        (afrs_ctx_set_route): _lib.AFRS_ROUTE_TABLE (default) or a forced one."""
        _check(_lib.lib().afrs_ctx_set_route(self._h, int(route)), "afrs_ctx_set_route")

    def close(self) -> None:
        if self._h:
            _lib.lib().afrs_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _is_cuda_tensor(x) -> bool:
    return hasattr(x, "is_cuda") and x.is_cuda


_torch = None


def _torch_mod():
    global _torch
    if _torch is None:
        import torch

        _torch = torch
    return _torch


def _dev_ptr(x) -> int:
    if x.dtype != _torch_mod().uint8 or not x.is_contiguous():
        raise AfrsError(_lib.AFRS_EINVAL, "tensor must be contiguous uint8")
    return x.data_ptr()


def _host_ptr(x: np.ndarray) -> int:
    if not isinstance(x, np.ndarray) or x.dtype != np.uint8 or not x.flags["C_CONTIGUOUS"]:
        raise AfrsError(_lib.AFRS_EINVAL, "host buffer must be a C-contiguous numpy uint8 array")
    return x.ctypes.data


_raw_stream = None


def _stream(x) -> int:
    """Handle of torch's current stream on the device of tensor ``x``.  Read
    through torch's raw-handle accessor where it exists: building a
    torch.cuda.Stream object costs about 2 us, a fifth of a small call."""
    global _raw_stream
    if _raw_stream is None:
        torch = _torch_mod()
        _raw_stream = getattr(torch._C, "_cuda_getCurrentRawStream", None) or (
            lambda d: torch.cuda.current_stream(d).cuda_stream)
    return _raw_stream(x.get_device())


def _nbytes(x) -> int:
    return x.numel() if _is_cuda_tensor(x) else x.size


class Codec:
    """Mirror of ``Rs::<N, T>`` (rs/src/lib.rs:20-45) running on the GPU."""

    def __init__(self, n: int, t: int, device: int = 0, context: "Context | None" = None):
        self.n, self.t = int(n), int(t)
        # A context's scratch serves one operation at a time; codecs that
        # should run concurrently on different streams take their own.
        self.ctx = context if context is not None else Context.get(device)

    def _sizes(self, shard_len: int, **bufs) -> None:
        want = {"message": (self.n - self.t) * shard_len, "parity": self.t * shard_len,
                "received": self.n * shard_len}
        for name, buf in bufs.items():
            if _nbytes(buf) != want[name]:
                raise AfrsError(_lib.AFRS_EINVAL, f"{name} has {_nbytes(buf)} bytes, expected {want[name]}")

    def encode_systematic_sharded(self, message, parity, workspace=None, shard_len: int = 0) -> None:
        self._sizes(shard_len, message=message, parity=parity)
        L = _lib.lib()
        if _is_cuda_tensor(message):
            _check(L.afrs_encode_dev(self.ctx.handle, self.n, self.t, _dev_ptr(message), _dev_ptr(parity),
                                     shard_len, 1, _stream(message)), "afrs_encode_dev")
        else:
            _check(L.afrs_encode(self.ctx.handle, self.n, self.t, _host_ptr(message), _host_ptr(parity),
                                 shard_len, 1), "afrs_encode")

    def encode_parity(self, message, parity, shard_len: int) -> None:
        """Encode into ``parity`` without reading it (parity treated as zero)."""
        self._sizes(shard_len, message=message, parity=parity)
        L = _lib.lib()
        if _is_cuda_tensor(message):
            _check(L.afrs_encode_dev(self.ctx.handle, self.n, self.t, _dev_ptr(message), _dev_ptr(parity),
                                     shard_len, 0, _stream(message)), "afrs_encode_dev")
        else:
            _check(L.afrs_encode(self.ctx.handle, self.n, self.t, _host_ptr(message), _host_ptr(parity),
                                 shard_len, 0), "afrs_encode")

    def recover_erasure_shards(self, received, workspace=None, shard_len: int = 0, erasure_positions=()) -> bool:
        self._sizes(shard_len, received=received)
        pos = np.ascontiguousarray(np.asarray(list(erasure_positions), dtype=np.int64))
        if pos.size and (pos.min() < 0 or pos.max() > 255):
            raise AfrsError(_lib.AFRS_EINVAL, "erasure positions must fit in u8")
        pos8 = pos.astype(np.uint8)
        pp = pos8.ctypes.data if pos8.size else None
        L = _lib.lib()
        if _is_cuda_tensor(received):
            r = L.afrs_recover_dev(self.ctx.handle, self.n, self.t, _dev_ptr(received), shard_len, pp, pos8.size,
                                   _stream(received))
        else:
            r = L.afrs_recover(self.ctx.handle, self.n, self.t, _host_ptr(received), shard_len, pp, pos8.size)
        return bool(_check(r, "recover_erasure_shards"))

    def recompute_data_from_parity_sharded(self, received, workspace=None, shard_len: int = 0) -> None:
        self._sizes(shard_len, received=received)
        if not _is_cuda_tensor(received):
            import torch

            d = torch.from_numpy(received).cuda(self.ctx.device)
            self.recompute_data_from_parity_sharded(d, None, shard_len)
            received[...] = d.cpu().numpy()
            return
        _check(_lib.lib().afrs_recompute_data_from_parity_dev(self.ctx.handle, self.n, self.t, _dev_ptr(received),
                                                              shard_len, _stream(received)),
               "recompute_data_from_parity")

    def syndrome_sharded(self, received, shard_len: int, syndrome=None):
        """Sharded Codec::compute_syndrome_scalar (codec.rs:269-301) of a uint8
        CUDA tensor of n shards: returns (syndrome, nonzero) where syndrome is a
        t*shard_len CUDA tensor (``syndrome`` if given) and nonzero a one-element
        int64 CUDA tensor counting its nonzero bytes (0 iff a codeword)."""
        import torch

        self._sizes(shard_len, received=received)
        if syndrome is None:
            syndrome = torch.empty(self.t * shard_len, dtype=torch.uint8, device=received.device)
        self._sizes(shard_len, parity=syndrome)
        nz = torch.zeros(1, dtype=torch.int64, device=received.device)
        _check(_lib.lib().afrs_syndrome_dev(self.ctx.handle, self.n, self.t, _dev_ptr(received), shard_len,
                                            _dev_ptr(syndrome), nz.data_ptr(), _stream(received)),
               "syndrome_sharded")
        return syndrome, nz

    def is_codeword(self, received, shard_len: int) -> bool:
        """True iff the n shards of ``received`` (CUDA tensor) form a codeword."""
        _, nz = self.syndrome_sharded(received, shard_len)
        return int(nz.item()) == 0


def fft_sharded(shards, shard_len: int, k: int, beta: int, device: int = 0) -> None:
    """Kernel::fft_sharded (rs/src/kernel/mod.rs:8-14) on a uint8 CUDA tensor."""
    ctx = Context.get(device)
    _check(_lib.lib().afrs_fft_sharded_dev(ctx.handle, _dev_ptr(shards), shard_len, k, beta, _stream(shards)),
           "fft_sharded")


def ifft_sharded(shards, shard_len: int, k: int, beta: int, device: int = 0) -> None:
    """Kernel::ifft_sharded (rs/src/kernel/mod.rs:15-21) on a uint8 CUDA tensor."""
    ctx = Context.get(device)
    _check(_lib.lib().afrs_ifft_sharded_dev(ctx.handle, _dev_ptr(shards), shard_len, k, beta, _stream(shards)),
           "ifft_sharded")


def scale(src, dst, scalar: int, device: int = 0) -> None:
    """Kernel::scale (rs/src/kernel/mod.rs:22): dst = scalar * src, bytewise."""
    ctx = Context.get(device)
    _check(_lib.lib().afrs_scale_dev(ctx.handle, _dev_ptr(src), _dev_ptr(dst), src.numel(), scalar, _stream(src)),
           "scale")


class Job:
    """One codeword of a batch: ``Job.encode(n, t, message, parity, shard_len)``
    or ``Job.recover(n, t, received, shard_len, positions)`` on uint8 CUDA
    tensors.  After ``run_batch`` its ``status`` is the C ABI's job status."""

    def __init__(self, op, n, t, src, dst, shard_len, positions=()):
        self.op, self.n, self.t, self.src, self.dst, self.shard_len = op, int(n), int(t), src, dst, int(shard_len)
        self.positions = [int(p) for p in positions]
        self.status = None

    @classmethod
    def encode(cls, n, t, message, parity, shard_len):
        return cls(_lib.AFRS_OP_ENCODE, n, t, message, parity, shard_len)

    @classmethod
    def recover(cls, n, t, received, shard_len, positions):
        return cls(_lib.AFRS_OP_RECOVER, n, t, None, received, shard_len, positions)

    @property
    def nbytes(self) -> int:
        return self.n * self.shard_len


# struct afrs_job of include/afrs.h: op, n, t, e (u32), shard_len, src, dst
# (64-bit) = 40 bytes, then positions[256], status (i32), reserved (u32).
_JOB_HEAD = struct.Struct("<IIIIQQQ")
_JOB_TAIL = 256 + 8
_JOB_STATUS = 296 // 4  # int32 index of status within a record
_JOB_WORDS = 304 // 4


def _job_record(j) -> bytes:
    """The 304 bytes of ``j`` as a struct afrs_job."""
    try:
        pos = bytes(j.positions[:256])
    except ValueError:
        raise AfrsError(_lib.AFRS_EINVAL, "erasure positions must fit in u8") from None
    src = _dev_ptr(j.src) if j.src is not None else 0
    dst = _dev_ptr(j.dst) if j.dst is not None else 0
    return _JOB_HEAD.pack(j.op, j.n, j.t, len(j.positions), j.shard_len, src, dst) + pos + bytes(_JOB_TAIL - len(pos))


def _job_array(jobs):
    """ctypes array of struct afrs_job for ``jobs``: one record packed per job
    and one copy into the array (a few microseconds per job less than setting
    the ctypes fields one by one, which matters when a server packs hundreds
    of requests per batch)."""
    n = max(len(jobs), 1)
    buf = b"".join(_job_record(j) for j in jobs) if jobs else bytes(ctypes.sizeof(_lib.AfrsJob))
    return (_lib.AfrsJob * n).from_buffer_copy(buf)


def _job_statuses(arr, count: int) -> list:
    """The status fields of the first ``count`` records of a job array."""
    words = np.frombuffer(arr, dtype=np.int32)
    return words[_JOB_STATUS:count * _JOB_WORDS:_JOB_WORDS].tolist()


def run_batch(jobs, device: int = 0, stream=None) -> list:
    """Enqueue every job in one batched launch (afrs_batch_dev) on the
    current torch stream (or ``stream``); returns the per-job statuses."""
    import torch

    arr = _job_array(jobs)
    ctx = Context.get(device)
    s = stream if stream is not None else torch.cuda.current_stream(device)
    _check(_lib.lib().afrs_batch_dev(ctx.handle, arr, len(jobs), s.cuda_stream), "afrs_batch_dev")
    out = _job_statuses(arr, len(jobs))
    for j, st in zip(jobs, out):
        j.status = st
    return out


class BatchPlan:
    """Jobs prepared once (afrs_batch_plan_create: validation, grouping and
    descriptor tables copied to the device) and launched any number of times
    with ``launch()`` (afrs_batch_plan_launch: kernels only, so the launch
    can be captured into a CUDA graph).  The plan runs on the jobs' buffers;
    it keeps references to them.  Launches of one plan must not overlap."""

    def __init__(self, jobs, device: int = 0, context: "Context | None" = None):
        self.jobs = list(jobs)
        self.ctx = context if context is not None else Context.get(device)
        arr = _job_array(self.jobs)
        self._h = ctypes.c_void_p()
        _check(_lib.lib().afrs_batch_plan_create(self.ctx.handle, arr, len(self.jobs), ctypes.byref(self._h)),
               "afrs_batch_plan_create")
        self.statuses = _job_statuses(arr, len(self.jobs))
        for j, st in zip(self.jobs, self.statuses):
            j.status = st

    def launch(self, stream=None) -> None:
        import torch

        s = stream if stream is not None else torch.cuda.current_stream()
        _check(_lib.lib().afrs_batch_plan_launch(self._h, s.cuda_stream), "afrs_batch_plan_launch")

    def close(self) -> None:
        if self._h:
            _lib.lib().afrs_batch_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
