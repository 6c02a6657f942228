"""B200 (sm_100a) sharded additive-FFT Reed-Solomon over GF(2^8).

Drop-in GPU path for the sharded encoder and erasure decoder of
vkomenda/additive-fft-reed-solomon.  The compute lives in libafrs_b200.so
(csrc/, C ABI in include/afrs.h); this package is the host-side mirror of the
reference codec API.
"""
from ._lib import LIB_PATH, build, lib  # noqa: F401
from .codec import AfrsError, BatchPlan, Codec, Context, Job, fft_sharded, ifft_sharded, run_batch, scale  # noqa: F401

# The reference's type names for the same codec (rs/src/lib.rs:20-45).
Rs = Codec
RsCuda = Codec
from . import serving  # noqa: F401,E402
