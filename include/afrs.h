/*
 * afrs.h - C ABI of the B200 (sm_100a) sharded additive-FFT Reed-Solomon
 * library, libafrs_b200.so.
 *
 * Drop-in boundary for the hot path of vkomenda/additive-fft-reed-solomon:
 * the sharded systematic encoder and the sharded erasure decoder over
 * GF(2^8) (poly 0x11d, Cantor-basis evaluation points).  Every entry point
 * takes plain pointers and sizes; results are bit-identical to the
 * reference on the same inputs.
 *
 * Layout (as in the reference): a codeword is n shards of shard_len bytes,
 * shard-major; shards 0..t-1 are parity, t..n-1 are message
 * (rs/src/codec.rs:504-523).  n and t are powers of two, 1 <= t < n <= 256
 * (rs/src/lib.rs:15-19).
 *
 * Return codes: AFRS_OK (0) or a negative AFRS_E* code.  The recover entry
 * points return 1 for the reference's `true`, 0 for its `false` (more
 * erasures than t), negative on error.  afrs_last_error() gives a message
 * for the calling thread's last error.
 */
#ifndef AFRS_H
#define AFRS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AFRS_OK 0
#define AFRS_EINVAL (-1)   /* bad n, t, shard length, or erasure positions */
#define AFRS_ECUDA (-2)    /* a CUDA call failed */
#define AFRS_ENOMEM (-3)   /* device or pinned allocation failed */
#define AFRS_ETIMEOUT (-4) /* a bounded device wait gave up */

typedef struct afrs_ctx afrs_ctx;

/* Context: device tables, a scratch arena for the host-buffer entry points
 * and a stream.  The reference's Codec is a zero-sized value
 * (rs/src/codec.rs:10-27, Codec::new :22-27); the context is its device-side
 * counterpart.  One context may be used from one thread at a time. */
int afrs_ctx_create(int device, afrs_ctx** out);
void afrs_ctx_destroy(afrs_ctx* ctx);
const char* afrs_last_error(void);

/* Replaces Codec::encode_systematic_sharded (rs/src/codec.rs:241-265) on
 * host buffers: message = (n-t)*shard_len bytes, parity = t*shard_len bytes.
 * accumulate != 0 reproduces the reference exactly: the result is
 * FFT_t(parity_in ^ sum of chunk IFFTs), i.e. the parity buffer is
 * XOR-accumulated as the reference does; accumulate == 0 treats parity_in as
 * zero, which is what every reference caller passes (encode bench:87,
 * rs/src/poly_11d_lut.rs:106).  Synchronous. */
int afrs_encode(afrs_ctx* ctx, uint32_t n, uint32_t t, const uint8_t* message, uint8_t* parity,
                size_t shard_len, int accumulate);

/* Replaces Codec::recover_erasure_shards (rs/src/codec.rs:479-569) on a
 * host buffer of n*shard_len bytes.  Rewrites only the erased shards.
 * Precondition (as in the reference, recover bench:128-132): the erased
 * shards are zero on entry; the decoder does not read them.  positions must
 * be distinct and < n (the reference does not check; here AFRS_EINVAL).
 * Returns 1 (recovered), 0 (e > t, nothing written), or < 0.  Synchronous. */
int afrs_recover(afrs_ctx* ctx, uint32_t n, uint32_t t, uint8_t* received, size_t shard_len,
                 const uint8_t* positions, size_t e);

/* Device-pointer variants of the two calls above, enqueued on `stream`
 * (a cudaStream_t; NULL = the legacy default stream).  Positions are read
 * from host memory during the call.  Encodes with t >= 32 and recovers with
 * n >= 32 keep intermediate rows in a device scratch buffer owned by the
 * context (except encodes with n <= 64 of at most 4 MiB per codeword, which
 * run as one launch without it): the first call of a size grows it (at most 1 GiB;
 * longer shards are processed in column batches), and calls that share a
 * context are ordered on that buffer even when they use different streams. */
int afrs_encode_dev(afrs_ctx* ctx, uint32_t n, uint32_t t, const uint8_t* d_message,
                    uint8_t* d_parity, size_t shard_len, int accumulate, void* stream);
int afrs_recover_dev(afrs_ctx* ctx, uint32_t n, uint32_t t, uint8_t* d_received,
                     size_t shard_len, const uint8_t* positions, size_t e, void* stream);

/* Replaces Codec::recompute_data_from_parity_sharded (rs/src/codec.rs:321-340),
 * n == 2t: rewrites the t message shards of d_received from its t parity
 * shards. */
int afrs_recompute_data_from_parity_dev(afrs_ctx* ctx, uint32_t n, uint32_t t, uint8_t* d_received,
                                        size_t shard_len, void* stream);

/* Sharded form of Codec::compute_syndrome_scalar (rs/src/codec.rs:269-301):
 * d_syndrome (t shards of shard_len bytes, not overlapping d_received) =
 * XOR over chunks i < n/t of IFFT_t(shards it..(i+1)t-1 of d_received,
 * omega_{it}); all zero iff d_received (n shards, parity first) is a
 * codeword.  If d_nonzero is not NULL, *d_nonzero (device memory) is set to
 * the number of nonzero syndrome bytes (0 for a codeword).  The reference has
 * only the scalar form (one column). */
int afrs_syndrome_dev(afrs_ctx* ctx, uint32_t n, uint32_t t, const uint8_t* d_received, size_t shard_len,
                      uint8_t* d_syndrome, unsigned long long* d_nonzero, void* stream);

/* The Kernel trait (rs/src/kernel/mod.rs:7-24) on device buffers:
 * fft_sharded / ifft_sharded over 2^k shards at coset beta, in place, and
 * scale (dst = scalar * src, dst may equal src). */
int afrs_fft_sharded_dev(afrs_ctx* ctx, uint8_t* d_shards, size_t shard_len, uint32_t k, uint8_t beta,
                         void* stream);
int afrs_ifft_sharded_dev(afrs_ctx* ctx, uint8_t* d_shards, size_t shard_len, uint32_t k, uint8_t beta,
                          void* stream);
int afrs_scale_dev(afrs_ctx* ctx, const uint8_t* d_src, uint8_t* d_dst, size_t len, uint8_t scalar,
                   void* stream);

/* Batched path: many independent codewords of any shapes in one call, run
 * grouped by shape on the specialised kernels, the groups concurrently
 * (no counterpart in the reference, whose methods take one codeword;
 * each job is one call of encode_systematic_sharded, rs/src/codec.rs:241-265,
 * or recover_erasure_shards, :479-569).  Device buffers.  Encode jobs write
 * parity (parity_in is treated as zero, i.e. accumulate = 0); recover jobs
 * rewrite the erased shards of dst (src is ignored; erased shards need not be
 * zero).  Each job's status is set during the call: encode 0 = queued; recover
 * 1 = queued, 0 = more erasures than t (nothing written, the reference's
 * false); < 0 = rejected (AFRS_EINVAL), nothing written.  The call returns
 * AFRS_OK once the batch is enqueued on `stream`, or < 0 when nothing was.
 * The descriptor tables and scratch live in the context, in two slots used
 * alternately: batches on different streams may run concurrently, and a call
 * waits on the host until the previous batch of its slot has finished.  A
 * slot's grouped scratch is at most 1 GiB; a batch that needs more runs its
 * grouped jobs in rounds that reuse it. */
#define AFRS_OP_ENCODE 0u
#define AFRS_OP_RECOVER 1u
typedef struct afrs_job {
  uint32_t op;      /* AFRS_OP_ENCODE or AFRS_OP_RECOVER */
  uint32_t n, t;    /* shards, parity shards */
  uint32_t e;       /* recover: number of erasures */
  size_t shard_len; /* bytes per shard */
  const uint8_t* src; /* encode: (n-t)*shard_len message bytes */
  uint8_t* dst;       /* encode: t*shard_len parity bytes; recover: n*shard_len codeword */
  uint8_t positions[256]; /* recover: erased shard indices (first e) */
  int32_t status;         /* out */
  uint32_t reserved;
} afrs_job;
int afrs_batch_dev(afrs_ctx* ctx, afrs_job* jobs, size_t count, void* stream);

/* A batch prepared once and launched many times (no counterpart in the
 * reference).  afrs_batch_plan_create validates the jobs as afrs_batch_dev
 * does (setting each job's status), groups them by shape and copies their
 * descriptor tables to device memory owned by the plan, synchronously; the
 * jobs' buffers are the ones the plan runs on, every launch.
 * afrs_batch_plan_launch enqueues the plan's kernels on `stream` (the group
 * streams of the plan's context fork from it and join back), with no host
 * work and no copy, so the launch can be captured into a CUDA graph and the
 * graph replayed.  Launches of one plan share its tables and scratch and
 * must not overlap on the GPU; the context must outlive its plans.
 * afrs_batch_plan_destroy waits for the device and frees the plan. */
typedef struct afrs_batch_plan afrs_batch_plan;
int afrs_batch_plan_create(afrs_ctx* ctx, afrs_job* jobs, size_t count, afrs_batch_plan** out);
int afrs_batch_plan_launch(afrs_batch_plan* plan, void* stream);
void afrs_batch_plan_destroy(afrs_batch_plan* plan);

/* Allocation-free erasure recovery.  No counterpart in the reference: it
 * exists for callers that cannot allocate device memory when they recover,
 * e.g. code inside CUDA stream capture (cudaMalloc is not allowed there),
 * serving loops that must never wait on the device-wide synchronisation an
 * allocation may take, and hosts that give the library a fixed memory
 * budget.  Same arguments and results as afrs_recover_dev, on the current
 * device, without a context.  Its scratch is a 32 MiB array of device
 * memory compiled into the library (held by every GPU that loads it, until
 * the process exits); shards that need more (n * ceil(shard_len/1024) * 2 KiB
 * > 32 MiB for n >= 32, e.g. n = 256 with shard_len > 64 KiB) are refused
 * with AFRS_EINVAL and a message in afrs_last_error().  The first call on a
 * device that launches work (valid arguments, 1 <= e <= t, shard_len > 0)
 * runs a set-up step: it looks up the array's device address and loads the
 * code of the recover kernels of every n (CUDA otherwise loads a kernel's
 * code at its first launch, which may allocate).  Make that first call
 * before any stream capture; after it, calls of any n and shard length
 * load and allocate nothing.  All calls share the one array: calls that
 * overlap on the GPU (different streams, or different host threads) race and
 * must be ordered by the caller.  No scratch word needs clearing between
 * calls: each call writes every word it reads. */
int afrs_recover_dev_noalloc(uint32_t n, uint32_t t, uint8_t* d_received, size_t shard_len,
                             const uint8_t* positions, size_t e, void* stream);

/* Library build information (kernel set, arch) for logs. */
const char* afrs_version(void);

/* How the host-buffer entry points (afrs_encode, afrs_recover) move data.
 * Staged: copy engines move shard columns in windows of about window_bytes
 * per codeword through device buffers (two windows in flight: copy-in,
 * kernels and copy-out overlap); runs of copied rows closer than merge_bytes
 * are merged into one copy.  Direct: when a buffer is page-locked and mapped,
 * the kernels read and write it themselves (exactly the rows the operation
 * needs).  AFRS_HOST_AUTO (default): recover direct when possible, encode
 * staged.  window_bytes / merge_bytes 0 select the defaults (4 MiB, 128 KiB);
 * merge_bytes = SIZE_MAX disables merging. */
#define AFRS_HOST_AUTO 0
#define AFRS_HOST_STAGED 1
#define AFRS_HOST_DIRECT 2
int afrs_ctx_set_staging(afrs_ctx* ctx, size_t window_bytes, size_t merge_bytes, int host_mode);

/* Largest device scratch (bytes) the context's encode and recover calls use
 * for the rows they keep between kernels; 0 restores the default, 1 GiB,
 * which is also the maximum.  Shards whose calls need more are processed in
 * column batches that each fit the cap, so a small cap bounds the context's
 * device memory at the price of more launches.  Values below 16 KiB (one
 * colword of an n = 256 recover) are refused with AFRS_EINVAL.  A
 * diagnostic and memory-budget knob; no counterpart in the reference, whose
 * calls take a caller-sized workspace (rs/src/codec.rs:241-247, :479-485). */
int afrs_ctx_set_work_cap(afrs_ctx* ctx, size_t bytes);

/* Kernel family of the context's per-call encodes and recovers.
 * AFRS_ROUTE_TABLE (default): per shape and shard length, the family the
 * library's tuned route table names (measured on a B200 by tune.py in the
 * package directory), and built-in rules where it names none.  The others
 * force one family, for tuning and diagnostics: GENERIC, the one-launch
 * kernel with runtime twiddles (rows must be compact; calls on host buffers
 * whose windows use a row pitch keep the specialised kernels); SPECIAL, the
 * kernels with compile-time twiddles, t <= 16 encodes with one warp per
 * 1024-column slice; SPECIAL_SPLIT, the same with the warps of a CTA
 * splitting one slice's chunks (t <= 16 encodes with n > 2t; otherwise as
 * SPECIAL); FUSED, the compile-time-twiddle kernels in one launch per call,
 * one CTA holding every row of a 1024-column slice (encodes with t = 32 or
 * 64, recovers with n = 32 .. 128; otherwise as SPECIAL); FEW, the
 * few-erasure recover (n >= 32 and 1 <= e <= 8: one pass over the surviving
 * shards and an e x e solve, no scratch; otherwise, and for encodes, as
 * TABLE).  Under TABLE (and in batches, afrs_batch_dev) every recover FEW
 * covers takes it: it measured faster than the other families at every such
 * shape and shard length.  Results are
 * identical on every route.  No counterpart in the reference, whose kernel
 * choice is a build-time CPU feature test (rs/build.rs:628-646). */
#define AFRS_ROUTE_TABLE 0
#define AFRS_ROUTE_GENERIC 1
#define AFRS_ROUTE_SPECIAL 2
#define AFRS_ROUTE_SPECIAL_SPLIT 3
#define AFRS_ROUTE_FUSED 4
#define AFRS_ROUTE_FEW 5
int afrs_ctx_set_route(afrs_ctx* ctx, int route);

/* Number of CUDA kernels this library has launched in this process, over
 * every context and entry point (a diagnostic for benchmarks and tests; no
 * counterpart in the reference). */
uint64_t afrs_kernel_launches(void);

/* Bytes the host-buffer entry points (afrs_encode, afrs_recover) have moved
 * host -> device and device -> host in this process: staging copies, or the
 * kernels' own reads and writes when the host buffers are page-locked and
 * mapped (a diagnostic; no counterpart in the reference). */
void afrs_staged_bytes(uint64_t* h2d, uint64_t* d2h);

#ifdef __cplusplus
}
#endif
#endif /* AFRS_H */
