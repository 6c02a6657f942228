// Internal interfaces between the C ABI (afrs_capi.cu) and the kernel files.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace afrs {

// Parameters of one recover launch, passed by value (kernel parameter space),
// so a launch needs no device allocation.
struct RecoverArgs {
  uint8_t* rx;       // n rows of L bytes, shard-major
  size_t L;          // shard length (columns processed)
  int n, t, e;       // shards, parity shards, erasures
  uint8_t pos[256];  // erased positions (first e entries)
  size_t pitch = 0;  // bytes between rows; 0 = L (the special kernels honour it)
  // n = 32 .. 128: kLayoutFused = one launch per call (the whole decoder per
  // CTA); n >= 32, e <= 8: kLayoutFew (or -1) = the few-erasure kernel;
  // otherwise the three phase kernels.
  int layout = -1;
};

struct EncodeArgs {
  const uint8_t* msg;  // (n - t) rows
  uint8_t* parity;     // t rows
  size_t L;
  int n, t;
  int accumulate;
  size_t pitch = 0;  // bytes between rows of msg and parity; 0 = L
  // t <= 16 encodes with several chunks: 1 = the warps of a CTA split one
  // slice's chunks, 0 = one warp per slice, -1 = chosen by the built-in rule.
  // t = 32, 64: kLayoutFused = one launch per call, else the phase kernels.
  int layout = -1;
};
// Layout value of the one-launch form of the specialised kernels.
constexpr int kLayoutFused = 2;
// Layout value of the few-erasure recover (one pass over the survivors and an
// e x e solve; n >= 32, 1 <= e <= 8).  With layout -1 the recover launcher
// takes it wherever the shape allows.
constexpr int kLayoutFew = 3;
inline bool few_recover_shape(int n, int e) { return n >= 32 && n <= 256 && e >= 1 && e <= 8; }
// Where a single call is faster on it than on the Leopard-form kernels
// (B200, CUDA graphs): every shape it covers, at every measured shard length
// (1 KiB .. 1 MiB; n = 256, 64 KiB shards: e = 1 7.8 vs 28.2 us, e = 8 27.8
// vs 30.1; 1 KiB, e = 8: 16.4 vs 16.5).
inline bool few_recover_wins(int n, int e, size_t) { return few_recover_shape(n, e); }
template <class A>
__host__ __device__ inline size_t row_pitch(const A& a) {
  return a.pitch ? a.pitch : a.L;
}

// Batched launch (batch.cu): device tables built by afrs_batch_dev.
struct BatchJob {
  const uint8_t* src;  // encode: message; recover: the codeword
  uint8_t* dst;        // encode: parity; recover: the codeword (same as src)
  size_t L;
  int op, n, t, e;     // op 0 = encode, 1 = recover
  uint32_t pos_off;    // erasure positions at pos_tab + pos_off
  uint32_t loc;        // locator slot of a recover job
};

struct BatchLaunch {
  const BatchJob* jobs;
  const uint2* tasks;    // (job, 256-column tile)
  int ntasks;
  const int* rec_jobs;   // indices of the recover jobs
  int nrec;
  const uint8_t* pos_tab;
  uint8_t* loc_tab;      // nrec * 768 bytes
  unsigned* counter;     // task counter (reset by the launch)
  int max_rows;          // largest 2n (recover) or 2t (encode) over the jobs
};

size_t batch_tiles(size_t L);
cudaError_t launch_batch(const BatchLaunch& b, cudaStream_t s);

// Generic kernels: any (n, t), runtime twiddles.
cudaError_t launch_encode_generic(const EncodeArgs& a, cudaStream_t s);
cudaError_t launch_recover_generic(const RecoverArgs& a, cudaStream_t s);
cudaError_t launch_transform_generic(uint8_t* shards, size_t L, int k, uint8_t beta, bool inverse,
                                     cudaStream_t s);
cudaError_t launch_recompute_generic(uint8_t* rx, size_t L, int t, cudaStream_t s);
cudaError_t launch_scale(const uint8_t* src, uint8_t* dst, size_t len, uint8_t c, cudaStream_t s);
// dst ^= src; *count += nonzero bytes of src (byte streams, any alignment).
cudaError_t launch_xor_into(uint8_t* dst, const uint8_t* src, size_t len, cudaStream_t s);
cudaError_t launch_count_nonzero(const uint8_t* src, size_t len, unsigned long long* count, cudaStream_t s);

// Per-call kernel routes (route.cu): the tuned table (route_table.inc,
// written by tune.py) for a shape and shard-length bucket, or -1 when it has
// no entry (the built-in rules decide).
enum Route : int { kRouteGeneric = 0, kRouteSpecial = 1, kRouteSpecialSplit = 2, kRouteFused = 3, kRouteFew = 4 };
// Shapes the one-launch specialised form (kRouteFused) covers.
inline bool fused_encode_shape(int n, int t) { return (t == 32 || t == 64) && t < n; }
inline bool fused_recover_shape(int n) { return n >= 32 && n <= 128; }
int route_encode(int n, int t, size_t L);
int route_recover(int n, size_t L);
// Bucket of a shard length in the table: 0 for L <= 64, else ceil(log2 L) - 6;
// -1 beyond the largest tuned length.
int route_bucket(size_t L);

// Device scratch for the phase kernels (bit-sliced intermediate rows).
struct ScratchArena {
  uint32_t* ptr;  // 16-byte aligned
  size_t bytes;
};

// Specialised kernels (compile-time twiddles).  Return cudaErrorNotSupported
// when no specialisation exists for the shape; the caller then uses the
// generic kernel.  With less scratch than scratch_bytes_*() the launchers
// process the shard in column batches; with none they need, they return
// cudaErrorMemoryAllocation.
cudaError_t launch_encode_special(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s);
cudaError_t launch_recover_special(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s);
// Loads the code of every recover kernel launch_recover_special may launch,
// on the current device, so that no later launch loads code lazily.
cudaError_t preload_recover_special();
size_t scratch_bytes_encode(int n, int t, size_t L);
// Sets the calling thread's afrs_last_error() message.
void set_last_error(const char* msg);
// Adds k to the process-wide count of kernels this library has launched
// (read back with afrs_kernel_launches()).
void count_launches(unsigned k);
// Raises kernel fn's dynamic shared-memory limit on the current device to at
// least `bytes`; the runtime call is made once per kernel, device and larger
// size (it costs about a microsecond, which small per-call launches notice).
cudaError_t ensure_smem_attr(const void* fn, size_t bytes);
size_t scratch_bytes_recover(int n, size_t L);

// Grouped launches of many codewords of one shape (afrs_batch_dev): op 0 =
// encode, 1 = recover, 2 = few-erasure recover (n >= 32, e <= 8, no
// scratch).  Each codeword gets a descriptor (job_desc_bytes, filled on the
// host) and its own scratch (job_scratch_bytes, the whole shard width); the
// descriptors are copied to device memory and launched per shape group.
bool jobs_supported(int op, int n, int t);
size_t job_desc_bytes(int op);
size_t job_scratch_bytes(int op, int n, int t, size_t L);
size_t job_colwords(size_t L);
void fill_enc_job(void* desc, const EncodeArgs& a, uint32_t* scratch);
void fill_rec_job(void* desc, const RecoverArgs& a, uint32_t* scratch);
cudaError_t launch_encode_jobs(int n, int t, const void* d_jobs, int count, size_t max_ncw, cudaStream_t s);
cudaError_t launch_recover_jobs(int n, void* d_jobs, int count, size_t max_ncw, cudaStream_t s);
// Few-erasure descriptor of one recover (the pattern's e x e solve, computed
// here); false when the pattern has none (the job then takes op 1).
bool fill_few_job(void* desc, const RecoverArgs& a);
// A group of few-erasure recovers of one n, each with 2^logt / 2 < e <= 2^logt.
cudaError_t launch_recover_few_jobs(int n, int logt, const void* d_jobs, int count, size_t max_ncw, cudaStream_t s);

}  // namespace afrs
