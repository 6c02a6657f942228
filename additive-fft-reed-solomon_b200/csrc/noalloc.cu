// Allocation-free erasure recovery: afrs_recover_dev_noalloc().
//
// Some callers cannot allocate device memory at the time they recover
// shards: code running inside CUDA stream capture (where cudaMalloc is not
// allowed), latency-critical serving loops that must never take the
// device-wide synchronisation a cudaMalloc/cudaFree may imply, and hosts
// that hand the library a fixed memory budget up front.  For them the
// recover path's scratch (the bit-sliced rows kept between its three
// kernels) lives in the fixed array below instead of the context's arena,
// and the entry point needs no afrs_ctx at all.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/afrs.h"
#include "afrs_internal.h"

namespace {

// 32 MiB: enough for one n = 256 codeword with 64 KiB shards.  Every GPU
// that loads this library holds the array until the process exits.
constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
uint32_t* g_scratch_ptr[kMaxDevices] = {};  // device address of the array, per device

int fail(int code, const char* fmt, ...) {
  char msg[256];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof msg, fmt, ap);
  va_end(ap);
  afrs::set_last_error(msg);  // read back with afrs_last_error()
  return code;
}

bool pow2(uint32_t v) { return v && !(v & (v - 1)); }

// The array's name is a host-side stand-in, not a device address; the
// device address is looked up once per device, with that device current.
// The same set-up step loads the code of every recover kernel on the device
// (CUDA otherwise loads a kernel's code at its first launch, which may
// allocate and is not allowed inside stream capture), so after the first
// call on a device no call of any shape loads or allocates anything.
int setup_current_device(uint32_t** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(AFRS_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(AFRS_EINVAL, "device %d beyond %d", dev, kMaxDevices);
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(AFRS_ECUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    e = afrs::preload_recover_special();
    if (e != cudaSuccess) return fail(AFRS_ECUDA, "loading the recover kernels: %s", cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_scratch_ptr[dev];
  return AFRS_OK;
}

}  // namespace

extern "C" int afrs_recover_dev_noalloc(uint32_t n, uint32_t t, uint8_t* d_received, size_t shard_len,
                                        const uint8_t* positions, size_t e, void* stream) {
  if (!pow2(n) || n < 2 || n > 256) return fail(AFRS_EINVAL, "n=%u must be a power of two in [2, 256]", n);
  if (!pow2(t) || t >= n) return fail(AFRS_EINVAL, "t=%u must be a power of two below n=%u", t, n);
  if (e > t) return 0;
  if (e == 0) return 1;
  if (!positions) return fail(AFRS_EINVAL, "positions is NULL with e=%zu", e);
  bool seen[256] = {};
  for (size_t i = 0; i < e; i++) {
    if (positions[i] >= n) return fail(AFRS_EINVAL, "erasure position %u >= n=%u", positions[i], n);
    if (seen[positions[i]]) return fail(AFRS_EINVAL, "duplicate erasure position %u", positions[i]);
    seen[positions[i]] = true;
  }
  if (shard_len == 0) return 1;
  if (!d_received) return fail(AFRS_EINVAL, "NULL buffer");
  const size_t need = afrs::scratch_bytes_recover((int)n, shard_len);
  if (need > kNoAllocScratchBytes)
    return fail(AFRS_EINVAL,
                "shard_len=%zu with n=%u needs %zu bytes of scratch; this entry point has %zu "
                "(use afrs_recover_dev for larger shards)",
                shard_len, n, need, kNoAllocScratchBytes);
  uint32_t* p = nullptr;
  int r = setup_current_device(&p);
  if (r) return r;
  afrs::ScratchArena sc{nullptr, 0};
  if (need) sc = afrs::ScratchArena{p, kNoAllocScratchBytes};
  afrs::RecoverArgs a{};
  a.rx = d_received;
  a.L = shard_len;
  a.n = (int)n;
  a.t = (int)t;
  a.e = (int)e;
  std::memcpy(a.pos, positions, e);
  cudaError_t err = afrs::launch_recover_special(a, sc, static_cast<cudaStream_t>(stream));
  if (err != cudaSuccess) return fail(AFRS_ECUDA, "recover launch: %s", cudaGetErrorString(err));
  return 1;
}
