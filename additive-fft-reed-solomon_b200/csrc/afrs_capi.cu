// C ABI of libafrs_b200.so (declared in include/afrs.h).
#include <cuda.h>  // driver types for cuPointerGetAttribute (resolved at run time, not linked)
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/afrs.h"
#include "afrs_internal.h"

struct afrs_ctx {
  int device;
  cudaStream_t stream;
  uint8_t* scratch;  // device staging for the host-buffer entry points
  size_t scratch_bytes;
  uint32_t* work;  // bit-sliced intermediate rows of the phase kernels
  size_t work_bytes;
  size_t work_cap;  // largest phase scratch used per call (afrs_ctx_set_work_cap)
  int route;        // forced per-call route (afrs_ctx_set_route): -1 = tuned table
  cudaEvent_t work_free;  // recorded after each use of `work`
  // Descriptor tables of afrs_batch_dev, two slots so that one batch can be
  // prepared while the previous one runs.
  uint8_t* batch_dev[2];
  size_t batch_dev_bytes[2];
  uint8_t* batch_host[2];  // pinned staging of those tables
  size_t batch_host_bytes[2];
  cudaEvent_t batch_free[2];  // recorded after each batch of the slot
  uint32_t* grp_scratch[2];   // scratch of the slot's grouped launches
  size_t grp_scratch_bytes[2];
  // Streams on which the shape groups of a batch run concurrently, forked
  // from and joined back into the caller's stream.
  cudaStream_t grp_stream[4];
  cudaEvent_t grp_fork, grp_join[4];
  int batch_slot;
  // Staged host-buffer path: copy streams and per-slot events.
  cudaStream_t copy_in, copy_out;
  cudaEvent_t ev_in[2], ev_cmp[2], ev_out[2];
  size_t window_bytes, merge_bytes;  // staging parameters (afrs_ctx_set_staging)
  int direct_mode;                   // AFRS_HOST_* (afrs_ctx_set_staging)
  std::recursive_mutex mu;
};

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? AFRS_ENOMEM : AFRS_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

bool pow2(uint32_t v) { return v && !(v & (v - 1)); }

int check_nt(uint32_t n, uint32_t t) {
  if (!pow2(n) || n > 256 || n < 2) return fail(AFRS_EINVAL, "n=%u must be a power of two in [2, 256]", n);
  if (!pow2(t) || t >= n) return fail(AFRS_EINVAL, "t=%u must be a power of two below n=%u", t, n);
  return AFRS_OK;
}

// Positions must be distinct and < n; the reference leaves this unchecked
// (a duplicate gives a zero denominator there, codec.rs:457-462).
int check_positions(uint32_t n, const uint8_t* pos, size_t e) {
  if (e && !pos) return fail(AFRS_EINVAL, "positions is NULL with e=%zu", e);
  bool seen[256] = {};
  for (size_t i = 0; i < e; i++) {
    if (pos[i] >= n) return fail(AFRS_EINVAL, "erasure position %u >= n=%u", pos[i], n);
    if (seen[pos[i]]) return fail(AFRS_EINVAL, "duplicate erasure position %u", pos[i]);
    seen[pos[i]] = true;
  }
  return AFRS_OK;
}

// Makes `dev` current for the call.  cudaSetDevice runs at least once per
// host thread and device even when `dev` is already the thread's device: in
// a thread that has made no CUDA call yet it binds the device's context,
// without which cudaPointerGetAttributes reports page-locked memory without
// its device address.  After that it runs only when the device changes
// (it costs a fraction of a microsecond on every small call otherwise).
struct DeviceGuard {
  int prev = -1;
  bool moved = false;
  explicit DeviceGuard(int dev) {
    thread_local int bound = -1;
    cudaGetDevice(&prev);
    if (prev != dev || bound != dev) {
      cudaSetDevice(dev);
      bound = dev;
      moved = prev != dev;
    }
  }
  ~DeviceGuard() {
    if (moved && prev >= 0) cudaSetDevice(prev);
  }
};

cudaError_t ensure_scratch(afrs_ctx* c, size_t bytes) {
  if (bytes <= c->scratch_bytes) return cudaSuccess;
  if (c->scratch) cudaFree(c->scratch);
  c->scratch = nullptr;
  c->scratch_bytes = 0;
  cudaError_t e = cudaMalloc(&c->scratch, bytes);
  if (e == cudaSuccess) c->scratch_bytes = bytes;
  return e;
}

// Largest phase scratch a context keeps (the launchers batch columns beyond it).
constexpr size_t kWorkCap = (size_t)1 << 30;
// Smallest cap afrs_ctx_set_work_cap accepts: one colword of the largest
// recover (n = 256: two buffers of 256 rows x 32 bytes).
constexpr size_t kMinWorkCap = (size_t)16 << 10;

// Grows the context's phase scratch to min(need, kWorkCap) and orders this
// call after the previous user of the scratch (calls on different streams
// would otherwise share it concurrently).
bool capturing(cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(s, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone;
}

// Inside a stream capture (CUDA graphs) the scratch must already be large
// enough (one call of the same shape before capturing grows it), and the
// ordering of the context's users is the caller's: the capture records no
// dependency on work outside the graph.
cudaError_t acquire_work(afrs_ctx* c, size_t need, cudaStream_t s, afrs::ScratchArena* out) {
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  if (need > c->work_cap) need = c->work_cap;
  const size_t usable = std::min(c->work_bytes, c->work_cap);
  if (capturing(s)) {
    if (need > usable) return cudaErrorStreamCaptureUnsupported;
    *out = afrs::ScratchArena{c->work, usable};
    return cudaSuccess;
  }
  if (need > c->work_bytes) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return e;
    if (c->work) cudaFree(c->work);
    c->work = nullptr;
    c->work_bytes = 0;
    e = cudaMalloc(reinterpret_cast<void**>(&c->work), need);
    if (e != cudaSuccess) return e;
    c->work_bytes = need;
  }
  cudaError_t e = cudaStreamWaitEvent(s, c->work_free, 0);
  if (e != cudaSuccess) return e;
  *out = afrs::ScratchArena{c->work, std::min(c->work_bytes, c->work_cap)};
  return cudaSuccess;
}

cudaError_t release_work(afrs_ctx* c, cudaStream_t s) {
  return capturing(s) ? cudaSuccess : cudaEventRecord(c->work_free, s);
}

// Built-in routing, used where the tuned table (route.cu) has no entry:
// shapes where the one-launch generic kernel was measured faster per call
// than the specialised ones (B200, codewords up to 4 MiB): encodes with
// t = 16 and n >= 32 (n = 32, 1 KiB shards: 6.2 vs 27.6 us; n = 64: 10 vs
// 26.5 us; n = 256: 33 vs 44 us), and encodes with t >= 32 and n <= 64, where
// three phase launches cost more than the work (n = 64, t = 32, 1 KiB: 8.2
// vs 13.9 us).  Beyond 4 MiB the generic kernel's time grows with the bytes
// and the specialised ones win (n = 32, t = 16, 1 MiB shards: 68 vs 28 us).
bool generic_encode_wins(const afrs::EncodeArgs& a) {
  if ((size_t)a.n * a.L > ((size_t)4 << 20)) return false;
  return a.t <= 16 ? a.t == 16 && a.n >= 32 : a.n <= 64;
}

// Route of one encode: the context's forced route, else the tuned table,
// else the built-in rule.  The generic kernel takes compact rows only.
int encode_route(const afrs_ctx* c, const afrs::EncodeArgs& a) {
  const bool compact = !a.pitch || a.pitch == a.L;
  int r = c->route >= 0 && c->route != afrs::kRouteFew ? c->route : afrs::route_encode(a.n, a.t, a.L);
  if (r < 0) return compact && generic_encode_wins(a) ? afrs::kRouteGeneric : -1;
  if (r == afrs::kRouteFused && !afrs::fused_encode_shape(a.n, a.t)) return afrs::kRouteSpecial;
  return r == afrs::kRouteGeneric && !compact ? afrs::kRouteSpecial : r;
}

int launch_encode(afrs_ctx* c, const afrs::EncodeArgs& a0, cudaStream_t s) {
  const int route = encode_route(c, a0);
  if (route == afrs::kRouteGeneric) {
    cudaError_t e = afrs::launch_encode_generic(a0, s);
    return e == cudaSuccess ? AFRS_OK : cuda_fail(e, "encode launch");
  }
  afrs::EncodeArgs a = a0;
  if (route >= 0)  // else the launcher's rule
    a.layout = route == afrs::kRouteSpecialSplit ? 1 : (route == afrs::kRouteFused ? afrs::kLayoutFused : 0);
  afrs::ScratchArena sc{nullptr, 0};
  cudaError_t e = cudaSuccess;
  const size_t need = route == afrs::kRouteFused ? 0 : afrs::scratch_bytes_encode(a.n, a.t, a.L);
  if (need && (e = acquire_work(c, need, s, &sc)) != cudaSuccess) return cuda_fail(e, "encode scratch");
  e = afrs::launch_encode_special(a, sc, s);
  if (e == cudaErrorNotSupported) e = afrs::launch_encode_generic(a, s);
  if (need && e == cudaSuccess) e = release_work(c, s);
  return e == cudaSuccess ? AFRS_OK : cuda_fail(e, "encode launch");
}

// Built-in rule where the table has no entry: recovers with n = 16 up to
// 4 MiB take the one-launch generic kernel (1 KiB shards: 10.3 vs 24.6 us;
// 256 KiB: 24.7 vs 26.9 us; 1 MiB: 74 vs 27 us).
bool generic_recover_wins(const afrs::RecoverArgs& a) {
  return a.n == 16 && (size_t)a.n * a.L <= ((size_t)4 << 20);
}

// Recovers of few erasures take the few-erasure kernel where it is faster
// (few_recover_wins), or wherever it applies when the context forces it: one
// pass over the survivors with no scratch, where the Leopard form runs two
// n-point transforms whatever e is.
int recover_route(const afrs_ctx* c, const afrs::RecoverArgs& a) {
  const bool compact = !a.pitch || a.pitch == a.L;
  if (c->route == afrs::kRouteFew ? afrs::few_recover_shape(a.n, a.e)
                                  : c->route < 0 && afrs::few_recover_wins(a.n, a.e, a.L))
    return afrs::kRouteFew;
  int r = c->route >= 0 && c->route != afrs::kRouteFew ? c->route : afrs::route_recover(a.n, a.L);
  if (r < 0) r = generic_recover_wins(a) ? afrs::kRouteGeneric : afrs::kRouteSpecial;
  if (r == afrs::kRouteFused && !afrs::fused_recover_shape(a.n)) return afrs::kRouteSpecial;
  return r == afrs::kRouteGeneric && !compact ? afrs::kRouteSpecial : r;
}

int launch_recover(afrs_ctx* c, const afrs::RecoverArgs& a0, cudaStream_t s) {
  const int route = recover_route(c, a0);
  if (route == afrs::kRouteGeneric) {
    cudaError_t e = afrs::launch_recover_generic(a0, s);
    return e == cudaSuccess ? AFRS_OK : cuda_fail(e, "recover launch");
  }
  afrs::RecoverArgs a = a0;
  a.layout = route == afrs::kRouteFused ? afrs::kLayoutFused : (route == afrs::kRouteFew ? afrs::kLayoutFew : 0);
  afrs::ScratchArena sc{nullptr, 0};
  cudaError_t e = cudaSuccess;
  const size_t need =
      route == afrs::kRouteFused || route == afrs::kRouteFew ? 0 : afrs::scratch_bytes_recover(a.n, a.L);
  if (need && (e = acquire_work(c, need, s, &sc)) != cudaSuccess) return cuda_fail(e, "recover scratch");
  e = afrs::launch_recover_special(a, sc, s);
  if (e == cudaErrorNotSupported) e = afrs::launch_recover_generic(a, s);
  if (need && e == cudaSuccess) e = release_work(c, s);
  return e == cudaSuccess ? AFRS_OK : cuda_fail(e, "recover launch");
}


// Waits for all three streams (also on error paths, so that no copy still
// references the caller's buffers after the call returns).
cudaError_t drain(afrs_ctx* c) {
  cudaError_t a = cudaStreamSynchronize(c->copy_in);
  cudaError_t b = cudaStreamSynchronize(c->stream);
  cudaError_t d = cudaStreamSynchronize(c->copy_out);
  return a != cudaSuccess ? a : (b != cudaSuccess ? b : d);
}

// ---- direct path for page-locked host buffers -------------------------------
// Page-locked host memory that is mapped into the device's address space can
// be read and written by the kernels themselves over PCIe: the decoder then
// reads exactly the surviving shards and writes exactly the erased ones (the
// encoder: message in, parity out), with no staging copies at all.  A range
// qualifies only if it lies inside one such allocation (checked with the
// driver's allocation-range attributes); anything else takes the staged path.
using PtrAttrFn = CUresult (*)(void*, CUpointer_attribute, CUdeviceptr);

PtrAttrFn ptr_attr_fn() {
  static PtrAttrFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      f = nullptr;
    }
    return reinterpret_cast<PtrAttrFn>(f);
  }();
  return fn;
}

// Device address of host range [p, p + bytes) when the kernels may access it
// directly, nullptr otherwise.
uint8_t* mapped_host_range(const void* p, size_t bytes) {
  PtrAttrFn fn = ptr_attr_fn();
  if (!fn || !p || !bytes) return nullptr;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
  CUdeviceptr start = 0;
  size_t size = 0;
  const CUdeviceptr hp = (CUdeviceptr)(uintptr_t)p;
  if (fn(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, hp) != CUDA_SUCCESS ||
      fn(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, hp) != CUDA_SUCCESS)
    return nullptr;
  if (hp < start || hp - start > size || bytes > size - (hp - start)) return nullptr;
  return static_cast<uint8_t*>(a.devicePointer);
}

// Runs `launch(args, arena, stream)` over column windows of the whole shard
// width: up to kDirectWindows windows of the same rows (pitch = full shard
// length) alternate between two streams, each with half of the scratch, so
// that one window's reads of host memory overlap another's writes.
constexpr int kDirectWindows = 4;

template <class Args, class Need, class Shift, class Launch>
int run_direct(afrs_ctx* c, const Args& a, Need need_for, Shift shift, Launch launch, const char* what) {
  const size_t L = a.L;
  size_t W = L;
  if (L >= 4096) W = ((L + kDirectWindows - 1) / kDirectWindows + 1023) / 1024 * 1024;
  const size_t need1 = need_for(W);
  cudaStream_t s0 = c->stream, s1 = c->copy_in;
  afrs::ScratchArena sc{nullptr, 0};
  cudaError_t e = cudaSuccess;
  if (need1 && (e = acquire_work(c, 2 * need1, s0, &sc)) != cudaSuccess) return cuda_fail(e, what);
  const size_t half = (sc.bytes / 2) & ~(size_t)255;
  const bool two = W < L && (!need1 || half >= need1);
  if (two && ((e = cudaEventRecord(c->ev_in[0], s0)) != cudaSuccess ||
              (e = cudaStreamWaitEvent(s1, c->ev_in[0], 0)) != cudaSuccess))
    return cuda_fail(e, what);
  int idx = 0;
  for (size_t c0 = 0; c0 < L && e == cudaSuccess; c0 += W, idx++) {
    const int k = two ? (idx & 1) : 0;
    Args w = a;
    shift(w, c0);
    w.L = (L - c0 < W) ? L - c0 : W;
    w.pitch = L;
    afrs::ScratchArena sub{nullptr, 0};
    if (need1) {
      sub.ptr = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(sc.ptr) + (size_t)k * half);
      sub.bytes = two ? half : sc.bytes;
    }
    e = launch(w, sub, k ? s1 : s0);
  }
  cudaError_t e2 = cudaSuccess;
  if (two && (e2 = cudaEventRecord(c->ev_in[1], s1)) == cudaSuccess) e2 = cudaStreamWaitEvent(s0, c->ev_in[1], 0);
  if (need1 && e2 == cudaSuccess) e2 = release_work(c, s0);
  cudaError_t e3 = drain(c);
  if (e == cudaSuccess) e = e2 != cudaSuccess ? e2 : e3;
  return e == cudaSuccess ? AFRS_OK : cuda_fail(e, what);
}

// ---- staged host-buffer path (afrs_encode, afrs_recover) -------------------
// The shard columns are cut into windows of W columns.  Window i uses staging
// slot i % 2 (a compact n x w block of device memory) and three streams:
// copy_in (host -> slot, only the rows the operation reads), the context
// stream (kernels, with shard_len = w) and copy_out (slot -> host, only the
// rows it writes).  Copy-in of window i+1 overlaps the kernels of window i and
// the copy-out of window i-1, and the two PCIe directions run at once; with
// page-locked caller buffers the copies are DMA straight to and from them.
// Rows move as runs of adjacent rows, one 2D copy per run (host pitch L,
// device pitch w); runs closer than kMergeBytes are merged and the rows in
// between are copied too, which is harmless: the decoder does not read
// erased rows, and survivor rows copied back hold the bytes they came with.
std::atomic<uint64_t> g_h2d_bytes{0}, g_d2h_bytes{0};

constexpr int kSlots = 2;
constexpr size_t kWindowBytes = (size_t)4 << 20;  // default n * W per window
constexpr size_t kMergeBytes = (size_t)128 << 10;  // default gap merged into a run

size_t window_cols(const afrs_ctx* c, uint32_t n, size_t L) {
  size_t W = c->window_bytes / n / 1024 * 1024;
  if (W < 1024) W = 1024;
  return W >= L ? L : W;
}

struct RowRun {
  uint32_t r0, rows;
};

// Runs of rows with sel[r] set, gaps of at most merge_bytes / w rows merged.
std::vector<RowRun> row_runs(const bool* sel, uint32_t n, size_t w, size_t merge_bytes) {
  std::vector<RowRun> runs;
  const size_t max_gap = w ? merge_bytes / w : 0;
  for (uint32_t r = 0; r < n; r++) {
    if (!sel[r]) continue;
    if (!runs.empty()) {
      RowRun& b = runs.back();
      const uint32_t end = b.r0 + b.rows;
      if (r - end <= max_gap) {
        b.rows = r + 1 - b.r0;
        continue;
      }
    }
    runs.push_back(RowRun{r, 1});
  }
  return runs;
}

cudaError_t copy_rows_h2d(uint8_t* dev, size_t w, const uint8_t* host, size_t L, size_t c0,
                          const std::vector<RowRun>& runs, cudaStream_t s) {
  for (const RowRun& q : runs) {
    cudaError_t e = cudaMemcpy2DAsync(dev + (size_t)q.r0 * w, w, host + (size_t)q.r0 * L + c0, L, w, q.rows,
                                      cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    g_h2d_bytes.fetch_add((uint64_t)w * q.rows, std::memory_order_relaxed);
  }
  return cudaSuccess;
}

cudaError_t copy_rows_d2h(uint8_t* host, size_t L, size_t c0, const uint8_t* dev, size_t w,
                          const std::vector<RowRun>& runs, cudaStream_t s) {
  for (const RowRun& q : runs) {
    cudaError_t e = cudaMemcpy2DAsync(host + (size_t)q.r0 * L + c0, L, dev + (size_t)q.r0 * w, w, w, q.rows,
                                      cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return e;
    g_d2h_bytes.fetch_add((uint64_t)w * q.rows, std::memory_order_relaxed);
  }
  return cudaSuccess;
}


// Runs `body(slot_base, w, c0)` per window with the copies around it.
// `in` / `out` describe the host rows (a codeword of `rows` rows) to stage.
template <class Launch>
int staged(afrs_ctx* c, uint32_t rows, size_t L, const uint8_t* h_in, const bool* sel_in, uint8_t* h_out,
           const bool* sel_out, Launch&& launch) {
  const size_t W = window_cols(c, rows, L);
  cudaError_t e = ensure_scratch(c, (size_t)kSlots * rows * W);
  if (e != cudaSuccess) return cuda_fail(e, "staging allocation");
  int slot = 0;
  for (size_t c0 = 0; c0 < L; c0 += W, slot ^= 1) {
    const size_t w = (L - c0 < W) ? L - c0 : W;
    uint8_t* base = c->scratch + (size_t)slot * rows * W;
    const std::vector<RowRun> rin = row_runs(sel_in, rows, w, c->merge_bytes),
                              rout = row_runs(sel_out, rows, w, c->merge_bytes);
    int r = AFRS_OK;
    if ((e = cudaStreamWaitEvent(c->copy_in, c->ev_out[slot], 0)) == cudaSuccess &&
        (e = copy_rows_h2d(base, w, h_in, L, c0, rin, c->copy_in)) == cudaSuccess &&
        (e = cudaEventRecord(c->ev_in[slot], c->copy_in)) == cudaSuccess &&
        (e = cudaStreamWaitEvent(c->stream, c->ev_in[slot], 0)) == cudaSuccess) {
      r = launch(base, w);
      if (r == AFRS_OK && (e = cudaEventRecord(c->ev_cmp[slot], c->stream)) == cudaSuccess &&
          (e = cudaStreamWaitEvent(c->copy_out, c->ev_cmp[slot], 0)) == cudaSuccess &&
          (e = copy_rows_d2h(h_out, L, c0, base, w, rout, c->copy_out)) == cudaSuccess)
        e = cudaEventRecord(c->ev_out[slot], c->copy_out);
    }
    if (r != AFRS_OK || e != cudaSuccess) {
      drain(c);
      return r != AFRS_OK ? r : cuda_fail(e, "staged copy");
    }
  }
  if ((e = drain(c)) != cudaSuccess) return cuda_fail(e, "staged operation");
  return AFRS_OK;
}

}  // namespace

namespace afrs {
void set_last_error(const char* msg) { snprintf(g_err, sizeof g_err, "%s", msg); }
std::atomic<uint64_t> g_launches{0};
void count_launches(unsigned k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
}  // namespace afrs

extern "C" {

const char* afrs_last_error(void) { return g_err; }

int afrs_ctx_set_staging(afrs_ctx* c, size_t window_bytes, size_t merge_bytes, int host_mode) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  if (host_mode < AFRS_HOST_AUTO || host_mode > AFRS_HOST_DIRECT)
    return fail(AFRS_EINVAL, "host_mode %d is not an AFRS_HOST_* value", host_mode);
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  c->direct_mode = host_mode;
  c->window_bytes = window_bytes ? window_bytes : kWindowBytes;
  c->merge_bytes = merge_bytes == (size_t)-1 ? 0 : (merge_bytes ? merge_bytes : kMergeBytes);
  return AFRS_OK;
}

int afrs_ctx_set_work_cap(afrs_ctx* c, size_t bytes) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  if (bytes && bytes < kMinWorkCap)
    return fail(AFRS_EINVAL, "work cap %zu is below the %zu-byte minimum", bytes, kMinWorkCap);
  if (bytes > kWorkCap) return fail(AFRS_EINVAL, "work cap %zu is above the %zu-byte maximum", bytes, kWorkCap);
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  c->work_cap = bytes ? bytes & ~(size_t)255 : kWorkCap;
  return AFRS_OK;
}

int afrs_ctx_set_route(afrs_ctx* c, int route) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  if (route < AFRS_ROUTE_TABLE || route > AFRS_ROUTE_FEW)
    return fail(AFRS_EINVAL, "route %d is not an AFRS_ROUTE_* value", route);
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  c->route = route == AFRS_ROUTE_TABLE ? -1 : route - AFRS_ROUTE_GENERIC;
  return AFRS_OK;
}

uint64_t afrs_kernel_launches(void) { return afrs::g_launches.load(std::memory_order_relaxed); }

void afrs_staged_bytes(uint64_t* h2d, uint64_t* d2h) {
  if (h2d) *h2d = g_h2d_bytes.load(std::memory_order_relaxed);
  if (d2h) *d2h = g_d2h_bytes.load(std::memory_order_relaxed);
}

const char* afrs_version(void) { return "afrs_b200 0.1 sm_100a (bit-sliced GF(2^8) additive FFT)"; }

int afrs_ctx_create(int device, afrs_ctx** out) {
  if (!out) return fail(AFRS_EINVAL, "out is NULL");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
  if (device < 0 || device >= count) return fail(AFRS_EINVAL, "device %d out of range (%d devices)", device, count);
  DeviceGuard g(device);
  afrs_ctx* c = new (std::nothrow) afrs_ctx;
  if (!c) return fail(AFRS_ENOMEM, "context allocation");
  c->device = device;
  c->scratch = nullptr;
  c->scratch_bytes = 0;
  c->work = nullptr;
  c->work_bytes = 0;
  c->work_cap = kWorkCap;
  c->route = -1;
  for (int i = 0; i < 2; i++) {
    c->batch_dev[i] = nullptr;
    c->batch_dev_bytes[i] = 0;
    c->batch_host[i] = nullptr;
    c->batch_host_bytes[i] = 0;
    c->grp_scratch[i] = nullptr;
    c->grp_scratch_bytes[i] = 0;
  }
  c->batch_slot = 0;
  c->window_bytes = kWindowBytes;
  c->merge_bytes = kMergeBytes;
  c->direct_mode = AFRS_HOST_AUTO;
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return cuda_fail(e, "cudaStreamCreate");
  }
  e = cudaEventCreateWithFlags(&c->work_free, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->batch_free[0], cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->batch_free[1], cudaEventDisableTiming);
  for (int i = 0; i < 2 && e == cudaSuccess; i++) {
    e = cudaEventCreateWithFlags(&c->ev_in[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_cmp[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_out[i], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy_in, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->grp_fork, cudaEventDisableTiming);
  for (int i = 0; i < 4 && e == cudaSuccess; i++) {
    e = cudaStreamCreateWithFlags(&c->grp_stream[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->grp_join[i], cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy_out, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    delete c;
    return cuda_fail(e, "cudaEventCreate");
  }
  *out = c;
  return AFRS_OK;
}

void afrs_ctx_destroy(afrs_ctx* c) {
  if (!c) return;
  DeviceGuard g(c->device);
  cudaDeviceSynchronize();
  if (c->scratch) cudaFree(c->scratch);
  if (c->work) cudaFree(c->work);
  for (int i = 0; i < 2; i++) {
    if (c->batch_dev[i]) cudaFree(c->batch_dev[i]);
    if (c->batch_host[i]) cudaFreeHost(c->batch_host[i]);
    if (c->grp_scratch[i]) cudaFree(c->grp_scratch[i]);
    cudaEventDestroy(c->batch_free[i]);
  }
  cudaEventDestroy(c->work_free);
  for (int i = 0; i < 2; i++) {
    cudaEventDestroy(c->ev_in[i]);
    cudaEventDestroy(c->ev_cmp[i]);
    cudaEventDestroy(c->ev_out[i]);
  }
  cudaStreamDestroy(c->copy_in);
  for (int i = 0; i < 4; i++) {
    cudaStreamDestroy(c->grp_stream[i]);
    cudaEventDestroy(c->grp_join[i]);
  }
  cudaEventDestroy(c->grp_fork);
  cudaStreamDestroy(c->copy_out);
  cudaStreamDestroy(c->stream);
  delete c;
}

int afrs_encode_dev(afrs_ctx* c, uint32_t n, uint32_t t, const uint8_t* d_message, uint8_t* d_parity,
                    size_t L, int accumulate, void* stream) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  int r = check_nt(n, t);
  if (r) return r;
  if (L == 0) return AFRS_OK;
  if (!d_message || !d_parity) return fail(AFRS_EINVAL, "NULL buffer");
  DeviceGuard g(c->device);
  afrs::EncodeArgs a{d_message, d_parity, L, (int)n, (int)t, accumulate ? 1 : 0};
  return launch_encode(c, a, static_cast<cudaStream_t>(stream));
}

int afrs_recover_dev(afrs_ctx* c, uint32_t n, uint32_t t, uint8_t* d_received, size_t L,
                     const uint8_t* positions, size_t e, void* stream) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  int r = check_nt(n, t);
  if (r) return r;
  if (e > t) return 0;
  if (e == 0) return 1;
  r = check_positions(n, positions, e);
  if (r) return r;
  if (L == 0) return 1;
  if (!d_received) return fail(AFRS_EINVAL, "NULL buffer");
  DeviceGuard g(c->device);
  afrs::RecoverArgs a{};
  a.rx = d_received;
  a.L = L;
  a.n = (int)n;
  a.t = (int)t;
  a.e = (int)e;
  std::memcpy(a.pos, positions, e);
  r = launch_recover(c, a, static_cast<cudaStream_t>(stream));
  return r ? r : 1;
}

int afrs_encode(afrs_ctx* c, uint32_t n, uint32_t t, const uint8_t* message, uint8_t* parity, size_t L,
                int accumulate) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  int r = check_nt(n, t);
  if (r) return r;
  if (L == 0) return AFRS_OK;
  if (!message || !parity) return fail(AFRS_EINVAL, "NULL buffer");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  DeviceGuard g(c->device);
  const uint32_t k = n - t;
  {
    const bool want = c->direct_mode == AFRS_HOST_DIRECT;
    uint8_t* dm = want ? mapped_host_range(message, (size_t)k * L) : nullptr;
    uint8_t* dp = dm ? mapped_host_range(parity, (size_t)t * L) : nullptr;
    if (dm && dp) {
      afrs::EncodeArgs a{dm, dp, L, (int)n, (int)t, accumulate ? 1 : 0};
      r = run_direct(
          c, a, [&](size_t W) { return afrs::scratch_bytes_encode((int)n, (int)t, W); },
          [](afrs::EncodeArgs& w, size_t c0) {
            w.msg += c0;
            w.parity += c0;
          },
          [](const afrs::EncodeArgs& w, const afrs::ScratchArena& sc, cudaStream_t s) {
            return afrs::launch_encode_special(w, sc, s);
          },
          "encode (page-locked buffers)");
      if (r) return r;
      g_h2d_bytes.fetch_add((uint64_t)(accumulate ? n : k) * L, std::memory_order_relaxed);
      g_d2h_bytes.fetch_add((uint64_t)t * L, std::memory_order_relaxed);
      return AFRS_OK;
    }
  }
  // Staged as one n-row block per window: message rows 0..k-1, parity rows
  // k..n-1.  The message and parity host buffers are separate, so each is
  // its own 2D copy.
  bool sel_msg[256] = {}, sel_par[256] = {};
  for (uint32_t r0 = 0; r0 < k; r0++) sel_msg[r0] = true;
  for (uint32_t r0 = 0; r0 < t; r0++) sel_par[r0] = true;
  const size_t W = window_cols(c, n, L);
  cudaError_t e = ensure_scratch(c, (size_t)kSlots * n * W);
  if (e != cudaSuccess) return cuda_fail(e, "staging allocation");
  int slot = 0;
  for (size_t c0 = 0; c0 < L; c0 += W, slot ^= 1) {
    const size_t w = (L - c0 < W) ? L - c0 : W;
    uint8_t* dm = c->scratch + (size_t)slot * n * W;
    uint8_t* dp = dm + (size_t)k * w;
    const std::vector<RowRun> rm = row_runs(sel_msg, k, w, c->merge_bytes),
                              rp = row_runs(sel_par, t, w, c->merge_bytes);
    r = AFRS_OK;
    if ((e = cudaStreamWaitEvent(c->copy_in, c->ev_out[slot], 0)) == cudaSuccess &&
        (e = copy_rows_h2d(dm, w, message, L, c0, rm, c->copy_in)) == cudaSuccess &&
        (!accumulate || (e = copy_rows_h2d(dp, w, parity, L, c0, rp, c->copy_in)) == cudaSuccess) &&
        (e = cudaEventRecord(c->ev_in[slot], c->copy_in)) == cudaSuccess &&
        (e = cudaStreamWaitEvent(c->stream, c->ev_in[slot], 0)) == cudaSuccess) {
      afrs::EncodeArgs a{dm, dp, w, (int)n, (int)t, accumulate ? 1 : 0};
      r = launch_encode(c, a, c->stream);
      if (r == AFRS_OK && (e = cudaEventRecord(c->ev_cmp[slot], c->stream)) == cudaSuccess &&
          (e = cudaStreamWaitEvent(c->copy_out, c->ev_cmp[slot], 0)) == cudaSuccess &&
          (e = copy_rows_d2h(parity, L, c0, dp, w, rp, c->copy_out)) == cudaSuccess)
        e = cudaEventRecord(c->ev_out[slot], c->copy_out);
    }
    if (r != AFRS_OK || e != cudaSuccess) {
      drain(c);
      return r != AFRS_OK ? r : cuda_fail(e, "encode staging");
    }
  }
  if ((e = drain(c)) != cudaSuccess) return cuda_fail(e, "encode");
  return AFRS_OK;
}

int afrs_recover(afrs_ctx* c, uint32_t n, uint32_t t, uint8_t* received, size_t L, const uint8_t* positions,
                 size_t e_count) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  int r = check_nt(n, t);
  if (r) return r;
  if (e_count > t) return 0;
  if (e_count == 0) return 1;
  r = check_positions(n, positions, e_count);
  if (r) return r;
  if (L == 0) return 1;
  if (!received) return fail(AFRS_EINVAL, "NULL buffer");
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  DeviceGuard g(c->device);
  // In: the surviving shards (the decoder reads no erased row).  Out: the
  // erased shards, the only ones that change.
  bool erased[256] = {}, survivor[256] = {};
  for (size_t j = 0; j < e_count; j++) erased[positions[j]] = true;
  for (uint32_t r0 = 0; r0 < n; r0++) survivor[r0] = !erased[r0];
  afrs::RecoverArgs a{};
  a.n = (int)n;
  a.t = (int)t;
  a.e = (int)e_count;
  std::memcpy(a.pos, positions, e_count);
  uint8_t* drx = c->direct_mode != AFRS_HOST_STAGED ? mapped_host_range(received, (size_t)n * L) : nullptr;
  if (drx) {
    a.rx = drx;
    a.L = L;
    // The few-erasure kernel, which the launcher takes where it wins, needs
    // no scratch.
    r = run_direct(
        c, a,
        [&](size_t W) {
          return afrs::few_recover_wins((int)n, (int)e_count, W) ? 0 : afrs::scratch_bytes_recover((int)n, W);
        },
        [](afrs::RecoverArgs& w, size_t c0) { w.rx += c0; },
        [](const afrs::RecoverArgs& w, const afrs::ScratchArena& sc, cudaStream_t s) {
          return afrs::launch_recover_special(w, sc, s);
        },
        "recover (page-locked buffers)");
    if (r) return r;
    g_h2d_bytes.fetch_add((uint64_t)(n - e_count) * L, std::memory_order_relaxed);
    g_d2h_bytes.fetch_add((uint64_t)e_count * L, std::memory_order_relaxed);
    return 1;
  }
  r = staged(c, n, L, received, survivor, received, erased, [&](uint8_t* base, size_t w) {
    a.rx = base;
    a.L = w;
    return launch_recover(c, a, c->stream);
  });
  return r == AFRS_OK ? 1 : r;
}

int afrs_recompute_data_from_parity_dev(afrs_ctx* c, uint32_t n, uint32_t t, uint8_t* d_received, size_t L,
                                        void* stream) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  int r = check_nt(n, t);
  if (r) return r;
  if (n != 2 * t) return fail(AFRS_EINVAL, "recompute needs n == 2t (n=%u, t=%u)", n, t);
  if (L == 0) return AFRS_OK;
  if (!d_received) return fail(AFRS_EINVAL, "NULL buffer");
  DeviceGuard g(c->device);
  cudaError_t e = afrs::launch_recompute_generic(d_received, L, (int)t, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? AFRS_OK : cuda_fail(e, "recompute launch");
}

static int transform_dev(afrs_ctx* c, uint8_t* d, size_t L, uint32_t k, uint8_t beta, bool inverse, void* stream) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  if (k > 8) return fail(AFRS_EINVAL, "k=%u must be in 0..=8", k);
  if (L == 0) return AFRS_OK;
  if (!d) return fail(AFRS_EINVAL, "NULL buffer");
  DeviceGuard g(c->device);
  cudaError_t e = afrs::launch_transform_generic(d, L, (int)k, beta, inverse, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? AFRS_OK : cuda_fail(e, "transform launch");
}

// Syndrome (codec.rs:269-301, sharded): XOR_i IFFT_t(chunk i, omega_it) =
// IFFT_t(parity) + acc with acc = XOR_{i>=1} IFFT_t(chunk i, omega_it), and
// the encoder gives E = FFT_t(acc), so the syndrome is IFFT_t(parity + E, 0):
// one encode (the fast kernels), one XOR pass and one t-point IFFT.
int afrs_syndrome_dev(afrs_ctx* c, uint32_t n, uint32_t t, const uint8_t* d_received, size_t L, uint8_t* d_syndrome,
                      unsigned long long* d_nonzero, void* stream) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  int r = check_nt(n, t);
  if (r) return r;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceGuard g(c->device);
  cudaError_t e;
  if (d_nonzero && (e = cudaMemsetAsync(d_nonzero, 0, sizeof(unsigned long long), s)) != cudaSuccess)
    return cuda_fail(e, "syndrome count reset");
  if (L == 0) return AFRS_OK;
  if (!d_received || !d_syndrome) return fail(AFRS_EINVAL, "NULL buffer");
  const size_t pb = (size_t)t * L;
  if (d_syndrome < d_received + (size_t)n * L && d_received < d_syndrome + pb)
    return fail(AFRS_EINVAL, "d_syndrome overlaps d_received");
  afrs::EncodeArgs a{d_received + pb, d_syndrome, L, (int)n, (int)t, 0};
  if ((r = launch_encode(c, a, s))) return r;
  if ((e = afrs::launch_xor_into(d_syndrome, d_received, pb, s)) != cudaSuccess) return cuda_fail(e, "syndrome xor");
  int k = 0;
  while ((1u << k) < t) k++;
  if (k > 0 && (e = afrs::launch_transform_generic(d_syndrome, L, k, 0, true, s)) != cudaSuccess)
    return cuda_fail(e, "syndrome ifft");
  if (d_nonzero && (e = afrs::launch_count_nonzero(d_syndrome, pb, d_nonzero, s)) != cudaSuccess)
    return cuda_fail(e, "syndrome count");
  return AFRS_OK;
}

int afrs_fft_sharded_dev(afrs_ctx* c, uint8_t* d, size_t L, uint32_t k, uint8_t beta, void* stream) {
  return transform_dev(c, d, L, k, beta, false, stream);
}

int afrs_ifft_sharded_dev(afrs_ctx* c, uint8_t* d, size_t L, uint32_t k, uint8_t beta, void* stream) {
  return transform_dev(c, d, L, k, beta, true, stream);
}

int afrs_scale_dev(afrs_ctx* c, const uint8_t* src, uint8_t* dst, size_t len, uint8_t scalar, void* stream) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  if (len == 0) return AFRS_OK;
  if (!src || !dst) return fail(AFRS_EINVAL, "NULL buffer");
  DeviceGuard g(c->device);
  cudaError_t e = afrs::launch_scale(src, dst, len, scalar, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? AFRS_OK : cuda_fail(e, "scale launch");
}

}  // extern "C"

namespace {

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

constexpr size_t kGroupScratchCap = (size_t)1 << 30;
// Smallest shape group (sum of n * shard_len) worth its own launches; a
// few-erasure group needs no scratch and is one launch.
constexpr size_t kGroupMinBytes = (size_t)8 << 20;
constexpr size_t kFewGroupMinBytes = (size_t)1 << 20;

// A job of a batch that runs through the grouped phase kernels.  The
// grouped scratch is reused in rounds: the jobs of one round hold at most
// kGroupScratchCap bytes of it, and a round starts once every group stream
// has finished the previous one.
struct GroupedJob {
  size_t job;      // index into the caller's array
  int op, n, t;    // shape key (op 2, few-erasure recover: t = log2 of its chunk size)
  size_t scratch;  // byte offset in the batch's grouped scratch
  int round;       // scratch round
  size_t few;      // op 2: offset of its descriptor in BatchPrep::few_desc
};

// One batch prepared on the host: which jobs run where, and the layout of
// its device tables (descriptors of the generic persistent kernel, then one
// descriptor array per shape group, then the task counter and the locator
// table, which are written on the device).
struct BatchPrep {
  std::vector<size_t> valid;  // accepted jobs (status set to queued)
  std::vector<afrs::BatchJob> bj;
  std::vector<uint2> tasks;
  std::vector<int> rec;
  std::vector<uint8_t> pos;
  std::vector<GroupedJob> grouped;
  std::vector<uint8_t> few_desc;  // descriptors of the few-erasure recovers
  struct Group {
    int op, n, t;
    size_t first, count, desc_off, max_ncw;
    int round;
  };
  std::vector<Group> groups;
  int rounds = 0;
  size_t grp_bytes = 0;  // grouped scratch (the largest round)
  int max_rows = 0;
  size_t o_jobs = 0, o_tasks = 0, o_rec = 0, o_pos = 0, o_cnt = 0, o_loc = 0;
  size_t upload = 0;  // bytes the host writes
  size_t total = 0;   // device table bytes
  bool empty() const { return bj.empty() && grouped.empty(); }
};

// Validates the jobs (setting each one's status), groups them by shape and
// lays out the tables.  Returns AFRS_OK or a negative code.
int batch_prepare(afrs_job* jobs, size_t count, BatchPrep* p) {
  for (size_t i = 0; i < count; i++) {
    afrs_job& j = jobs[i];
    j.status = AFRS_EINVAL;
    if (j.op != AFRS_OP_ENCODE && j.op != AFRS_OP_RECOVER) continue;
    if (!pow2(j.n) || j.n < 2 || j.n > 256 || !pow2(j.t) || j.t >= j.n) continue;
    const bool enc = j.op == AFRS_OP_ENCODE;
    if (!enc) {
      if (j.e > j.t) {
        j.status = 0;
        continue;
      }
      bool seen[256] = {}, ok = true;
      for (uint32_t q = 0; q < j.e; q++) {
        if (j.positions[q] >= j.n || seen[j.positions[q]]) ok = false;
        else seen[j.positions[q]] = true;
      }
      if (!ok) continue;
      if (j.e == 0 || j.shard_len == 0) {
        j.status = 1;
        continue;
      }
      if (!j.dst) continue;
    } else {
      if (j.shard_len == 0) {
        j.status = 0;
        continue;
      }
      if (!j.src || !j.dst) continue;
    }
    j.status = enc ? 0 : 1;
    p->valid.push_back(i);
  }
  // A shape group (encode: n, t; recover: n) runs on the specialised kernels
  // when it holds enough bytes to fill the GPU; its jobs take scratch in
  // rounds of at most kGroupScratchCap bytes, assigned in shape order so that
  // a group spans few rounds.  The rest (small groups, shapes without grouped
  // kernels, a job whose scratch alone exceeds the cap) share one launch of
  // the generic persistent kernel, which runs concurrently with the groups.
  // Recovers of at most 8 erasures with n >= 32 form their own groups (op 2,
  // keyed by n and the chunk size 2^ceil(log2 e)) on the few-erasure kernel.
  auto key = [&](const afrs_job& j) {
    if (j.op == AFRS_OP_ENCODE) return std::make_tuple(0, (int)j.n, (int)j.t);
    if (!afrs::few_recover_shape((int)j.n, (int)j.e)) return std::make_tuple(1, (int)j.n, 0);
    int lt = 0;
    while ((1u << lt) < j.e) lt++;
    return std::make_tuple(2, (int)j.n, lt);
  };
  std::map<std::tuple<int, int, int>, size_t> group_bytes;
  for (size_t i : p->valid) group_bytes[key(jobs[i])] += (size_t)jobs[i].n * jobs[i].shard_len;
  std::vector<size_t> order(p->valid);
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return key(jobs[x]) < key(jobs[y]); });
  std::vector<bool> grouped(count, false);
  size_t round_bytes = 0;
  for (size_t i : order) {
    const afrs_job& j = jobs[i];
    const int op = std::get<0>(key(j));
    if (!afrs::jobs_supported(op, (int)j.n, (int)j.t) ||
        group_bytes[key(j)] < (op == 2 ? kFewGroupMinBytes : kGroupMinBytes))
      continue;
    size_t few = 0;
    if (op == 2) {
      afrs::RecoverArgs a{};
      a.rx = j.dst;
      a.L = j.shard_len;
      a.n = (int)j.n;
      a.t = (int)j.t;
      a.e = (int)j.e;
      std::memcpy(a.pos, j.positions, j.e);
      few = p->few_desc.size();
      p->few_desc.resize(few + afrs::job_desc_bytes(2));
      if (!afrs::fill_few_job(p->few_desc.data() + few, a)) {
        p->few_desc.resize(few);
        continue;
      }
    }
    const size_t need = align256(afrs::job_scratch_bytes(op, (int)j.n, (int)j.t, j.shard_len));
    if (need > kGroupScratchCap) continue;
    if (round_bytes + need > kGroupScratchCap) {
      p->rounds++;
      round_bytes = 0;
    }
    p->grouped.push_back(GroupedJob{i, op, (int)j.n, std::get<2>(key(j)), round_bytes, p->rounds, few});
    round_bytes += need;
    p->grp_bytes = std::max(p->grp_bytes, round_bytes);
    grouped[i] = true;
  }
  if (!p->grouped.empty()) p->rounds++;
  for (size_t i : p->valid) {
    if (grouped[i]) continue;
    const afrs_job& j = jobs[i];
    const bool enc = j.op == AFRS_OP_ENCODE;
    const int op = enc ? 0 : 1;
    afrs::BatchJob b{};
    b.src = j.src;
    b.dst = j.dst;
    b.L = j.shard_len;
    b.op = op;
    b.n = (int)j.n;
    b.t = (int)j.t;
    b.e = (int)j.e;
    b.pos_off = (uint32_t)p->pos.size();
    if (!enc) {
      b.loc = (uint32_t)p->rec.size();
      p->rec.push_back((int)p->bj.size());
      p->pos.insert(p->pos.end(), j.positions, j.positions + j.e);
      p->max_rows = std::max(p->max_rows, 2 * (int)j.n);
    } else {
      p->max_rows = std::max(p->max_rows, (int)j.t * ((int)(j.n / j.t) - 1 > 1 ? 2 : 1));
    }
    const size_t tiles = afrs::batch_tiles(j.shard_len);
    for (size_t q = 0; q < tiles; q++) p->tasks.push_back(make_uint2((unsigned)p->bj.size(), (unsigned)q));
    p->bj.push_back(b);
  }
  if (p->tasks.size() > (size_t)INT32_MAX) {
    for (size_t i : p->valid) jobs[i].status = AFRS_EINVAL;
    return fail(AFRS_EINVAL, "too many tiles");
  }
  // Jobs sorted by round and shape (stable: caller order within a shape);
  // the descriptors of one shape group of a round form one array.
  std::stable_sort(p->grouped.begin(), p->grouped.end(), [](const GroupedJob& x, const GroupedJob& y) {
    return std::make_tuple(x.round, x.op, x.n, x.t) < std::make_tuple(y.round, y.op, y.n, y.t);
  });
  p->o_jobs = 0;
  p->o_tasks = align256(p->o_jobs + p->bj.size() * sizeof(afrs::BatchJob));
  p->o_rec = align256(p->o_tasks + p->tasks.size() * sizeof(uint2));
  p->o_pos = align256(p->o_rec + p->rec.size() * sizeof(int));
  size_t o_grp = align256(p->o_pos + p->pos.size() + 1);
  auto& groups = p->groups;
  for (size_t q = 0; q < p->grouped.size(); q++) {
    const GroupedJob& g = p->grouped[q];
    if (groups.empty() || groups.back().op != g.op || groups.back().n != g.n || groups.back().t != g.t ||
        groups.back().round != g.round) {
      if (!groups.empty()) o_grp = align256(o_grp + groups.back().count * afrs::job_desc_bytes(groups.back().op));
      groups.push_back(BatchPrep::Group{g.op, g.n, g.t, q, 0, o_grp, 0, g.round});
    }
    groups.back().count++;
    groups.back().max_ncw = std::max(groups.back().max_ncw, afrs::job_colwords(jobs[g.job].shard_len));
  }
  if (!groups.empty()) o_grp = align256(o_grp + groups.back().count * afrs::job_desc_bytes(groups.back().op));
  p->o_cnt = o_grp;
  p->upload = p->o_cnt;  // the locator table and the counter are written on the device
  p->o_loc = align256(p->o_cnt + sizeof(unsigned));
  p->total = align256(p->o_loc + p->rec.size() * 768);
  return AFRS_OK;
}

// Writes the batch's tables (host staging h, p.upload bytes) for grouped
// scratch at device address `scratch`.
void batch_fill(const BatchPrep& p, const afrs_job* jobs, uint8_t* h, uint8_t* scratch) {
  if (!p.bj.empty()) std::memcpy(h + p.o_jobs, p.bj.data(), p.bj.size() * sizeof(afrs::BatchJob));
  if (!p.tasks.empty()) std::memcpy(h + p.o_tasks, p.tasks.data(), p.tasks.size() * sizeof(uint2));
  if (!p.rec.empty()) std::memcpy(h + p.o_rec, p.rec.data(), p.rec.size() * sizeof(int));
  if (!p.pos.empty()) std::memcpy(h + p.o_pos, p.pos.data(), p.pos.size());
  for (const BatchPrep::Group& gr : p.groups) {
    const size_t sz = afrs::job_desc_bytes(gr.op);
    for (size_t q = 0; q < gr.count; q++) {
      const GroupedJob& gj = p.grouped[gr.first + q];
      const afrs_job& j = jobs[gj.job];
      uint32_t* sc = reinterpret_cast<uint32_t*>(scratch + gj.scratch);
      void* desc = h + gr.desc_off + q * sz;
      if (gr.op == 2) {
        std::memcpy(desc, p.few_desc.data() + gj.few, sz);
      } else if (gr.op == 0) {
        afrs::EncodeArgs a{j.src, j.dst, j.shard_len, (int)j.n, (int)j.t, 0};
        afrs::fill_enc_job(desc, a, sc);
      } else {
        afrs::RecoverArgs a{};
        a.rx = j.dst;
        a.L = j.shard_len;
        a.n = (int)j.n;
        a.t = (int)j.t;
        a.e = (int)j.e;
        std::memcpy(a.pos, j.positions, j.e);
        afrs::fill_rec_job(desc, a, sc);
      }
    }
  }
}

// Enqueues the kernels of a prepared batch whose tables are at `d` (device):
// the group streams fork from `s`, the generic persistent kernel runs on
// `s`, the shape groups (largest first) round-robin on the group streams,
// and every forked stream is joined back into `s`, also after a failure.
// Only kernel launches and event records: capturable in a CUDA graph.
cudaError_t batch_enqueue(afrs_ctx* c, const BatchPrep& p, uint8_t* d, cudaStream_t s, const char** what) {
  const int nstreams = (int)std::min<size_t>(4, p.groups.size());
  int forked = 0;
  cudaError_t e = cudaSuccess;
  *what = "batch fork";
  if (nstreams) e = cudaEventRecord(c->grp_fork, s);
  for (int k = 0; k < nstreams && e == cudaSuccess; k++)
    if ((e = cudaStreamWaitEvent(c->grp_stream[k], c->grp_fork, 0)) == cudaSuccess) forked = k + 1;
  if (e == cudaSuccess && !p.bj.empty()) {
    afrs::BatchLaunch bl{};
    bl.jobs = reinterpret_cast<const afrs::BatchJob*>(d + p.o_jobs);
    bl.tasks = reinterpret_cast<const uint2*>(d + p.o_tasks);
    bl.ntasks = (int)p.tasks.size();
    bl.rec_jobs = reinterpret_cast<const int*>(d + p.o_rec);
    bl.nrec = (int)p.rec.size();
    bl.pos_tab = d + p.o_pos;
    bl.loc_tab = d + p.o_loc;
    bl.counter = reinterpret_cast<unsigned*>(d + p.o_cnt);
    bl.max_rows = p.max_rows;
    e = afrs::launch_batch(bl, s);
    *what = "batch launch";
  }
  // Rounds of grouped jobs: within a round the groups (largest first) go
  // round-robin to the group streams; a round reuses the previous round's
  // scratch, so every group stream first waits for all of them.
  for (int r = 0; r < p.rounds && e == cudaSuccess; r++) {
    if (r > 0) {
      *what = "batch round barrier";
      for (int k = 0; k < nstreams && e == cudaSuccess; k++) e = cudaEventRecord(c->grp_join[k], c->grp_stream[k]);
      for (int k = 0; k < nstreams && e == cudaSuccess; k++)
        for (int k2 = 0; k2 < nstreams && e == cudaSuccess; k2++)
          if (k2 != k) e = cudaStreamWaitEvent(c->grp_stream[k], c->grp_join[k2], 0);
    }
    const auto& groups = p.groups;
    std::vector<size_t> order;
    for (size_t q = 0; q < groups.size(); q++)
      if (groups[q].round == r) order.push_back(q);
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
      return groups[x].count * groups[x].max_ncw * groups[x].n > groups[y].count * groups[y].max_ncw * groups[y].n;
    });
    for (size_t q = 0; q < order.size() && e == cudaSuccess; q++) {
      const BatchPrep::Group& gr = groups[order[q]];
      cudaStream_t gs = c->grp_stream[q % nstreams];
      if (gr.op == 0)
        e = afrs::launch_encode_jobs(gr.n, gr.t, d + gr.desc_off, (int)gr.count, gr.max_ncw, gs);
      else if (gr.op == 1)
        e = afrs::launch_recover_jobs(gr.n, d + gr.desc_off, (int)gr.count, gr.max_ncw, gs);
      else
        e = afrs::launch_recover_few_jobs(gr.n, gr.t, d + gr.desc_off, (int)gr.count, gr.max_ncw, gs);
      *what = "batch group launch";
    }
  }
  for (int k = 0; k < forked; k++) {
    cudaError_t je = cudaEventRecord(c->grp_join[k], c->grp_stream[k]);
    if (je == cudaSuccess) je = cudaStreamWaitEvent(s, c->grp_join[k], 0);
    if (e == cudaSuccess && je != cudaSuccess) {
      e = je;
      *what = "batch join";
    }
  }
  return e;
}

}  // namespace

// A prepared batch (afrs_batch_plan_*): the tables and grouped scratch live
// on the device for the plan's lifetime, so a launch enqueues kernels only.
struct afrs_batch_plan {
  afrs_ctx* ctx;
  BatchPrep prep;
  uint8_t* tables;   // prep.total bytes
  uint8_t* scratch;  // prep.grp_bytes bytes
};

extern "C" {

int afrs_batch_dev(afrs_ctx* c, afrs_job* jobs, size_t count, void* stream) {
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  if (count && !jobs) return fail(AFRS_EINVAL, "jobs is NULL");
  if (count > (size_t)1 << 24) return fail(AFRS_EINVAL, "too many jobs (%zu)", count);
  BatchPrep p;
  int r = batch_prepare(jobs, count, &p);
  if (r) return r;
  if (p.empty()) return AFRS_OK;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  DeviceGuard g(c->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // A failure before anything is enqueued leaves every accepted job unrun.
  auto bail = [&](cudaError_t err, const char* what) -> int {
    const int rr = cuda_fail(err, what);
    for (size_t i : p.valid) jobs[i].status = rr;
    return rr;
  };
  const int slot = c->batch_slot;
  c->batch_slot ^= 1;
  // The slot's previous batch must be done with its staging, tables and scratch.
  cudaError_t e = cudaEventSynchronize(c->batch_free[slot]);
  if (e != cudaSuccess) return bail(e, "batch wait");
  if (p.total > c->batch_dev_bytes[slot]) {
    if (c->batch_dev[slot]) cudaFree(c->batch_dev[slot]);
    c->batch_dev[slot] = nullptr;
    c->batch_dev_bytes[slot] = 0;
    if ((e = cudaMalloc(&c->batch_dev[slot], p.total * 2)) != cudaSuccess) return bail(e, "batch tables");
    c->batch_dev_bytes[slot] = p.total * 2;
  }
  if (p.upload > c->batch_host_bytes[slot]) {
    if (c->batch_host[slot]) cudaFreeHost(c->batch_host[slot]);
    c->batch_host[slot] = nullptr;
    c->batch_host_bytes[slot] = 0;
    if ((e = cudaMallocHost(&c->batch_host[slot], p.upload * 2)) != cudaSuccess) return bail(e, "batch staging");
    c->batch_host_bytes[slot] = p.upload * 2;
  }
  if (p.grp_bytes > c->grp_scratch_bytes[slot]) {
    if (c->grp_scratch[slot]) cudaFree(c->grp_scratch[slot]);
    c->grp_scratch[slot] = nullptr;
    c->grp_scratch_bytes[slot] = 0;
    const size_t want = std::min(kGroupScratchCap, p.grp_bytes * 2);
    if ((e = cudaMalloc(reinterpret_cast<void**>(&c->grp_scratch[slot]), want)) != cudaSuccess)
      return bail(e, "batch scratch");
    c->grp_scratch_bytes[slot] = want;
  }
  uint8_t* h = c->batch_host[slot];
  batch_fill(p, jobs, h, reinterpret_cast<uint8_t*>(c->grp_scratch[slot]));
  uint8_t* d = c->batch_dev[slot];
  // Every exit from here on records batch_free[slot] on `s` (the next call on
  // this slot waits for it before it rewrites the slot's staging and
  // tables) and on failure marks the jobs as not run; batch_enqueue joins
  // every group stream it forked.
  auto finish = [&](cudaError_t err, const char* what) -> int {
    if (err != cudaSuccess)
      for (size_t i : p.valid) jobs[i].status = AFRS_ECUDA;
    cudaError_t re = cudaEventRecord(c->batch_free[slot], s);
    if (err == cudaSuccess && re != cudaSuccess) {
      err = re;
      what = "batch record";
    }
    return err == cudaSuccess ? AFRS_OK : cuda_fail(err, what);
  };
  if ((e = cudaMemcpyAsync(d, h, p.upload, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return finish(e, "batch upload");
  const char* what = "";
  e = batch_enqueue(c, p, d, s, &what);
  return finish(e, what);
}

int afrs_batch_plan_create(afrs_ctx* c, afrs_job* jobs, size_t count, afrs_batch_plan** out) {
  if (!out) return fail(AFRS_EINVAL, "out is NULL");
  *out = nullptr;
  if (!c) return fail(AFRS_EINVAL, "ctx is NULL");
  if (count && !jobs) return fail(AFRS_EINVAL, "jobs is NULL");
  if (count > (size_t)1 << 24) return fail(AFRS_EINVAL, "too many jobs (%zu)", count);
  afrs_batch_plan* pl = new (std::nothrow) afrs_batch_plan{};
  if (!pl) return fail(AFRS_ENOMEM, "plan allocation");
  pl->ctx = c;
  int r = batch_prepare(jobs, count, &pl->prep);
  if (r) {
    delete pl;
    return r;
  }
  if (!pl->prep.empty()) {
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    DeviceGuard g(c->device);
    const BatchPrep& p = pl->prep;
    cudaError_t e = cudaMalloc(&pl->tables, p.total);
    const char* what = "plan tables";
    if (e == cudaSuccess && p.grp_bytes) {
      e = cudaMalloc(&pl->scratch, p.grp_bytes);
      what = "plan scratch";
    }
    if (e == cudaSuccess) {
      std::vector<uint8_t> h(p.upload);
      batch_fill(p, jobs, h.data(), pl->scratch);
      e = cudaMemcpy(pl->tables, h.data(), p.upload, cudaMemcpyHostToDevice);
      what = "plan upload";
    }
    if (e != cudaSuccess) {
      r = cuda_fail(e, what);
      for (size_t i : p.valid) jobs[i].status = r;
      if (pl->tables) cudaFree(pl->tables);
      if (pl->scratch) cudaFree(pl->scratch);
      delete pl;
      return r;
    }
  }
  *out = pl;
  return AFRS_OK;
}

int afrs_batch_plan_launch(afrs_batch_plan* pl, void* stream) {
  if (!pl) return fail(AFRS_EINVAL, "plan is NULL");
  if (pl->prep.empty()) return AFRS_OK;
  afrs_ctx* c = pl->ctx;
  std::lock_guard<std::recursive_mutex> lk(c->mu);
  DeviceGuard g(c->device);
  const char* what = "";
  cudaError_t e = batch_enqueue(c, pl->prep, pl->tables, static_cast<cudaStream_t>(stream), &what);
  return e == cudaSuccess ? AFRS_OK : cuda_fail(e, what);
}

void afrs_batch_plan_destroy(afrs_batch_plan* pl) {
  if (!pl) return;
  if (pl->tables || pl->scratch) {
    DeviceGuard g(pl->ctx->device);
    cudaDeviceSynchronize();  // no launch of the plan may still read its tables
    if (pl->tables) cudaFree(pl->tables);
    if (pl->scratch) cudaFree(pl->scratch);
  }
  delete pl;
}

}  // extern "C"
