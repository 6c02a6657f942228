// Compile-time-twiddle kernels (the throughput path): templates shared by
// the special_*.cu translation units, which instantiate them per shape.
//
// Every twiddle of an additive FFT level depends only on the level, the
// coset beta and the row bits above the level (rs/src/kernel/lut_kernel.rs:
// 28-82), so once a thread's rows are fixed at compile time every multiply
// is a fixed XOR network over bit-sliced planes (gf_device.cuh).
//
// Transforms of 2^k rows, k >= 5, run as three phase kernels (radix 16 x
// 2^(k-4)):
//   bottom pass (b1): levels 0..3 on 16 contiguous rows (group g = row >> 4);
//   top pass (p2):    levels 4..k-1 on rows {b + 16 m};
//   bottom pass (b3) of the next transform.
// The code of a bottom pass depends on g (its twiddles do), so each CTA runs
// one g (blockIdx.y) over many columns: every fetched instruction is used by
// all warps of the CTA.  A bottom group is shared by two warps, 8 rows per
// warp: levels 0..2 stay inside a warp and level 3 goes through shared
// memory, which halves the registers per thread and the code per variant.
// (A single kernel holding all rows of a column tile in shared memory runs
// each variant once per tile and is bound by instruction fetch: ~800 KB of
// straight-line code for n = 256.)
// Between phases the rows stay bit-sliced in a scratch buffer (1 GiB at most;
// L2-resident for small codewords); longer shards are processed in column
// batches.  For some shapes a one-launch form (k_enc_fused, k_rec_fused)
// holds all rows of a slice in one CTA instead; the route table picks it
// where it measured faster (short shards).
// Transforms with k <= 4 run entirely inside one thread.
#pragma once
#include <cooperative_groups.h>

#include <array>
#include <cstring>
#include <utility>

#include "afrs_internal.h"
#include "gf_device.cuh"
#include "io.cuh"

namespace afrs {
namespace spec {

static __constant__ FieldTables c_tab = make_field_tables();

constexpr int kThreads = 256;

// ---- butterflies and compile-time blocks ---------------------------------

template <int TW>
__device__ __forceinline__ void bf_fwd(uint32_t (&a)[8], uint32_t (&b)[8]) {
  if constexpr (TW != 0) mul_xor_c<static_cast<uint8_t>(TW)>(a, b);
#pragma unroll
  for (int p = 0; p < 8; p++) b[p] ^= a[p];
}

template <int TW>
__device__ __forceinline__ void bf_inv(uint32_t (&a)[8], uint32_t (&b)[8]) {
#pragma unroll
  for (int p = 0; p < 8; p++) b[p] ^= a[p];
  if constexpr (TW != 0) mul_xor_c<static_cast<uint8_t>(TW)>(a, b);
}

// Levels [L0, L0 + RLOG) of a transform at coset BETA on NR = 2^RLOG rows in
// registers; register row r is global row (HI << (L0 + RLOG)) | (r << L0) |
// (bits below L0, which no twiddle of these levels depends on).
template <int L0, int RLOG, int HI, int BETA, int NR>
__device__ __forceinline__ void block_fft(uint32_t (&x)[NR][8]) {
  static_assert(NR == (1 << RLOG), "rows");
  static_for<RLOG>([&](auto s) {
    constexpr int lv = RLOG - 1 - decltype(s)::value;
    static_for<NR / 2>([&](auto q) {
      constexpr int qq = decltype(q)::value;
      constexpr int i = ((qq >> lv) << (lv + 1)) | (qq & ((1 << lv) - 1));
      constexpr int j = L0 + lv;
      constexpr int row = (HI << (L0 + RLOG)) | (i << L0);
      constexpr int tw = twiddle_c(j, static_cast<uint8_t>(BETA), row & ~((2 << j) - 1));
      bf_fwd<tw>(x[i], x[i + (1 << lv)]);
    });
  });
}

template <int L0, int RLOG, int HI, int BETA, int NR>
__device__ __forceinline__ void block_ifft(uint32_t (&x)[NR][8]) {
  static_assert(NR == (1 << RLOG), "rows");
  static_for<RLOG>([&](auto s) {
    constexpr int lv = decltype(s)::value;
    static_for<NR / 2>([&](auto q) {
      constexpr int qq = decltype(q)::value;
      constexpr int i = ((qq >> lv) << (lv + 1)) | (qq & ((1 << lv) - 1));
      constexpr int j = L0 + lv;
      constexpr int row = (HI << (L0 + RLOG)) | (i << L0);
      constexpr int tw = twiddle_c(j, static_cast<uint8_t>(BETA), row & ~((2 << j) - 1));
      bf_inv<tw>(x[i], x[i + (1 << lv)]);
    });
  });
}

// x <- (I + D) x on NR rows in registers, D the formal derivative in the
// LCH basis (d[m] = sum over clear bits j of m of c[m + 2^j]).  In-place
// order: i = 1 .. NR-1, rows [i - w, i) ^= rows [i, i + w), w = lowbit(i);
// sources are never modified before they are read.
template <int NR>
__device__ __forceinline__ void one_plus_derivative(uint32_t (&x)[NR][8]) {
  static_for<NR - 1>([&](auto s) {
    constexpr int i = decltype(s)::value + 1;
    constexpr int w = i & -i;
    static_for<w>([&](auto u) {
      constexpr int o = decltype(u)::value;
#pragma unroll
      for (int p = 0; p < 8; p++) x[i - w + o][p] ^= x[i + o][p];
    });
  });
}

// Bit-sliced shared-memory tile: row r, plane p, colword w at
// sm[(r * 8 + p) * CW + w]; a warp reading one (row, plane) over 32 colwords
// touches 32 consecutive words.
template <int CW>
__device__ __forceinline__ void sload(const uint32_t* sm, int row, int w, uint32_t (&x)[8]) {
#pragma unroll
  for (int p = 0; p < 8; p++) x[p] = sm[(row * 8 + p) * CW + w];
}
template <int CW>
__device__ __forceinline__ void sstore(uint32_t* sm, int row, int w, const uint32_t (&x)[8]) {
#pragma unroll
  for (int p = 0; p < 8; p++) sm[(row * 8 + p) * CW + w] = x[p];
}

// Shard row <-> bit-sliced planes for global colword w (io.cuh layout).
// Row r starts at base + r * pitch; columns [0, L) exist.
__device__ __forceinline__ void gload(const uint8_t* base, size_t row, size_t pitch, size_t L, size_t w,
                                      uint32_t (&x)[8], const ShiftMul& km) {
  load_cw(base + row * pitch, L, w, x);
  transpose8f(x, km);
}
__device__ __forceinline__ void gstore(uint8_t* base, size_t row, size_t pitch, size_t L, size_t w,
                                       uint32_t (&x)[8], const ShiftMul& km) {
  transpose8f(x, km);
  store_cw(base + row * pitch, L, w, x);
}

// y <- c * y for c = g^a (g = 2), a in [0, 254] uniform across the warp:
// a = 16 h + l and c = g^l * g^(16 h), two multiplies by compile-time
// constants picked from 16 each (about 32 LOP3 instead of the ~85 of the
// branch-free shift-and-add).  The phase kernels scale lambda and Forney
// rows this way: with the operations of several codewords sharing the GPU
// it measured 2.3 % faster than the shift-and-add, which a bottom pass run
// alone prefers by 3 % (its uniform branches cost latency, the extra LOP3
// cost ALU issue).
template <int C>
__device__ __forceinline__ void mul_by_c(uint32_t (&y)[8]) {
  if constexpr (C != 1) {
    uint32_t r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    mul_xor_c<static_cast<uint8_t>(C)>(r, y);
#pragma unroll
    for (int p = 0; p < 8; p++) y[p] = r[p];
  }
}
__device__ __forceinline__ void scale_log(uint32_t (&y)[8], int a) {
  dispatch<0, 15>(a >> 4, [&](auto h) { mul_by_c<kField.exp[16 * decltype(h)::value]>(y); });
  dispatch<0, 15>(a & 15, [&](auto l) { mul_by_c<kField.exp[decltype(l)::value]>(y); });
}
// x <- c * x for a runtime constant c (branch-free shift-and-add).
__device__ __forceinline__ void scale_rt(uint32_t (&x)[8], uint32_t c) {
  uint32_t r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  mul_xor_rt(r, x, c);
#pragma unroll
  for (int p = 0; p < 8; p++) x[p] = r[p];
}

template <int NR>
__device__ __forceinline__ void zero_rows(uint32_t (&x)[NR][8]) {
#pragma unroll
  for (int r = 0; r < NR; r++)
#pragma unroll
    for (int p = 0; p < 8; p++) x[r][p] = 0;
}

// ---- encode, t <= 16: one warp per 1024-column slice ----------------------
// codec.rs:241-265: parity = FFT_t(parity_in? ^ sum_c IFFT_t(chunk c, omega_ct), 0),
// chunk c = message shards (c-1)t .. ct-1, c = 1 .. n/t - 1.
// t <= 16 with more than one chunk: the CTA's warps share one 1024-column
// slice and split its chunks (warp w takes chunks w + 1, w + 1 + W, ...),
// each XOR-accumulating its chunk IFFTs in its own shared-memory rows; the
// rows are then summed over the warps and warp 0 runs the final FFT.  (One
// warp running all n/t - 1 chunks of a slice made the time of a small
// codeword the serial latency of its chunks.)
template <int LOGN, int LOGT>
__device__ __forceinline__ void enc_small_split_body(const EncodeArgs& a, unsigned bx, uint32_t* sm) {
  constexpr int N = 1 << LOGN, T = 1 << LOGT, C = N / T - 1, W = kThreads / 32;
  constexpr int WU = C < W ? C : W;  // warps that get chunks
  constexpr int kRows = T * 8 * 32;  // words of one warp's accumulator
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if ((size_t)bx * 1024 >= a.L) return;  // the whole CTA
  const size_t cw = (size_t)bx * 32 + lane;
  const ShiftMul km = make_shift_mul();
  if (warp < WU) {
    uint32_t* wacc = sm + warp * kRows;
    for (int c = 1 + warp; c <= C; c += W) {
      uint32_t x[T][8];
#pragma unroll
      for (int r = 0; r < T; r++) gload(a.msg, (size_t)(c - 1) * T + r, row_pitch(a), a.L, cw, x[r], km);
      if constexpr (LOGT > 0) {
        dispatch<1, C>(c, [&](auto cc) {
          constexpr int CC = decltype(cc)::value;
          block_ifft<0, LOGT, 0, omega_c(CC * T), T>(x);
        });
      }
      const bool first = c == 1 + warp;
#pragma unroll
      for (int r = 0; r < T; r++) {
        uint32_t y[8];
        if (first) {
#pragma unroll
          for (int p = 0; p < 8; p++) y[p] = x[r][p];
        } else {
          sload<32>(wacc, r, lane, y);
#pragma unroll
          for (int p = 0; p < 8; p++) y[p] ^= x[r][p];
        }
        sstore<32>(wacc, r, lane, y);
      }
    }
  }
  __syncthreads();
  for (int r = warp; r < T; r += W) {
    uint32_t y[8];
    sload<32>(sm, r, lane, y);
    for (int w = 1; w < WU; w++) {
      uint32_t z[8];
      sload<32>(sm + w * kRows, r, lane, z);
#pragma unroll
      for (int p = 0; p < 8; p++) y[p] ^= z[p];
    }
    sstore<32>(sm, r, lane, y);
  }
  __syncthreads();
  // Warp 0 runs the final FFT; the warps then transpose and store one parity
  // row each (warp 0 alone storing all T rows was the CTA's serial tail).
  if (warp == 0) {
    uint32_t f[T][8];
#pragma unroll
    for (int r = 0; r < T; r++) {
      sload<32>(sm, r, lane, f[r]);
      if (a.accumulate) {
        uint32_t y[8];
        gload(a.parity, r, row_pitch(a), a.L, cw, y, km);
#pragma unroll
        for (int p = 0; p < 8; p++) f[r][p] ^= y[p];
      }
    }
    block_fft<0, LOGT, 0, 0, T>(f);
#pragma unroll
    for (int r = 0; r < T; r++) sstore<32>(sm, r, lane, f[r]);
  }
  __syncthreads();
  for (int r = warp; r < T; r += W) {
    uint32_t y[8];
    sload<32>(sm, r, lane, y);
    gstore(a.parity, r, row_pitch(a), a.L, cw, y, km);
  }
}

// Layout of the t <= 16 encode.  With more than one chunk and few slices of
// 1024 columns (or t < 16, where the per-warp accumulators are small), the
// warps of a CTA split the chunks of one slice; otherwise each warp takes a
// slice of its own and runs all its chunks (at t = 16 and long shards that is
// faster: n = 256, 1 MiB shards: 280 vs 465 us).
template <int LOGN, int LOGT>
inline bool enc_small_split(size_t slices) {
  constexpr int T = 1 << LOGT, C = ((1 << LOGN) >> LOGT) - 1;
  return C > 1 && (T < 16 || slices <= 128);
}
// CTAs and dynamic shared memory of either layout.
template <int LOGN, int LOGT>
inline unsigned enc_small_ctas(size_t slices, bool split) {
  return (unsigned)(split ? slices : (slices + kThreads / 32 - 1) / (kThreads / 32));
}
template <int LOGN, int LOGT>
constexpr size_t enc_small_smem(bool split) {
  constexpr int T = 1 << LOGT, C = ((1 << LOGN) >> LOGT) - 1, W = kThreads / 32;
  return split ? (size_t)(C < W ? C : W) * T * 8 * 32 * 4 : (T == 16 ? (size_t)W * 16 * 8 * 32 * 4 : 0);
}

template <int LOGN, int LOGT, bool kSplit>
__device__ __forceinline__ void enc_small_body(const EncodeArgs& a, unsigned bx, uint32_t* sm) {
  constexpr int N = 1 << LOGN, T = 1 << LOGT, C = N / T - 1;
  if constexpr (kSplit && C > 1) {
    enc_small_split_body<LOGN, LOGT>(a, bx, sm);
    return;
  }
  constexpr bool kSmemAcc = (T == 16);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t slice = (size_t)bx * (kThreads / 32) + warp;
  if (slice * 1024 >= a.L) return;
  const size_t cw = slice * 32 + lane;
  const ShiftMul km = make_shift_mul();
  uint32_t* wacc = sm + warp * (T * 8 * 32);  // per-warp accumulator when kSmemAcc
  uint32_t acc[kSmemAcc ? 1 : T][8];
  if constexpr (kSmemAcc) {
    for (int r = 0; r < T; r++) {
      uint32_t z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      sstore<32>(wacc, r, lane, z);
    }
  } else {
    zero_rows(acc);
  }
  for (int c = 1; c <= C; c++) {
    uint32_t x[T][8];
#pragma unroll
    for (int r = 0; r < T; r++) gload(a.msg, (size_t)(c - 1) * T + r, row_pitch(a), a.L, cw, x[r], km);
    if constexpr (LOGT > 0) {
      dispatch<1, C>(c, [&](auto cc) {
        constexpr int CC = decltype(cc)::value;
        block_ifft<0, LOGT, 0, omega_c(CC * T), T>(x);
      });
    }
    if constexpr (kSmemAcc) {
#pragma unroll
      for (int r = 0; r < T; r++) {
        uint32_t y[8];
        sload<32>(wacc, r, lane, y);
#pragma unroll
        for (int p = 0; p < 8; p++) y[p] ^= x[r][p];
        sstore<32>(wacc, r, lane, y);
      }
    } else {
#pragma unroll
      for (int r = 0; r < T; r++)
#pragma unroll
        for (int p = 0; p < 8; p++) acc[r][p] ^= x[r][p];
    }
  }
  uint32_t f[T][8];
#pragma unroll
  for (int r = 0; r < T; r++) {
    if constexpr (kSmemAcc)
      sload<32>(wacc, r, lane, f[r]);
    else
#pragma unroll
      for (int p = 0; p < 8; p++) f[r][p] = acc[r][p];
    if (a.accumulate) {
      uint32_t y[8];
      gload(a.parity, r, row_pitch(a), a.L, cw, y, km);
#pragma unroll
      for (int p = 0; p < 8; p++) f[r][p] ^= y[p];
    }
  }
  block_fft<0, LOGT, 0, 0, T>(f);
#pragma unroll
  for (int r = 0; r < T; r++) gstore(a.parity, r, row_pitch(a), a.L, cw, f[r], km);
}


// ---- bit-sliced scratch ---------------------------------------------------
// Row r, colword w of a batch of ncw colwords: planes 0..3 as one 16-byte
// word at ((r * 2 + 0) * ncw + w) and planes 4..7 at ((r * 2 + 1) * ncw + w),
// so that a warp over 32 consecutive colwords moves 512 contiguous bytes per
// instruction.
__device__ __forceinline__ void xload(const uint32_t* s, size_t ncw, int r, size_t w, uint32_t (&x)[8]) {
  const uint4* q = reinterpret_cast<const uint4*>(s);
  uint4 a = q[(size_t)(2 * r) * ncw + w], b = q[(size_t)(2 * r + 1) * ncw + w];
  x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
  x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
}
__device__ __forceinline__ void xstore(uint32_t* s, size_t ncw, int r, size_t w, const uint32_t (&x)[8]) {
  uint4* q = reinterpret_cast<uint4*>(s);
  q[(size_t)(2 * r) * ncw + w] = make_uint4(x[0], x[1], x[2], x[3]);
  q[(size_t)(2 * r + 1) * ncw + w] = make_uint4(x[4], x[5], x[6], x[7]);
}

// One batch of colwords [cw0, cw0 + ncw) of a phase kernel.
struct Batch {
  uint32_t* s1;  // scratch (bit-sliced rows)
  uint32_t* s2;  // second scratch (recover)
  size_t ncw;    // colwords in the batch
  size_t cw0;    // first global colword of the batch
};

constexpr int kPhaseThreads = 128;

// Programmatic dependent launch inside one operation: b1 and p2 let the next
// kernel be scheduled once every CTA has finished its arithmetic (just before
// its final stores), which hides the launch gap; p2 and b3 block in
// griddep_wait() until the previous kernel has completed and its writes are
// visible (a no-op when a kernel is launched without the attribute).  A
// trigger at kernel entry measured slower when two operations share the GPU:
// the early-scheduled CTAs hold SM slots while they wait.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// cp.async copy of 16 bytes from global (device or mapped host) memory to
// shared memory.
__device__ __forceinline__ void cp_async16(uint4* dst, const uint8_t* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

// ---- encode, t >= 32 -------------------------------------------------------
template <int LOGN, int LOGT, bool kSplit>
__global__ void __launch_bounds__(kThreads) k_enc_small(EncodeArgs a) {
  extern __shared__ uint32_t sm[];
  enc_small_body<LOGN, LOGT, kSplit>(a, blockIdx.x, sm);
}

// E2: top levels for rows {b + 16 m} (b = blockIdx.y): IFFT top of every
// chunk, accumulated, plus parity_in, then FFT top at 0; written to scratch
// rows b + 16 m (chunk 1's rows, read above by this thread only).
template <int LOGN, int LOGT>
__device__ __forceinline__ void enc_p2_body(const EncodeArgs& a, const Batch& bt, unsigned bx, int by) {
  constexpr int N = 1 << LOGN, T = 1 << LOGT, C = N / T - 1, TL = LOGT - 4, TR = 1 << TL;
  griddep_wait();
  const size_t w = (size_t)bx * kPhaseThreads + threadIdx.x;
  if (w >= bt.ncw) return;
  const int b = by;
  uint32_t acc[TR][8];
  zero_rows(acc);
  for (int c = 1; c <= C; c++) {
    uint32_t y[TR][8];
#pragma unroll
    for (int m = 0; m < TR; m++) xload(bt.s1, bt.ncw, (c - 1) * T + b + 16 * m, w, y[m]);
    dispatch<1, C>(c, [&](auto cc) {
      constexpr int CC = decltype(cc)::value;
      block_ifft<4, TL, 0, omega_c(CC * T), TR>(y);
    });
#pragma unroll
    for (int m = 0; m < TR; m++)
#pragma unroll
      for (int p = 0; p < 8; p++) acc[m][p] ^= y[m][p];
  }
  if (a.accumulate) {
    const ShiftMul km = make_shift_mul();
#pragma unroll
    for (int m = 0; m < TR; m++) {
      uint32_t q[8];
      gload(a.parity, b + 16 * m, row_pitch(a), a.L, bt.cw0 + w, q, km);
#pragma unroll
      for (int p = 0; p < 8; p++) acc[m][p] ^= q[p];
    }
  }
  block_fft<4, TL, 0, 0, TR>(acc);
  griddep_trigger();
#pragma unroll
  for (int m = 0; m < TR; m++) xstore(bt.s1, bt.ncw, b + 16 * m, w, acc[m]);
}
template <int LOGN, int LOGT>
__global__ void __launch_bounds__(kPhaseThreads) k_enc_p2(EncodeArgs a, Batch bt) {
  enc_p2_body<LOGN, LOGT>(a, bt, blockIdx.x, blockIdx.y);
}


// ---- bottom passes split over several warps -------------------------------
// A 16-row bottom group (levels 0..3) is shared by WG = 16 / RW warps of a
// CTA: warp q of the group holds rows 16g + RW q + i (i < RW) of the same 32
// colwords.  The LR = log2(RW) lowest levels run inside each warp (a
// warp-uniform compile-time variant), the higher ones pair row i of warp q
// with row i of warp q ^ 2^(j - LR) through shared memory.  Exchanges (and
// their barriers) are CTA-uniform code; only the combine step, whose twiddle
// depends on the warp, is dispatched per warp.  Fewer rows per warp means
// fewer registers, less code per warp and more warps per launch, but one more
// exchange level: RW = 4 measured slower than RW = 8 for n = 256 with 64 KiB
// shards (encode 31.1 vs 25.7 us, recover 54.0 vs 43.8 us) and within 5 %
// for 1-4 MiB shards.
constexpr int kSplitThreads = 128;  // 4 warps
constexpr int kRowsPerWarp = 8;

template <int RW>
struct Split {
  static_assert(RW == 4 || RW == 8, "rows per warp");
  static constexpr int WG = 16 / RW;                 // warps per row group
  static constexpr int LR = RW == 8 ? 3 : 2;         // levels inside a warp
  static constexpr int CW = 32 * (4 / WG);           // colwords per CTA
  static constexpr size_t kStage = (size_t)RW * 32 * kSplitThreads;
};

// Stage slot of row i (half hf) of thread tid in a CTA of NT threads.
template <int NT = kSplitThreads>
__device__ __forceinline__ uint4* sl(uint32_t* st, int i, int hf, int tid) {
  return reinterpret_cast<uint4*>(st) + (i * 2 + hf) * NT + tid;
}
template <int NT = kSplitThreads>
__device__ __forceinline__ void s_get(uint32_t* st, int i, int tid, uint32_t (&x)[8]) {
  const uint4 a = *sl<NT>(st, i, 0, tid), b = *sl<NT>(st, i, 1, tid);
  x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
  x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
}
template <int NT = kSplitThreads>
__device__ __forceinline__ void s_put(uint32_t* st, int i, int tid, const uint32_t (&x)[8]) {
  *sl<NT>(st, i, 0, tid) = make_uint4(x[0], x[1], x[2], x[3]);
  *sl<NT>(st, i, 1, tid) = make_uint4(x[4], x[5], x[6], x[7]);
}

// Rows first_row + i (i < RW) of colword w into the calling thread's slots
// (cp.async where 16-byte aligned and in bounds); bit i of skip stages zero.
template <int RW, int NT = kSplitThreads>
__device__ __forceinline__ void stage_rows(uint32_t* st, const uint8_t* base, size_t first_row, size_t pitch,
                                           size_t L, size_t w, uint32_t skip) {
  const size_t c = cw_col(w);
  const int tid = threadIdx.x;
#pragma unroll
  for (int i = 0; i < RW; i++) {
#pragma unroll
    for (int hf = 0; hf < 2; hf++) {
      uint4* dst = sl<NT>(st, i, hf, tid);
      if ((skip >> i) & 1) {
        *dst = make_uint4(0, 0, 0, 0);
        continue;
      }
      const size_t col = c + 512 * hf;
      const uint8_t* row = base + (first_row + i) * pitch;
      if (col + 16 <= L && ((reinterpret_cast<uintptr_t>(row + col) & 15) == 0)) {
        cp_async16(dst, row + col);
      } else {
        uint32_t x[4];
        load16(row, col, L, x);
        *dst = make_uint4(x[0], x[1], x[2], x[3]);
      }
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// CTA-uniform: every thread publishes its rows in its own slots.  The leading
// barrier orders it after all earlier reads of the stage.
template <int RW, int NT = kSplitThreads>
__device__ __forceinline__ void xchg_put(uint32_t* st, const uint32_t (&x)[RW][8]) {
  __syncthreads();
#pragma unroll
  for (int i = 0; i < RW; i++) s_put<NT>(st, i, threadIdx.x, x[i]);
  __syncthreads();
}

// Cross-warp IFFT level: (g0, g1) = (row i of the low warp, row i of the high
// warp) -> (g0 + T (g0 + g1), g0 + g1); H = 1 for the high warp.
template <int TW, int H, int RW, int NT = kSplitThreads>
__device__ __forceinline__ void combine_ifft(uint32_t* st, uint32_t (&x)[RW][8], int ptid) {
#pragma unroll
  for (int i = 0; i < RW; i++) {
    uint32_t y[8];
    s_get<NT>(st, i, ptid, y);
    if constexpr (H == 0) {
      uint32_t d[8];
#pragma unroll
      for (int p = 0; p < 8; p++) d[p] = x[i][p] ^ y[p];
      if constexpr (TW != 0) mul_xor_c<static_cast<uint8_t>(TW)>(x[i], d);
    } else {
#pragma unroll
      for (int p = 0; p < 8; p++) x[i][p] ^= y[p];
    }
  }
}

// Cross-warp FFT level: (a, b) -> (a + T b, a + (T + 1) b).
template <int TW, int H, int RW, int NT = kSplitThreads>
__device__ __forceinline__ void combine_fft(uint32_t* st, uint32_t (&x)[RW][8], int ptid) {
#pragma unroll
  for (int i = 0; i < RW; i++) {
    uint32_t y[8];
    s_get<NT>(st, i, ptid, y);
    if constexpr (H == 0) {
      if constexpr (TW != 0) mul_xor_c<static_cast<uint8_t>(TW)>(x[i], y);
    } else {
      uint32_t m[8];
#pragma unroll
      for (int p = 0; p < 8; p++) m[p] = y[p] ^ x[i][p];
      if constexpr (TW != 0) mul_xor_c<static_cast<uint8_t>(TW)>(m, x[i]);
#pragma unroll
      for (int p = 0; p < 8; p++) x[i][p] = m[p];
    }
  }
}

template <int RW>
struct SplitPos {
  int q;        // warp within its row group
  size_t w;     // colword
  bool active;  // w inside the batch
};
template <int RW>
__device__ __forceinline__ SplitPos<RW> split_pos(size_t ncw, unsigned bx) {
  const int warp = threadIdx.x >> 5;
  SplitPos<RW> p;
  p.q = warp % Split<RW>::WG;
  p.w = (size_t)bx * Split<RW>::CW + (warp / Split<RW>::WG) * 32 + (threadIdx.x & 31);
  p.active = p.w < ncw;
  return p;
}

// Drops from L2, without writing them back, the scratch lines of rows
// [r0, r0 + RW) of the calling warp's colwords [w0, w0 + 32): once the last
// pass has read them they are dead (every operation writes its scratch before
// it reads it), and otherwise L2 writes them back to DRAM when it evicts
// them.  A warp owns whole lines only when its 32 colwords are all in the
// batch and every (row, half) region starts on a 128-byte boundary (ncw a
// multiple of 8); otherwise nothing is dropped.  Call it only after the
// warp's loads of those rows have been consumed.
template <int RW>
__device__ __forceinline__ void discard_rows(const uint32_t* s, size_t ncw, int r0, size_t w0) {
  if (ncw % 8 != 0 || w0 + 32 > ncw) return;
  const uint4* q = reinterpret_cast<const uint4*>(s);
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = lane; k < 8 * RW; k += 32) {  // 2 RW regions x 4 lines of 128 bytes
    const uint4* p = q + (size_t)(2 * r0 + (k >> 2)) * ncw + w0 + 8 * (k & 3);
    asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
  }
}

// E1 (split): bottom IFFT of chunk c, group g; blockIdx.y = (c - 1) * (t/16) + g.
template <int LOGN, int LOGT>
__device__ __forceinline__ void enc_b1_body(const EncodeArgs& a, const Batch& bt, unsigned bx, int by, uint32_t* st) {
  constexpr int RW = kRowsPerWarp, WG = Split<RW>::WG, LR = Split<RW>::LR;
  constexpr int N = 1 << LOGN, T = 1 << LOGT, C = N / T - 1, G = T / 16;
  const SplitPos<RW> q = split_pos<RW>(bt.ncw, bx);
  const ShiftMul km = make_shift_mul();
  const int v = by, c = v / G + 1, g = v % G;
  const size_t row0 = (size_t)(c - 1) * T + 16 * g + RW * q.q;
  uint32_t x[RW][8];
  zero_rows(x);
  if (q.active) {
    stage_rows<RW>(st, a.msg, row0, row_pitch(a), a.L, bt.cw0 + q.w, 0);
#pragma unroll 1
    for (int i = 0; i < RW; i++) {
      uint32_t y[8];
      s_get(st, i, threadIdx.x, y);
      transpose8f(y, km);
      s_put(st, i, threadIdx.x, y);
    }
#pragma unroll
    for (int i = 0; i < RW; i++) s_get(st, i, threadIdx.x, x[i]);
  }
  const int vq = v * WG + q.q;
  dispatch<0, C * G * WG - 1>(vq, [&](auto vv) {
    constexpr int V = decltype(vv)::value / WG, Q = decltype(vv)::value % WG;
    block_ifft<0, LR, (V % G) * WG + Q, omega_c((V / G + 1) * T), RW>(x);
  });
  static_for<4 - LR>([&](auto jj) {
    constexpr int J = LR + decltype(jj)::value;
    xchg_put<RW>(st, x);
    dispatch<0, C * G * WG - 1>(vq, [&](auto vv) {
      constexpr int V = decltype(vv)::value / WG, Q = decltype(vv)::value % WG;
      constexpr int TW = twiddle_c(J, omega_c((V / G + 1) * T), (16 * (V % G) + RW * Q) & ~((2 << J) - 1));
      combine_ifft<TW, (Q >> (J - LR)) & 1, RW>(st, x, threadIdx.x ^ (32 << (J - LR)));
    });
  });
  griddep_trigger();
  if (q.active) {
#pragma unroll
    for (int i = 0; i < RW; i++) xstore(bt.s1, bt.ncw, (int)row0 + i, q.w, x[i]);
  }
}

// E3 (split): bottom FFT of group g = blockIdx.y, store of parity rows.
template <int LOGN, int LOGT>
__device__ __forceinline__ void enc_b3_body(const EncodeArgs& a, const Batch& bt, unsigned bx, int by, uint32_t* st) {
  griddep_wait();
  constexpr int RW = kRowsPerWarp, WG = Split<RW>::WG, LR = Split<RW>::LR;
  constexpr int T = 1 << LOGT, G = T / 16;
  const SplitPos<RW> q = split_pos<RW>(bt.ncw, bx);
  const ShiftMul km = make_shift_mul();
  const int g = by;
  const int row0 = 16 * g + RW * q.q;
  uint32_t x[RW][8];
  zero_rows(x);
  if (q.active) {
#pragma unroll
    for (int i = 0; i < RW; i++) xload(bt.s1, bt.ncw, row0 + i, q.w, x[i]);
  }
  const int gq = g * WG + q.q;
  static_for<4 - LR>([&](auto jj) {
    constexpr int J = 3 - decltype(jj)::value;
    xchg_put<RW>(st, x);
    dispatch<0, G * WG - 1>(gq, [&](auto vv) {
      constexpr int GG = decltype(vv)::value / WG, Q = decltype(vv)::value % WG;
      constexpr int TW = twiddle_c(J, 0, (16 * GG + RW * Q) & ~((2 << J) - 1));
      combine_fft<TW, (Q >> (J - LR)) & 1, RW>(st, x, threadIdx.x ^ (32 << (J - LR)));
    });
  });
  __syncthreads();  // partners' reads of the stage are done
  // The scratch rows were stored to shared memory before the barriers above.
  discard_rows<RW>(bt.s1, bt.ncw, row0, q.w - (threadIdx.x & 31));
  dispatch<0, G * WG - 1>(gq, [&](auto vv) {
    constexpr int VV = decltype(vv)::value;
    block_fft<0, LR, VV, 0, RW>(x);
  });
  if (q.active) {
#pragma unroll
    for (int i = 0; i < RW; i++) s_put(st, i, threadIdx.x, x[i]);
#pragma unroll 1
    for (int i = 0; i < RW; i++) {
      uint32_t y[8];
      s_get(st, i, threadIdx.x, y);
      gstore(a.parity, row0 + i, row_pitch(a), a.L, bt.cw0 + q.w, y, km);
    }
  }
}

template <int LOGN, int LOGT>
__global__ void __launch_bounds__(kSplitThreads, 4) k_enc_b1(EncodeArgs a, Batch bt) {
  extern __shared__ uint32_t st[];
  enc_b1_body<LOGN, LOGT>(a, bt, blockIdx.x, blockIdx.y, st);
}
template <int LOGN, int LOGT>
__global__ void __launch_bounds__(kSplitThreads, 4) k_enc_b3(EncodeArgs a, Batch bt) {
  extern __shared__ uint32_t st[];
  enc_b3_body<LOGN, LOGT>(a, bt, blockIdx.x, blockIdx.y, st);
}

// Grouped launches (afrs_batch_dev): many codewords of one shape (codeword
// blockIdx.y in the bottom passes, blockIdx.z in the others), each with its
// own scratch holding its whole shard width.  Blocks beyond a codeword's
// colwords leave before any barrier.
struct EncJob {
  EncodeArgs a;
  uint32_t* s1;
  size_t ncw;
};
// The bottom passes of a group put the codeword in blockIdx.y and the row
// group (the code variant) in blockIdx.z, so that CTAs launched together
// run one variant across codewords: with short shards most column blocks of
// a codeword exit at once, and codeword-major order then kept every variant
// in flight on every SM (instruction fetch: 13.9 stall cycles per issue).
template <int LOGN, int LOGT>
__global__ void __launch_bounds__(kSplitThreads, 4) k_enc_b1_jobs(const EncJob* __restrict__ jobs) {
  extern __shared__ uint32_t st[];
  const EncJob& j = jobs[blockIdx.y];
  if ((size_t)blockIdx.x * Split<kRowsPerWarp>::CW >= j.ncw) return;
  enc_b1_body<LOGN, LOGT>(j.a, Batch{j.s1, nullptr, j.ncw, 0}, blockIdx.x, blockIdx.z, st);
}
template <int LOGN, int LOGT>
__global__ void __launch_bounds__(kPhaseThreads) k_enc_p2_jobs(const EncJob* __restrict__ jobs) {
  const EncJob& j = jobs[blockIdx.z];
  enc_p2_body<LOGN, LOGT>(j.a, Batch{j.s1, nullptr, j.ncw, 0}, blockIdx.x, blockIdx.y);
}
template <int LOGN, int LOGT>
__global__ void __launch_bounds__(kSplitThreads, 4) k_enc_b3_jobs(const EncJob* __restrict__ jobs) {
  extern __shared__ uint32_t st[];
  const EncJob& j = jobs[blockIdx.y];
  if ((size_t)blockIdx.x * Split<kRowsPerWarp>::CW >= j.ncw) return;
  enc_b3_body<LOGN, LOGT>(j.a, Batch{j.s1, nullptr, j.ncw, 0}, blockIdx.x, blockIdx.z, st);
}

// Grouped t <= 16 encode: one warp per 1024-column slice of codeword blockIdx.z.
template <int LOGN, int LOGT, bool kSplit>
__global__ void __launch_bounds__(kThreads) k_enc_small_jobs(const EncJob* __restrict__ jobs) {
  extern __shared__ uint32_t sm[];
  const EncJob& j = jobs[blockIdx.z];
  if ((size_t)blockIdx.x * (kSplit ? 1 : kThreads / 32) * 1024 >= j.a.L) return;
  enc_small_body<LOGN, LOGT, kSplit>(j.a, blockIdx.x, sm);
}

// ---- recover ------------------------------------------------------------
// Leopard-form decoder (the same map as rs/src/codec.rs:479-569 on every
// input whose erased rows are zero): y = lambda .* r over survivors,
// c = IFFT_n(y, 0), x = (I + D) c, z = FFT_n(x, 0), r[p] = z[p] / lambda'(omega_p).
// The identity term only adds FFT_n(c) = y to z, and y is zero on erased
// rows, so the erased outputs equal those of FFT_n(D c).

// n <= 16: one warp per 1024-column slice, the whole codeword column in registers.
template <int LOGN>
__device__ __forceinline__ void rec_small_body(const RecoverArgs& a, unsigned bx) {
  constexpr int N = 1 << LOGN;
  __shared__ uint8_t s_er[256], s_lam[256], s_ilp[256];
  if (threadIdx.x < 32) erasure_locator_warp(a, c_tab, s_er, s_lam, s_ilp);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t slice = (size_t)bx * (kThreads / 32) + warp;
  if (slice * 1024 >= a.L) return;
  const size_t cw = slice * 32 + lane;
  const ShiftMul km = make_shift_mul();
  uint32_t x[N][8];
#pragma unroll
  for (int r = 0; r < N; r++) {
    if (s_er[r]) {
#pragma unroll
      for (int p = 0; p < 8; p++) x[r][p] = 0;
    } else {
      gload(a.rx, r, row_pitch(a), a.L, cw, x[r], km);
      scale_rt(x[r], c_tab.exp[s_lam[r]]);
    }
  }
  block_ifft<0, LOGN, 0, 0, N>(x);
  one_plus_derivative<N>(x);
  block_fft<0, LOGN, 0, 0, N>(x);
#pragma unroll
  for (int r = 0; r < N; r++) {
    if (s_er[r]) {
      scale_rt(x[r], c_tab.exp[s_ilp[r]]);
      gstore(a.rx, r, row_pitch(a), a.L, cw, x[r], km);
    }
  }
}


// n >= 32: three phase kernels.  With c' = IFFT_bot(y) and c = IFFT_top(c'),
// the derivative splits over the row bits, D = D_top + D_bot, and D_bot
// commutes with the top butterflies (its row pairs differ below every top
// level, where no top twiddle depends), while FFT_top(c) = c'.  So
//   FFT_n(D c) = FFT_bot(u + D_bot c'),  u = FFT_top(D_top c),
// and with u' = FFT_top((I + D_top) c) = u + c' this is exactly
//   FFT_n(D c) = FFT_bot(u' + (I + D_bot) c'),
// where both I + D terms are computed in place (one_plus_derivative).
//   R1: y = lambda .* r on group g, c' = IFFT_bot  -> s1
//   R2: rows {b + 16m}: u' = FFT_top((I + D_top) IFFT_top(c'))  -> s2
//   R3: group g with erasures: FFT_bot(s2 + (I + D_bot) s1), Forney, store.
// Erasure locator of one recover call, computed on the host by the launcher
// and passed to the kernels as a parameter (constant bank): erased flags,
// log lambda(omega_x) and log 1/lambda'(omega_x).  Same log-domain
// Walsh-Hadamard computation as erasure_locator_warp (io.cuh), mod 255.
struct LocTable {
  uint8_t er[256], lam[256], ilp[256];
};

inline int host_mod255(int v) {
  v %= 255;
  return v < 0 ? v + 255 : v;
}

// Integer Walsh-Hadamard transform, no reduction: the transform is linear
// over the integers, so reducing mod 255 once at the end equals reducing at
// every step.  |inputs| <= 64516 (254 * 254) and n <= 256 keep every value
// within 32 bits.
inline void host_fwht(int* v, int n) {
  for (int h = 1; h < n; h <<= 1)
    for (int i = 0; i < n; i += 2 * h)
      for (int j = i; j < i + h; j++) {
        const int x = v[j], y = v[j + h];
        v[j] = x + y;
        v[j + h] = x - y;
      }
}

// Transform of log(omega_x) (0 at x = 0) mod 255 for n = 2^k points; it
// depends on n only, so it is computed once per n.
inline const int* host_log_omega_wht(int n) {
  static const std::array<std::array<int, 256>, 9> tabs = [] {
    std::array<std::array<int, 256>, 9> t{};
    for (int k = 0; k <= 8; k++) {
      const int m = 1 << k;
      int v[256] = {};
      for (int x = 1; x < m; x++) v[x] = kField.log[kField.omega[x]];
      host_fwht(v, m);
      for (int x = 0; x < m; x++) t[k][x] = host_mod255(v[x]);
    }
    return t;
  }();
  return tabs[__builtin_ctz((unsigned)n)].data();
}

inline void host_locator(const RecoverArgs& a, LocTable* t) {
  const int n = a.n;
  int ve[256] = {};
  *t = LocTable{};
  for (int j = 0; j < a.e; j++) {
    t->er[a.pos[j]] = 1;
    ve[a.pos[j]] = 1;
  }
  host_fwht(ve, n);
  const int* wl = host_log_omega_wht(n);
  for (int x = 0; x < n; x++) ve[x] = host_mod255(ve[x]) * wl[x];
  host_fwht(ve, n);
  const int k = __builtin_ctz((unsigned)n);
  const int ninv = (1 << (8 - k)) % 255;
  for (int x = 0; x < n; x++) {
    const int sv = host_mod255(host_mod255(ve[x]) * ninv);
    t->lam[x] = (uint8_t)sv;
    t->ilp[x] = (uint8_t)host_mod255(255 - sv);
  }
}

// The column windows and batches of one call, and repeated calls with one
// erasure pattern, share a locator: each host thread keeps its last one.
inline const LocTable& cached_locator(const RecoverArgs& a) {
  thread_local LocTable t;
  thread_local int n = 0, e = -1;
  thread_local uint8_t pos[256];
  if (a.n != n || a.e != e || std::memcmp(pos, a.pos, (size_t)a.e) != 0) {
    host_locator(a, &t);
    n = a.n;
    e = a.e;
    std::memcpy(pos, a.pos, (size_t)a.e);
  }
  return t;
}

template <int LOGN>
__global__ void __launch_bounds__(kThreads) k_rec_small(RecoverArgs a) {
  rec_small_body<LOGN>(a, blockIdx.x);
}

template <int LOGN>
__device__ __forceinline__ void rec_p2_body(const RecoverArgs& a, const Batch& bt, unsigned bx, int by) {
  constexpr int TL = LOGN - 4, TR = 1 << TL;
  griddep_wait();
  const size_t w = (size_t)bx * kPhaseThreads + threadIdx.x;
  if (w >= bt.ncw) return;
  const int b = by;
  uint32_t y[TR][8];
#pragma unroll
  for (int m = 0; m < TR; m++) xload(bt.s1, bt.ncw, b + 16 * m, w, y[m]);
  block_ifft<4, TL, 0, 0, TR>(y);
  one_plus_derivative<TR>(y);
  block_fft<4, TL, 0, 0, TR>(y);
  griddep_trigger();
#pragma unroll
  for (int m = 0; m < TR; m++) xstore(bt.s2, bt.ncw, b + 16 * m, w, y[m]);
}
template <int LOGN>
__global__ void __launch_bounds__(kPhaseThreads) k_rec_p2(RecoverArgs a, Batch bt) {
  rec_p2_body<LOGN>(a, bt, blockIdx.x, blockIdx.y);
}

// blockIdx.y indexes the list of groups holding at least one erasure.
struct GroupList {
  int count;
  uint8_t g[16];
};


// R1 (split): lambda-scale + bottom IFFT of group g = blockIdx.y.
template <int LOGN>
__device__ __forceinline__ void rec_b1_body(const RecoverArgs& a, const Batch& bt, unsigned bx, int by, uint32_t* st,
                                            const LocTable& loc) {
  constexpr int RW = kRowsPerWarp, WG = Split<RW>::WG, LR = Split<RW>::LR;
  constexpr int G = (1 << LOGN) / 16;
  const SplitPos<RW> q = split_pos<RW>(bt.ncw, bx);
  const ShiftMul km = make_shift_mul();
  const int g = by;
  const int row0 = 16 * g + RW * q.q;
  uint32_t x[RW][8];
  zero_rows(x);
  if (q.active) {
    uint32_t skip = 0;
#pragma unroll
    for (int i = 0; i < RW; i++) skip |= (uint32_t)(loc.er[row0 + i] != 0) << i;
    stage_rows<RW>(st, a.rx, row0, row_pitch(a), a.L, bt.cw0 + q.w, skip);
#pragma unroll 1
    for (int i = 0; i < RW; i++) {
      if ((skip >> i) & 1) continue;
      uint32_t y[8];
      s_get(st, i, threadIdx.x, y);
      transpose8f(y, km);
      scale_log(y, loc.lam[row0 + i]);
      s_put(st, i, threadIdx.x, y);
    }
#pragma unroll
    for (int i = 0; i < RW; i++) s_get(st, i, threadIdx.x, x[i]);
  }
  const int gq = g * WG + q.q;
  dispatch<0, G * WG - 1>(gq, [&](auto vv) {
    constexpr int VV = decltype(vv)::value;
    block_ifft<0, LR, VV, 0, RW>(x);
  });
  static_for<4 - LR>([&](auto jj) {
    constexpr int J = LR + decltype(jj)::value;
    xchg_put<RW>(st, x);
    dispatch<0, G * WG - 1>(gq, [&](auto vv) {
      constexpr int GG = decltype(vv)::value / WG, Q = decltype(vv)::value % WG;
      constexpr int TW = twiddle_c(J, 0, (16 * GG + RW * Q) & ~((2 << J) - 1));
      combine_ifft<TW, (Q >> (J - LR)) & 1, RW>(st, x, threadIdx.x ^ (32 << (J - LR)));
    });
  });
  griddep_trigger();
  if (q.active) {
#pragma unroll
    for (int i = 0; i < RW; i++) xstore(bt.s1, bt.ncw, row0 + i, q.w, x[i]);
  }
}

// R3 (split): x = s2 + (I + D_bot) s1 on group g, bottom FFT, Forney, store
// the erased rows.  (I + D_bot) = (I + D over the in-warp bits) applied in
// registers, plus, for each cross-warp bit j that is clear in the warp's rows,
// the ORIGINAL row i of the warp whose rows have bit j set.
template <int LOGN>
__device__ __forceinline__ void rec_b3_body(const RecoverArgs& a, const Batch& bt, unsigned bx, int g, uint32_t* st,
                                            const LocTable& loc) {
  griddep_wait();
  constexpr int RW = kRowsPerWarp, WG = Split<RW>::WG, LR = Split<RW>::LR;
  constexpr int G = (1 << LOGN) / 16;
  const SplitPos<RW> q = split_pos<RW>(bt.ncw, bx);
  const ShiftMul km = make_shift_mul();
  const int row0 = 16 * g + RW * q.q;
  const int tid = threadIdx.x;
  uint32_t x[RW][8];
  zero_rows(x);
  if (q.active) {
#pragma unroll
    for (int i = 0; i < RW; i++) xload(bt.s1, bt.ncw, row0 + i, q.w, x[i]);
  }
#pragma unroll
  for (int i = 0; i < RW; i++) s_put(st, i, tid, x[i]);  // original c' for the partners
  __syncthreads();
  one_plus_derivative<RW>(x);
#pragma unroll
  for (int j = LR; j < 4; j++) {
    if ((q.q >> (j - LR)) & 1) continue;
    const int ptid = tid ^ (32 << (j - LR));
#pragma unroll
    for (int i = 0; i < RW; i++) {
      uint32_t y[8];
      s_get(st, i, ptid, y);
#pragma unroll
      for (int p = 0; p < 8; p++) x[i][p] ^= y[p];
    }
  }
  if (q.active) {
#pragma unroll
    for (int i = 0; i < RW; i++) {
      uint32_t u[8];
      xload(bt.s2, bt.ncw, row0 + i, q.w, u);
#pragma unroll
      for (int p = 0; p < 8; p++) x[i][p] ^= u[p];
    }
  }
  const int gq = g * WG + q.q;
  static_for<4 - LR>([&](auto jj) {
    constexpr int J = 3 - decltype(jj)::value;
    xchg_put<RW>(st, x);
    dispatch<0, G * WG - 1>(gq, [&](auto vv) {
      constexpr int GG = decltype(vv)::value / WG, Q = decltype(vv)::value % WG;
      constexpr int TW = twiddle_c(J, 0, (16 * GG + RW * Q) & ~((2 << J) - 1));
      combine_fft<TW, (Q >> (J - LR)) & 1, RW>(st, x, tid ^ (32 << (J - LR)));
    });
  });
  __syncthreads();  // partners' reads of the stage are done
  // Both scratch buffers' rows were consumed into x, which was stored to
  // shared memory before the barriers above.
  discard_rows<RW>(bt.s1, bt.ncw, row0, q.w - (tid & 31));
  discard_rows<RW>(bt.s2, bt.ncw, row0, q.w - (tid & 31));
  dispatch<0, G * WG - 1>(gq, [&](auto vv) {
    constexpr int VV = decltype(vv)::value;
    block_fft<0, LR, VV, 0, RW>(x);
  });
  if (q.active) {
#pragma unroll
    for (int i = 0; i < RW; i++) s_put(st, i, tid, x[i]);
#pragma unroll 1
    for (int i = 0; i < RW; i++) {
      const int r = row0 + i;
      if (!loc.er[r]) continue;
      uint32_t y[8];
      s_get(st, i, tid, y);
      scale_log(y, loc.ilp[r]);
      gstore(a.rx, r, row_pitch(a), a.L, bt.cw0 + q.w, y, km);
    }
  }
}

template <int LOGN>
__global__ void __launch_bounds__(kSplitThreads, 4) k_rec_b1(RecoverArgs a, Batch bt, const __grid_constant__ LocTable loc) {
  extern __shared__ uint32_t st[];
  rec_b1_body<LOGN>(a, bt, blockIdx.x, blockIdx.y, st, loc);
}
template <int LOGN>
__global__ void __launch_bounds__(kSplitThreads, 4)
    k_rec_b3(RecoverArgs a, Batch bt, GroupList gl, const __grid_constant__ LocTable loc) {
  extern __shared__ uint32_t st[];
  rec_b3_body<LOGN>(a, bt, blockIdx.x, gl.g[blockIdx.y], st, loc);
}

// ---- one launch per call for short shards ---------------------------------
// Encodes with t = 32 or 64 and recovers with n = 32 .. 128: one CTA per
// 1024-column slice holds every row of a transform for its 32 colwords, 8
// rows per warp (t / 8 or n / 8 warps).  Levels 0..2 run inside a warp and
// the higher ones pair warps through shared memory, as level 3 does in the
// bottom passes; there is no scratch and no second launch.  Every warp runs
// its own compile-time variant of each level, so a CTA fetches the code of
// all of them: the route table picks this form where the three dependent
// launches and scratch round trips of the phase kernels cost more (short
// shards).  A partial last slice is handled by the bounds of the row loads
// and stores.
template <int ROWS>
constexpr int fused_threads() {
  return ROWS / kRowsPerWarp * 32;
}
template <int ROWS>
constexpr size_t fused_smem() {
  return (size_t)kRowsPerWarp * 32 * fused_threads<ROWS>();
}

// IFFT levels [3, LOG) at coset BETA over the warps of the CTA (warp q holds
// rows 8q .. 8q + 7 of the transform).
template <int LOG, int BETA, int NT>
__device__ __forceinline__ void fused_ifft_top(uint32_t* st, uint32_t (&x)[kRowsPerWarp][8], int q) {
  constexpr int RW = kRowsPerWarp, NW = NT / 32;
  static_for<LOG - 3>([&](auto jj) {
    constexpr int J = 3 + decltype(jj)::value;
    xchg_put<RW, NT>(st, x);
    dispatch<0, NW - 1>(q, [&](auto vv) {
      constexpr int Q = decltype(vv)::value;
      constexpr int TW = twiddle_c(J, static_cast<uint8_t>(BETA), (RW * Q) & ~((2 << J) - 1));
      combine_ifft<TW, (Q >> (J - 3)) & 1, RW, NT>(st, x, threadIdx.x ^ (32 << (J - 3)));
    });
  });
}

// FFT levels LOG - 1 .. 3 at coset 0 over the warps of the CTA.
template <int LOG, int NT>
__device__ __forceinline__ void fused_fft_top(uint32_t* st, uint32_t (&x)[kRowsPerWarp][8], int q) {
  constexpr int RW = kRowsPerWarp, NW = NT / 32;
  static_for<LOG - 3>([&](auto jj) {
    constexpr int J = LOG - 1 - decltype(jj)::value;
    xchg_put<RW, NT>(st, x);
    dispatch<0, NW - 1>(q, [&](auto vv) {
      constexpr int Q = decltype(vv)::value;
      constexpr int TW = twiddle_c(J, 0, (RW * Q) & ~((2 << J) - 1));
      combine_fft<TW, (Q >> (J - 3)) & 1, RW, NT>(st, x, threadIdx.x ^ (32 << (J - 3)));
    });
  });
}

// Rows row0 .. row0 + 7 of `base` (colword w) into x, bit-sliced; the rows
// with a bit set in `skip` are zero.  Starts with a barrier (the stage may
// still be read by partner warps).
template <int NT>
__device__ __forceinline__ void fused_load(uint32_t* st, const uint8_t* base, size_t row0, size_t pitch, size_t L,
                                           size_t w, uint32_t skip, uint32_t (&x)[kRowsPerWarp][8],
                                           const ShiftMul& km) {
  constexpr int RW = kRowsPerWarp;
  __syncthreads();
  stage_rows<RW, NT>(st, base, row0, pitch, L, w, skip);
#pragma unroll 1
  for (int i = 0; i < RW; i++) {
    uint32_t y[8];
    s_get<NT>(st, i, threadIdx.x, y);
    transpose8f(y, km);
    s_put<NT>(st, i, threadIdx.x, y);
  }
#pragma unroll
  for (int i = 0; i < RW; i++) s_get<NT>(st, i, threadIdx.x, x[i]);
}

// codec.rs:241-265 in one launch: parity = FFT_t(parity_in? + sum_c
// IFFT_t(chunk c, omega_ct), 0), the accumulator in registers.
template <int LOGN, int LOGT>
__device__ __forceinline__ void enc_fused_body(const EncodeArgs& a, unsigned bx, uint32_t* st) {
  constexpr int RW = kRowsPerWarp, T = 1 << LOGT, C = (1 << LOGN) / T - 1;
  constexpr int NT = fused_threads<T>(), NW = NT / 32;
  const int tid = threadIdx.x, q = tid >> 5;
  const size_t w = (size_t)bx * 32 + (tid & 31);
  const ShiftMul km = make_shift_mul();
  uint32_t acc[RW][8];
  static_for<C>([&](auto cc) {
    constexpr int c = decltype(cc)::value + 1;
    uint32_t x[RW][8];
    fused_load<NT>(st, a.msg, (size_t)(c - 1) * T + RW * q, row_pitch(a), a.L, w, 0, x, km);
    dispatch<0, NW - 1>(q, [&](auto vv) { block_ifft<0, 3, decltype(vv)::value, omega_c(c * T), RW>(x); });
    fused_ifft_top<LOGT, omega_c(c * T), NT>(st, x, q);
#pragma unroll
    for (int i = 0; i < RW; i++)
#pragma unroll
      for (int p = 0; p < 8; p++) acc[i][p] = c == 1 ? x[i][p] : acc[i][p] ^ x[i][p];
  });
  if (a.accumulate) {
    uint32_t x[RW][8];
    fused_load<NT>(st, a.parity, (size_t)RW * q, row_pitch(a), a.L, w, 0, x, km);
#pragma unroll
    for (int i = 0; i < RW; i++)
#pragma unroll
      for (int p = 0; p < 8; p++) acc[i][p] ^= x[i][p];
  }
  fused_fft_top<LOGT, NT>(st, acc, q);
  dispatch<0, NW - 1>(q, [&](auto vv) { block_fft<0, 3, decltype(vv)::value, 0, RW>(acc); });
  __syncthreads();  // partners' reads of the stage are done
#pragma unroll
  for (int i = 0; i < RW; i++) s_put<NT>(st, i, tid, acc[i]);
#pragma unroll 1
  for (int i = 0; i < RW; i++) {
    uint32_t y[8];
    s_get<NT>(st, i, tid, y);
    gstore(a.parity, (size_t)RW * q + i, row_pitch(a), a.L, w, y, km);
  }
}

// The decoder of the three recover phases in one launch: y = lambda .* r,
// c = IFFT_n(y), (I + D) c, FFT_n, Forney on the erased rows (whose y is
// zero, so the identity term adds nothing there).
template <int LOGN>
__device__ __forceinline__ void rec_fused_body(const RecoverArgs& a, unsigned bx, uint32_t* st, const LocTable& loc) {
  constexpr int RW = kRowsPerWarp, NT = fused_threads<(1 << LOGN)>(), NW = NT / 32;
  const int tid = threadIdx.x, q = tid >> 5, row0 = RW * q;
  const size_t w = (size_t)bx * 32 + (tid & 31);
  const ShiftMul km = make_shift_mul();
  uint32_t x[RW][8];
  uint32_t skip = 0;
#pragma unroll
  for (int i = 0; i < RW; i++) skip |= (uint32_t)(loc.er[row0 + i] != 0) << i;
  stage_rows<RW, NT>(st, a.rx, row0, row_pitch(a), a.L, w, skip);
#pragma unroll 1
  for (int i = 0; i < RW; i++) {
    if ((skip >> i) & 1) continue;
    uint32_t y[8];
    s_get<NT>(st, i, tid, y);
    transpose8f(y, km);
    scale_log(y, loc.lam[row0 + i]);
    s_put<NT>(st, i, tid, y);
  }
#pragma unroll
  for (int i = 0; i < RW; i++) s_get<NT>(st, i, tid, x[i]);
  dispatch<0, NW - 1>(q, [&](auto vv) { block_ifft<0, 3, decltype(vv)::value, 0, RW>(x); });
  fused_ifft_top<LOGN, 0, NT>(st, x, q);
  // (I + D): the in-warp bits in registers; for each warp bit clear in this
  // warp's rows, the original rows of the partner warp that has it set.
  __syncthreads();  // partners' reads of the stage are done
#pragma unroll
  for (int i = 0; i < RW; i++) s_put<NT>(st, i, tid, x[i]);
  __syncthreads();
  one_plus_derivative<RW>(x);
#pragma unroll
  for (int j = 3; j < LOGN; j++) {
    if ((q >> (j - 3)) & 1) continue;
    const int ptid = tid ^ (32 << (j - 3));
#pragma unroll
    for (int i = 0; i < RW; i++) {
      uint32_t y[8];
      s_get<NT>(st, i, ptid, y);
#pragma unroll
      for (int p = 0; p < 8; p++) x[i][p] ^= y[p];
    }
  }
  fused_fft_top<LOGN, NT>(st, x, q);
  dispatch<0, NW - 1>(q, [&](auto vv) { block_fft<0, 3, decltype(vv)::value, 0, RW>(x); });
  __syncthreads();  // partners' reads of the stage are done
#pragma unroll
  for (int i = 0; i < RW; i++) s_put<NT>(st, i, tid, x[i]);
#pragma unroll 1
  for (int i = 0; i < RW; i++) {
    const int r = row0 + i;
    if (!loc.er[r]) continue;
    uint32_t y[8];
    s_get<NT>(st, i, tid, y);
    scale_log(y, loc.ilp[r]);
    gstore(a.rx, (size_t)r, row_pitch(a), a.L, w, y, km);
  }
}

template <int LOGN, int LOGT>
__global__ void __launch_bounds__(fused_threads<(1 << LOGT)>(), 1) k_enc_fused(EncodeArgs a) {
  extern __shared__ uint32_t st[];
  enc_fused_body<LOGN, LOGT>(a, blockIdx.x, st);
}
template <int LOGN>
__global__ void __launch_bounds__(fused_threads<(1 << LOGN)>(), 1)
    k_rec_fused(RecoverArgs a, const __grid_constant__ LocTable loc) {
  extern __shared__ uint32_t st[];
  rec_fused_body<LOGN>(a, blockIdx.x, st, loc);
}

// Grouped recover (see EncJob): gmask bit g is set when row group g holds an
// erasure of this codeword; the last pass runs only those groups.
struct RecJob {
  RecoverArgs a;
  uint32_t* s1;
  uint32_t* s2;
  size_t ncw;
  uint32_t gmask;
  LocTable loc;
};
// Grouped n <= 16 recover (the whole column in registers, own locator).
template <int LOGN>
__global__ void __launch_bounds__(kThreads) k_rec_small_jobs(const RecJob* __restrict__ jobs) {
  const RecJob& j = jobs[blockIdx.z];
  if ((size_t)blockIdx.x * (kThreads / 32) * 1024 >= j.a.L) return;
  rec_small_body<LOGN>(j.a, blockIdx.x);
}

// The erasure tables of every codeword of a group, one warp per codeword
// (the same log-domain tables host_locator computes for a single call).
static __global__ void __launch_bounds__(32) k_rec_jobs_locator(RecJob* __restrict__ jobs) {
  __shared__ uint8_t s_er[256], s_lam[256], s_ilp[256];
  RecJob& j = jobs[blockIdx.x];
  erasure_locator_warp(j.a, c_tab, s_er, s_lam, s_ilp);
  __syncwarp();
  for (int i = threadIdx.x; i < j.a.n; i += 32) {
    j.loc.er[i] = s_er[i];
    j.loc.lam[i] = s_lam[i];
    j.loc.ilp[i] = s_ilp[i];
  }
}
template <int LOGN>
__global__ void __launch_bounds__(kSplitThreads, 4) k_rec_b1_jobs(const RecJob* __restrict__ jobs) {
  extern __shared__ uint32_t st[];
  const RecJob& j = jobs[blockIdx.y];
  if ((size_t)blockIdx.x * Split<kRowsPerWarp>::CW >= j.ncw) return;
  rec_b1_body<LOGN>(j.a, Batch{j.s1, j.s2, j.ncw, 0}, blockIdx.x, blockIdx.z, st, j.loc);
}
template <int LOGN>
__global__ void __launch_bounds__(kPhaseThreads) k_rec_p2_jobs(const RecJob* __restrict__ jobs) {
  const RecJob& j = jobs[blockIdx.z];
  rec_p2_body<LOGN>(j.a, Batch{j.s1, j.s2, j.ncw, 0}, blockIdx.x, blockIdx.y);
}
template <int LOGN>
__global__ void __launch_bounds__(kSplitThreads, 4) k_rec_b3_jobs(const RecJob* __restrict__ jobs) {
  extern __shared__ uint32_t st[];
  const RecJob& j = jobs[blockIdx.y];
  if ((size_t)blockIdx.x * Split<kRowsPerWarp>::CW >= j.ncw || !((j.gmask >> blockIdx.z) & 1u)) return;
  rec_b3_body<LOGN>(j.a, Batch{j.s1, j.s2, j.ncw, 0}, blockIdx.x, blockIdx.z, st, j.loc);
}

// ---- recover, few erasures ------------------------------------------------
// For 1 <= e <= 8 erasures: T = 2^ceil(log2 e) and the n/T chunks of T rows at
// cosets omega_{iT}.  S = xor_i IFFT_T(chunk i, omega_{iT}) equals the top T
// coefficients (n - T .. n - 1) of the word's polynomial in the LCH basis of
// the Cantor basis: X_{uT + v} = X_{uT} X_v, X_{uT} is constant on each
// chunk's coset, and its sum over the cosets is 1 for u = n/T - 1 and 0
// below.  The decoder's output (rs/src/codec.rs:479-569, the Leopard form of
// the phase kernels above) is the polynomial of degree < n - e through the
// surviving rows, whose coefficients n - e .. n - 1 vanish.  With the erased
// rows read as zero, S = S_known + V x over the erased values x, so
// x = V_R^{-1} S_known[R] for the rows R = T - e .. T - 1 of S, on every input.
// V_R^{-1} depends only on the erasure pattern and is computed on the host;
// the kernel is one pass over the survivors (the chunk IFFTs of the t <= 16
// encoder) and an e x e multiply by runtime constants, with no scratch.
constexpr int kFewMax = 8;
struct FewTable {
  uint32_t er[8];    // erased rows, bit r of er[r / 32]
  uint64_t m[8][8];  // output j, plane p: bit 8 r + q takes plane q of S[T - e + r]
  uint8_t row[8];    // row of output j
  int e;
};

inline int few_logt(int e) {
  int l = 0;
  while ((1 << l) < e) l++;
  return l;
}

// IFFT of T = 2^logt bytes at coset beta: the map block_ifft applies to
// bit-sliced rows (bf_inv: b ^= a, a ^= s_j(beta + omega_base) b).
inline void host_ifft_bytes(uint8_t* v, int logt, uint8_t beta) {
  const int T = 1 << logt;
  for (int lv = 0; lv < logt; lv++)
    for (int i = 0; i < T; i++) {
      if ((i >> lv) & 1) continue;
      const int j = i + (1 << lv);
      const uint8_t tw = kField.spv[lv][static_cast<uint8_t>(beta ^ kField.omega[i & ~((2 << lv) - 1)])];
      v[j] ^= v[i];
      v[i] ^= gf_mul(tw, v[j]);
    }
}

inline uint8_t host_gf_mul(uint8_t a, uint8_t b) {
  return a && b ? kField.exp[kField.log[a] + kField.log[b]] : 0;
}

// The table of one erasure pattern; false when V_R is singular, which the
// argument above rules out (the caller then runs the phase kernels).
inline bool host_few_table(const RecoverArgs& a, FewTable* ft) {
  const int e = a.e, lt = few_logt(e), T = 1 << lt, r0 = T - e;
  *ft = FewTable{};
  ft->e = e;
  uint8_t aug[kFewMax][2 * kFewMax] = {};  // [V_R | I]
  for (int j = 0; j < e; j++) {
    const int p = a.pos[j];
    ft->er[p >> 5] |= 1u << (p & 31);
    ft->row[j] = static_cast<uint8_t>(p);
    uint8_t u[kFewMax] = {};
    u[p & (T - 1)] = 1;
    host_ifft_bytes(u, lt, kField.omega[p & ~(T - 1)]);
    for (int r = 0; r < e; r++) aug[r][j] = u[r0 + r];
    aug[j][e + j] = 1;
  }
  for (int c = 0; c < e; c++) {  // Gauss-Jordan over GF(2^8)
    int piv = c;
    while (piv < e && !aug[piv][c]) piv++;
    if (piv == e) return false;
    if (piv != c)
      for (int k = 0; k < 2 * e; k++) std::swap(aug[piv][k], aug[c][k]);
    const uint8_t inv = kField.exp[255 - kField.log[aug[c][c]]];
    for (int k = 0; k < 2 * e; k++) aug[c][k] = host_gf_mul(aug[c][k], inv);
    for (int r = 0; r < e; r++) {
      const uint8_t f = aug[r][c];
      if (r == c || !f) continue;
      for (int k = 0; k < 2 * e; k++) aug[r][k] ^= host_gf_mul(f, aug[c][k]);
    }
  }
  // Coefficient b = V_R^{-1}[j][r]: byte q of `cols` is b * 2^q; after an 8x8
  // bit transpose, byte p holds bit p of every b * 2^q, i.e. the planes q of
  // S[r0 + r] that plane p of output j takes.
  for (int j = 0; j < e; j++)
    for (int r = 0; r < e; r++) {
      uint8_t b = aug[j][e + r];
      uint64_t cols = 0;
      for (int q = 0; q < 8; q++) {
        cols |= static_cast<uint64_t>(b) << (8 * q);
        b = static_cast<uint8_t>((b << 1) ^ ((b & 0x80) ? 0x1d : 0));
      }
      uint64_t t = (cols ^ (cols >> 7)) & 0x00AA00AA00AA00AAull;
      cols ^= t ^ (t << 7);
      t = (cols ^ (cols >> 14)) & 0x0000CCCC0000CCCCull;
      cols ^= t ^ (t << 14);
      t = (cols ^ (cols >> 28)) & 0x00000000F0F0F0F0ull;
      cols ^= t ^ (t << 28);
      for (int p = 0; p < 8; p++) ft->m[j][p] |= ((cols >> (8 * p)) & 0xff) << (8 * r);
    }
  return true;
}

// Repeated calls with one erasure pattern (and the column windows of one
// call) share a table: each host thread keeps its last one.  nullptr when
// the pattern has none.
inline const FewTable* cached_few_table(const RecoverArgs& a) {
  thread_local FewTable t;
  thread_local bool ok = false;
  thread_local int e = -1;
  thread_local uint8_t pos[kFewMax];
  if (a.e != e || std::memcmp(pos, a.pos, (size_t)a.e) != 0) {
    ok = host_few_table(a, &t);
    e = a.e;
    std::memcpy(pos, a.pos, (size_t)a.e);
  }
  return ok ? &t : nullptr;
}

// One CTA, or a cluster of nc CTAs, per 1024-column slice: the cluster's
// warps split the chunks (warp g = rank * 8 + w takes chunks g, g + 8 nc,
// ...) and XOR-accumulate their IFFTs in shared memory; each CTA sums its
// warps' rows, CTA 0 adds the other CTAs' sums through distributed shared
// memory, then its warp j computes erased row j.  With T = 1 the chunk IFFT
// is the identity and the bit transpose is linear, so raw bytes are XORed and
// transposed once.  Clusters give short shards (few slices) more SMs.
template <int LOGN, int LOGT>
__device__ __forceinline__ void rec_few_body(const RecoverArgs& a, const FewTable& ft, unsigned bx, unsigned rank,
                                             unsigned nc, uint32_t* sm) {
  constexpr int N = 1 << LOGN, T = 1 << LOGT, NC = N / T, W = kThreads / 32;
  constexpr int kRows = T * 8 * 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if ((size_t)bx * 1024 >= a.L) return;  // the whole CTA (the whole cluster: bx is shared)
  const int g0 = (int)rank * W;            // this CTA's first warp in the cluster
  const int WU = NC - g0 < W ? (NC - g0 > 0 ? NC - g0 : 0) : W;  // its warps that get chunks
  const size_t cw = (size_t)bx * 32 + lane;
  const ShiftMul km = make_shift_mul();
  const size_t pitch = row_pitch(a);
  // T = 8 accumulates in the warp's shared-memory rows, so that two CTAs
  // fit an SM (at most 128 registers).
  constexpr bool kSmemAcc = LOGT >= 3;
  if (warp < WU) {
    uint32_t* wacc = sm + warp * kRows;
    uint32_t acc[kSmemAcc ? 1 : T][8];
    zero_rows(acc);
    for (int c = g0 + warp; c < NC; c += W * (int)nc) {
      uint32_t x[T][8];
#pragma unroll
      for (int r = 0; r < T; r++) {
        const int row = c * T + r;
        if ((ft.er[row >> 5] >> (row & 31)) & 1u) {
#pragma unroll
          for (int p = 0; p < 8; p++) x[r][p] = 0;
        } else if constexpr (LOGT == 0) {
          load_cw(a.rx + (size_t)row * pitch, a.L, cw, x[r]);
        } else {
          gload(a.rx, row, pitch, a.L, cw, x[r], km);
        }
      }
      if constexpr (LOGT > 0) {
        dispatch<0, NC - 1>(c, [&](auto cc) {
          constexpr int CC = decltype(cc)::value;
          block_ifft<0, LOGT, 0, omega_c(CC * T), T>(x);
        });
      }
      if constexpr (kSmemAcc) {
        const bool first = c == g0 + warp;
#pragma unroll
        for (int r = 0; r < T; r++) {
          if (!first) {
            uint32_t y[8];
            sload<32>(wacc, r, lane, y);
#pragma unroll
            for (int p = 0; p < 8; p++) x[r][p] ^= y[p];
          }
          sstore<32>(wacc, r, lane, x[r]);
        }
      } else {
#pragma unroll
        for (int r = 0; r < T; r++)
#pragma unroll
          for (int p = 0; p < 8; p++) acc[r][p] ^= x[r][p];
      }
    }
    if constexpr (!kSmemAcc) {
      if constexpr (LOGT == 0) transpose8f(acc[0], km);
#pragma unroll
      for (int r = 0; r < T; r++) sstore<32>(wacc, r, lane, acc[r]);
    }
  }
  __syncthreads();
  for (int r = warp; r < T; r += W) {
    uint32_t y[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int w = 0; w < WU; w++) {
      uint32_t z[8];
      sload<32>(sm + w * kRows, r, lane, z);
#pragma unroll
      for (int p = 0; p < 8; p++) y[p] ^= z[p];
    }
    sstore<32>(sm, r, lane, y);
  }
  if (nc > 1) {
    // Every CTA's sums are in its region 0; CTA 0 reads the others' (their
    // shared memory stays live until the second barrier).
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    if (rank == 0) {
      for (int r = warp; r < T; r += W) {
        uint32_t y[8];
        sload<32>(sm, r, lane, y);
        for (unsigned k = 1; k < nc; k++) {
          uint32_t z[8];
          sload<32>(cluster.map_shared_rank(sm, k), r, lane, z);
#pragma unroll
          for (int p = 0; p < 8; p++) y[p] ^= z[p];
        }
        sstore<32>(sm, r, lane, y);
      }
    }
    cluster.sync();
    if (rank != 0) return;
  } else {
    __syncthreads();
  }
  if (warp >= ft.e) return;
  const int r0 = T - ft.e;
  uint32_t y[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int r = 0; r < T; r++) {
    if (r < r0) continue;
    uint32_t s[8];
    sload<32>(sm, r, lane, s);
#pragma unroll
    for (int p = 0; p < 8; p++) {
      const uint32_t mm = static_cast<uint32_t>(ft.m[warp][p] >> (8 * (r - r0)));
#pragma unroll
      for (int q = 0; q < 8; q++)
        if ((mm >> q) & 1u) y[p] ^= s[q];  // warp-uniform: a predicated XOR
    }
  }
  gstore(a.rx, ft.row[warp], pitch, a.L, cw, y, km);
}

// CTAs per SM the few-erasure kernels are compiled for (register caps 64,
// 85, 128, 128 for T = 1, 2, 4, 8; without caps ptxas takes up to 174).
constexpr int few_min_ctas(int logt) { return logt == 0 ? 4 : (logt == 1 ? 3 : 2); }

template <int LOGN, int LOGT>
__global__ void __launch_bounds__(kThreads, few_min_ctas(LOGT)) k_rec_few(RecoverArgs a, const __grid_constant__ FewTable ft) {
  extern __shared__ uint32_t sm[];
  const unsigned nc = cooperative_groups::this_cluster().num_blocks();
  rec_few_body<LOGN, LOGT>(a, ft, blockIdx.x / nc, blockIdx.x % nc, nc, sm);
}

template <int LOGN, int LOGT>
constexpr size_t few_smem() {
  constexpr int NC = (1 << LOGN) >> LOGT, W = kThreads / 32;
  return (size_t)(NC < W ? NC : W) * (1 << LOGT) * 8 * 32 * 4;
}

// Grouped few-erasure recovers (afrs_batch_dev): codewords of one n and one
// chunk size T, blockIdx.y = codeword, each with the table of its pattern.
struct FewJob {
  RecoverArgs a;
  FewTable ft;
};
template <int LOGN, int LOGT>
__global__ void __launch_bounds__(kThreads, few_min_ctas(LOGT)) k_rec_few_jobs(const FewJob* __restrict__ jobs) {
  extern __shared__ uint32_t sm[];
  const FewJob& j = jobs[blockIdx.y];
  if ((size_t)blockIdx.x * 1024 >= j.a.L) return;
  rec_few_body<LOGN, LOGT>(j.a, j.ft, blockIdx.x, 0, 1, sm);
}

// ---- launchers ------------------------------------------------------------

// Launch that may start before the previous kernel on the stream has
// finished (programmatic stream serialization); the kernel must begin with
// griddep_wait() before it touches that kernel's output.
template <class... KArgs, class... Args>
cudaError_t launch_dependent(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                             Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

// Scratch budget per column batch.  Larger batches mean fewer launches and
// fuller waves, which outweighs keeping the scratch inside L2: n = 256 with
// 4 MiB shards, recover 1856 us (128 MiB) -> 1623 (256) -> 1463 (512) ->
// 1407 us (1 GiB).
constexpr size_t kScratchBudget = (size_t)1 << 30;

// Colwords covering L bytes in the io.cuh layout (whole 1024-column slices).
inline size_t total_colwords(size_t L) { return (L + 1023) / 1024 * 32; }

inline size_t batch_colwords(size_t rows_per_buffer, int buffers, size_t scratch_bytes, size_t total_cw) {
  const size_t per_cw = rows_per_buffer * 32 * (size_t)buffers;
  size_t cap = scratch_bytes < kScratchBudget ? scratch_bytes : kScratchBudget;
  size_t cw = cap / per_cw;
  if (cw > total_cw) cw = total_cw;
  return cw;
}

template <int LOGN, int LOGT>
cudaError_t launch_enc(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s) {
  if constexpr (LOGT <= 4) {
    constexpr int C = ((1 << LOGN) >> LOGT) - 1;
    const size_t slices = (a.L + 1023) / 1024;
    const bool split = a.layout >= 0 ? (a.layout != 0 && C > 1) : enc_small_split<LOGN, LOGT>(slices);
    const size_t smem = enc_small_smem<LOGN, LOGT>(split);
    auto fn = split ? k_enc_small<LOGN, LOGT, true> : k_enc_small<LOGN, LOGT, false>;
    if (smem > (48 << 10)) {
      cudaError_t e = ensure_smem_attr(reinterpret_cast<const void*>(fn), smem);
      if (e != cudaSuccess) return e;
    }
    fn<<<enc_small_ctas<LOGN, LOGT>(slices, split), kThreads, smem, s>>>(a);
    count_launches(1);
    return cudaGetLastError();
  } else {
    constexpr int N = 1 << LOGN, T = 1 << LOGT, C = N / T - 1, G = T / 16;
    if constexpr (LOGT == 5 || LOGT == 6) {
      const size_t slices = (a.L + 1023) / 1024;
      if (a.layout == kLayoutFused && slices <= 0x7fffffff) {
        constexpr size_t smem = fused_smem<T>();
        if constexpr (smem > (48 << 10)) {
          cudaError_t e = ensure_smem_attr(reinterpret_cast<const void*>(k_enc_fused<LOGN, LOGT>), smem);
          if (e != cudaSuccess) return e;
        }
        k_enc_fused<LOGN, LOGT><<<(unsigned)slices, fused_threads<T>(), smem, s>>>(a);
        count_launches(1);
        return cudaGetLastError();
      }
    }
    const size_t total_cw = total_colwords(a.L);
    const size_t bcw = batch_colwords(N - T, 1, sc.bytes, total_cw);
    if (bcw == 0) return cudaErrorMemoryAllocation;
    for (size_t cw0 = 0; cw0 < total_cw; cw0 += bcw) {
      Batch bt{sc.ptr, nullptr, (total_cw - cw0 < bcw ? total_cw - cw0 : bcw), cw0};
      const unsigned gx = (unsigned)((bt.ncw + kPhaseThreads - 1) / kPhaseThreads);
      constexpr int SCW = Split<kRowsPerWarp>::CW;
      constexpr size_t kStage = Split<kRowsPerWarp>::kStage;
      const unsigned gs = (unsigned)((bt.ncw + SCW - 1) / SCW);
      k_enc_b1<LOGN, LOGT><<<dim3(gs, C * G), kSplitThreads, kStage, s>>>(a, bt);
      cudaError_t e = launch_dependent(k_enc_p2<LOGN, LOGT>, dim3(gx, 16), dim3(kPhaseThreads), 0, s, a, bt);
      if (e == cudaSuccess)
        e = launch_dependent(k_enc_b3<LOGN, LOGT>, dim3(gs, G), dim3(kSplitThreads), kStage, s, a, bt);
      if (e != cudaSuccess) return e;
      count_launches(3);
    }
    return cudaGetLastError();
  }
}

template <int LOGN, int LOGT>
cudaError_t launch_rec_few_t(const RecoverArgs& a, const FewTable& ft, cudaStream_t s) {
  constexpr size_t smem = few_smem<LOGN, LOGT>();
  if constexpr (smem > (48 << 10)) {
    cudaError_t e = ensure_smem_attr(reinterpret_cast<const void*>(k_rec_few<LOGN, LOGT>), smem);
    if (e != cudaSuccess) return e;
  }
  // Clusters of up to 8 CTAs per slice while the slices alone would leave
  // SMs idle (below two CTAs per SM), each warp keeping at least one chunk
  // and four rows (n = 32 and 64 measured slower with smaller shares: the
  // cluster barriers cost more than the rows); one CTA per slice otherwise.
  const size_t slices = (a.L + 1023) / 1024;
  constexpr unsigned kChunkCap = (unsigned)(((1 << LOGN) >> LOGT) + kThreads / 32 - 1) / (kThreads / 32);
  constexpr unsigned kRowCap = (1u << LOGN) / 32;
  constexpr unsigned kCap = kChunkCap < kRowCap ? kChunkCap : kRowCap;
  unsigned nc = 1;
  while (nc < 8 && 2 * nc <= kCap && slices * nc < 2 * 148) nc *= 2;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(slices * nc));
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = nc;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, k_rec_few<LOGN, LOGT>, a, ft);
  count_launches(1);
  return e;
}
template <int LOGN>
cudaError_t launch_rec_few(const RecoverArgs& a, const FewTable& ft, cudaStream_t s) {
  if (a.L == 0) return cudaSuccess;
  switch (few_logt(a.e)) {
    case 0: return launch_rec_few_t<LOGN, 0>(a, ft, s);
    case 1: return launch_rec_few_t<LOGN, 1>(a, ft, s);
    case 2: return launch_rec_few_t<LOGN, 2>(a, ft, s);
    case 3: return launch_rec_few_t<LOGN, 3>(a, ft, s);
    default: return cudaErrorNotSupported;
  }
}

template <int LOGN, int LOGT>
cudaError_t launch_rec_few_jobs_t(const FewJob* d, int count, size_t max_ncw, cudaStream_t s) {
  constexpr size_t smem = few_smem<LOGN, LOGT>();
  if constexpr (smem > (48 << 10)) {
    cudaError_t e = ensure_smem_attr(reinterpret_cast<const void*>(k_rec_few_jobs<LOGN, LOGT>), smem);
    if (e != cudaSuccess) return e;
  }
  const unsigned slices = (unsigned)((max_ncw + 31) / 32);
  for (int j0 = 0; j0 < count; j0 += 65535) {
    const unsigned cnt = (unsigned)(count - j0 < 65535 ? count - j0 : 65535);
    k_rec_few_jobs<LOGN, LOGT><<<dim3(slices, cnt), kThreads, smem, s>>>(d + j0);
    count_launches(1);
  }
  return cudaGetLastError();
}
// Every codeword of the group has 2^logt / 2 < e <= 2^logt erasures.
template <int LOGN>
cudaError_t launch_rec_few_jobs(const FewJob* d, int count, size_t max_ncw, int logt, cudaStream_t s) {
  if constexpr (LOGN >= 5) {
    if (count <= 0 || max_ncw == 0) return cudaSuccess;
    switch (logt) {
      case 0: return launch_rec_few_jobs_t<LOGN, 0>(d, count, max_ncw, s);
      case 1: return launch_rec_few_jobs_t<LOGN, 1>(d, count, max_ncw, s);
      case 2: return launch_rec_few_jobs_t<LOGN, 2>(d, count, max_ncw, s);
      case 3: return launch_rec_few_jobs_t<LOGN, 3>(d, count, max_ncw, s);
      default: return cudaErrorNotSupported;
    }
  } else {
    return cudaErrorNotSupported;
  }
}

template <int LOGN>
cudaError_t launch_rec(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s) {
  if constexpr (LOGN >= 5) {
    // Few erasures: one pass, no scratch (by default where it wins; layout 0
    // or kLayoutFused keep the Leopard-form kernels).
    if (((a.layout == kLayoutFew && few_recover_shape(1 << LOGN, a.e)) ||
         (a.layout < 0 && few_recover_wins(1 << LOGN, a.e, a.L))) &&
        (a.L + 1023) / 1024 <= 0x7fffffff) {
      if (const FewTable* ft = cached_few_table(a)) return launch_rec_few<LOGN>(a, *ft, s);
    }
  }
  if constexpr (LOGN <= 4) {
    const size_t slices = (a.L + 1023) / 1024;
    k_rec_small<LOGN><<<(unsigned)((slices + 7) / 8), kThreads, 0, s>>>(a);
    count_launches(1);
    return cudaGetLastError();
  } else {
    constexpr int N = 1 << LOGN, G = N / 16;
    if constexpr (LOGN <= 7) {
      const size_t slices = (a.L + 1023) / 1024;
      if (a.layout == kLayoutFused && slices <= 0x7fffffff) {
        constexpr size_t smem = fused_smem<N>();
        if constexpr (smem > (48 << 10)) {
          cudaError_t e = ensure_smem_attr(reinterpret_cast<const void*>(k_rec_fused<LOGN>), smem);
          if (e != cudaSuccess) return e;
        }
        k_rec_fused<LOGN><<<(unsigned)slices, fused_threads<N>(), smem, s>>>(a, cached_locator(a));
        count_launches(1);
        return cudaGetLastError();
      }
    }
    GroupList gl{};
    bool has[16] = {};
    for (int j = 0; j < a.e; j++) has[a.pos[j] >> 4] = true;
    for (int g = 0; g < G; g++)
      if (has[g]) gl.g[gl.count++] = (uint8_t)g;
    const size_t total_cw = total_colwords(a.L);
    const LocTable& loc = cached_locator(a);
    const size_t bcw = batch_colwords(N, 2, sc.bytes, total_cw);
    if (bcw == 0) return cudaErrorMemoryAllocation;

    for (size_t cw0 = 0; cw0 < total_cw; cw0 += bcw) {
      const size_t ncw = total_cw - cw0 < bcw ? total_cw - cw0 : bcw;
      Batch bt{sc.ptr, sc.ptr + (size_t)N * ncw * 8, ncw, cw0};
      const unsigned gx = (unsigned)((ncw + kPhaseThreads - 1) / kPhaseThreads);
      constexpr int SCW = Split<kRowsPerWarp>::CW;
      constexpr size_t kStage = Split<kRowsPerWarp>::kStage;
      const unsigned gs = (unsigned)((ncw + SCW - 1) / SCW);
      k_rec_b1<LOGN><<<dim3(gs, G), kSplitThreads, kStage, s>>>(a, bt, loc);
      cudaError_t e = launch_dependent(k_rec_p2<LOGN>, dim3(gx, 16), dim3(kPhaseThreads), 0, s, a, bt);
      if (e == cudaSuccess)
        e = launch_dependent(k_rec_b3<LOGN>, dim3(gs, gl.count), dim3(kSplitThreads), kStage, s, a, bt, gl, loc);
      if (e != cudaSuccess) return e;
      count_launches(3);
    }
    return cudaGetLastError();
  }
}

// Grouped launches: `count` codewords of one shape, descriptors in device
// memory; max_ncw = the largest codeword's colwords.
template <int LOGN, int LOGT>
cudaError_t launch_enc_jobs(const EncJob* d, int count, size_t max_ncw, cudaStream_t s) {
  if constexpr (LOGT <= 4) {
    // The layout rule counts the slices of the whole group: many codewords
    // fill the GPU as slices do (t = 16: one warp per slice once the group
    // holds more than 128).
    const size_t slices = (max_ncw + 31) / 32;
    const bool split = enc_small_split<LOGN, LOGT>(slices * (size_t)count);
    const size_t smem = enc_small_smem<LOGN, LOGT>(split);
    auto fn = split ? k_enc_small_jobs<LOGN, LOGT, true> : k_enc_small_jobs<LOGN, LOGT, false>;
    if (smem > (48 << 10)) {
      cudaError_t e = ensure_smem_attr(reinterpret_cast<const void*>(fn), smem);
      if (e != cudaSuccess) return e;
    }
    for (int j0 = 0; j0 < count; j0 += 65535) {
      const unsigned cnt = (unsigned)(count - j0 < 65535 ? count - j0 : 65535);
      fn<<<dim3(enc_small_ctas<LOGN, LOGT>(slices, split), 1, cnt), kThreads, smem, s>>>(d + j0);
      count_launches(1);
    }
    return cudaGetLastError();
  } else {
    constexpr int N = 1 << LOGN, T = 1 << LOGT, C = N / T - 1, G = T / 16;
    constexpr int SCW = Split<kRowsPerWarp>::CW;
    constexpr size_t kStage = Split<kRowsPerWarp>::kStage;
    const unsigned gs = (unsigned)((max_ncw + SCW - 1) / SCW);
    const unsigned gx = (unsigned)((max_ncw + kPhaseThreads - 1) / kPhaseThreads);
    for (int j0 = 0; j0 < count; j0 += 65535) {
      const unsigned cnt = (unsigned)(count - j0 < 65535 ? count - j0 : 65535);
      k_enc_b1_jobs<LOGN, LOGT><<<dim3(gs, cnt, C * G), kSplitThreads, kStage, s>>>(d + j0);
      cudaError_t e = launch_dependent(k_enc_p2_jobs<LOGN, LOGT>, dim3(gx, 16, cnt), dim3(kPhaseThreads), 0, s,
                                       d + j0);
      if (e == cudaSuccess)
        e = launch_dependent(k_enc_b3_jobs<LOGN, LOGT>, dim3(gs, cnt, G), dim3(kSplitThreads), kStage, s, d + j0);
      if (e != cudaSuccess) return e;
      count_launches(3);
    }
    return cudaGetLastError();
  }
}

template <int LOGN>
cudaError_t launch_rec_jobs(RecJob* d, int count, size_t max_ncw, cudaStream_t s) {
  if constexpr (LOGN <= 4) {
    const size_t slices = (max_ncw + 31) / 32;
    for (int j0 = 0; j0 < count; j0 += 65535) {
      const unsigned cnt = (unsigned)(count - j0 < 65535 ? count - j0 : 65535);
      k_rec_small_jobs<LOGN><<<dim3((unsigned)((slices + 7) / 8), 1, cnt), kThreads, 0, s>>>(d + j0);
      count_launches(1);
    }
    return cudaGetLastError();
  } else {
    constexpr int G = (1 << LOGN) / 16;
    constexpr int SCW = Split<kRowsPerWarp>::CW;
    constexpr size_t kStage = Split<kRowsPerWarp>::kStage;
    const unsigned gs = (unsigned)((max_ncw + SCW - 1) / SCW);
    const unsigned gx = (unsigned)((max_ncw + kPhaseThreads - 1) / kPhaseThreads);
    for (int j0 = 0; j0 < count; j0 += 65535) {
      const unsigned cnt = (unsigned)(count - j0 < 65535 ? count - j0 : 65535);
      k_rec_jobs_locator<<<cnt, 32, 0, s>>>(d + j0);
      k_rec_b1_jobs<LOGN><<<dim3(gs, cnt, G), kSplitThreads, kStage, s>>>(d + j0);
      cudaError_t e = launch_dependent(k_rec_p2_jobs<LOGN>, dim3(gx, 16, cnt), dim3(kPhaseThreads), 0, s, d + j0);
      if (e == cudaSuccess)
        e = launch_dependent(k_rec_b3_jobs<LOGN>, dim3(gs, cnt, G), dim3(kSplitThreads), kStage, s, d + j0);
      if (e != cudaSuccess) return e;
      count_launches(4);
    }
    return cudaGetLastError();
  }
}

// Loads the module code of the recover kernels of one n (CUDA loads kernel
// code lazily, at a kernel's first launch, and that load may allocate):
// querying a kernel's attributes loads it.
template <int LOGN>
cudaError_t preload_rec() {
  cudaFuncAttributes fa;
  if constexpr (LOGN <= 4) {
    return cudaFuncGetAttributes(&fa, k_rec_small<LOGN>);
  } else {
    cudaError_t e = cudaFuncGetAttributes(&fa, k_rec_b1<LOGN>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_rec_p2<LOGN>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_rec_b3<LOGN>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_rec_few<LOGN, 0>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_rec_few<LOGN, 1>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_rec_few<LOGN, 2>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_rec_few<LOGN, 3>);
    return e;
  }
}

// Scratch bytes a call needs for one batch covering the whole shard
// (callers may provide less: the launchers then batch the columns).
inline size_t scratch_full_bytes_enc(int n, int t, size_t L) {
  return t >= 32 ? (size_t)(n - t) * total_colwords(L) * 32 : 0;
}
inline size_t scratch_full_bytes_rec(int n, size_t L) { return n >= 32 ? (size_t)2 * n * total_colwords(L) * 32 : 0; }

// Per-shape entry points, one translation unit each (special_enc_*.cu,
// special_rec_*.cu) so that the build parallelises.
#define AFRS_DECLARE_ENC(LN, LT)                                                                   \
  cudaError_t launch_enc_##LN##_##LT(const EncodeArgs& a, const ScratchArena& sc, cudaStream_t s); \
  cudaError_t launch_enc_jobs_##LN##_##LT(const EncJob* d, int count, size_t max_ncw, cudaStream_t s);
#define AFRS_DECLARE_REC(LN)                                                                          \
  cudaError_t launch_rec_##LN(const RecoverArgs& a, const ScratchArena& sc, cudaStream_t s);        \
  cudaError_t launch_rec_jobs_##LN(RecJob* d, int count, size_t max_ncw, cudaStream_t s);            \
  cudaError_t launch_rec_few_jobs_##LN(const FewJob* d, int count, size_t max_ncw, int logt, cudaStream_t s); \
  cudaError_t preload_rec_##LN();
AFRS_DECLARE_ENC(1, 0)
AFRS_DECLARE_ENC(2, 0)
AFRS_DECLARE_ENC(2, 1)
AFRS_DECLARE_ENC(3, 0)
AFRS_DECLARE_ENC(3, 1)
AFRS_DECLARE_ENC(3, 2)
AFRS_DECLARE_ENC(4, 0)
AFRS_DECLARE_ENC(4, 1)
AFRS_DECLARE_ENC(4, 2)
AFRS_DECLARE_ENC(4, 3)
AFRS_DECLARE_ENC(5, 0)
AFRS_DECLARE_ENC(5, 1)
AFRS_DECLARE_ENC(5, 2)
AFRS_DECLARE_ENC(5, 3)
AFRS_DECLARE_ENC(5, 4)
AFRS_DECLARE_ENC(6, 0)
AFRS_DECLARE_ENC(6, 1)
AFRS_DECLARE_ENC(6, 2)
AFRS_DECLARE_ENC(6, 3)
AFRS_DECLARE_ENC(6, 4)
AFRS_DECLARE_ENC(6, 5)
AFRS_DECLARE_ENC(7, 0)
AFRS_DECLARE_ENC(7, 1)
AFRS_DECLARE_ENC(7, 2)
AFRS_DECLARE_ENC(7, 3)
AFRS_DECLARE_ENC(7, 4)
AFRS_DECLARE_ENC(7, 5)
AFRS_DECLARE_ENC(7, 6)
AFRS_DECLARE_ENC(8, 0)
AFRS_DECLARE_ENC(8, 1)
AFRS_DECLARE_ENC(8, 2)
AFRS_DECLARE_ENC(8, 3)
AFRS_DECLARE_ENC(8, 4)
AFRS_DECLARE_ENC(8, 5)
AFRS_DECLARE_ENC(8, 6)
AFRS_DECLARE_ENC(8, 7)
AFRS_DECLARE_REC(1)
AFRS_DECLARE_REC(2)
AFRS_DECLARE_REC(3)
AFRS_DECLARE_REC(4)
AFRS_DECLARE_REC(5)
AFRS_DECLARE_REC(6)
AFRS_DECLARE_REC(7)
AFRS_DECLARE_REC(8)
#undef AFRS_DECLARE_ENC
#undef AFRS_DECLARE_REC

}  // namespace spec
}  // namespace afrs
