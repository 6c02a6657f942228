// Compile-time-twiddle kernels (the throughput path): templates shared by
// the special_*.cu translation units, which instantiate them per shape.
//
// Every twiddle of an additive FFT level depends only on the level, the
// coset beta and the row bits above the level (rs/src/kernel/lut_kernel.rs:
// 28-82), so once the thread's rows are fixed at compile time every
// multiply is a fixed XOR network over bit-sliced planes (gf_device.cuh).
// A warp owns 32 colwords (1024 byte-columns); rows are split between warps,
// and a warp-uniform row group selects its compile-time variant.
//
// Two-level schedule for 2^k rows, k >= 5 (radix 16 x 2^(k-4)):
//   bottom pass: levels 0..3 on 16 contiguous rows (group g = row >> 4),
//                one warp per group, variant chosen by g;
//   top pass:    levels 4..k-1 on rows {b + 16 m}, uniform code for every b.
// Transforms with k <= 4 run entirely inside one thread.
#pragma once
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

// Runtime v in [LO, HI] -> f(integral_constant<v>) by binary search; v is
// warp-uniform at every call site, so the branches do not diverge.
template <int LO, int HI, typename F>
__device__ __forceinline__ void dispatch(int v, F&& f) {
  if constexpr (LO == HI) {
    f(std::integral_constant<int, LO>{});
  } else {
    constexpr int MID = (LO + HI) / 2;
    if (v <= MID)
      dispatch<LO, MID>(v, f);
    else
      dispatch<MID + 1, HI>(v, f);
  }
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

__device__ __forceinline__ void gload(const uint8_t* base, size_t row, size_t L, size_t col, uint32_t (&x)[8]) {
  load32(base + row * L, col, L, x);
  transpose8(x);
}
__device__ __forceinline__ void gstore(uint8_t* base, size_t row, size_t L, size_t col, uint32_t (&x)[8]) {
  transpose8(x);
  store32(base + row * L, col, L, x);
}

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
template <int LOGN, int LOGT>
__global__ void __launch_bounds__(kThreads) k_enc_small(EncodeArgs a) {
  constexpr int N = 1 << LOGN, T = 1 << LOGT, C = N / T - 1;
  constexpr bool kSmemAcc = (T == 16);
  extern __shared__ uint32_t sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t slice = (size_t)blockIdx.x * (kThreads / 32) + warp;
  if (slice * 1024 >= a.L) return;
  const size_t col = (slice * 32 + lane) * 32;
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
    for (int r = 0; r < T; r++) gload(a.msg, (size_t)(c - 1) * T + r, a.L, col, x[r]);
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
      gload(a.parity, r, a.L, col, y);
#pragma unroll
      for (int p = 0; p < 8; p++) f[r][p] ^= y[p];
    }
  }
  block_fft<0, LOGT, 0, 0, T>(f);
#pragma unroll
  for (int r = 0; r < T; r++) gstore(a.parity, r, a.L, col, f[r]);
}

// ---- encode, t >= 32: one CTA per 1024-column slice -----------------------
// Chunks are processed in waves of 128/t (128 rows of shared memory):
// bottom IFFT pass per (chunk, group) warp, then top IFFT pass accumulating
// into registers; finally top FFT, bottom FFT and store.
template <int LOGN, int LOGT>
__global__ void __launch_bounds__(kThreads, 1) k_enc_large(EncodeArgs a) {
  constexpr int N = 1 << LOGN, T = 1 << LOGT, C = N / T - 1;
  constexpr int G = T / 16, WC = 128 / T, TL = LOGT - 4, TR = 1 << TL;
  constexpr int WAVES = (C + WC - 1) / WC;
  extern __shared__ uint32_t sm[];  // 128 rows x 8 planes x 32 colwords
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t col = ((size_t)blockIdx.x * 32 + lane) * 32;

  uint32_t acc[WAVES > 1 ? 2 : 1][WAVES > 1 ? TR : 1][8];
  if constexpr (WAVES > 1) {
#pragma unroll
    for (int s = 0; s < 2; s++) zero_rows(acc[s]);
  }
  for (int wv = 0; wv < WAVES; wv++) {
    {  // bottom IFFT: warp -> (chunk in wave, group)
      const int ci = warp / G, g = warp % G;
      const int c = 1 + wv * WC + ci;
      if (c <= C) {
        uint32_t x[16][8];
#pragma unroll
        for (int i = 0; i < 16; i++) gload(a.msg, (size_t)(c - 1) * T + 16 * g + i, a.L, col, x[i]);
        dispatch<0, C * G - 1>((c - 1) * G + g, [&](auto v) {
          constexpr int V = decltype(v)::value;
          constexpr int CC = V / G + 1, GG = V % G;
          block_ifft<0, 4, GG, omega_c(CC * T), 16>(x);
        });
#pragma unroll
        for (int i = 0; i < 16; i++) sstore<32>(sm, ci * T + 16 * g + i, lane, x[i]);
      }
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < 2; s++) {  // top IFFT for b = warp + 8 s
      const int b = warp + 8 * s;
      uint32_t part[TR][8];
      zero_rows(part);
      for (int ci = 0; ci < WC; ci++) {
        const int c = 1 + wv * WC + ci;
        if (c > C) break;
        uint32_t y[TR][8];
#pragma unroll
        for (int m = 0; m < TR; m++) sload<32>(sm, ci * T + b + 16 * m, lane, y[m]);
        dispatch<1, C>(c, [&](auto cc) {
          constexpr int CC = decltype(cc)::value;
          block_ifft<4, TL, 0, omega_c(CC * T), TR>(y);
        });
#pragma unroll
        for (int m = 0; m < TR; m++)
#pragma unroll
          for (int p = 0; p < 8; p++) part[m][p] ^= y[m][p];
      }
      if constexpr (WAVES > 1) {
#pragma unroll
        for (int m = 0; m < TR; m++)
#pragma unroll
          for (int p = 0; p < 8; p++) acc[s][m][p] ^= part[m][p];
      } else {
        // single wave: finish this b now (parity_in, top FFT, back to smem)
        if (a.accumulate) {
#pragma unroll
          for (int m = 0; m < TR; m++) {
            uint32_t q[8];
            gload(a.parity, b + 16 * m, a.L, col, q);
#pragma unroll
            for (int p = 0; p < 8; p++) part[m][p] ^= q[p];
          }
        }
        __syncwarp();
        block_fft<4, TL, 0, 0, TR>(part);
        // rows b + 16m of chunk 0's region were read above by this thread only
#pragma unroll
        for (int m = 0; m < TR; m++) sstore<32>(sm, b + 16 * m, lane, part[m]);
      }
    }
    __syncthreads();
  }
  if constexpr (WAVES > 1) {
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const int b = warp + 8 * s;
      if (a.accumulate) {
#pragma unroll
        for (int m = 0; m < TR; m++) {
          uint32_t q[8];
          gload(a.parity, b + 16 * m, a.L, col, q);
#pragma unroll
          for (int p = 0; p < 8; p++) acc[s][m][p] ^= q[p];
        }
      }
      block_fft<4, TL, 0, 0, TR>(acc[s]);
#pragma unroll
      for (int m = 0; m < TR; m++) sstore<32>(sm, b + 16 * m, lane, acc[s][m]);
    }
    __syncthreads();
  }
  if (warp < G) {  // bottom FFT and store
    const int g = warp;
    uint32_t x[16][8];
#pragma unroll
    for (int i = 0; i < 16; i++) sload<32>(sm, 16 * g + i, lane, x[i]);
    dispatch<0, G - 1>(g, [&](auto v) {
      constexpr int GG = decltype(v)::value;
      block_fft<0, 4, GG, 0, 16>(x);
    });
#pragma unroll
    for (int i = 0; i < 16; i++) gstore(a.parity, 16 * g + i, a.L, col, x[i]);
  }
}

// ---- recover ------------------------------------------------------------
// Leopard-form decoder (the same map as rs/src/codec.rs:479-569 on every
// input whose erased rows are zero): y = lambda .* r over survivors,
// c = IFFT_n(y, 0), x = (I + D) c, z = FFT_n(x, 0), r[p] = z[p] / lambda'(omega_p).
// The identity term only adds FFT_n(c) = y to z, and y is zero on erased
// rows, so the erased outputs equal those of FFT_n(D c).

// n <= 16: one warp per 1024-column slice, the whole codeword column in registers.
template <int LOGN>
__global__ void __launch_bounds__(kThreads) k_rec_small(RecoverArgs a) {
  constexpr int N = 1 << LOGN;
  __shared__ uint8_t s_er[256], s_lam[256], s_ilp[256];
  if (threadIdx.x < 32) erasure_locator_warp(a, c_tab, s_er, s_lam, s_ilp);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t slice = (size_t)blockIdx.x * (kThreads / 32) + warp;
  if (slice * 1024 >= a.L) return;
  const size_t col = (slice * 32 + lane) * 32;
  uint32_t x[N][8];
#pragma unroll
  for (int r = 0; r < N; r++) {
    if (s_er[r]) {
#pragma unroll
      for (int p = 0; p < 8; p++) x[r][p] = 0;
    } else {
      gload(a.rx, r, a.L, col, x[r]);
      scale_rt(x[r], s_lam[r]);
    }
  }
  block_ifft<0, LOGN, 0, 0, N>(x);
  one_plus_derivative<N>(x);
  block_fft<0, LOGN, 0, 0, N>(x);
#pragma unroll
  for (int r = 0; r < N; r++) {
    if (s_er[r]) {
      scale_rt(x[r], s_ilp[r]);
      gstore(a.rx, r, a.L, col, x[r]);
    }
  }
}

// n >= 32: one CTA per slice of CW colwords, all n rows bit-sliced in shared
// memory.  The derivative splits over the row bits: D = D_top + D_bot, with
// D_top acting on bits >= 4 (local to a top task) and D_bot on bits < 4
// (read from the other tasks' rows in shared memory).  Top tasks run in
// rounds of 16 colwords so that no task overwrites rows another task of the
// same round still has to read.
template <int LOGN, int CW>
__global__ void __launch_bounds__(kThreads, 1) k_rec_large(RecoverArgs a) {
  constexpr int N = 1 << LOGN, G = N / 16, TL = LOGN - 4, TR = 1 << TL;
  extern __shared__ uint32_t sm[];  // N rows x 8 planes x CW colwords
  __shared__ uint8_t s_er[256], s_lam[256], s_ilp[256];
  if (threadIdx.x < 32) erasure_locator_warp(a, c_tab, s_er, s_lam, s_ilp);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t col0 = (size_t)blockIdx.x * CW * 32;

  // bottom IFFT: warp-uniform group g, lane = colword
  for (int g = warp; g < G; g += kThreads / 32) {
    if (lane < CW) {
      const size_t col = col0 + (size_t)lane * 32;
      uint32_t x[16][8];
#pragma unroll
      for (int i = 0; i < 16; i++) {
        const int r = 16 * g + i;
        if (s_er[r]) {
#pragma unroll
          for (int p = 0; p < 8; p++) x[i][p] = 0;
        } else {
          gload(a.rx, r, a.L, col, x[i]);
          scale_rt(x[i], s_lam[r]);
        }
      }
      dispatch<0, G - 1>(g, [&](auto v) {
        constexpr int GG = decltype(v)::value;
        block_ifft<0, 4, GG, 0, 16>(x);
      });
#pragma unroll
      for (int i = 0; i < 16; i++) sstore<CW>(sm, 16 * g + i, lane, x[i]);
    }
  }
  __syncthreads();

  // top pass in rounds of 16 colwords: task (b, w) = (tid / 16, 16 * round + tid % 16)
  for (int w0 = 0; w0 < CW; w0 += 16) {
    const int b = threadIdx.x >> 4;
    const int w = w0 + (threadIdx.x & 15);
    const bool active = w < CW;
    uint32_t y[TR][8];
    if (active) {
#pragma unroll
      for (int m = 0; m < TR; m++) sload<CW>(sm, b + 16 * m, w, y[m]);
      block_ifft<4, TL, 0, 0, TR>(y);
#pragma unroll
      for (int m = 0; m < TR; m++) sstore<CW>(sm, b + 16 * m, w, y[m]);  // c, own rows
    }
    __syncthreads();
    if (active) {
      one_plus_derivative<TR>(y);  // (I + D_top) on the top index m
#pragma unroll
      for (int j = 0; j < 4; j++) {  // + D_bot: rows b + 2^j for clear bits j of b
        if ((b >> j) & 1) continue;
#pragma unroll
        for (int m = 0; m < TR; m++) {
          uint32_t q[8];
          sload<CW>(sm, b + (1 << j) + 16 * m, w, q);
#pragma unroll
          for (int p = 0; p < 8; p++) y[m][p] ^= q[p];
        }
      }
    }
    __syncthreads();
    if (active) {
      block_fft<4, TL, 0, 0, TR>(y);
#pragma unroll
      for (int m = 0; m < TR; m++) sstore<CW>(sm, b + 16 * m, w, y[m]);
    }
  }
  __syncthreads();

  // bottom FFT, Forney scale, store the erased rows
  for (int g = warp; g < G; g += kThreads / 32) {
    bool any = false;
#pragma unroll
    for (int i = 0; i < 16; i++) any |= s_er[16 * g + i] != 0;
    if (!any || lane >= CW) continue;
    const size_t col = col0 + (size_t)lane * 32;
    uint32_t x[16][8];
#pragma unroll
    for (int i = 0; i < 16; i++) sload<CW>(sm, 16 * g + i, lane, x[i]);
    dispatch<0, G - 1>(g, [&](auto v) {
      constexpr int GG = decltype(v)::value;
      block_fft<0, 4, GG, 0, 16>(x);
    });
#pragma unroll
    for (int i = 0; i < 16; i++) {
      const int r = 16 * g + i;
      if (s_er[r]) {
        scale_rt(x[i], s_ilp[r]);
        gstore(a.rx, r, a.L, col, x[i]);
      }
    }
  }
}

// ---- launchers ------------------------------------------------------------

template <int LOGN, int LOGT>
cudaError_t launch_enc(const EncodeArgs& a, cudaStream_t s) {
  if constexpr (LOGT <= 4) {
    constexpr size_t smem = (LOGT == 4) ? (size_t)8 * 16 * 8 * 32 * 4 : 0;
    auto fn = k_enc_small<LOGN, LOGT>;
    if (smem) {
      cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
    }
    const size_t slices = (a.L + 1023) / 1024;
    fn<<<(unsigned)((slices + 7) / 8), kThreads, smem, s>>>(a);
  } else {
    constexpr size_t smem = (size_t)128 * 8 * 32 * 4;
    auto fn = k_enc_large<LOGN, LOGT>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    fn<<<(unsigned)((a.L + 1023) / 1024), kThreads, smem, s>>>(a);
  }
  return cudaGetLastError();
}

template <int LOGN>
cudaError_t launch_rec(const RecoverArgs& a, cudaStream_t s) {
  if constexpr (LOGN <= 4) {
    const size_t slices = (a.L + 1023) / 1024;
    k_rec_small<LOGN><<<(unsigned)((slices + 7) / 8), kThreads, 0, s>>>(a);
  } else {
    constexpr int CW = LOGN == 8 ? 24 : 32;
    constexpr size_t smem = (size_t)(1 << LOGN) * 8 * CW * 4;
    auto fn = k_rec_large<LOGN, CW>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    fn<<<(unsigned)((a.L + CW * 32 - 1) / (CW * 32)), kThreads, smem, s>>>(a);
  }
  return cudaGetLastError();
}

// Per-shape entry points, one translation unit each (special_enc_*.cu,
// special_rec_*.cu) so that the build parallelises.
#define AFRS_DECLARE_ENC(LN, LT) cudaError_t launch_enc_##LN##_##LT(const EncodeArgs& a, cudaStream_t s);
#define AFRS_DECLARE_REC(LN) cudaError_t launch_rec_##LN(const RecoverArgs& a, cudaStream_t s);
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
