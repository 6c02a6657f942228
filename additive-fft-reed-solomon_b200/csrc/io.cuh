// Global-memory row access and the erasure locator shared by the kernels.
#pragma once
#include <cstdint>

#include "afrs_internal.h"
#include "gf_device.cuh"

namespace afrs {

// 32 bytes of one shard row starting at byte column `col`, zero beyond L.
// 16-byte vector loads when the run is in bounds and aligned, bytes otherwise.
__device__ __forceinline__ void load32(const uint8_t* row, size_t col, size_t L, uint32_t (&x)[8]) {
  const uint8_t* p = row + col;
  if (col + 32 <= L && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
    uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
    uint4 b = __ldg(reinterpret_cast<const uint4*>(p) + 1);
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
    return;
  }
#pragma unroll
  for (int w = 0; w < 8; w++) {
    uint32_t v = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      size_t c = col + 4 * w + q;
      uint32_t byte = c < L ? p[4 * w + q] : 0u;
      v |= byte << (8 * q);
    }
    x[w] = v;
  }
}

__device__ __forceinline__ void store32(uint8_t* row, size_t col, size_t L, const uint32_t (&x)[8]) {
  uint8_t* p = row + col;
  if (col + 32 <= L && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
    reinterpret_cast<uint4*>(p)[0] = make_uint4(x[0], x[1], x[2], x[3]);
    reinterpret_cast<uint4*>(p)[1] = make_uint4(x[4], x[5], x[6], x[7]);
    return;
  }
#pragma unroll
  for (int w = 0; w < 8; w++) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      size_t c = col + 4 * w + q;
      if (c < L) p[4 * w + q] = static_cast<uint8_t>(x[w] >> (8 * q));
    }
  }
}

// Colword w (32 byte-columns) of a shard row, in the layout the specialised
// kernels use: 16 bytes at column 1024*(w/32) + 16*(w%32) and 16 bytes 512
// columns further.  A warp over 32 consecutive colwords then reads or writes
// 512 contiguous bytes per instruction.  x[0..3] hold the first 16 bytes,
// x[4..7] the second; columns at or beyond L read as zero and are not written.
__device__ __forceinline__ size_t cw_col(size_t w) { return (w >> 5) * 1024 + (w & 31) * 16; }

__device__ __forceinline__ void load16(const uint8_t* row, size_t col, size_t L, uint32_t* x) {
  const uint8_t* p = row + col;
  if (col + 16 <= L && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
    uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
    x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
    return;
  }
#pragma unroll
  for (int w = 0; w < 4; w++) {
    uint32_t v = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      size_t c = col + 4 * w + q;
      uint32_t byte = c < L ? p[4 * w + q] : 0u;
      v |= byte << (8 * q);
    }
    x[w] = v;
  }
}

__device__ __forceinline__ void store16(uint8_t* row, size_t col, size_t L, const uint32_t* x) {
  uint8_t* p = row + col;
  if (col + 16 <= L && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
    *reinterpret_cast<uint4*>(p) = make_uint4(x[0], x[1], x[2], x[3]);
    return;
  }
#pragma unroll
  for (int w = 0; w < 4; w++) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      size_t c = col + 4 * w + q;
      if (c < L) p[4 * w + q] = static_cast<uint8_t>(x[w] >> (8 * q));
    }
  }
}

__device__ __forceinline__ void load_cw(const uint8_t* row, size_t L, size_t w, uint32_t (&x)[8]) {
  const size_t c = cw_col(w);
  load16(row, c, L, x);
  load16(row, c + 512, L, x + 4);
}

__device__ __forceinline__ void store_cw(uint8_t* row, size_t L, size_t w, const uint32_t (&x)[8]) {
  const size_t c = cw_col(w);
  store16(row, c, L, x);
  store16(row, c + 512, L, x + 4);
}

// Erasure locator in the log domain, computed by one warp with shuffles.
// S[x] = sum_{p in E} log(omega_x + omega_p) mod 255 is the XOR-convolution
// of the erasure indicator with LOGW[x] = log(omega_x) (omega_x + omega_p =
// omega_{x^p}); it is evaluated with Walsh-Hadamard transforms mod 255
// (2^8 = 1 mod 255, so 1/n = 2^(8 - log n)).  Outputs, for x < n:
//   er[x]  = 1 if x is erased
//   lam[x] = log lambda(omega_x) = S[x] (meaningful for surviving x)
//   ilp[x] = log 1/lambda'(omega_x) = -S[x] mod 255 (used for erased x),
//            where lambda'(omega_p) = prod_{q != p}(omega_p + omega_q)
//            (rs/src/codec.rs:436-465 computes the same values directly).
// Lane l owns indices 8l .. 8l+7.  Levels h < n only, so indices >= n
// never mix into indices < n.
// v mod 255 for 0 <= v < 65536 without a division: 256 = 1 (mod 255), so
// folding the high byte onto the low byte keeps the residue.
__device__ __forceinline__ int mod255(int v) {
  v = (v & 255) + (v >> 8);  // < 511
  v = (v & 255) + (v >> 8);  // < 256
  return v >= 255 ? v - 255 : v;
}

__device__ __forceinline__ void fwht_warp(int (&v)[8], int n, int lane) {
#pragma unroll
  for (int h = 1; h < 8; h <<= 1) {
    if (h >= n) break;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      if (i & h) continue;
      int a = v[i], b = v[i + h];
      v[i] = mod255(a + b);
      v[i + h] = mod255(a - b + 255);
    }
  }
  for (int h = 8; h < n; h <<= 1) {
    const int lm = h >> 3;
    const bool upper = (lane & lm) != 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      int other = __shfl_xor_sync(0xffffffffu, v[i], lm);
      v[i] = upper ? mod255(other - v[i] + 255) : mod255(v[i] + other);
    }
  }
}

template <typename Tab>
__device__ void erasure_locator_warp(const RecoverArgs& a, const Tab& tab, uint8_t* er, uint8_t* lam, uint8_t* ilp) {
  const int lane = threadIdx.x & 31;
  const int n = a.n;
  for (int x = lane; x < 256; x += 32) er[x] = 0;
  __syncwarp();
  for (int j = lane; j < a.e; j += 32) er[a.pos[j]] = 1;
  __syncwarp();
  int ve[8], vl[8];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int x = 8 * lane + i;
    ve[i] = (x < n) ? er[x] : 0;
    vl[i] = (x < n && x > 0) ? tab.log[tab.omega[x]] : 0;
  }
  fwht_warp(ve, n, lane);
  fwht_warp(vl, n, lane);
#pragma unroll
  for (int i = 0; i < 8; i++) ve[i] = mod255(ve[i] * vl[i]);
  fwht_warp(ve, n, lane);
  const int k = __ffs(n) - 1;
  const int ninv = (1 << (8 - k)) % 255;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const int x = 8 * lane + i;
    if (x < n) {
      const int s = mod255(ve[i] * ninv);
      lam[x] = static_cast<uint8_t>(s);
      ilp[x] = static_cast<uint8_t>(mod255(255 - s));
    }
  }
}

}  // namespace afrs
