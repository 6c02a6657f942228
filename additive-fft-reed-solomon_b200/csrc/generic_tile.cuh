// Generic (runtime-twiddle) tile routines: one CTA of kThreads threads
// works on a tile of 32*kCW byte-columns of every shard it needs, bit-sliced
// in shared memory, butterfly levels as parallel sweeps over the tile.  Used
// by the generic kernels (any n, t) and by the batched kernel, which runs
// many codewords of different shapes in one launch.
#pragma once
#include "afrs_internal.h"
#include "gf_device.cuh"
#include "io.cuh"  // load32 / store32

namespace afrs {
namespace gtile {

static __constant__ FieldTables c_field = make_field_tables();


constexpr int kThreads = 256;
constexpr int kCW = 8;                    // colwords per CTA (256 byte-columns)
constexpr int kRowStride = 8 * kCW + 1;   // words per bit-sliced row (+1: bank skew)

__device__ __forceinline__ void lds8(const uint32_t* base, int row, int cw, uint32_t (&x)[8]) {
  const uint32_t* r = base + row * kRowStride + cw;
#pragma unroll
  for (int p = 0; p < 8; p++) x[p] = r[p * kCW];
}
__device__ __forceinline__ void sts8(uint32_t* base, int row, int cw, const uint32_t (&x)[8]) {
  uint32_t* r = base + row * kRowStride + cw;
#pragma unroll
  for (int p = 0; p < 8; p++) r[p * kCW] = x[p];
}

// One additive FFT (inverse=false) or IFFT over 2^k bit-sliced rows in
// shared memory at coset beta (rs/src/kernel/lut_kernel.rs:28-82): level j
// pairs rows (i, i + 2^j) inside blocks of 2^(j+1) rows with twiddle
// s_j(beta + omega_blockstart).  Ends with a barrier.
static __device__ void transform_smem(uint32_t* s, int k, uint8_t beta, bool inverse, int cw, int pw, int P) {
  const int npairs = k > 0 ? (1 << (k - 1)) : 0;
  for (int step = 0; step < k; step++) {
    const int j = inverse ? step : k - 1 - step;
    const int half = 1 << j;
    for (int q = pw; q < npairs; q += P) {
      const int blk = q >> j;
      const int ia = (blk << (j + 1)) | (q & (half - 1));
      const uint8_t tw = c_field.spv[j][static_cast<uint8_t>(beta ^ c_field.omega[blk << (j + 1)])];
      uint32_t a[8], b[8];
      lds8(s, ia, cw, a);
      lds8(s, ia + half, cw, b);
      if (inverse) {
#pragma unroll
        for (int p = 0; p < 8; p++) b[p] ^= a[p];
        if (tw) mul_xor_rt(a, b, tw);
      } else {
        if (tw) mul_xor_rt(a, b, tw);
#pragma unroll
        for (int p = 0; p < 8; p++) b[p] ^= a[p];
      }
      sts8(s, ia, cw, a);
      sts8(s, ia + half, cw, b);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ void scale_planes(uint32_t (&x)[8], uint32_t c) {
  uint32_t r[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  mul_xor_rt(r, x, c);
#pragma unroll
  for (int p = 0; p < 8; p++) x[p] = r[p];
}

// codec.rs:241-265: parity = FFT_t(parity_in? ^ sum_i IFFT_t(chunk_i, omega_(i+1)t), 0)
// One 256-column tile (index `tile`) of an encode; sm holds 2t rows.
static __device__ void tile_encode(const EncodeArgs& a, size_t tile, uint32_t* sm) {
  const int t = a.t, n = a.n;
  const int k = __ffs(t) - 1;
  const int chunks = n / t - 1;
  uint32_t* acc = sm;
  uint32_t* buf = sm + t * kRowStride;
  const int cw = threadIdx.x % kCW, pw = threadIdx.x / kCW, P = kThreads / kCW;
  const size_t col = tile * 32 * kCW + 32 * cw;
  for (int c = 0; c < chunks; c++) {
    uint32_t* dst = c == 0 ? acc : buf;
    for (int r = pw; r < t; r += P) {
      uint32_t x[8];
      load32(a.msg + (size_t)(c * t + r) * a.L, col, a.L, x);
      transpose8(x);
      sts8(dst, r, cw, x);
    }
    __syncthreads();
    transform_smem(dst, k, c_field.omega[(c + 1) * t], true, cw, pw, P);
    if (c > 0) {
      for (int r = pw; r < t; r += P) {
        uint32_t x[8], y[8];
        lds8(acc, r, cw, x);
        lds8(buf, r, cw, y);
#pragma unroll
        for (int p = 0; p < 8; p++) x[p] ^= y[p];
        sts8(acc, r, cw, x);
      }
      __syncthreads();
    }
  }
  if (a.accumulate) {
    for (int r = pw; r < t; r += P) {
      uint32_t x[8], y[8];
      load32(a.parity + (size_t)r * a.L, col, a.L, y);
      transpose8(y);
      lds8(acc, r, cw, x);
#pragma unroll
      for (int p = 0; p < 8; p++) x[p] ^= y[p];
      sts8(acc, r, cw, x);
    }
    __syncthreads();
  }
  transform_smem(acc, k, 0, false, cw, pw, P);
  for (int r = pw; r < t; r += P) {
    uint32_t x[8];
    lds8(acc, r, cw, x);
    transpose8(x);
    store32(a.parity + (size_t)r * a.L, col, a.L, x);
  }
}

// Erasure locator in the log domain (per CTA, in shared memory):
// S[i] = sum_{p in E} log(omega_i + omega_p) mod 255 = (1_E (*) LOGW)[i], a
// XOR-convolution computed with Walsh-Hadamard transforms mod 255
// (2^8 = 1 mod 255, so 1/n = 2^(8-k) mod 255).  Gives lambda(omega_i) =
// exp(S[i]) for surviving i and 1/lambda'(omega_p) = exp(-S[p]) for erased
// p (lambda'(omega_p) = prod_{q != p}(omega_p + omega_q), codec.rs:457-462).
static __device__ void fwht255(int* v, int n) {
  for (int h = 1; h < n; h <<= 1) {
    for (int q = threadIdx.x; q < n / 2; q += blockDim.x) {
      int i = ((q / h) * 2 * h) + (q % h);
      int x = v[i], y = v[i + h];
      v[i] = (x + y) % 255;
      v[i + h] = (x - y + 255) % 255;
    }
    __syncthreads();
  }
}

static __device__ void erasure_locator(int n, int e, const uint8_t* pos, uint8_t* s_erased, uint8_t* s_lam,
                                uint8_t* s_ilp, int* s_x, int* s_y) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_erased[i] = 0;
  __syncthreads();
  for (int j = threadIdx.x; j < e; j += blockDim.x) s_erased[pos[j]] = 1;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    s_x[i] = s_erased[i];
    s_y[i] = i ? c_field.log[c_field.omega[i]] : 0;
  }
  __syncthreads();
  fwht255(s_x, n);
  fwht255(s_y, n);
  const int k = __ffs(n) - 1;
  const int ninv = (1 << (8 - k)) % 255;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_x[i] = (s_x[i] * s_y[i]) % 255;
  __syncthreads();
  fwht255(s_x, n);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    int sv = (s_x[i] * ninv) % 255;
    s_lam[i] = s_erased[i] ? 0 : c_field.exp[sv];
    s_ilp[i] = c_field.exp[(255 - sv) % 255];
  }
  __syncthreads();
}

// Erasure decoder in the Leopard form, the same map as codec.rs:479-569 on
// every input whose erased rows are zero: y = lambda .* r (survivors),
// c = IFFT_n(y, 0), d = formal derivative of c (d[m] = sum over clear bits j
// of m of c[m + 2^j]), z = FFT_n(d, 0), r[p] = z[p] / lambda'(omega_p).
// One 256-column tile of a recover of the n shards at rx; sm holds 2n rows.
// s_erased / s_lam / s_ilp come from erasure_locator (lambda values).
static __device__ void tile_recover(uint8_t* rx, size_t L, int n, int e, const uint8_t* pos, size_t tile, uint32_t* sm,
                             const uint8_t* s_erased, const uint8_t* s_lam, const uint8_t* s_ilp) {
  const int k = __ffs(n) - 1;
  uint32_t* A = sm;
  uint32_t* B = sm + n * kRowStride;
  const int cw = threadIdx.x % kCW, pw = threadIdx.x / kCW, P = kThreads / kCW;
  const size_t col = tile * 32 * kCW + 32 * cw;
  for (int r = pw; r < n; r += P) {
    uint32_t x[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (!s_erased[r]) {
      load32(rx + (size_t)r * L, col, L, x);
      transpose8(x);
      scale_planes(x, s_lam[r]);
    }
    sts8(A, r, cw, x);
  }
  __syncthreads();
  transform_smem(A, k, 0, true, cw, pw, P);
  for (int m = pw; m < n; m += P) {
    uint32_t d[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int j = 0; j < k; j++) {
      if ((m >> j) & 1) continue;
      uint32_t y[8];
      lds8(A, m + (1 << j), cw, y);
#pragma unroll
      for (int p = 0; p < 8; p++) d[p] ^= y[p];
    }
    sts8(B, m, cw, d);
  }
  __syncthreads();
  transform_smem(B, k, 0, false, cw, pw, P);
  for (int j = pw; j < e; j += P) {
    const int p = pos[j];
    uint32_t x[8];
    lds8(B, p, cw, x);
    scale_planes(x, s_ilp[p]);
    transpose8(x);
    store32(rx + (size_t)p * L, col, L, x);
  }
}

}  // namespace gtile
}  // namespace afrs
