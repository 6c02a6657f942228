// Generic sharded-RS kernels: any power-of-two (n, t) with t < n <= 256,
// runtime twiddles.  One CTA owns a tile of 32*CW byte-columns of every
// shard it needs, bit-sliced in shared memory; butterfly levels run as
// parallel sweeps over that tile.  These kernels are the coverage path; the
// shapes that matter for throughput have compile-time-twiddle kernels in
// special_kernels.cu.
#include <map>
#include <mutex>
#include <utility>

#include "afrs_internal.h"
#include "generic_tile.cuh"

namespace afrs {

namespace {

using namespace gtile;

__global__ void __launch_bounds__(kThreads) k_encode_generic(EncodeArgs a) {
  extern __shared__ uint32_t sm[];
  tile_encode(a, blockIdx.x, sm);
}

__global__ void __launch_bounds__(kThreads) k_recover_generic(RecoverArgs a) {
  extern __shared__ uint32_t sm[];
  __shared__ uint8_t s_erased[256], s_lam[256], s_ilp[256];
  __shared__ int s_x[256], s_y[256];
  erasure_locator(a.n, a.e, a.pos, s_erased, s_lam, s_ilp, s_x, s_y);
  tile_recover(a.rx, a.L, a.n, a.e, a.pos, blockIdx.x, sm, s_erased, s_lam, s_ilp);
}

// Kernel::fft_sharded / ifft_sharded (rs/src/kernel/mod.rs:7-24) on 2^k rows.
__global__ void __launch_bounds__(kThreads) k_transform_generic(uint8_t* shards, size_t L, int k, uint8_t beta,
                                                                 bool inverse) {
  extern __shared__ uint32_t sm[];
  const int rows = 1 << k;
  const int cw = threadIdx.x % kCW, pw = threadIdx.x / kCW, P = kThreads / kCW;
  const size_t col = (size_t)blockIdx.x * 32 * kCW + 32 * cw;
  for (int r = pw; r < rows; r += P) {
    uint32_t x[8];
    load32(shards + (size_t)r * L, col, L, x);
    transpose8(x);
    sts8(sm, r, cw, x);
  }
  __syncthreads();
  transform_smem(sm, k, beta, inverse, cw, pw, P);
  for (int r = pw; r < rows; r += P) {
    uint32_t x[8];
    lds8(sm, r, cw, x);
    transpose8(x);
    store32(shards + (size_t)r * L, col, L, x);
  }
}

// codec.rs:321-340 (n = 2t): message = FFT_t(IFFT_t(parity, 0), omega_t).
__global__ void __launch_bounds__(kThreads) k_recompute_generic(uint8_t* rx, size_t L, int t) {
  extern __shared__ uint32_t sm[];
  const int k = __ffs(t) - 1;
  const int cw = threadIdx.x % kCW, pw = threadIdx.x / kCW, P = kThreads / kCW;
  const size_t col = (size_t)blockIdx.x * 32 * kCW + 32 * cw;
  for (int r = pw; r < t; r += P) {
    uint32_t x[8];
    load32(rx + (size_t)r * L, col, L, x);
    transpose8(x);
    sts8(sm, r, cw, x);
  }
  __syncthreads();
  transform_smem(sm, k, 0, true, cw, pw, P);
  transform_smem(sm, k, c_field.omega[t], false, cw, pw, P);
  for (int r = pw; r < t; r += P) {
    uint32_t x[8];
    lds8(sm, r, cw, x);
    transpose8(x);
    store32(rx + (size_t)(t + r) * L, col, L, x);
  }
}

// Kernel::scale (gfni_kernel.rs:153-195): dst = c * src, bytewise through
// log/exp tables held in shared memory.
__global__ void k_scale(const uint8_t* src, uint8_t* dst, size_t len, uint8_t c) {
  __shared__ uint8_t s_mul[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    s_mul[i] = (i == 0 || c == 0) ? 0 : c_field.exp[c_field.log[i] + c_field.log[c]];
  __syncthreads();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = s_mul[src[i]];
}

size_t slices(size_t L) { return (L + 32 * kCW - 1) / (32 * kCW); }

cudaError_t set_smem(const void* fn, size_t bytes) { return ensure_smem_attr(fn, bytes); }

// dst ^= src over len bytes.
__global__ void k_xor_into(uint8_t* __restrict__ dst, const uint8_t* __restrict__ src, size_t len) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool vec = ((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 15) == 0;
  size_t done = 0;
  if (vec) {
    const size_t nv = len / 16;
    uint4* d = reinterpret_cast<uint4*>(dst);
    const uint4* q = reinterpret_cast<const uint4*>(src);
    for (size_t v = i; v < nv; v += stride) {
      uint4 a = d[v];
      const uint4 b = q[v];
      a.x ^= b.x;
      a.y ^= b.y;
      a.z ^= b.z;
      a.w ^= b.w;
      d[v] = a;
    }
    done = nv * 16;
  }
  for (size_t b = done + i; b < len; b += stride) dst[b] ^= src[b];
}

// *count += number of nonzero bytes in src[0, len).
__global__ void k_count_nonzero(const uint8_t* __restrict__ src, size_t len, unsigned long long* count) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned c = 0;
  size_t done = 0;
  if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
    const size_t nv = len / 16;
    const uint4* q = reinterpret_cast<const uint4*>(src);
    for (size_t v = i; v < nv; v += stride) {
      const uint4 b = q[v];
      const uint32_t w[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
      for (int k = 0; k < 4; k++)
#pragma unroll
        for (int j = 0; j < 4; j++) c += ((w[k] >> (8 * j)) & 0xFF) != 0;
    }
    done = nv * 16;
  }
  for (size_t b = done + i; b < len; b += stride) c += src[b] != 0;
  c = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

}  // namespace

cudaError_t launch_encode_generic(const EncodeArgs& a, cudaStream_t s) {
  const int rows = a.t * (a.n / a.t - 1 > 1 ? 2 : 1);
  const size_t smem = (size_t)rows * kRowStride * 4;
  cudaError_t err = set_smem((const void*)k_encode_generic, smem);
  if (err != cudaSuccess) return err;
  k_encode_generic<<<(unsigned)slices(a.L), kThreads, smem, s>>>(a);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_recover_generic(const RecoverArgs& a, cudaStream_t s) {
  const size_t smem = (size_t)2 * a.n * kRowStride * 4;
  cudaError_t err = set_smem((const void*)k_recover_generic, smem);
  if (err != cudaSuccess) return err;
  k_recover_generic<<<(unsigned)slices(a.L), kThreads, smem, s>>>(a);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_transform_generic(uint8_t* shards, size_t L, int k, uint8_t beta, bool inverse,
                                     cudaStream_t s) {
  const size_t smem = (size_t)(1 << k) * kRowStride * 4;
  cudaError_t err = set_smem((const void*)k_transform_generic, smem);
  if (err != cudaSuccess) return err;
  k_transform_generic<<<(unsigned)slices(L), kThreads, smem, s>>>(shards, L, k, beta, inverse);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_recompute_generic(uint8_t* rx, size_t L, int t, cudaStream_t s) {
  const size_t smem = (size_t)t * kRowStride * 4;
  cudaError_t err = set_smem((const void*)k_recompute_generic, smem);
  if (err != cudaSuccess) return err;
  k_recompute_generic<<<(unsigned)slices(L), kThreads, smem, s>>>(rx, L, t);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_scale(const uint8_t* src, uint8_t* dst, size_t len, uint8_t c, cudaStream_t s) {
  size_t blocks = (len + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks == 0) return cudaSuccess;
  k_scale<<<(unsigned)blocks, 256, 0, s>>>(src, dst, len, c);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t ensure_smem_attr(const void* fn, size_t bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> set;
  std::lock_guard<std::mutex> lk(mu);
  size_t& have = set[{fn, dev}];
  if (bytes <= have) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) have = bytes;
  return e;
}

}  // namespace afrs

namespace afrs {
namespace {
unsigned stream_grid(size_t work) {
  size_t blocks = (work + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  return (unsigned)(blocks ? blocks : 1);
}
}  // namespace

cudaError_t launch_xor_into(uint8_t* dst, const uint8_t* src, size_t len, cudaStream_t s) {
  if (len == 0) return cudaSuccess;
  k_xor_into<<<stream_grid(len / 16 + 1), 256, 0, s>>>(dst, src, len);
  count_launches(1);
  return cudaGetLastError();
}

cudaError_t launch_count_nonzero(const uint8_t* src, size_t len, unsigned long long* count, cudaStream_t s) {
  if (len == 0) return cudaSuccess;
  k_count_nonzero<<<stream_grid(len / 16 + 1), 256, 0, s>>>(src, len, count);
  count_launches(1);
  return cudaGetLastError();
}
}  // namespace afrs
