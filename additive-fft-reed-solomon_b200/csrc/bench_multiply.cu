// Multiply-strategy benchmark (a standalone program, not part of the library).
//
// One bottom pass of the n = 256 transforms (levels 0..3 of the inverse FFT
// at beta = 0 on every 16-row group, rs/src/kernel/lut_kernel.rs:28-82) over
// 256 shards of 64 KiB, out of place, with four ways of multiplying by a
// twiddle:
//   network   bit-sliced rows, twiddles known at compile time: an XOR network
//             per twiddle (the phase kernels of special.cuh);
//   shiftadd  bit-sliced rows, runtime twiddle, shift-and-add over the planes
//             (gf_device.cuh mul_xor_rt, ~85 LOP3);
//   uniform   bit-sliced rows, runtime warp-uniform twiddle, two XOR networks
//             picked by its logarithm (mul_xor_uniform below);
//   logexp    bytes, no bit slicing: t*x = exp[log x + log t] per byte from
//             tables in shared memory (the reference's LUT kernel,
//             rs/src/poly_11d_lut.rs:10-17).
// Every variant's output is compared with the network variant's.
//
//   make -C additive-fft-reed-solomon_b200/csrc bench_multiply
//   additive-fft-reed-solomon_b200/_build/bench_multiply
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gf_device.cuh"
#include "io.cuh"

namespace afrs {
void count_launches(unsigned) {}
}

using namespace afrs;

#define CK(x)                                                                              \
  do {                                                                                     \
    cudaError_t e_ = (x);                                                                  \
    if (e_ != cudaSuccess) {                                                               \
      fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
      exit(1);                                                                             \
    }                                                                                      \
  } while (0)

namespace {

constexpr int kRows = 256, kGroup = 16;
constexpr size_t kL = 65536;
static __constant__ FieldTables c_mt = make_field_tables();

// acc ^= c * b for a constant c = g^lg (g = 2, lg = log c in [0, 254]) that
// is the same in every lane of the warp: lg = 16 h + l and c = g^(16 h) g^l,
// two compile-time XOR networks picked from 16 each (about 36 LOP3 instead
// of mul_xor_rt's ~85, plus eight uniform branches).
__device__ __forceinline__ void mul_xor_uniform(uint32_t (&acc)[8], const uint32_t (&b)[8], int lg) {
  uint32_t y[8];
  dispatch<0, 15>(lg >> 4, [&](auto h) {
    constexpr uint8_t C = kField.exp[16 * decltype(h)::value];
    if constexpr (C == 1) {
#pragma unroll
      for (int p = 0; p < 8; p++) y[p] = b[p];
    } else {
#pragma unroll
      for (int p = 0; p < 8; p++) y[p] = 0;
      mul_xor_c<C>(y, b);
    }
  });
  dispatch<0, 15>(lg & 15, [&](auto l) { mul_xor_c<kField.exp[decltype(l)::value]>(acc, y); });
}

// Twiddle of level j for rows base..: s_j(omega_base) (beta = 0).
__host__ __device__ inline uint8_t twiddle_rt(const FieldTables& f, int j, int row_base) {
  return f.spv[j][f.omega[row_base & 255]];
}

// Levels 0..3 of the IFFT on the 16 rows of group g, compile-time twiddles.
template <int G>
__device__ __forceinline__ void group_ifft_c(uint32_t (&x)[kGroup][8]) {
  static_for<4>([&](auto s) {
    constexpr int lv = decltype(s)::value;
    static_for<8>([&](auto q) {
      constexpr int qq = decltype(q)::value;
      constexpr int i = ((qq >> lv) << (lv + 1)) | (qq & ((1 << lv) - 1));
      constexpr int tw = twiddle_c(lv, 0, (16 * G + i) & ~((2 << lv) - 1));
#pragma unroll
      for (int p = 0; p < 8; p++) x[i + (1 << lv)][p] ^= x[i][p];
      if constexpr (tw != 0) mul_xor_c<static_cast<uint8_t>(tw)>(x[i], x[i + (1 << lv)]);
    });
  });
}

// Runtime twiddles; MODE 0 shift-and-add, 1 two networks.
template <int MODE>
__device__ __forceinline__ void group_ifft_r(uint32_t (&x)[kGroup][8], int g) {
#pragma unroll
  for (int lv = 0; lv < 4; lv++) {
#pragma unroll
    for (int qq = 0; qq < 8; qq++) {
      const int i = ((qq >> lv) << (lv + 1)) | (qq & ((1 << lv) - 1));
      const uint8_t tw = twiddle_rt(c_mt, lv, (16 * g + i) & ~((2 << lv) - 1));
#pragma unroll
      for (int p = 0; p < 8; p++) x[i + (1 << lv)][p] ^= x[i][p];
      if (tw) {
        if (MODE == 0)
          mul_xor_rt(x[i], x[i + (1 << lv)], tw);
        else
          mul_xor_uniform(x[i], x[i + (1 << lv)], c_mt.log[tw]);
      }
    }
  }
}

// Bit-sliced variants: thread = colword w, CTA row group g = blockIdx.y
// (warp-uniform twiddles), 16 rows in registers.
template <int MODE>  // 0 network, 1 shiftadd, 2 uniform
__global__ void __launch_bounds__(128) k_mul_sliced(const uint8_t* __restrict__ in, uint8_t* __restrict__ out) {
  const size_t w = (size_t)blockIdx.x * 128 + threadIdx.x;
  const int g = blockIdx.y;
  uint32_t x[kGroup][8];
#pragma unroll
  for (int r = 0; r < kGroup; r++) {
    load_cw(in + (size_t)(16 * g + r) * kL, kL, w, x[r]);
    transpose8(x[r]);
  }
  if constexpr (MODE == 0)
    dispatch<0, kRows / kGroup - 1>(g, [&](auto gg) { group_ifft_c<decltype(gg)::value>(x); });
  else
    group_ifft_r<MODE - 1>(x, g);
#pragma unroll
  for (int r = 0; r < kGroup; r++) {
    transpose8(x[r]);
    store_cw(out + (size_t)(16 * g + r) * kL, kL, w, x[r]);
  }
}

// Bytes: thread = one 4-byte word of every row of group g.  exp has 1024
// entries, zero from 510 on, and log[0] = 512, so a zero byte maps to zero.
__device__ __forceinline__ uint32_t mul_bytes(uint32_t v, int lt, const uint16_t* lg, const uint8_t* ex) {
  uint32_t r = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) r |= (uint32_t)ex[lg[(v >> (8 * q)) & 255] + lt] << (8 * q);
  return r;
}

__global__ void __launch_bounds__(256) k_mul_logexp(const uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
  __shared__ uint16_t s_log[256];
  __shared__ uint8_t s_exp[1024];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) s_log[i] = i ? c_mt.log[i] : 512;
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) s_exp[i] = i < 510 ? c_mt.exp[i] : 0;
  __syncthreads();
  const size_t words = kL / 4;
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int g = blockIdx.y;
  uint32_t x[kGroup];
#pragma unroll
  for (int r = 0; r < kGroup; r++) x[r] = in[(size_t)(16 * g + r) * words + c];
#pragma unroll
  for (int lv = 0; lv < 4; lv++) {
#pragma unroll
    for (int qq = 0; qq < 8; qq++) {
      const int i = ((qq >> lv) << (lv + 1)) | (qq & ((1 << lv) - 1));
      const uint8_t tw = twiddle_rt(c_mt, lv, (16 * g + i) & ~((2 << lv) - 1));
      x[i + (1 << lv)] ^= x[i];
      if (tw) x[i] ^= mul_bytes(x[i + (1 << lv)], c_mt.log[tw], s_log, s_exp);
    }
  }
#pragma unroll
  for (int r = 0; r < kGroup; r++) out[(size_t)(16 * g + r) * words + c] = x[r];
}

}  // namespace

int main() {
  const size_t bytes = (size_t)kRows * kL;
  std::vector<uint8_t> h(bytes), ref(bytes), got(bytes);
  uint64_t s = 0x9E3779B97F4A7C15ull;
  for (size_t i = 0; i < bytes; i++) {  // SplitMix64
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    h[i] = (uint8_t)(z ^ (z >> 31));
  }
  uint8_t *d_in, *d_out;
  CK(cudaMalloc(&d_in, bytes));
  CK(cudaMalloc(&d_out, bytes));
  CK(cudaMemcpy(d_in, h.data(), bytes, cudaMemcpyHostToDevice));
  const dim3 gs((unsigned)(kL / 1024 * 32 / 128), kRows / kGroup), gb((unsigned)(kL / 4 / 256), kRows / kGroup);
  auto launch = [&](int v) {
    switch (v) {
      case 0: k_mul_sliced<0><<<gs, 128>>>(d_in, d_out); break;
      case 1: k_mul_sliced<1><<<gs, 128>>>(d_in, d_out); break;
      case 2: k_mul_sliced<2><<<gs, 128>>>(d_in, d_out); break;
      default:
        k_mul_logexp<<<gb, 256>>>(reinterpret_cast<const uint32_t*>(d_in), reinterpret_cast<uint32_t*>(d_out));
    }
  };
  const char* names[] = {"network", "shiftadd", "uniform", "logexp"};
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  printf("bottom IFFT pass (levels 0..3, 16 groups of 16 rows), 256 shards x 64 KiB, in %zu B + out %zu B\n", bytes,
         bytes);
  for (int v = 0; v < 4; v++) {
    CK(cudaMemset(d_out, 0, bytes));
    launch(v);
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(v == 0 ? ref.data() : got.data(), d_out, bytes, cudaMemcpyDeviceToHost));
    const bool same = v == 0 || std::memcmp(ref.data(), got.data(), bytes) == 0;
    for (int i = 0; i < 5; i++) launch(v);
    const int reps = 50;
    CK(cudaEventRecord(a));
    for (int i = 0; i < reps; i++) launch(v);
    CK(cudaEventRecord(b));
    CK(cudaEventSynchronize(b));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, a, b));
    const double us = ms * 1e3 / reps;
    printf("%-9s %8.2f us  %7.1f GB/s (in + out)  %s\n", names[v], us, 2.0 * bytes / us / 1e3,
           same ? "output equal to network" : "OUTPUT DIFFERS");
    if (!same) return 1;
  }
  return 0;
}
