// GF(2^8) arithmetic for the sharded additive-FFT Reed-Solomon kernels.
//
// Field: GF(2^8) modulo x^8 + x^4 + x^3 + x^2 + 1 (0x11d), generator 2
// (gf2p8/src/poly_11d.rs:18-21).  Evaluation points omega_i are the XOR of
// the Cantor basis elements selected by the bits of i (gf2p8/src/field.rs:
// 218-226); the twiddle of butterfly level j at coset beta is s_j(beta)
// (rs/src/kernel/lut_kernel.rs:28-82, field.rs:312-336).  All tables are
// computed at compile time from these definitions.
//
// Data on the device is bit-sliced: a "colword" is 32 byte-columns of one
// shard, held as 8 uint32 planes, plane p carrying bit p of each of the 32
// bytes.  Multiplying by a constant is then an 8x8 GF(2) matrix applied with
// XORs, the same map the reference's GFNI affine instruction applies per byte
// (rs/src/kernel/gfni_kernel.rs:15-76).
#pragma once
#include <cstdint>
#include <utility>

namespace afrs {

constexpr uint8_t gf_mul(uint8_t a8, uint8_t b8) {
  uint32_t a = a8, b = b8, r = 0;
  for (int i = 0; i < 8; i++) {
    if (b & 1) r ^= a;
    a <<= 1;
    if (a & 0x100) a ^= 0x11d;
    b >>= 1;
  }
  return static_cast<uint8_t>(r);
}

constexpr bool gf_trace(uint8_t a) {
  uint8_t t = a, s = a;
  for (int i = 0; i < 7; i++) {
    t = gf_mul(t, t);
    s ^= t;
  }
  return (s & 1) != 0;
}

struct FieldTables {
  uint8_t basis[8];
  uint8_t omega[256];
  uint8_t spv[9][256];  // spv[j][x] = s_j(x)
  uint8_t log[256];     // log[0] unused (0)
  uint8_t exp[512];     // exp[i] = 2^(i mod 255)
};

constexpr FieldTables make_field_tables() {
  FieldTables t{};
  // Cantor basis: v0 = 1, v_i^2 + v_i = v_{i-1}, choosing the trace-0 root
  // (gf2p8/src/field.rs:174-198).
  uint8_t cur = 1;
  t.basis[0] = 1;
  for (int len = 1; len < 8; len++) {
    uint8_t x = 0;
    for (int c = 0; c < 256; c++) {
      uint8_t cc = static_cast<uint8_t>(c);
      if (static_cast<uint8_t>(gf_mul(cc, cc) ^ cc) == cur) {
        x = cc;
        break;
      }
    }
    cur = gf_trace(x) ? static_cast<uint8_t>(x ^ 1) : x;
    t.basis[len] = cur;
  }
  for (int i = 0; i < 256; i++) {
    uint8_t p = 0;
    for (int b = 0; b < 8; b++)
      if ((i >> b) & 1) p ^= t.basis[b];
    t.omega[i] = p;
  }
  for (int x = 0; x < 256; x++) t.spv[0][x] = static_cast<uint8_t>(x);
  for (int j = 0; j < 8; j++) {
    uint8_t bj = t.spv[j][t.basis[j]];
    for (int x = 0; x < 256; x++) {
      uint8_t s = t.spv[j][x];
      t.spv[j + 1][x] = gf_mul(s, static_cast<uint8_t>(s ^ bj));
    }
  }
  uint8_t v = 1;
  for (int i = 0; i < 255; i++) {
    t.exp[i] = v;
    t.log[v] = static_cast<uint8_t>(i);
    v = gf_mul(v, 2);
  }
  for (int i = 255; i < 512; i++) t.exp[i] = t.exp[i - 255];
  return t;
}

inline constexpr FieldTables kField = make_field_tables();

constexpr uint8_t omega_c(int i) { return kField.omega[i & 255]; }
// Twiddle of level j for the butterfly block whose first row is `row_base`
// (bits <= j clear) inside a transform at coset beta: s_j(beta + omega_row_base).
constexpr uint8_t twiddle_c(int j, uint8_t beta, int row_base) {
  return kField.spv[j][static_cast<uint8_t>(beta ^ kField.omega[row_base & 255])];
}

// Bit-sliced multiply matrix of c: column j (byte j of the result) = c * 2^j.
constexpr uint64_t mul_columns(uint8_t c) {
  uint64_t m = 0;
  for (int j = 0; j < 8; j++) m |= static_cast<uint64_t>(gf_mul(c, static_cast<uint8_t>(1u << j))) << (8 * j);
  return m;
}

// ---- compile-time loops -------------------------------------------------
template <int... Is, typename F>
__device__ __forceinline__ void static_for_impl(std::integer_sequence<int, Is...>, F&& f) {
  (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void static_for(F&& f) {
  static_for_impl(std::make_integer_sequence<int, N>{}, static_cast<F&&>(f));
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

// ---- bit-sliced primitives ----------------------------------------------
using Planes = uint32_t[8];

// acc ^= C * b, C known at compile time: plane i of the product is the XOR
// of the planes j whose column C*2^j has bit i set.
template <uint8_t C>
__host__ __device__ __forceinline__ void mul_xor_c(uint32_t (&acc)[8], const uint32_t (&b)[8]) {
  constexpr uint64_t M = mul_columns(C);
#pragma unroll
  for (int i = 0; i < 8; i++) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      if ((M >> (8 * j + i)) & 1) acc[i] ^= b[j];
    }
  }
}

// x <- 2 * x (poly 0x11d: x^8 = x^4 + x^3 + x^2 + 1).
__host__ __device__ __forceinline__ void xtime(uint32_t (&x)[8]) {
  uint32_t h = x[7];
  x[7] = x[6];
  x[6] = x[5];
  x[5] = x[4];
  x[4] = x[3] ^ h;
  x[3] = x[2] ^ h;
  x[2] = x[1] ^ h;
  x[1] = x[0];
  x[0] = h;
}

// acc ^= c * b for a runtime constant c (shift-and-add over the planes).
__host__ __device__ __forceinline__ void mul_xor_rt(uint32_t (&acc)[8], const uint32_t (&b)[8], uint32_t c) {
  uint32_t cur[8];
#pragma unroll
  for (int i = 0; i < 8; i++) cur[i] = b[i];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    uint32_t m = 0u - ((c >> j) & 1u);
#pragma unroll
    for (int i = 0; i < 8; i++) acc[i] ^= cur[i] & m;
    if (j < 7) xtime(cur);
  }
}

// 8x8 bit transpose in each byte lane of eight words.  Applied to eight
// words of raw bytes (word w = bytes 4w..4w+3 of a 32-byte run) it yields
// the planes: plane b, bit 8q+w = bit b of byte 4w+q.  It is an involution,
// so the same routine turns planes back into bytes.
__host__ __device__ __forceinline__ void transpose8(uint32_t (&x)[8]) {
#pragma unroll
  for (int w = 0; w < 4; w++) {
    uint32_t t = ((x[w] >> 4) ^ x[w + 4]) & 0x0F0F0F0Fu;
    x[w + 4] ^= t;
    x[w] ^= t << 4;
  }
#pragma unroll
  for (int w = 0; w < 8; w++) {
    if (w & 2) continue;
    uint32_t t = ((x[w] >> 2) ^ x[w + 2]) & 0x33333333u;
    x[w + 2] ^= t;
    x[w] ^= t << 2;
  }
#pragma unroll
  for (int w = 0; w < 8; w += 2) {
    uint32_t t = ((x[w] >> 1) ^ x[w + 1]) & 0x55555555u;
    x[w + 1] ^= t;
    x[w] ^= t << 1;
  }
}

// transpose8 with its shifts issued as integer multiplies, which execute on
// the FMA pipe while the XOR/AND work occupies the ALU pipe (the bit-sliced
// kernels are bound by the ALU pipe).  Left shifts by s are products by 2^s;
// right shifts by s are the high words of products by 2^(32-s).  The factors
// come from ShiftMul registers whose values the compiler cannot see, so it
// keeps them as multiplies.
struct ShiftMul {
  uint32_t l1, l2, l4, r1, r2, r4;
};

__device__ __forceinline__ ShiftMul make_shift_mul() {
  ShiftMul m;
  asm("mov.u32 %0, 2;" : "=r"(m.l1));
  asm("mov.u32 %0, 4;" : "=r"(m.l2));
  asm("mov.u32 %0, 16;" : "=r"(m.l4));
  asm("mov.u32 %0, 0x80000000;" : "=r"(m.r1));
  asm("mov.u32 %0, 0x40000000;" : "=r"(m.r2));
  asm("mov.u32 %0, 0x10000000;" : "=r"(m.r4));
  return m;
}

__device__ __forceinline__ void transpose8f(uint32_t (&x)[8], const ShiftMul& k) {
#pragma unroll
  for (int w = 0; w < 4; w++) {
    uint32_t t = (__umulhi(x[w], k.r4) ^ x[w + 4]) & 0x0F0F0F0Fu;
    x[w + 4] ^= t;
    x[w] ^= t * k.l4;
  }
#pragma unroll
  for (int w = 0; w < 8; w++) {
    if (w & 2) continue;
    uint32_t t = (__umulhi(x[w], k.r2) ^ x[w + 2]) & 0x33333333u;
    x[w + 2] ^= t;
    x[w] ^= t * k.l2;
  }
#pragma unroll
  for (int w = 0; w < 8; w += 2) {
    uint32_t t = (__umulhi(x[w], k.r1) ^ x[w + 1]) & 0x55555555u;
    x[w + 1] ^= t;
    x[w] ^= t * k.l1;
  }
}

}  // namespace afrs
