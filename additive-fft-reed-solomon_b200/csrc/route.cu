// Per-call kernel routes from the tuned table (route_table.inc).
//
// For each shape and shard-length bucket the table names the kernel family
// that was fastest per call on a B200 when tune.py measured it: the
// one-launch generic kernel (runtime twiddles), the specialised kernels
// (compile-time twiddles: the register kernels for t <= 16 encodes and
// n <= 16 recovers, the three phase kernels otherwise), or, for t <= 16
// encodes with several chunks, the specialised kernel with the warps of a
// CTA splitting a slice's chunks.  Entries of -1 were not measured (the
// built-in rules of afrs_capi.cu decide there).
#include <cstdint>

#include "afrs_internal.h"

namespace afrs {
namespace {
#include "route_table.inc"
}  // namespace

int route_bucket(size_t L) {
  if (L <= 64) return 0;
  int b = 0;
  while (((size_t)64 << b) < L) b++;  // ceil(log2 L) - 6
  return b < kRouteBuckets ? b : -1;
}

int route_encode(int n, int t, size_t L) {
  const int b = route_bucket(L);
  if (b < 0 || n < 2 || n > 256 || t < 1 || t >= n) return -1;
  return kEncRoute[__builtin_ctz((unsigned)n)][__builtin_ctz((unsigned)t)][b];
}

int route_recover(int n, size_t L) {
  const int b = route_bucket(L);
  if (b < 0 || n < 2 || n > 256) return -1;
  return kRecRoute[__builtin_ctz((unsigned)n)][b];
}

}  // namespace afrs
