/*
 * CPU baseline: a C restatement of the reference's AVX-512 GFNI kernel
 * (rs/src/kernel/gfni_kernel.rs) driven by the reference codec's call
 * sequence (rs/src/codec.rs:241-265 encode, :479-569 recover).
 *
 * TEST / MEASUREMENT INFRASTRUCTURE ONLY: bench.py times it as the
 * "cpu_baseline" (kind "port") and as the --impl reference arm, because the
 * reference itself is Rust and no Rust toolchain exists on these machines.
 * It is also checked bit-exact against the LUT oracle in the CPU tests.
 */
#define _POSIX_C_SOURCE 200809L
#include <immintrin.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "afrs_oracle.h"

/* gfni_kernel.rs:15-44 */
static inline void bfly_fwd(uint8_t* a, uint8_t* b, size_t len, __m512i mat) {
  size_t i = 0;
  for (; i + 64 <= len; i += 64) {
    __m512i va = _mm512_loadu_si512((const void*)(a + i));
    __m512i vb = _mm512_loadu_si512((const void*)(b + i));
    __m512i t = _mm512_gf2p8affine_epi64_epi8(vb, mat, 0);
    va = _mm512_xor_si512(va, t);
    vb = _mm512_xor_si512(vb, va);
    _mm512_storeu_si512((void*)(a + i), va);
    _mm512_storeu_si512((void*)(b + i), vb);
  }
  if (i < len) {
    __mmask64 k = (1ULL << (len - i)) - 1;
    __m512i va = _mm512_maskz_loadu_epi8(k, a + i);
    __m512i vb = _mm512_maskz_loadu_epi8(k, b + i);
    __m512i t = _mm512_gf2p8affine_epi64_epi8(vb, mat, 0);
    va = _mm512_xor_si512(va, t);
    vb = _mm512_xor_si512(vb, va);
    _mm512_mask_storeu_epi8(a + i, k, va);
    _mm512_mask_storeu_epi8(b + i, k, vb);
  }
}

/* gfni_kernel.rs:47-76 */
static inline void bfly_inv(uint8_t* a, uint8_t* b, size_t len, __m512i mat) {
  size_t i = 0;
  for (; i + 64 <= len; i += 64) {
    __m512i va = _mm512_loadu_si512((const void*)(a + i));
    __m512i vb = _mm512_loadu_si512((const void*)(b + i));
    vb = _mm512_xor_si512(vb, va);
    __m512i t = _mm512_gf2p8affine_epi64_epi8(vb, mat, 0);
    va = _mm512_xor_si512(va, t);
    _mm512_storeu_si512((void*)(a + i), va);
    _mm512_storeu_si512((void*)(b + i), vb);
  }
  if (i < len) {
    __mmask64 k = (1ULL << (len - i)) - 1;
    __m512i va = _mm512_maskz_loadu_epi8(k, a + i);
    __m512i vb = _mm512_maskz_loadu_epi8(k, b + i);
    vb = _mm512_xor_si512(vb, va);
    __m512i t = _mm512_gf2p8affine_epi64_epi8(vb, mat, 0);
    va = _mm512_xor_si512(va, t);
    _mm512_mask_storeu_epi8(a + i, k, va);
    _mm512_mask_storeu_epi8(b + i, k, vb);
  }
}

/* Twiddle-zero blocks of the generated beta = 0 code reduce to b ^= a
 * (rs/build.rs:290-300, :343-353). */
static inline void xor_into(const uint8_t* a, uint8_t* b, size_t len) {
  size_t i = 0;
  for (; i + 64 <= len; i += 64) {
    __m512i va = _mm512_loadu_si512((const void*)(a + i));
    __m512i vb = _mm512_loadu_si512((const void*)(b + i));
    _mm512_storeu_si512((void*)(b + i), _mm512_xor_si512(va, vb));
  }
  for (; i < len; i++) b[i] ^= a[i];
}

static __m512i mat_of(uint8_t tw) {
  return _mm512_set1_epi64((long long)orc_get_tables()->gfni_mul[tw]);
}

/* gfni_kernel.rs:79-107 (recursive, beta != 0) and the generated beta = 0
 * variants (build.rs:387-413), which skip the multiply on zero twiddles. */
static void fft_gfni(uint8_t* s, size_t L, int k, uint8_t beta, int unrolled) {
  if (k == 0) return;
  const orc_tables* t = orc_get_tables();
  size_t half = (size_t)1 << (k - 1);
  uint8_t tw = t->spv[k - 1][beta];
  if (unrolled && tw == 0) {
    for (size_t i = 0; i < half; i++) xor_into(s + i * L, s + (i + half) * L, L);
  } else {
    __m512i m = mat_of(tw);
    for (size_t i = 0; i < half; i++) bfly_fwd(s + i * L, s + (i + half) * L, L, m);
  }
  fft_gfni(s, L, k - 1, beta, unrolled);
  fft_gfni(s + half * L, L, k - 1, (uint8_t)(beta ^ t->cantor_basis[k - 1]), unrolled);
}

/* gfni_kernel.rs:110-150 and build.rs:415-438. */
static void ifft_gfni(uint8_t* s, size_t L, int k, uint8_t beta, int unrolled) {
  if (k == 0) return;
  const orc_tables* t = orc_get_tables();
  size_t half = (size_t)1 << (k - 1);
  ifft_gfni(s, L, k - 1, beta, unrolled);
  ifft_gfni(s + half * L, L, k - 1, (uint8_t)(beta ^ t->cantor_basis[k - 1]), unrolled);
  uint8_t tw = t->spv[k - 1][beta];
  if (unrolled && tw == 0) {
    for (size_t i = 0; i < half; i++) xor_into(s + i * L, s + (i + half) * L, L);
  } else {
    __m512i m = mat_of(tw);
    for (size_t i = 0; i < half; i++) bfly_inv(s + i * L, s + (i + half) * L, L, m);
  }
}

/* Kernel trait dispatch (gfni_kernel.rs:200-281): beta = 0 -> unrolled. */
void gfb_fft_sharded(uint8_t* s, size_t L, int k, uint8_t beta) { fft_gfni(s, L, k, beta, beta == 0); }
void gfb_ifft_sharded(uint8_t* s, size_t L, int k, uint8_t beta) { ifft_gfni(s, L, k, beta, beta == 0); }

/* gfni_kernel.rs:153-195 */
void gfb_scale(const uint8_t* src, uint8_t* dst, size_t len, uint8_t c) {
  __m512i m = mat_of(c);
  size_t i = 0;
  for (; i + 64 <= len; i += 64) {
    __m512i v = _mm512_loadu_si512((const void*)(src + i));
    _mm512_storeu_si512((void*)(dst + i), _mm512_gf2p8affine_epi64_epi8(v, m, 0));
  }
  if (i < len) {
    __mmask64 k = (1ULL << (len - i)) - 1;
    __m512i v = _mm512_maskz_loadu_epi8(k, src + i);
    _mm512_mask_storeu_epi8(dst + i, k, _mm512_gf2p8affine_epi64_epi8(v, m, 0));
  }
}

/* rs/src/codec.rs:241-265 with the GFNI kernel. */
void gfb_encode(int n, int t, const uint8_t* msg, uint8_t* parity, uint8_t* ws, size_t L) {
  const orc_tables* tb = orc_get_tables();
  int tl = __builtin_ctz((unsigned)t);
  size_t bytes = (size_t)t * L;
  for (int i = 0; i < (n - t) / t; i++) {
    memcpy(ws, msg + (size_t)i * bytes, bytes);
    gfb_ifft_sharded(ws, L, tl, tb->subspace[(i + 1) * t]);
    xor_into(ws, parity, bytes);
  }
  gfb_fft_sharded(parity, L, tl, 0);
}

/* rs/src/codec.rs:479-569 with the GFNI kernel. */
int gfb_recover(int n, int t, uint8_t* received, uint8_t* ws, size_t L, const uint8_t* pos,
                size_t e) {
  const orc_tables* tb = orc_get_tables();
  if (e > (size_t)t) return 0;
  if (e == 0 || t == 0) return 1;
  int tl = __builtin_ctz((unsigned)t), nl = __builtin_ctz((unsigned)n);
  size_t bytes = (size_t)t * L;
  uint8_t lambda[257], denoms[256];
  memset(lambda, 0, sizeof lambda);
  orc_erasure_locator_and_denominators(n, pos, e, lambda, denoms);
  memcpy(ws, received, bytes);
  gfb_ifft_sharded(ws, L, tl, 0);
  for (int c = 1; c < n / t; c++) {
    uint8_t* tmp = ws + bytes;
    memcpy(tmp, received + (size_t)c * bytes, bytes);
    gfb_ifft_sharded(tmp, L, tl, tb->subspace[c * t]);
    xor_into(tmp, ws, bytes);
  }
  memset(ws + bytes, 0, (size_t)(n - t) * L);
  uint8_t lev[256];
  for (int i = 0; i < n; i++) {
    uint8_t p = tb->subspace[i], v = lambda[e];
    for (size_t j = e; j-- > 0;) v = (uint8_t)(orc_mul_lut(v, p) ^ lambda[j]);
    lev[i] = v;
  }
  gfb_fft_sharded(ws, L, nl, 0);
  for (int i = 0; i < n; i++) gfb_scale(ws + (size_t)i * L, ws + (size_t)i * L, L, lev[i]);
  gfb_ifft_sharded(ws, L, nl, 0);
  memmove(ws, ws + bytes, e * L);
  memset(ws + e * L, 0, ((size_t)n - e) * L);
  gfb_fft_sharded(ws, L, nl, 0);
  for (size_t j = 0; j < e; j++) {
    size_t p = pos[j];
    gfb_scale(ws + p * L, received + p * L, L, tb->inv[denoms[j]]);
  }
  return 1;
}

/* ---- timing harness (bounded samples; used by bench.py) ---- */

typedef struct {
  int op, n, t, iters;
  size_t L;
  uint64_t seed;
  double busy_s;
  double bytes;
  int ok;
} gfb_job;

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* Fisher-Yates prefix, as in the reference recover bench (recover bench:119-126). */
static void pick_erasures(int n, int e, uint64_t* s, uint8_t* out) {
  uint8_t perm[256];
  for (int i = 0; i < n; i++) perm[i] = (uint8_t)i;
  for (int i = 0; i < e; i++) {
    int j = i + (int)(orc_splitmix64(s) % (uint64_t)(n - i));
    uint8_t tmp = perm[i];
    perm[i] = perm[j];
    perm[j] = tmp;
  }
  memcpy(out, perm, (size_t)e);
}

static void* run_job(void* arg) {
  gfb_job* j = (gfb_job*)arg;
  size_t L = j->L;
  int n = j->n, t = j->t;
  uint8_t* cw = (uint8_t*)aligned_alloc(64, ((size_t)n * L + 63) / 64 * 64);
  uint8_t* ws = (uint8_t*)aligned_alloc(64, ((size_t)n * L + 63) / 64 * 64);
  uint8_t* keep = (uint8_t*)malloc((size_t)t * L);
  j->ok = 0;
  if (!cw || !ws || !keep) goto out;
  orc_fill_random(cw + (size_t)t * L, (size_t)(n - t) * L, j->seed);
  memset(cw, 0, (size_t)t * L);
  gfb_encode(n, t, cw + (size_t)t * L, cw, ws, L);
  uint64_t s = j->seed ^ 0xabcdefULL;
  uint8_t pos[256];
  double busy = 0;
  j->ok = 1;
  for (int it = 0; it < j->iters; it++) {
    if (j->op == 0) {
      memset(cw, 0, (size_t)t * L); /* the reference bench hands encode a zeroed parity buffer */
      double t0 = now_s();
      gfb_encode(n, t, cw + (size_t)t * L, cw, ws, L);
      busy += now_s() - t0;
    } else {
      pick_erasures(n, t, &s, pos);
      for (int q = 0; q < t; q++) {
        memcpy(keep + (size_t)q * L, cw + (size_t)pos[q] * L, L);
        memset(cw + (size_t)pos[q] * L, 0, L);
      }
      double t0 = now_s();
      gfb_recover(n, t, cw, ws, L, pos, (size_t)t);
      busy += now_s() - t0;
      for (int q = 0; q < t; q++)
        if (memcmp(keep + (size_t)q * L, cw + (size_t)pos[q] * L, L) != 0) j->ok = 0;
    }
  }
  j->busy_s = busy;
  j->bytes = (double)j->iters * (double)n * (double)L;
out:
  free(cw);
  free(ws);
  free(keep);
  return NULL;
}

/* Runs `iters` operations (op 0 = encode, 1 = recover of t random erasures)
 * of one (n, t, L) codeword per thread on `nthreads` threads.  Returns the
 * aggregate throughput in bytes/s (n*L bytes per operation, summed over
 * threads, each thread's bytes over its own busy time), or a negative value
 * on failure (allocation, or a recover that did not round-trip). */
double gfb_throughput(int op, int n, int t, size_t L, int iters, int nthreads, uint64_t seed) {
  if (nthreads < 1 || nthreads > 256) return -1.0;
  gfb_job jobs[256];
  pthread_t th[256];
  for (int i = 0; i < nthreads; i++) {
    jobs[i] = (gfb_job){op, n, t, iters, L, seed + 7919u * (uint64_t)i, 0, 0, 0};
    if (pthread_create(&th[i], NULL, run_job, &jobs[i]) != 0) return -2.0;
  }
  double rate = 0;
  int ok = 1;
  for (int i = 0; i < nthreads; i++) {
    pthread_join(th[i], NULL);
    if (!jobs[i].ok || jobs[i].busy_s <= 0) ok = 0;
    else rate += jobs[i].bytes / jobs[i].busy_s;
  }
  return ok ? rate : -3.0;
}
