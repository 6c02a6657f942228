/*
 * CPU oracle for the sharded additive-FFT Reed-Solomon path over GF(2^8).
 * TEST INFRASTRUCTURE ONLY (see afrs_oracle.h).  Reference file:line
 * citations are relative to the vkomenda/additive-fft-reed-solomon tree.
 */
#include "afrs_oracle.h"

#include <stdlib.h>
#include <string.h>

#define POLY 0x11d
#define PRIM 2

static orc_tables g_tab;
static int g_ready = 0;

/* gf2p8/src/field.rs:22-37 (shift-and-add multiply modulo POLY). */
uint8_t orc_mul_slow(uint8_t a8, uint8_t b8) {
  uint16_t a = a8, b = b8, res = 0;
  for (int i = 0; i < 8; i++) {
    if (b & 1) res ^= a;
    a <<= 1;
    if (a & 0x100) a ^= POLY;
    b >>= 1;
  }
  return (uint8_t)res;
}

/* gf2p8/src/field.rs:122-130. */
int orc_trace(uint8_t a) {
  uint8_t t = a, sum = a;
  for (int i = 0; i < 7; i++) {
    t = orc_mul_slow(t, t);
    sum ^= t;
  }
  return (sum & 1) != 0;
}

/* gf2p8/src/field.rs:134-147: first x (by value) with x^2 + x = a. */
int orc_solve_quadratic(uint8_t a, uint8_t* x) {
  if (orc_trace(a)) return 0;
  for (int i = 0; i < 256; i++) {
    uint8_t c = (uint8_t)i;
    if ((uint8_t)(orc_mul_slow(c, c) ^ c) == a) {
      *x = c;
      return 1;
    }
  }
  return 0;
}

/* gf2p8/src/bit_matrix.rs:8-16 applied to the byte rows of a GFNI u64
 * (bit_matrix.rs:80-82 stores row r in byte 7-r, big-endian). */
uint8_t orc_bitmatrix_apply(uint64_t gfni_mat, uint8_t v) {
  uint8_t res = 0;
  for (int i = 0; i < 8; i++) {
    uint8_t row = (uint8_t)(gfni_mat >> (8 * (7 - i)));
    res |= (uint8_t)((__builtin_popcount((unsigned)(v & row)) & 1) << i);
  }
  return res;
}

/* gf2p8/src/field.rs:150-157 (columns mul(a, 1<<i), transposed to rows),
 * bit_matrix.rs:19-31 (transpose) and :80-82 (to_gfni_u64). */
uint64_t orc_mul_matrix(uint8_t a) {
  uint8_t cols[8], rows[8];
  for (int i = 0; i < 8; i++) cols[i] = orc_mul_slow(a, (uint8_t)(1u << i));
  for (int r = 0; r < 8; r++) {
    uint8_t rv = 0;
    for (int c = 0; c < 8; c++) rv |= (uint8_t)(((cols[c] >> r) & 1) << c);
    rows[r] = rv;
  }
  uint64_t m = 0;
  for (int r = 0; r < 8; r++) m = (m << 8) | rows[r];
  return m;
}

static void build_tables(void) {
  orc_tables* t = &g_tab;
  memset(t, 0, sizeof *t);
  /* gf2p8/src/field.rs:68-88 */
  uint8_t x = 1;
  for (int i = 0; i < 255; i++) {
    t->exp[i] = x;
    t->log[x] = (uint8_t)i;
    x = orc_mul_slow(x, PRIM);
  }
  for (int i = 0; i < 255; i++) t->exp[255 + i] = t->exp[i];
  /* gf2p8/src/field.rs:90-102 */
  for (int i = 1; i < 256; i++) t->inv[i] = t->exp[255 - t->log[i]];
  /* gf2p8/src/field.rs:174-198: v0 = 1, v_i^2 + v_i = v_{i-1}, trace-0 root. */
  uint8_t cur = 1;
  int len = 0;
  t->cantor_basis[len++] = cur;
  uint8_t nx;
  while (len < 8 && orc_solve_quadratic(cur, &nx)) {
    cur = orc_trace(nx) ? (uint8_t)(nx ^ 1) : nx;
    t->cantor_basis[len++] = cur;
  }
  /* gf2p8/src/field.rs:218-226 */
  for (int i = 0; i < 256; i++) {
    uint8_t p = 0;
    for (int b = 0; b < 8; b++)
      if ((i >> b) & 1) p ^= t->cantor_basis[b];
    t->subspace[i] = p;
  }
  /* gf2p8/src/field.rs:312-336: s_0(x) = x, s_{j+1}(x) = s_j(x)(s_j(x) + s_j(v_j)). */
  for (int v = 0; v < 256; v++) t->spv[0][v] = (uint8_t)v;
  for (int j = 0; j < 8; j++) {
    uint8_t bj = t->spv[j][t->cantor_basis[j]];
    for (int v = 0; v < 256; v++) {
      uint8_t s = t->spv[j][v];
      t->spv[j + 1][v] = orc_mul_slow(s, (uint8_t)(s ^ bj));
    }
  }
  /* gf2p8/src/field.rs:381-395 */
  uint16_t masks[9];
  masks[0] = 1;
  for (int j = 0; j < 8; j++) masks[j + 1] = (uint16_t)((masks[j] << 1) ^ masks[j]);
  for (int j = 0; j < 9; j++) t->spc[j] = (uint8_t)(masks[j] >> 1);
  /* gf2p8/src/field.rs:159-161 */
  for (int i = 0; i < 256; i++) t->gfni_mul[i] = orc_mul_matrix((uint8_t)i);
  g_ready = 1;
}

const orc_tables* orc_get_tables(void) {
  if (!g_ready) build_tables();
  return &g_tab;
}

/* rs/src/poly_11d_lut.rs:10-17 */
uint8_t orc_mul_lut(uint8_t a, uint8_t b) {
  const orc_tables* t = orc_get_tables();
  if (a == 0 || b == 0) return 0;
  return t->exp[t->log[a] + t->log[b]];
}

/* gf2p8/src/field.rs:339-361 */
void orc_normalization_factors(uint8_t out[256]) {
  const orc_tables* t = orc_get_tables();
  uint8_t img[8];
  for (int i = 0; i < 8; i++) img[i] = t->spv[i][t->cantor_basis[i]];
  for (int i = 0; i < 256; i++) {
    uint8_t p = 1;
    for (int j = 0; j < 8; j++)
      if ((i >> j) & 1) p = orc_mul_slow(p, img[j]);
    out[i] = t->inv[p];
  }
}

/* gf2p8/src/field.rs:364-377 (product of the non-zero span_by_gray_code(i)). */
void orc_deriv_subspace_polys(uint8_t out[9]) {
  const orc_tables* t = orc_get_tables();
  for (int i = 0; i < 9; i++) {
    uint8_t d = 1;
    int size = 1 << i;
    uint8_t span[256];
    span[0] = 0;
    for (int m = 1; m < size; m++) {
      int lsb = __builtin_ctz((unsigned)m);
      span[m] = span[m ^ (1 << lsb)] ^ t->cantor_basis[lsb];
    }
    for (int m = 0; m < size; m++)
      if (span[m]) d = orc_mul_slow(d, span[m]);
    out[i] = d;
  }
}

static void make_mul_lut(uint8_t c, uint8_t lut[256]) {
  for (int i = 0; i < 256; i++) lut[i] = orc_mul_lut(c, (uint8_t)i);
}

/* rs/src/kernel/lut_kernel.rs:12-18 */
static void butterfly_fwd(uint8_t* a, uint8_t* b, size_t len, const uint8_t* lut) {
  for (size_t i = 0; i < len; i++) {
    a[i] ^= lut[b[i]];
    b[i] ^= a[i];
  }
}

/* rs/src/kernel/lut_kernel.rs:21-26 */
static void butterfly_inv(uint8_t* a, uint8_t* b, size_t len, const uint8_t* lut) {
  for (size_t i = 0; i < len; i++) {
    b[i] ^= a[i];
    a[i] ^= lut[b[i]];
  }
}

/* rs/src/kernel/lut_kernel.rs:28-50.  The generated beta = 0 code of
 * rs/build.rs:126-179 evaluates the same twiddles (s_0(beta) = beta), so one
 * recursion covers both the unrolled and the recursive reference paths. */
void orc_fft_sharded(uint8_t* shards, size_t L, int k, uint8_t beta) {
  if (k == 0) return;
  const orc_tables* t = orc_get_tables();
  size_t half = (size_t)1 << (k - 1);
  uint8_t lut[256];
  make_mul_lut(t->spv[k - 1][beta], lut);
  for (size_t i = 0; i < half; i++) butterfly_fwd(shards + i * L, shards + (i + half) * L, L, lut);
  orc_fft_sharded(shards, L, k - 1, beta);
  orc_fft_sharded(shards + half * L, L, k - 1, (uint8_t)(beta ^ t->cantor_basis[k - 1]));
}

/* rs/src/kernel/lut_kernel.rs:52-78 */
void orc_ifft_sharded(uint8_t* shards, size_t L, int k, uint8_t beta) {
  if (k == 0) return;
  const orc_tables* t = orc_get_tables();
  size_t half = (size_t)1 << (k - 1);
  orc_ifft_sharded(shards, L, k - 1, beta);
  orc_ifft_sharded(shards + half * L, L, k - 1, (uint8_t)(beta ^ t->cantor_basis[k - 1]));
  uint8_t lut[256];
  make_mul_lut(t->spv[k - 1][beta], lut);
  for (size_t i = 0; i < half; i++) butterfly_inv(shards + i * L, shards + (i + half) * L, L, lut);
}

/* rs/src/kernel/lut_kernel.rs:80-86 */
void orc_scale(const uint8_t* src, uint8_t* dst, size_t len, uint8_t c) {
  uint8_t lut[256];
  make_mul_lut(c, lut);
  for (size_t i = 0; i < len; i++) dst[i] = lut[src[i]];
}

/* rs/src/poly_arith.rs:129-162 (LNH Algorithm 1). */
void orc_fft_scalar(uint8_t* d, int k, uint8_t beta) {
  if (k == 0) return;
  const orc_tables* t = orc_get_tables();
  int half = 1 << (k - 1);
  uint8_t tw = t->spv[k - 1][beta];
  for (int i = 0; i < half; i++) {
    uint8_t g0 = (uint8_t)(d[i] ^ orc_mul_slow(tw, d[i + half]));
    uint8_t g1 = (uint8_t)(g0 ^ d[i + half]);
    d[i] = g0;
    d[i + half] = g1;
  }
  orc_fft_scalar(d, k - 1, beta);
  orc_fft_scalar(d + half, k - 1, (uint8_t)(beta ^ t->cantor_basis[k - 1]));
}

/* rs/src/poly_arith.rs:165-189 (LNH Algorithm 2). */
void orc_ifft_scalar(uint8_t* e, int k, uint8_t beta) {
  if (k == 0) return;
  const orc_tables* t = orc_get_tables();
  int half = 1 << (k - 1);
  orc_ifft_scalar(e, k - 1, beta);
  orc_ifft_scalar(e + half, k - 1, (uint8_t)(beta ^ t->cantor_basis[k - 1]));
  uint8_t tw = t->spv[k - 1][beta];
  for (int i = 0; i < half; i++) {
    uint8_t h = (uint8_t)(e[i] ^ e[i + half]);
    e[i] = (uint8_t)(e[i] ^ orc_mul_slow(tw, h));
    e[i + half] = h;
  }
}

static int ilog2(int v) { return __builtin_ctz((unsigned)v); }

/* rs/src/codec.rs:222-239 */
void orc_encode_systematic_scalar(int n, int t, const uint8_t* message, uint8_t* parity) {
  const orc_tables* tb = orc_get_tables();
  int tl = ilog2(t);
  uint8_t ws[256];
  memset(parity, 0, (size_t)t);
  for (int i = 0; i < (n - t) / t; i++) {
    memcpy(ws, message + i * t, (size_t)t);
    orc_ifft_scalar(ws, tl, tb->subspace[(i + 1) * t]);
    for (int j = 0; j < t; j++) parity[j] ^= ws[j];
  }
  orc_fft_scalar(parity, tl, 0);
}

/* rs/src/codec.rs:241-265.  Parity is XOR-accumulated, as in the reference. */
void orc_encode_systematic_sharded(int n, int t, const uint8_t* message, uint8_t* parity,
                                   uint8_t* ws, size_t L) {
  const orc_tables* tb = orc_get_tables();
  int tl = ilog2(t);
  size_t tl_bytes = (size_t)t * L;
  for (int i = 0; i < (n - t) / t; i++) {
    memcpy(ws, message + (size_t)i * tl_bytes, tl_bytes);
    orc_ifft_sharded(ws, L, tl, tb->subspace[(i + 1) * t]);
    for (size_t j = 0; j < tl_bytes; j++) parity[j] ^= ws[j];
  }
  orc_fft_sharded(parity, L, tl, 0);
}

/* rs/src/codec.rs:436-465 */
void orc_erasure_locator_and_denominators(int n, const uint8_t* pos, size_t e, uint8_t* lambda,
                                          uint8_t* denoms) {
  const orc_tables* tb = orc_get_tables();
  uint8_t pts[256];
  memset(pts, 0, sizeof pts);
  for (size_t k = 0; k < e; k++) pts[k] = tb->subspace[pos[k]];
  memset(lambda, 0, (size_t)n);
  lambda[0] = 1;
  for (size_t k = 0; k < e; k++) {
    uint8_t p = pts[k];
    for (size_t j = k + 1; j >= 1; j--) lambda[j] = (uint8_t)(lambda[j - 1] ^ orc_mul_lut(p, lambda[j]));
    lambda[0] = orc_mul_lut(p, lambda[0]);
  }
  memset(denoms, 0, (size_t)n);
  for (size_t j = 0; j < e; j++) {
    uint8_t acc = 1;
    for (size_t i = 0; i < e; i++)
      if (i != j) acc = orc_mul_lut(acc, (uint8_t)(pts[j] ^ pts[i]));
    denoms[j] = acc;
  }
}

/* rs/src/codec.rs:479-569 */
int orc_recover_erasure_shards(int n, int t, uint8_t* received, uint8_t* ws, size_t L,
                               const uint8_t* pos, size_t e) {
  const orc_tables* tb = orc_get_tables();
  if (e > (size_t)t) return 0;
  if (e == 0 || t == 0) return 1;
  int tl = ilog2(t), nl = ilog2(n);
  size_t tb_bytes = (size_t)t * L;
  /* lambda has degree e <= t < n; one spare slot keeps lambda[e] in range
   * when e == n - 1 would be reached (it cannot: e <= t <= n/2). */
  uint8_t lambda[257], denoms[256];
  memset(lambda, 0, sizeof lambda);
  orc_erasure_locator_and_denominators(n, pos, e, lambda, denoms);

  memcpy(ws, received, tb_bytes);
  orc_ifft_sharded(ws, L, tl, 0);
  for (int c = 1; c < n / t; c++) {
    uint8_t* tmp = ws + tb_bytes;
    memcpy(tmp, received + (size_t)c * tb_bytes, tb_bytes);
    orc_ifft_sharded(tmp, L, tl, tb->subspace[c * t]);
    for (size_t j = 0; j < tb_bytes; j++) ws[j] ^= tmp[j];
  }
  memset(ws + tb_bytes, 0, (size_t)(n - t) * L);

  uint8_t lev[256];
  for (int i = 0; i < n; i++) {
    uint8_t p = tb->subspace[i];
    uint8_t v = lambda[e];
    for (size_t j = e; j-- > 0;) v = (uint8_t)(orc_mul_lut(v, p) ^ lambda[j]);
    lev[i] = v;
  }
  orc_fft_sharded(ws, L, nl, 0);
  for (int i = 0; i < n; i++) orc_scale(ws + (size_t)i * L, ws + (size_t)i * L, L, lev[i]);
  orc_ifft_sharded(ws, L, nl, 0);
  memmove(ws, ws + tb_bytes, e * L);
  memset(ws + e * L, 0, ((size_t)n - e) * L);
  orc_fft_sharded(ws, L, nl, 0);
  for (size_t j = 0; j < e; j++) {
    size_t p = pos[j];
    orc_scale(ws + p * L, received + p * L, L, tb->inv[denoms[j]]);
  }
  return 1;
}

/* rs/src/codec.rs:321-340 */
void orc_recompute_data_from_parity_sharded(int n, int t, uint8_t* received, uint8_t* ws,
                                            size_t L) {
  const orc_tables* tb = orc_get_tables();
  (void)n;
  int tl = ilog2(t);
  size_t bytes = (size_t)t * L;
  memcpy(ws, received, bytes);
  orc_ifft_sharded(ws, L, tl, 0);
  orc_fft_sharded(ws, L, tl, tb->subspace[t]);
  memcpy(received + bytes, ws, bytes);
}

/* Leopard-form erasure decoder over the same field and basis: y = lambda .* r
 * (erased rows ignored), c = IFFT_n(y), d = formal derivative of c in the
 * LCH basis (d[i - 2^j] ^= c[i] for each set bit j of i; s_j' = 1 for this
 * Cantor basis, field.rs:364-377 / test poly_11d.rs:204-213), z = FFT_n(d),
 * out_p = z_p / lambda'(omega_p). */
int orc_recover_leopard_form(int n, int t, uint8_t* received, size_t L, const uint8_t* pos,
                             size_t e) {
  const orc_tables* tb = orc_get_tables();
  if (e > (size_t)t) return 0;
  if (e == 0 || t == 0) return 1;
  int nl = ilog2(n);
  uint8_t erased[256];
  memset(erased, 0, sizeof erased);
  for (size_t j = 0; j < e; j++) erased[pos[j]] = 1;
  uint8_t lev[256];
  for (int i = 0; i < n; i++) {
    uint8_t v = 1;
    for (size_t j = 0; j < e; j++) v = orc_mul_lut(v, (uint8_t)(tb->subspace[i] ^ tb->subspace[pos[j]]));
    lev[i] = v;
  }
  uint8_t* w = (uint8_t*)calloc((size_t)n * L, 1);
  uint8_t* d = (uint8_t*)calloc((size_t)n * L, 1);
  if (!w || !d) {
    free(w);
    free(d);
    return -1;
  }
  for (int i = 0; i < n; i++)
    if (!erased[i]) orc_scale(received + (size_t)i * L, w + (size_t)i * L, L, lev[i]);
  orc_ifft_sharded(w, L, nl, 0);
  for (int i = 1; i < n; i++)
    for (int j = 0; j < nl; j++)
      if ((i >> j) & 1) {
        uint8_t* dst = d + (size_t)(i - (1 << j)) * L;
        const uint8_t* src = w + (size_t)i * L;
        for (size_t c = 0; c < L; c++) dst[c] ^= src[c];
      }
  orc_fft_sharded(d, L, nl, 0);
  for (size_t j = 0; j < e; j++) {
    size_t p = pos[j];
    /* lambda'(omega_p) = prod_{q != p} (omega_p + omega_q) */
    uint8_t dp = 1;
    for (size_t q = 0; q < e; q++)
      if (q != j) dp = orc_mul_lut(dp, (uint8_t)(tb->subspace[p] ^ tb->subspace[pos[q]]));
    orc_scale(d + p * L, received + p * L, L, tb->inv[dp]);
  }
  free(w);
  free(d);
  return 1;
}

uint64_t orc_splitmix64(uint64_t* s) {
  uint64_t z = (*s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

void orc_fill_random(uint8_t* buf, size_t len, uint64_t seed) {
  uint64_t s = seed;
  size_t i = 0;
  while (i + 8 <= len) {
    uint64_t v = orc_splitmix64(&s);
    memcpy(buf + i, &v, 8);
    i += 8;
  }
  if (i < len) {
    uint64_t v = orc_splitmix64(&s);
    memcpy(buf + i, &v, len - i);
  }
}
