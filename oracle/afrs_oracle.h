/*
 * CPU oracle for the sharded additive-FFT Reed-Solomon path over GF(2^8).
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker used by tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py.  The product
 * (the CUDA library under additive-fft-reed-solomon_b200/) never links,
 * loads or calls it.
 *
 * It restates, function by function, the reference crate
 * vkomenda/additive-fft-reed-solomon (Rust; no Rust toolchain exists on this
 * machine, so the reference itself cannot be built or run here).  Every
 * function cites the reference file:line it follows.  Parity is pinned by the
 * reference's own known-answer and property tests, restated in
 * tests/test_oracle.py (the reference commits no golden codeword bytes).
 */
#ifndef AFRS_ORACLE_H
#define AFRS_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Tables generated the way rs/build.rs:549-601 generates them. */
typedef struct {
  uint8_t exp[510];          /* EXP_TABLE, doubled (gf2p8/src/field.rs:68-88) */
  uint8_t log[256];          /* LOG_TABLE */
  uint8_t inv[256];          /* INV_TABLE, inv[0] = 0 (field.rs:90-102) */
  uint8_t cantor_basis[8];   /* CANTOR_BASIS (field.rs:174-198) */
  uint8_t subspace[256];     /* CANTOR_SUBSPACE, omega_i (field.rs:218-226) */
  uint8_t spv[9][256];       /* SUBSPACE_POLY_VALUES s_j(x) (field.rs:312-336) */
  uint8_t spc[9];            /* SUBSPACE_POLY_COEFFS (field.rs:381-395) */
  uint64_t gfni_mul[256];    /* GFNI_MUL_TABLE (field.rs:150-161, bit_matrix.rs:80-82) */
} orc_tables;

const orc_tables* orc_get_tables(void);

uint8_t orc_mul_slow(uint8_t a, uint8_t b);      /* field.rs:22-37 */
uint8_t orc_mul_lut(uint8_t a, uint8_t b);       /* poly_11d_lut.rs:10-17 */
int orc_trace(uint8_t a);                        /* field.rs:122-130 */
int orc_solve_quadratic(uint8_t a, uint8_t* x);  /* field.rs:134-147; returns 0 if none */
uint64_t orc_mul_matrix(uint8_t a);              /* into_mul_matrix + to_gfni_u64 */
uint8_t orc_bitmatrix_apply(uint64_t gfni_mat, uint8_t v); /* bit_matrix.rs:8-16 */
void orc_normalization_factors(uint8_t out[256]);          /* field.rs:339-361 */
void orc_deriv_subspace_polys(uint8_t out[9]);             /* field.rs:364-377 */

/* Sharded LUT transforms (rs/src/kernel/lut_kernel.rs:52-120). */
void orc_fft_sharded(uint8_t* shards, size_t shard_len, int k, uint8_t beta);
void orc_ifft_sharded(uint8_t* shards, size_t shard_len, int k, uint8_t beta);
void orc_scale(const uint8_t* src, uint8_t* dst, size_t len, uint8_t c);

/* Scalar transforms (rs/src/poly_arith.rs:129-189). */
void orc_fft_scalar(uint8_t* coeffs, int k, uint8_t beta);
void orc_ifft_scalar(uint8_t* evals, int k, uint8_t beta);

/* Codec (rs/src/codec.rs). n = N, t = T, powers of two, t < n <= 256. */
void orc_encode_systematic_scalar(int n, int t, const uint8_t* message, uint8_t* parity);
void orc_encode_systematic_sharded(int n, int t, const uint8_t* message, uint8_t* parity,
                                   uint8_t* workspace, size_t shard_len);
void orc_erasure_locator_and_denominators(int n, const uint8_t* positions, size_t e,
                                          uint8_t* lambda, uint8_t* denoms);
int orc_recover_erasure_shards(int n, int t, uint8_t* received, uint8_t* workspace,
                               size_t shard_len, const uint8_t* positions, size_t e);
void orc_recompute_data_from_parity_sharded(int n, int t, uint8_t* received, uint8_t* workspace,
                                            size_t shard_len);

/* Independent restatement of the erasure decoder in the Leopard form
 * (lambda-scale, IFFT_n, formal derivative, FFT_n, divide by lambda').  Used
 * only by the tests, to show that this form and the reference form are the
 * same map on every input whose erased rows are zero. */
int orc_recover_leopard_form(int n, int t, uint8_t* received, size_t shard_len,
                             const uint8_t* positions, size_t e);

/* Deterministic generator: SplitMix64 (Steele, Lea, Flood 2014). */
uint64_t orc_splitmix64(uint64_t* state);
void orc_fill_random(uint8_t* buf, size_t len, uint64_t seed);

#ifdef __cplusplus
}
#endif
#endif
