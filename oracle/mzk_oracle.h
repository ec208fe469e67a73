/*
 * mzk_oracle.h — CPU restatement of the midnight-zk prover core.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product in midnight-zk_b200/: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load it.  Nothing in the
 * product links or calls it.
 *
 * Layouts are the reference's in-memory layouts:
 *   Fr  (midnight's `Fq`, scalar field r)  : 4 x u64 little-endian, Montgomery R = 2^256
 *                                            (curves/src/bls12_381/fq.rs:25-29)
 *   Fp  (base field p)                     : 6 x u64 little-endian, Montgomery R = 2^384
 *                                            (curves/src/bls12_381/fp.rs:96-98)
 *   G1 affine  : {x: Fp, y: Fp}, identity = all-zero (blst_p1_affine, g1.rs:34, :761-763)
 *   G1 jacobian: {x, y, z: Fp}, identity = z == 0     (blst_p1, g1.rs:495)
 *
 * The arithmetic of the external `blst` crate (curves/Cargo.toml:16, "0.3.15",
 * unpinned, source not vendored) is restated from published mathematics:
 * Montgomery CIOS multiplication, Jacobian formulas from the Explicit-Formulas
 * Database, Fermat inversion.  The algorithms of the reference itself
 * (msm_best, the FFTs, EvaluationDomain) follow the reference files cited at
 * each function in mzk_oracle.c.
 */
#ifndef MZK_ORACLE_H
#define MZK_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Fr ---------------------------------------------------------------- */
void or_fr_mul(uint64_t out[4], const uint64_t a[4], const uint64_t b[4]);
void or_fr_add(uint64_t out[4], const uint64_t a[4], const uint64_t b[4]);
void or_fr_sub(uint64_t out[4], const uint64_t a[4], const uint64_t b[4]);
void or_fr_neg(uint64_t out[4], const uint64_t a[4]);
void or_fr_inv(uint64_t out[4], const uint64_t a[4]);
void or_fr_from_canonical(uint64_t out[4], const uint64_t a[4]); /* a < r */
void or_fr_to_canonical(uint64_t out[4], const uint64_t a[4]);
void or_fr_const(int which, uint64_t out[4]); /* 0:R(one) 1:R2 2:ROOT_OF_UNITY 3:ZETA 4:ROOT_OF_UNITY_INV 5:DELTA 6:GENERATOR */

/* ---- Fp ---------------------------------------------------------------- */
void or_fp_mul(uint64_t out[6], const uint64_t a[6], const uint64_t b[6]);
void or_fp_add(uint64_t out[6], const uint64_t a[6], const uint64_t b[6]);
void or_fp_sub(uint64_t out[6], const uint64_t a[6], const uint64_t b[6]);
void or_fp_inv(uint64_t out[6], const uint64_t a[6]);
void or_fp_from_canonical(uint64_t out[6], const uint64_t a[6]);
void or_fp_to_canonical(uint64_t out[6], const uint64_t a[6]);
void or_fp_const(int which, uint64_t out[6]); /* 0:R(one) 1:R2 2:B=4 */

/* ---- G1 ---------------------------------------------------------------- */
void or_g1_generator(uint64_t out_affine[12]);
void or_g1_add(uint64_t out[18], const uint64_t a[18], const uint64_t b[18]);
void or_g1_double(uint64_t out[18], const uint64_t a[18]);
void or_g1_to_affine(uint64_t out[12], const uint64_t jac[18]);
void or_g1_from_affine(uint64_t out[18], const uint64_t aff[12]);
int  or_g1_is_on_curve_affine(const uint64_t aff[12]);
/* scalar in Montgomery form (as stored in Fq) */
void or_g1_mul(uint64_t out_affine[12], const uint64_t aff[12], const uint64_t scalar_mont[4]);
/* 48-byte compressed encoding (ZCash BLS12-381 format) */
void or_g1_compress(uint8_t out[48], const uint64_t aff[12]);
/* from_compressed: 0 ok, 1 bad encoding, 2 not on the curve, 3 not in G1 */
int or_g1_decompress(uint64_t out[12], const uint8_t in[48], int check_subgroup);

/* ---- MSM ---------------------------------------------------------------- */
/* naive sum of double-and-add products, result affine */
void or_msm_naive(uint64_t out_affine[12], const uint64_t *scalars, const uint64_t *bases, size_t n);
/* restatement of curves::msm::msm_best (curves/src/msm.rs:460-532), result affine */
void or_msm_best(uint64_t out_affine[12], const uint64_t *scalars, const uint64_t *bases, size_t n, int threads);
/* restatement of proofs::poly::kzg::msm::msm_specific's zero filter + msm_best (kzg/msm.rs:174-201) */
void or_msm_specific(uint64_t out_affine[12], const uint64_t *scalars, const uint64_t *bases, size_t n, int threads);
int  or_booth_index(size_t window_index, size_t window_size, const uint8_t el[32]);
/* sum_i s_i * r_i over Fr (Montgomery in, Montgomery out) */
void or_fr_inner_product(uint64_t out[4], const uint64_t *s, const uint64_t *r, size_t n, int threads);

/* ---- seeded synthetic inputs ---------------------------------------------- */
uint64_t or_rand64(uint64_t seed, uint64_t ctr);
/* uniform Fr elements in Montgomery form, element i depends only on (seed, i) */
void or_rand_fr(uint64_t *out, uint64_t seed, uint64_t first, size_t n, int threads);
/* affine bases [r_i]G with r_i = or_rand_fr(seed, i) */
void or_gen_bases(uint64_t *out_affine, uint64_t seed, uint64_t first, size_t n, int threads);

/* ---- FFT (curves/src/fft.rs) ------------------------------------------------ */
void or_compute_twiddles(uint64_t *out, const uint64_t omega[4], uint32_t log_n);
void or_best_fft(uint64_t *a, const uint64_t *twiddles, uint32_t log_n, int threads);
void or_fft_dif_pruned(uint64_t *a, const uint64_t *twiddles, uint32_t log_n, size_t n_real, int threads);
void or_dft_naive(uint64_t *out, const uint64_t *a, const uint64_t omega[4], size_t n);
/* eval_polynomial, proofs/src/utils/arithmetic.rs:59-87 */
void or_eval_polynomial(uint64_t out[4], const uint64_t *poly, size_t n, const uint64_t point[4], int threads);

/* ---- EvaluationDomain (proofs/src/poly/domain.rs) ---------------------------- */
typedef struct or_domain or_domain;
or_domain *or_domain_new(uint32_t j, uint32_t k);
void or_domain_free(or_domain *d);
uint32_t or_domain_k(const or_domain *d);
uint32_t or_domain_extended_k(const or_domain *d);
/* 0 omega 1 omega_inv 2 extended_omega 3 g_coset 4 g_coset_inv 5 ifft_divisor
   6 extended_ifft_divisor 7 t_evaluations[0] (more via index) */
void or_domain_get(const or_domain *d, int which, int idx, uint64_t out[4]);
void or_domain_lagrange_to_coeff(const or_domain *d, uint64_t *a, int threads);
void or_domain_coeff_to_lagrange(const or_domain *d, uint64_t *a, int threads);
/* in: n coeffs, out: 2^extended_k values */
void or_domain_coeff_to_extended(const or_domain *d, const uint64_t *in, uint64_t *out, int threads);
void or_domain_extended_to_coeff(const or_domain *d, uint64_t *a, int threads);
/* in: 2^extended_k values (destroyed), out: n values */
void or_domain_extended_to_lagrange(const or_domain *d, uint64_t *a, uint64_t *out, int threads);
void or_domain_divide_by_vanishing_poly(const or_domain *d, uint64_t *a, int threads);

/* ---- quotient numerator (proofs/src/plonk/evaluation.rs:818-1114) ----------
 * Restated for the circuit shape of the single-proof configuration: one
 * standard gate q_l a + q_r b + q_m a b + q_o c + q_c, permutation sets over
 * advice/fixed columns, at most one logup lookup with one input column and one
 * helper, no trashcans.  All columns are extended-domain (coset) evaluations
 * of length 2^extended_k, Fr Montgomery. */
/* grand products and running sums (permutation and logup arguments) */
void or_fr_batch_invert(uint64_t *a, size_t n); /* ff BatchInvert: zeros stay zero */
void or_permutation_z(const uint64_t *const *values, const uint64_t *const *sigmas, uint32_t n_cols,
                      uint32_t chunk_len, uint32_t k, const uint64_t omega[4], const uint64_t beta[4],
                      const uint64_t gamma[4], uint32_t blinding_factors, const uint64_t *blinds,
                      uint64_t *const *z_out);
void or_logup(const uint64_t *const *inputs, const uint32_t *chunk_cols, uint32_t n_chunks, const uint64_t *table,
              const uint64_t *selector, const uint64_t *multiplicities, size_t n, const uint64_t beta[4],
              uint32_t blinding_factors, const uint64_t *blinds, uint64_t *const *helpers_out,
              uint64_t *aggregator_out);
unsigned long long or_fr_mul_counter(int on); /* count Fr multiplications (single thread) */
void or_fr_mul_vec(const uint64_t *a, const uint64_t *b, uint64_t *out, size_t n);
void or_kate_division(const uint64_t *a, size_t n, const uint64_t b[4], uint64_t *q);
void or_g1_suffix_sum(const uint64_t *in, size_t n, uint64_t *out);
void or_srs_setup(const uint64_t s[4], uint32_t k, const uint64_t omega[4], uint64_t *g, uint64_t *lag,
                  uint64_t *delta, uint64_t *ddelta);
void or_poly_inner_product(const uint64_t *const *polys, const size_t *lens, size_t m, const uint64_t *scalars,
                           uint64_t *out, size_t out_len);

typedef struct {
    uint32_t k, extended_k;
    const uint64_t *const *advice; uint32_t n_advice;
    const uint64_t *const *fixed; uint32_t n_fixed;
    uint32_t gate_fixed[5];   /* q_l, q_r, q_m, q_o, q_c */
    uint32_t gate_advice[3];  /* a, b, c */
    uint32_t n_perm_cols;
    const uint32_t *perm_col_kind;   /* 0 advice, 1 fixed, 2 instance */
    const uint32_t *perm_col_index;
    const uint64_t *const *perm_sigma; /* n_perm_cols cosets */
    uint32_t n_perm_sets;
    const uint64_t *const *perm_z;     /* n_perm_sets cosets */
    uint32_t chunk_len;                /* cs.degree() - 2 */
    uint32_t blinding_factors;
    int has_lookup;
    uint32_t lookup_input_advice, lookup_table_fixed;
    int32_t lookup_selector_fixed;     /* -1: constant one */
    const uint64_t *lookup_h, *lookup_z, *lookup_m;
    const uint64_t *l0, *l_last, *l_active;
    uint64_t y[4], beta[4], gamma[4], theta[4];
    uint64_t extended_omega[4], g_coset[4];
    const uint64_t *const *instance; uint32_t n_instance; /* permutation columns of kind 2 */
} or_quotient_desc;
/* out[i] = numerator nu at extended row i; divide != 0 multiplies by the
 * inverted vanishing polynomial (divide_by_vanishing_poly, domain.rs:361). */
void or_quotient_eval(const or_quotient_desc *d, const or_domain *dom, int divide, uint64_t *out, int threads);
/* the same with the custom gates' value of every row given (gates as flattened programs) */
void or_quotient_eval_gates(const or_quotient_desc *d, const or_domain *dom, int divide, const uint64_t *gate_values,
                            uint64_t *out, int threads);

#ifdef __cplusplus
}
#endif
#endif
