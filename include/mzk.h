/*
 * mzk.h — C ABI of the B200 (sm_100a) prover core for midnight-zk.
 *
 * Plain pointers and sizes only.  Memory layouts are the reference's own
 * in-memory layouts, so a Rust caller passes its slices unchanged:
 *   Fr (midnight `Fq`)   4 x u64 LE, Montgomery R = 2^256   (curves/src/bls12_381/fq.rs:25-29)
 *   Fp                   6 x u64 LE, Montgomery R = 2^384   (curves/src/bls12_381/fp.rs:96-98)
 *   G1Affine             {x, y: Fp}, identity all-zero       (blst_p1_affine, g1.rs:34)
 *   G1Projective         {x, y, z: Fp} Jacobian, identity z=0 (blst_p1, g1.rs:495)
 *
 * Every function returns 0 on success or an MZK_ERR_* code; mzk_last_error()
 * gives the message of the calling thread's last failure.  All entry points
 * are thread-safe; calls on one context are serialised.  The reference panics
 * on length mismatch (curves/src/msm.rs:461, proofs/src/poly/domain.rs:250);
 * the Rust binding turns a non-zero status into that panic.
 */
#ifndef MZK_H
#define MZK_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MZK_OK 0
#define MZK_ERR_ARG 1
#define MZK_ERR_OOM 2
#define MZK_ERR_CUDA 3
#define MZK_ERR_TIMEOUT 4
#define MZK_ERR_STATE 5

typedef struct mzk_ctx mzk_ctx;

/* ---- context ---------------------------------------------------------- */
int mzk_ctx_create(int device, mzk_ctx **out);
int mzk_ctx_destroy(mzk_ctx *ctx);
const char *mzk_last_error(void);
const char *mzk_version(void);
/* kernels this library launched on ctx since creation */
uint64_t mzk_ctx_launch_count(const mzk_ctx *ctx);
/* the stream every call of ctx runs on (cudaStream_t as void*) */
void *mzk_ctx_stream(mzk_ctx *ctx);
int mzk_ctx_synchronize(mzk_ctx *ctx);
/* Per-phase device timing (CUDA events on the launching stream).  Phases of
 * the MSM: 0 histogram, 1 scan, 2 scatter, 3 accumulate, 4 fixup, 5 reduce.
 * Turning profiling on resets the totals. */
int mzk_ctx_set_profiling(mzk_ctx *ctx, int on);
int mzk_ctx_phase_stats(mzk_ctx *ctx, double *ms_out, uint64_t *count_out, int max_phases);
/* create_proof wall time per Fiat-Shamir phase since the last reset, summed
 * over calls: 0 set-up, 1 advice, 2 multiplicities, 3 permutation / logup
 * products, 4 cosets + quotient + limbs, 5 evaluations + linearization,
 * 6 q polynomials + f, 7 q evaluations, 8 final polynomial + pi, and 9 the
 * MSMs inside phases 1-8; reset != 0 zeroes the totals after reading. */
int mzk_ctx_prove_phase_stats(mzk_ctx *ctx, double *ms_out, uint64_t *calls, int max_phases, int reset);
/* Integer multiply-add throughput of this GPU (IMAD/s, carry-chained
 * mad.lo.cc/madc.hi pairs as the field code issues them) and 12-limb
 * Montgomery multiplications per second, measured by microbenchmark kernels.
 * variants (may be NULL): [0] independent mad.lo+mad.hi, [1] carry-chained
 * pairs, [2] independent mad.lo only (IMAD/s), [3] mixed XYZZ additions per
 * second with operands in registers. */
int mzk_probe_imad_peak(mzk_ctx *ctx, double *imad_per_s, double *fp_mul_per_s, double variants[4]);

/* Self-check of the field code: squares n device Fp values (12 x u32
 * Montgomery, lazily reduced in [0, 2p)) with the dedicated squaring and with
 * the general multiplication, and counts the values whose results differ in
 * any limb (expected 0). */
int mzk_probe_fp_sqr_check(mzk_ctx *ctx, const uint64_t *d_values, size_t n, uint64_t *mismatches);

/* Batch-affine bucket additions (the accumulation scheme of the reference's
 * batch_add / Schedule, curves/src/msm.rs:58-144) per second on this GPU:
 * each thread adds a point to each of B affine accumulators held in local
 * memory, the B additions sharing one inversion by Montgomery's trick (6
 * multiplications per addition plus the inversion's share).  out[0..3]: B =
 * 16, 32, 64, 128 with a Fermat inversion; out[4..7]: the same with the
 * binary extended Euclidean inversion.  A microbenchmark (no gathers, no
 * bucket bookkeeping) that bounds the scheme against the mixed XYZZ
 * addition that mzk_probe_imad_peak's variants[3] measures. */
int mzk_probe_batch_affine(mzk_ctx *ctx, double out[8]);

/* Self-check of the binary extended Euclidean inversion used by the batch
 * inversion's per-block step and the batch-affine probe: for n device Fp
 * values, counts those whose inverse differs from the Fermat power or does
 * not give a^-1 a = 1 (expected 0; zeros are skipped). */
int mzk_probe_fp_inv_check(mzk_ctx *ctx, const uint64_t *d_values, size_t n, uint64_t *mismatches);

/* Captured CUDA graphs of this context: captures made and replays run (the
 * proof core's per-proof NTT sequences). */
int mzk_ctx_graph_stats(mzk_ctx *ctx, uint64_t *captures, uint64_t *replays);

/* ---- autotuner -------------------------------------------------------------
 * The reference fixes its choices in code: the window width c = ceil(ln n)
 * (curves/src/msm.rs:464-470) and the blst/msm_best cut-over at 2^19 points
 * (proofs/src/poly/kzg/msm.rs:187-190).  Here the MSM window width and the
 * NTT pass split are chosen per log2 size by timing the candidates on the
 * device; every choice gives the same results, only the speed differs.
 * Without a tuned entry the cost model / even split apply; mzk_msm_set_window
 * overrides everything.  A context created with the environment variable
 * MZK_TUNE_FILE set loads that table (a malformed file fails the creation). */
#define MZK_TUNE_MSM_WINDOW 0 /* value: window width c in [5, 24] */
#define MZK_TUNE_NTT_SPLIT 1  /* value: 1 even, 2 largest passes first, 3 largest passes last */
/* Time the window widths c_model-2 .. c_model+2 for each log2 size in
 * msm_log_n on the first 2^L device scalars and bases (both holding at least
 * 2^max(L) elements), and the three NTT splits for each log2 size in ntt_log_n
 * (a forward transform of random data); keep the fastest.  reps: timed runs
 * per candidate after one warm-up.  msm_ms / ntt_ms (may be NULL): the best
 * time per size. */
int mzk_autotune(mzk_ctx *ctx, const uint64_t *d_scalars, const uint64_t *d_bases, const uint32_t *msm_log_n,
                 size_t n_msm, const uint32_t *ntt_log_n, size_t n_ntt, int reps, double *msm_ms, double *ntt_ms);
int mzk_autotune_get(mzk_ctx *ctx, int kind, uint32_t log_n, int *value); /* 0 = not tuned */
int mzk_autotune_set(mzk_ctx *ctx, int kind, uint32_t log_n, int value);  /* 0 clears the entry */
/* the table as text lines "msm_c <log_n> <c>" / "ntt_split <log_n> <mode>" */
int mzk_autotune_save(mzk_ctx *ctx, const char *path);
int mzk_autotune_load(mzk_ctx *ctx, const char *path);

/* ---- device memory helpers (for callers without a CUDA runtime) ---------- */
int mzk_device_alloc(mzk_ctx *ctx, size_t bytes, void **out);
int mzk_device_free(mzk_ctx *ctx, void *ptr);
int mzk_memcpy_h2d(mzk_ctx *ctx, void *dst, const void *src, size_t bytes);
int mzk_memcpy_d2h(mzk_ctx *ctx, void *dst, const void *src, size_t bytes);

/* ---- G1 multi-scalar multiplication ------------------------------------ */
/*
 * out = sum_i scalars[i] * bases[i] as a G1Projective (18 u64: x, y, z with
 * z = 1 in Montgomery form, or all zero for the identity), bit-identical in
 * affine form to the reference.
 *
 * Replaces curves::msm::msm_best<G1Affine> (curves/src/msm.rs:460) and
 * proofs::poly::kzg::msm::msm_specific<G1Affine> (proofs/src/poly/kzg/msm.rs:174):
 * zero scalars and identity bases contribute nothing, n == 0 gives the identity.
 * scalars: n x 4 u64 (Fq, Montgomery); bases: n x 12 u64 (G1Affine). HOST pointers.
 */
int mzk_msm_g1(mzk_ctx *ctx, const uint64_t *scalars, const uint64_t *bases, size_t n, uint64_t out[18]);
/* Host-side sum of `count` points in the MSM result layout (z = 1 or all
 * zero), normalised the same way: the final add of a point-split MSM, whose
 * ranks each return the partial sum of their slice of the points. */
int mzk_g1_sum_host(const uint64_t *points, size_t count, uint64_t out[18]);
/* Same with DEVICE pointers (inputs resident in HBM, e.g. a device SRS). */
int mzk_msm_g1_device(mzk_ctx *ctx, const uint64_t *d_scalars, const uint64_t *d_bases, size_t n, uint64_t out[18]);
/*
 * Allocation-free MSM for callers that cannot allocate device memory (a host
 * framework that owns all GPU memory and passes an operation only its inputs
 * and outputs, or code running where the CUDA allocator must not be called).
 * No counterpart in the reference.  Same inputs and result as
 * mzk_msm_g1_device, but it needs no context and calls no allocator: its
 * scratch is one fixed device array of about 21 MB inside this library, held
 * by every GPU that loads it until the process exits.  n must not exceed
 * 65536 (larger n returns MZK_ERR_ARG).  The first call on a device looks up
 * that array's device address; with CUDA's
 * lazy module loading that first call is also when the module and its array
 * are loaded onto the device, so make it before the host reserves the rest of
 * the device's memory.  Runs on `stream` (NULL: the default stream), which
 * must belong to the current device (whose copy of the array is used), and
 * returns when the result is on the host.  All calls on one device share its
 * array: they are serialised by a host lock per device, and GPU work of two
 * calls that overlapped would race on it.
 */
int mzk_msm_g1_noalloc(const uint64_t *d_scalars, const uint64_t *d_bases, size_t n, uint64_t out[18], void *stream);
/* Batched MSMs over one shared device SRS: item m is
 * sum_i scalars_m[i] * bases[base_offset_m + i] for i < n_m (commit_many's
 * `bases[..size]` prefix, proofs/src/poly/kzg/mod.rs:98-103, with any offset).
 * All items are sorted together and accumulated in one load-balanced launch.
 * out: count x 18 u64 G1Projective results, in item order. */
typedef struct {
    const uint64_t *d_scalars; /* n x 4 u64 Fq, DEVICE */
    uint64_t base_offset;
    uint64_t n;
} mzk_msm_batch_item;
int mzk_msm_g1_batch_device(mzk_ctx *ctx, const uint64_t *d_bases, size_t bases_len, const mzk_msm_batch_item *items,
                            size_t count, uint64_t *out);

/* Fixed-base window tables for a resident SRS.  Row j of a table of width c
 * holds [2^(c j)] of every base (row 0 the bases, len points per row); an MSM
 * of width c over such bases needs no per-window bucket sets: window w of
 * point i reads row w, every window's digits go to one bucket set, and the
 * window sums need no doublings.  Same results as without the table.
 * mzk_msm_table_rows(c): rows a table of width c needs.
 * mzk_msm_window_table: fills rows 1 .. rows-1 of d_table (DEVICE, rows x len
 * affine points) from row 0, which the caller has written.
 * mzk_msm_g1_batch_table_device: mzk_msm_g1_batch_device over a table (items
 * index row 0); items of at least min_n points use the table at width c,
 * smaller ones run as usual on row 0. */
int mzk_msm_table_rows(int c);
int mzk_msm_window_table(mzk_ctx *ctx, uint64_t *d_table, size_t len, int c, size_t rows);
int mzk_msm_g1_batch_table_device(mzk_ctx *ctx, const uint64_t *d_table, size_t len, int c, size_t rows,
                                  size_t min_n, const mzk_msm_batch_item *items, size_t count, uint64_t *out);
/* Window width override (0 = automatic), for tuning and tests. */
int mzk_msm_set_window(mzk_ctx *ctx, int c);
int mzk_msm_pick_window(size_t n);
/* Window width, window count and bucket entries (non-zero digits) of the last MSM. */
int mzk_msm_last_shape(mzk_ctx *ctx, int *c, int *windows, uint64_t *entries);

/* ---- EvaluationDomain (proofs/src/poly/domain.rs) ----------------------- */
typedef struct mzk_domain mzk_domain;
/* EvaluationDomain::new(j, k) (domain.rs:54-167): n = 2^k, extended domain
 * 2^extended_k >= n * (j - 1), coset generator zeta; twiddle tables on ctx's GPU. */
int mzk_domain_create(mzk_ctx *ctx, uint32_t j, uint32_t k, mzk_domain **out);
/* destroy a domain (and the keys built over it) before the context it was created on */
int mzk_domain_destroy(mzk_domain *d);
int mzk_domain_shape(const mzk_domain *d, uint32_t *k, uint32_t *extended_k);
/* domain constants (Montgomery Fr): 0 omega, 1 omega_inv, 2 extended_omega,
 * 3 extended_omega_inv, 4 g_coset (zeta), 5 g_coset_inv (zeta^2),
 * 6 ifft_divisor, 7 extended_ifft_divisor, 8 t_evaluations[idx] (inverted) */
int mzk_domain_constant(const mzk_domain *d, int which, int idx, uint64_t out[4]);
/* Operations (op codes) and the reference methods they replace:
 *   0 coeff_to_lagrange      in n      -> out n       (domain.rs:268)
 *   1 lagrange_to_coeff      in n      -> out n       (domain.rs:249)
 *   2 coeff_to_extended      in n      -> out 2^ext_k (domain.rs:285)
 *   3 extended_to_coeff      in 2^ext_k-> out 2^ext_k (domain.rs:312)
 *   4 extended_to_lagrange   in 2^ext_k-> out n       (domain.rs:335)
 *   5 divide_by_vanishing_poly in 2^ext_k -> out 2^ext_k (domain.rs:361)
 * Elements are Fr (4 x u64 Montgomery).  mzk_domain_op takes HOST buffers
 * (in and out may be the same buffer when the lengths agree). */
int mzk_domain_op(mzk_ctx *ctx, mzk_domain *d, int op, const uint64_t *in, uint64_t *out);
/* DEVICE buffers; in == out allowed for ops 0, 1, 3, 5; op 4 overwrites in. */
int mzk_domain_op_device(mzk_ctx *ctx, mzk_domain *d, int op, const uint64_t *d_in, uint64_t *d_out);
/* The same operation (0-3) on `count` polynomials of the domain: d_in[i] ->
 * d_out[i] (HOST arrays of DEVICE pointers; d_in[i] == d_out[i] allowed),
 * the transforms' passes launched together, up to 64 polynomials per launch,
 * where a small domain alone fills few of the GPU's blocks (the evaluator's
 * per-polynomial coeff_to_extended and lagrange_to_coeff calls,
 * evaluation.rs:846-960, prover.rs:634-771).  Same results as one call each. */
int mzk_domain_op_batch_device(mzk_ctx *ctx, mzk_domain *d, int op, const uint64_t *const *d_in,
                               uint64_t *const *d_out, size_t count);

/* ---- quotient evaluation (proofs/src/plonk/evaluation.rs:818-1114) ------ */
/* Custom gates of any circuit as the reference flattens them
 * (FlatGraphEvaluator, proofs/src/plonk/evaluation.rs:148-213; evaluated per
 * row as evaluate_chunk, :530-651).  Each row has one values buffer: the
 * constants, the challenge slots (beta, theta, trash_challenge, y) and the
 * previous value (zero: the gates come first), the column reads, then the
 * intermediates; result_idx holds the Horner-in-y combination of every gate
 * polynomial.  Column types as ColumnRead (:163-181): 0 fixed, 1 advice,
 * 2 instance.  Ops in FlatOpKind order (:134-143), operand indices into the
 * values buffer: dst = a+b, a-b, a*b, a^2, 2a, -a, a*b+c.  At most 256 values
 * and 32 rotations; every index is checked before anything runs. */
#define MZK_FLAT_ADD 0
#define MZK_FLAT_SUB 1
#define MZK_FLAT_MUL 2
#define MZK_FLAT_SQUARE 3
#define MZK_FLAT_DOUBLE 4
#define MZK_FLAT_NEGATE 5
#define MZK_FLAT_MULADD 6
typedef struct { uint32_t col_type, col_idx, rot_idx, dst; } mzk_column_read;
typedef struct { uint32_t kind, dst, a, b, c; } mzk_flat_op;
typedef struct {
    const uint64_t *constants; uint32_t n_constants; /* HOST, Montgomery Fr, values [0, n_constants) */
    const int32_t *rotations; uint32_t n_rotations;  /* row offsets of the original domain */
    const mzk_column_read *reads; uint32_t n_reads;
    const mzk_flat_op *ops; uint32_t n_ops;
    uint32_t values_len;
    uint32_t beta_idx, theta_idx, trash_challenge_idx, y_idx, previous_value_idx, result_idx;
} mzk_flat_graph;
/* A logup argument of any shape (Evaluator::lookups_flat, evaluation.rs:
 * 686-767; its constraint terms :1034-1090): one program per helper column
 * (per chunk of input expressions) computing, in its values buffer, the sum of
 * the partial products sum_j prod_{k!=j} (f_k + beta), the product
 * prod_j (f_j + beta), the compressed table + beta and the selector; outputs
 * holds those four value indices per helper (the table and selector are read
 * from the first helper's program, as the reference does). */
typedef struct {
    uint32_t n_helpers;
    const mzk_flat_graph *programs;   /* n_helpers */
    const uint32_t *outputs;          /* n_helpers x 4: sum_partial_products, product, table, selector */
    const uint64_t *const *helpers;   /* n_helpers extended cosets, DEVICE */
    const uint64_t *aggregator;       /* Z, extended coset, DEVICE */
    const uint64_t *multiplicities;   /* m, extended coset, DEVICE */
} mzk_lookup_arg;
/* A trash argument (trash/prover.rs; its constraint term evaluation.rs:
 * 1093-1109): the program compresses the constraint expressions with the
 * trash challenge (result_idx), the term is compressed - (1 - q) trash. */
typedef struct {
    mzk_flat_graph program;
    uint32_t selector_fixed;          /* fixed column q */
    const uint64_t *trash;            /* trash polynomial, extended coset, DEVICE */
} mzk_trash_arg;

/* Columns are extended-domain (coset) evaluations, 2^extended_k Fr each,
 * DEVICE pointers, given through HOST arrays of pointers.  Circuit shape: one
 * standard gate q_l a + q_r b + q_m a b + q_o c + q_c, or any custom gates given
 * as a flattened program (`gates`), permutation sets over advice/fixed columns
 * (chunk_len = cs.degree() - 2 columns each), then either the built-in logup
 * lookup (one input column, one helper: has_lookup) or lookups and trashcans
 * of any shape as programs (`lookups`, `trash`).  Limits: 16 advice, 16 fixed,
 * 4 instance, 16 permutation columns, 8 sets, 8 lookups of 8 helpers each,
 * 8 trashcans.  extended_omega and
 * g_coset are taken from the domain (the fields exist for layout parity with
 * the CPU restatement). */
typedef struct {
    uint32_t k, extended_k;
    const uint64_t *const *advice; uint32_t n_advice;
    const uint64_t *const *fixed; uint32_t n_fixed;
    uint32_t gate_fixed[5];   /* q_l, q_r, q_m, q_o, q_c */
    uint32_t gate_advice[3];  /* a, b, c */
    uint32_t n_perm_cols;
    const uint32_t *perm_col_kind;     /* 0 advice, 1 fixed, 2 instance */
    const uint32_t *perm_col_index;
    const uint64_t *const *perm_sigma; /* permutation_pk_cosets, one per column */
    uint32_t n_perm_sets;
    const uint64_t *const *perm_z;     /* permutation product cosets, one per set */
    uint32_t chunk_len;
    uint32_t blinding_factors;
    int has_lookup;
    uint32_t lookup_input_advice, lookup_table_fixed;
    int32_t lookup_selector_fixed;     /* -1: constant one (no selector) */
    const uint64_t *lookup_h, *lookup_z, *lookup_m; /* helper, aggregator, multiplicities */
    const uint64_t *l0, *l_last, *l_active;
    uint64_t y[4], beta[4], gamma[4], theta[4];
    uint64_t extended_omega[4], g_coset[4];
    /* custom gates as a flattened program (null: the standard gate above);
     * instance columns (extended coset, DEVICE) and the trash challenge are
     * read by programs only */
    const mzk_flat_graph *gates;
    const uint64_t *const *instance; uint32_t n_instance;
    uint64_t trash_challenge[4];
    /* lookups and trashcans of any shape as programs (used when has_lookup
     * is 0): their terms follow the permutation terms in the reference's order */
    uint32_t n_lookups; const mzk_lookup_arg *lookups;
    uint32_t n_trash; const mzk_trash_arg *trash;
} mzk_quotient_desc;
/* d_out (2^extended_k Fr) = nu(X) on the extended coset; with divide != 0,
 * h(X) = nu(X) / (X^n - 1) (evaluate_numerator + divide_by_vanishing_poly,
 * proofs/src/plonk/prover.rs:664, :713). */
int mzk_quotient_eval_device(mzk_ctx *ctx, mzk_domain *d, const mzk_quotient_desc *desc, int divide, uint64_t *d_out);

/* compute_h_poly (proofs/src/plonk/prover.rs:701-771) on the device, without
 * the transcript writes: h = nu / t, extended_to_coeff, truncated to
 * (n-1)*qdeg and split into qdeg limbs of n - 1 coefficients, inter-limb
 * blinding with the caller's `blinds` ((qdeg-1) x 4 u64 Montgomery, host;
 * blind_quotient_limbs draws them from OsRng, prover.rs:774-785), every limb
 * padded to n and committed against the monomial SRS d_srs_g[0..n).
 * out_commitments: qdeg x 18 u64 G1Projective (host); d_limbs_out: optional
 * DEVICE buffer of qdeg x n Fr receiving the limbs.  qdeg = j - 1 of the domain. */
int mzk_compute_h_poly_device(mzk_ctx *ctx, mzk_domain *d, const mzk_quotient_desc *desc, const uint64_t *d_srs_g,
                              size_t srs_len, const uint64_t *blinds, uint64_t *out_commitments, uint64_t *d_limbs_out);

/* ---- device part of create_proof (proofs/src/plonk/prover.rs:432) ------- */
/* Circuit shape of the single-proof configuration: advice a, b, c under the
 * gate q_l a + q_r b + q_m a b + q_o c + q_c, one permutation set over a, b, c,
 * one logup lookup of a into the fixed table column (selector column 6),
 * degree 5 (j = 5: four quotient limbs).  Resident proving-key data: */
typedef struct {
    uint32_t k;
    const uint64_t *fixed_ext[7];  /* q_l, q_r, q_m, q_o, q_c, table, lookup selector (extended coset), DEVICE */
    const uint64_t *sigma_ext[3];  /* permutation_pk_cosets of a, b, c, DEVICE */
    const uint64_t *l0_ext, *l_last_ext, *l_active_ext;
    const uint64_t *srs;           /* DEVICE G1Affine array holding the four bases below */
    uint64_t srs_len;              /* points in srs */
    uint64_t off_g, off_lagrange, off_lagrange_delta, off_lagrange_double_delta; /* ParamsKZG::bases, params.rs:83-93 */
    uint32_t blinding_factors;     /* at most 8 */
    /* Lagrange forms (DEVICE, n each), read only for jobs whose z / h / Z the
     * device derives (null perm_z, lookup_h, lookup_Z): */
    const uint64_t *sigma_lagrange[3];  /* permutation polynomials of a, b, c */
    const uint64_t *table_lagrange;     /* lookup table column */
    const uint64_t *selector_lagrange;  /* lookup selector column */
    /* srs_table_c > 0: srs is row 0 of a window table of that width with
     * srs_table_rows rows of srs_len points (mzk_msm_window_table); MSMs of
     * at least srs_table_min_n points use it */
    int32_t srs_table_c;
    uint32_t srs_table_rows;
    uint64_t srs_table_min_n;
} mzk_proving_key_desc;
/* One proof's witness (Lagrange form, DEVICE, n Fr each) and challenges.
 * perm_z null: the device derives z (permutation/prover.rs:81-255) from a, b,
 * c and the key's sigma_lagrange with perm_blinds; lookup_h and lookup_Z both
 * null: it derives them (logup/prover.rs:195-300; the compressed input of the
 * single input expression is a itself) with lookup_blinds. */
typedef struct {
    const uint64_t *advice[3];     /* a, b, c */
    const uint64_t *perm_z;        /* permutation product, or null */
    const uint64_t *lookup_m, *lookup_h, *lookup_Z; /* logup multiplicities, helper, aggregator (h, Z or null) */
    uint64_t y[4], beta[4], gamma[4], theta[4];
    uint64_t quotient_blinds[3][4];
    uint64_t perm_blinds[8][4];    /* blinding rows of a derived z */
    uint64_t lookup_blinds[8][4];  /* blinding rows of a derived Z */
} mzk_proof_job;
/* For each job: commitments (out: count x 11 x 18 u64 G1Projective, in the
 * order a, b, c, m (delta), z (delta), Z (double delta), h, quotient limbs
 * 0..3), lagrange_to_coeff and coeff_to_extended of the seven witness
 * polynomials, compute_h_poly.  All jobs' MSMs run as two batched MSMs, or,
 * with MZK_PROVE_MSM_PER_CALL in flags, each as its own call (the plain
 * one-call-at-a-time form; same results). */
#define MZK_PROVE_MSM_PER_CALL 1u
/* launch each proof's NTT sequence kernel by kernel instead of replaying a
 * captured CUDA graph (same kernels, same results) */
#define MZK_PROVE_NO_GRAPHS 2u
int mzk_prove_core_device(mzk_ctx *ctx, mzk_domain *d, const mzk_proving_key_desc *pk, const mzk_proof_job *jobs,
                          size_t count, uint32_t flags, uint64_t *out);

/* ---- Fiat-Shamir transcript (proofs/src/transcript) --------------------- */
/* CircuitTranscript<Blake2bState> (transcript/mod.rs:83-150,
 * implementors.rs:13-30, 138-185): keyed BLAKE2b-512; points are absorbed and
 * written compressed (48 bytes), scalars as 32 little-endian canonical bytes;
 * a squeezed challenge is the digest reduced mod r.  Points use the MSM
 * result layout (18 u64: x, y, z with z = 1 in Montgomery form, or all zero
 * for the identity); scalars are Fr (4 u64 Montgomery).  Host only. */
typedef struct mzk_transcript mzk_transcript;
int mzk_transcript_create(mzk_transcript **out);
int mzk_transcript_destroy(mzk_transcript *t);
int mzk_transcript_common_fr(mzk_transcript *t, const uint64_t v[4]);    /* Transcript::common */
int mzk_transcript_write_fr(mzk_transcript *t, const uint64_t v[4]);     /* Transcript::write */
int mzk_transcript_write_point(mzk_transcript *t, const uint64_t p[18]); /* Transcript::write */
int mzk_transcript_squeeze(mzk_transcript *t, uint64_t out[4]);          /* squeeze_challenge */
/* the proof bytes written so far (Transcript::finalize); *len = their count */
int mzk_transcript_proof(const mzk_transcript *t, uint8_t *out, size_t cap, size_t *len);
/* VerifyingKey::from_parts's transcript_repr (proofs/src/plonk/mod.rs:227-284):
 * Blake2b-512 personalised "Halo2-Verify-Key" over the version byte, k, the
 * fixed and permutation commitments (uncompressed, each list after its u32
 * length) and `pinned` = format!("{:?}", domain.pinned()) followed by
 * format!("{:?}", cs.pinned()) as the caller renders them, then
 * from_uniform_bytes.  Commitments in the 18-u64 point layout. */
int mzk_vk_transcript_repr(uint32_t k, const uint64_t *fixed_coms, size_t n_fixed, const uint64_t *perm_coms,
                           size_t n_perm, const uint8_t *pinned, size_t pinned_len, uint64_t out[4]);

/* ---- keygen and create_proof (proofs/src/plonk/{keygen,prover}.rs) ------- */
/* A column query of ConstraintSystem::advice_queries / fixed_queries. */
typedef struct { uint32_t column; int32_t rotation; } mzk_query;
/* A logup lookup whose input expression is one advice column (queried at
 * rotation 0) and whose table expression is one fixed column, with a fixed
 * selector column or none (selector_fixed = -1: the constant one). */
typedef struct { uint32_t input_advice, table_fixed; int32_t selector_fixed; } mzk_lookup_shape;
/* A lookup of n_inputs parallel tuples of advice columns into one tuple of
 * fixed columns (width 1..4 columns each, queried at rotation 0; 1..8
 * inputs), every tuple compressed with theta by Horner in its order as the
 * reference compresses lookup expressions; the inputs are split into helper
 * chunks by degree (Argument::chunk_by_degree, logup.rs:223-337: at most
 * next_pow2(degree - 1) inputs per helper), one helper polynomial each.
 * With mzk_circuit_desc.lookup_tuples given it replaces the shape's input
 * and table columns (the shape's selector still applies). */
typedef struct {
    uint32_t width, n_inputs;
    uint32_t input_advice[8][4];
    uint32_t table_fixed[4];
} mzk_lookup_tuple;
/* The constraint system a key is built for.  Gates: any custom gates as the
 * reference flattens them (`gates`, an mzk_flat_graph whose result is the
 * Horner-in-y combination of every gate polynomial, evaluation.rs:148-213;
 * every (column, rotation) it reads must be in the query lists), or, with
 * gates null, the standard gate q_l a + q_r b + q_m a b + q_o c + q_c over
 * fixed columns gate_fixed and advice columns gate_advice (each queried at
 * rotation 0).
 * Permutation columns: kind 0 advice, 1 fixed, 2 instance; sets of degree - 2 columns.
 * The query lists and their order are the reference's (they fix the order
 * of the evaluations in the proof).  Limits: 16 advice, 16 fixed, 16
 * permutation columns (8 sets), at most 8 lookups (each one advice column
 * or expression, or a tuple of them, into one fixed table column or a tuple
 * of them; their multiplicities, helpers and aggregators
 * are committed, evaluated and opened lookup by lookup, as logup/prover.rs
 * does), at most 4 instance columns (the reference's default, without the
 * committed-instances feature: every proof's instance values are absorbed
 * into its transcript, compute_instances, prover.rs:475-539; gates may read
 * them, `col_type` 2, at their queried rotations, and permutation columns of
 * kind 2 are instance columns), at most 8 trashcans (trash/prover.rs: each an
 * mzk_trash_arg whose program compresses the constraint expressions with the
 * trash challenge, reading only queried columns, and whose selector is a
 * fixed column queried at rotation 0; its `trash` pointer is not used here:
 * the prover computes, commits, evaluates and opens the trash column), and
 * simple selectors: with `gates` given, n_gate_polys > 0 lists each gate
 * polynomial in order (Gate::polynomials of every gate) by the value slot
 * that holds it in the gates program (gate_poly_values; the operand the
 * program folds into its Horner chain in y) and by its simple selector's
 * fixed column (gate_poly_selector, -1 for none).  Those fixed columns are
 * evaluated as one in the identities and are neither written to the
 * transcript nor opened; their polynomials enter the linearization, scaled by
 * the identity (partially_evaluate_identities, plonk/mod.rs:502-608;
 * compute_linearization_poly, linearization/prover.rs:41-86). */
typedef struct {
    uint32_t degree;                   /* cs.degree() (plonk/circuit.rs:2174-2199), 3..9 */
    uint32_t blinding_factors;         /* cs.blinding_factors() (circuit.rs:2203-2245) */
    uint32_t n_advice, n_fixed;
    const mzk_query *advice_queries; uint32_t n_advice_queries;
    const mzk_query *fixed_queries; uint32_t n_fixed_queries;
    uint32_t gate_fixed[5], gate_advice[3];
    const mzk_flat_graph *gates;       /* null: the standard gate above */
    uint32_t n_perm_cols;
    const uint32_t *perm_col_kind, *perm_col_index;
    uint32_t n_lookups;
    const mzk_lookup_shape *lookups;
    uint32_t n_instance;               /* instance columns (0..4) */
    const mzk_query *instance_queries; uint32_t n_instance_queries;
    uint32_t n_trash; const mzk_trash_arg *trash;
    uint32_t n_gate_polys;
    const uint32_t *gate_poly_values;  /* value slot of each gate polynomial in `gates` */
    const int32_t *gate_poly_selector; /* its simple selector's fixed column, or -1 */
    const mzk_lookup_tuple *lookup_tuples; /* null, or one per lookup */
    /* null, or every lookup input element as an expression: the programs of
     * lookup 0's input tuples element by element, then lookup 1's, ...
     * (n_inputs x width each, 1 x 1 without lookup_tuples), each evaluating
     * one input expression (BatchedArgument's input_expressions, logup.rs:
     * 47-58: any product or sum of fixed, advice and instance queries at any
     * rotation) into result_idx; it then replaces input_advice.  A program
     * that only reads an advice column at rotation 0 is that column. */
    const mzk_flat_graph *lookup_input_programs;
} mzk_circuit_desc;
/* ParamsKZG's bases (params.rs:83-93) inside one DEVICE G1Affine buffer;
 * table_c > 0: srs is row 0 of a window table of that width and table_rows
 * rows of srs_len points (mzk_msm_window_table), used by MSMs of at least
 * table_min_n points. */
typedef struct {
    const uint64_t *srs;
    uint64_t srs_len;
    uint64_t off_g, off_lagrange, off_lagrange_delta, off_lagrange_double_delta;
    int32_t table_c;
    uint32_t table_rows;
    uint64_t table_min_n;
} mzk_srs_desc;
typedef struct mzk_plonk_key mzk_plonk_key;
/* keygen_vk + keygen_pk (plonk/keygen.rs:227-359) on the device for domain d
 * (2^k rows, created with j = degree): the fixed columns' polynomials and
 * extended cosets, the permutation polynomials of build_pk
 * (permutation/keygen.rs:138-185; cell (c, r) holds delta^c' omega^r' of the
 * cell (c', r') it maps to), their polynomials and cosets, l0, l_last and
 * l_active_row (keygen.rs:361-404), the fixed and permutation commitments
 * (Lagrange basis) and the VK's transcript_repr (mzk_vk_transcript_repr).
 * fixed_values: n_fixed HOST columns of 2^k Fr (Lagrange form); perm_mapping:
 * HOST n_perm_cols x 2^k x 2 u32 (column, row) pairs (Assembly::mapping), or
 * null for the identity.  The key keeps pointers to d and to the SRS buffer:
 * both must outlive it. */
int mzk_keygen(mzk_ctx *ctx, mzk_domain *d, const mzk_circuit_desc *cs, const mzk_srs_desc *srs,
               const uint64_t *const *fixed_values, const uint32_t *perm_mapping, const uint8_t *pinned,
               size_t pinned_len, mzk_plonk_key **out);
/* The same with the permutation polynomials' Lagrange values given (n_perm_cols
 * HOST columns of 2^k Fr) instead of the copy mapping: a ProvingKey read from
 * its file holds these (ProvingKey::read, plonk/mod.rs:421-453,
 * permutation.rs:153-166). */
int mzk_keygen_from_values(mzk_ctx *ctx, mzk_domain *d, const mzk_circuit_desc *cs, const mzk_srs_desc *srs,
                           const uint64_t *const *fixed_values, const uint64_t *const *perm_values,
                           const uint8_t *pinned, size_t pinned_len, mzk_plonk_key **out);
int mzk_plonk_key_destroy(mzk_plonk_key *key);
/* Key files (VerifyingKey::write / ProvingKey::write, plonk/mod.rs:95-113,
 * 391-399; readers :120-196, :418-453) in SerdeFormat (utils/helpers.rs:
 * 17-28): Processed writes commitments compressed (48 bytes), RawBytes and
 * RawBytesUnchecked uncompressed (96 bytes); the polynomial slices of a PK
 * are always raw Montgomery limbs (u32 big-endian counts and lengths).  A VK
 * file is version 0x03, k, a u32 little-endian count and the fixed
 * commitments, then the permutation commitments; a PK file is its VK file,
 * the fixed columns' values and the permutation polynomials' values.
 * mzk_vk_write / mzk_pk_write: *len = the file's size; out may be null to ask
 * for it.  mzk_pk_read: a key from a PK file for the constraint system cs
 * (the reader's ConcreteCircuit::configure) over domain d and the SRS, with
 * the file's commitments (decoded and checked: encoding, x, y < p, curve and
 * subgroup; RawBytesUnchecked checks nothing) and values (below r unless
 * RawBytesUnchecked), as ProvingKey::read derives the rest. */
#define MZK_SERDE_PROCESSED 0
#define MZK_SERDE_RAW 1
#define MZK_SERDE_RAW_UNCHECKED 2
int mzk_vk_write(const mzk_plonk_key *key, int format, uint8_t *out, size_t cap, size_t *len);
int mzk_pk_write(mzk_ctx *ctx, const mzk_plonk_key *key, int format, uint8_t *out, size_t cap, size_t *len);
int mzk_pk_read(mzk_ctx *ctx, mzk_domain *d, const mzk_circuit_desc *cs, const mzk_srs_desc *srs,
                const uint8_t *bytes, size_t len, int format, const uint8_t *pinned, size_t pinned_len,
                mzk_plonk_key **out);
/* The transcript operations of one proof of this key, in order: one code per
 * operation (MZK_TR_*).  A caller holding its own transcript object (the
 * reference's CircuitTranscript) replays a proof into it with these: a
 * point is 48 proof bytes, a scalar 32, a squeeze reads nothing.  A key with
 * instance columns also absorbs, right after the VK's repr, each instance
 * column's length and values (common, not in the proof bytes; the caller
 * holds them): those operations depend on the request and are not listed. */
#define MZK_TR_COMMON_FR 0   /* the VK's transcript_repr (not in the proof bytes) */
#define MZK_TR_WRITE_POINT 1
#define MZK_TR_WRITE_FR 2
#define MZK_TR_SQUEEZE 3
int mzk_plonk_key_transcript_layout(const mzk_plonk_key *key, uint8_t *ops, size_t cap, size_t *len);
/* repr (optional): transcript_repr; proof_len: bytes of one proof;
 * n_blinds: the rng draws one proof takes (the order under
 * mzk_create_proofs) */
int mzk_plonk_key_info(const mzk_plonk_key *key, uint64_t repr[4], size_t *proof_len, size_t *n_blinds);
/* the VK commitments: fixed n_fixed x 18 u64, permutation n_perm_cols x 18 u64 */
int mzk_plonk_key_commitments(const mzk_plonk_key *key, uint64_t *fixed, uint64_t *perm);
/* the SRS description the key was built over */
int mzk_plonk_key_srs(const mzk_plonk_key *key, mzk_srs_desc *out);
/* One proof: the advice columns (2^k Fr each in Lagrange form; rows from
 * 2^k - blinding_factors - 1 on are replaced by blinding values), HOST or
 * DEVICE pointers, and the rng draws in the reference's order: the blinding
 * rows of every advice column (prover.rs:606-617, bf + 1 each), the
 * multiplicity blinds of every lookup (prover.rs:122-123, bf + 1 each), the
 * permutation blinds of every set (:165-167, bf each), the logup blinds of
 * every lookup (:168, bf each), then the degree - 2 quotient-limb blinds
 * (blind_quotient_limbs draws those from OsRng, prover.rs:774-785; taking them
 * from the caller makes proofs reproducible).  proof_out receives the
 * transcript bytes (Transcript::finalize).  instance / instance_len: the
 * values of each instance column of the key (HOST, Montgomery Fr, at most
 * n - blinding_factors - 1 each, else MZK_ERR_ARG as Error::InstanceTooLarge;
 * rows past a column's values are zero); null when the key has none. */
typedef struct {
    const mzk_plonk_key *key;
    const uint64_t *const *advice;
    int advice_on_device;
    const uint64_t *blinds;  /* HOST, n_blinds Fr */
    uint8_t *proof_out;      /* HOST, at least proof_len bytes */
    const uint64_t *const *instance;
    const uint64_t *instance_len;
} mzk_proof_request;
/* create_proof (plonk/prover.rs:432-473) for `count` proofs, any keys over
 * one SRS buffer: each phase of the reference's Fiat-Shamir order (advice
 * commitments, theta; multiplicities, beta, gamma; permutation products and
 * logup helper / aggregator, trash challenge, y; quotient limbs, x;
 * evaluations; multi_open with f, x3, the q evaluations, x4 and pi,
 * kzg/mod.rs:110-289) runs for every proof before the next, its MSMs as one
 * batched MSM (or, with MZK_PROVE_MSM_PER_CALL, one call each); the
 * polynomial transforms of all proofs of one domain run together (or, with
 * MZK_PROVE_NO_GRAPHS, proof by proof, kernel by kernel).  Flags:
 * MZK_PROVE_MSM_PER_CALL, MZK_PROVE_NO_GRAPHS (above) and: */
#define MZK_PROVE_SELF_CHECK 4u /* also check L'(x) = -C (prover.rs:404-408): an unsatisfied witness fails */
int mzk_create_proofs(mzk_ctx *ctx, const mzk_proof_request *reqs, size_t count, uint32_t flags);

/* ---- column scans: grand products, running sums, evaluations ------------- */
/* All arrays are DEVICE arrays of Fr (4 x u64 Montgomery) unless marked host. */

/* ff 0.13 BatchInvert (used by permutation/prover.rs:139, logup/prover.rs:221,
 * 232): every non-zero element of a[0..n) replaced by its inverse, zeros kept. */
int mzk_batch_invert_device(mzk_ctx *ctx, uint64_t *a, size_t n);
/* eval_polynomial (proofs/src/utils/arithmetic.rs:59-87): out (host) =
 * sum_i poly[i] point^i. */
int mzk_eval_polynomial_device(mzk_ctx *ctx, const uint64_t *poly, size_t n, const uint64_t point[4],
                               uint64_t out[4]);
/* kate_division (utils/arithmetic.rs:106-125): q[0..n-1) = a(X) / (X - b). */
int mzk_kate_division_device(mzk_ctx *ctx, const uint64_t *a, size_t n, const uint64_t b[4], uint64_t *q);
/* poly_inner_product of multi_open (proofs/src/poly/kzg/mod.rs:125-147):
 * out[i] = sum_p scalars[p] * polys[p][i], each polynomial zero-extended to
 * out_len = the longest length.  polys: m device pointers (host array), lens:
 * their lengths (host), scalars: m Fr (host). */
int mzk_poly_inner_product_device(mzk_ctx *ctx, const uint64_t *const *polys, const size_t *lens, size_t m,
                                  const uint64_t *scalars, uint64_t *out, size_t out_len);

/* Permutation argument, permutation/prover.rs:81-255: the z polynomial of each
 * set of chunk_len columns (Lagrange form, n = 2^k values each), blinding rows
 * from blinds (host, n_sets x blinding_factors Fr), sets chained as in the
 * reference.  values[j], sigmas[j]: column j and its permutation polynomial. */
typedef struct {
    uint32_t n_cols;
    const uint64_t *const *values;  /* n_cols device arrays */
    const uint64_t *const *sigmas;  /* n_cols device arrays */
    uint32_t chunk_len;             /* cs.degree() - 2, at most 8 */
    uint32_t blinding_factors;
    const uint64_t *blinds;         /* host */
    uint64_t beta[4], gamma[4];
    uint64_t *const *z_out;         /* ceil(n_cols / chunk_len) device arrays */
} mzk_permutation_desc;
int mzk_permutation_z_device(mzk_ctx *ctx, mzk_domain *d, const mzk_permutation_desc *desc);

/* Logup argument, logup/prover.rs:195-300: helper h_c = sum over the chunk's
 * compressed input columns of 1/(f + beta), and the aggregator (running sum of
 * selector * sum_c h_c - m / (t + beta), n - blinding_factors rows, then the
 * blinding values). */
typedef struct {
    uint32_t n_chunks;               /* at most 8 */
    const uint32_t *chunk_cols;      /* host: columns per chunk */
    const uint64_t *const *inputs;   /* compressed input columns, chunk by chunk */
    const uint64_t *table;           /* compressed table expression */
    const uint64_t *selector;
    const uint64_t *multiplicities;
    uint32_t blinding_factors;
    const uint64_t *blinds;          /* host, blinding_factors Fr */
    uint64_t beta[4];
    uint64_t *const *helpers_out;    /* n_chunks device arrays */
    uint64_t *aggregator_out;
} mzk_logup_desc;
int mzk_logup_device(mzk_ctx *ctx, mzk_domain *d, const mzk_logup_desc *desc);

/* ---- KZG setup on the device ------------------------------------------- */
/* ParamsKZG::unsafe_setup (proofs/src/poly/kzg/params.rs:160-209), G1 part,
 * for the secret s (host Fr, Montgomery; the reference draws it from its rng)
 * and the domain's n = 2^k: g[i] = [s^i]G, g_lagrange[i] = [L_i(s)]G with
 * L_i(s) = (s^n - 1)/n * w^i/(s - w^i), g_lagrange_delta = suffix sums of
 * g_lagrange and g_lagrange_double_delta = suffix sums of those
 * (suffix_sum, params.rs:47-57).  Outputs: DEVICE G1Affine arrays of n points,
 * any of them null when not wanted.  The G2 elements are not produced. */
int mzk_srs_setup_device(mzk_ctx *ctx, mzk_domain *d, const uint64_t s[4], uint64_t *g, uint64_t *g_lagrange,
                         uint64_t *g_lagrange_delta, uint64_t *g_lagrange_double_delta);
/* g_to_lagrange (proofs/src/utils/arithmetic.rs:34-54): out[i] = (1/n)
 * sum_j w^(-ij) g[j] for the domain's n = 2^k (DEVICE G1Affine arrays). */
int mzk_g1_to_lagrange_device(mzk_ctx *ctx, mzk_domain *d, const uint64_t *g, uint64_t *out);
/* ParamsKZG::downsize (params.rs:96-107) for the domain's k: g_lagrange =
 * g_to_lagrange(g[0..n)), then its two suffix sums (outputs may be null). */
int mzk_srs_downsize_device(mzk_ctx *ctx, mzk_domain *d, const uint64_t *g, uint64_t *g_lagrange,
                            uint64_t *g_lagrange_delta, uint64_t *g_lagrange_double_delta);
/* suffix_sum (params.rs:47-57): out[i] = sum_{j >= i} in[j], n DEVICE G1Affine. */
int mzk_g1_suffix_sum_device(mzk_ctx *ctx, const uint64_t *in, size_t n, uint64_t *out);
/* G1Affine::from_compressed (curves/src/bls12_381/g1.rs:367-376) of n 48-byte
 * ZCash encodings (DEVICE, contiguous) into n DEVICE G1Affine; status
 * (optional DEVICE n bytes): 0 ok, 1 bad encoding, 2 not on the curve, 3 not
 * in G1 (checked when check_subgroup != 0); invalid points are written as the
 * identity and counted in *n_invalid (host, optional). */
int mzk_g1_decompress_device(mzk_ctx *ctx, const uint8_t *in, size_t n, int check_subgroup, uint64_t *out,
                             uint8_t *status, uint64_t *n_invalid);
/* G1Affine::to_compressed (curves/src/bls12_381/g1.rs:326-334; ZCash format:
 * x big-endian, 0x80 compressed, 0x40 identity, 0x20 the larger y) of n
 * DEVICE points into n x 48 DEVICE bytes. */
int mzk_g1_compress_device(mzk_ctx *ctx, const uint64_t *points, size_t n, uint8_t *out);
/* ParamsKZG::write_custom(.., SerdeFormat::Processed) (proofs/src/poly/kzg/
 * params.rs:260-281), G1 part: out (host, at least 4 + 96 n bytes) = k as u32
 * little-endian, n compressed g, n compressed g_lagrange (n = 2^k, DEVICE
 * inputs); the caller appends the two G2 elements. */
int mzk_srs_write_processed(mzk_ctx *ctx, const uint64_t *g, const uint64_t *g_lagrange, size_t n, uint8_t *out,
                            size_t out_len);
/* ParamsKZG::read_custom with SerdeFormat::Processed (params.rs:283-350), G1
 * part: bytes (host) = k as u32 LE, 2^k compressed g, 2^k compressed
 * g_lagrange (the G2 elements that follow are not read).  Points are
 * decompressed and checked on the device; the delta bases are derived as the
 * reference does after reading.  Outputs: DEVICE arrays of capacity points
 * (any may be null); returns MZK_ERR_ARG on a short buffer, 2^k > capacity or
 * an invalid point encoding. */
int mzk_srs_read_processed(mzk_ctx *ctx, const uint8_t *bytes, size_t len, size_t capacity, uint32_t *k_out,
                           uint64_t *g, uint64_t *g_lagrange, uint64_t *g_lagrange_delta,
                           uint64_t *g_lagrange_double_delta);

/* ---- proving service (continuous batching over create_proof) ------------ */
/* No reference counterpart: the reference proves one call at a time.
 * `lanes` worker threads (1..8), each with its own device context, serve one
 * request queue of create_proof requests (mzk_proof_request, any keys).  An
 * idle lane takes a wave: queued requests oldest first whose keys share the
 * first one's SRS buffer, while the wave holds fewer than max_batch proofs,
 * its device scratch stays within mem_budget_bytes / lanes and that of all
 * proofs in flight within mem_budget_bytes (0: no limit; a proof larger than
 * that runs alone when nothing else is in flight), run as one
 * mzk_create_proofs call with `flags`; requests arriving while a wave runs
 * start beside it on the device.  max_batch = 1 with one lane and
 * MZK_PROVE_MSM_PER_CALL is the plain one-call-at-a-time prover.  A
 * request's witness, blinds and output buffer must stay valid until its
 * wait returns. */
typedef struct mzk_server mzk_server;
int mzk_server_create(mzk_ctx *ctx, uint32_t max_batch, uint32_t lanes, uint64_t mem_budget_bytes,
                      uint32_t flags /* MZK_PROVE_* of every wave */, mzk_server **out);
/* caps the rows (sum of 2^k) of one wave (0: no cap, the default); a wave's
 * duration grows with its rows, so the cap bounds how long a request that
 * arrives meanwhile waits behind it.  A single request larger than the cap
 * still runs, alone. */
int mzk_server_set_wave_rows(mzk_server *s, uint64_t max_rows);
int mzk_server_submit(mzk_server *s, const mzk_proof_request *req, uint64_t *ticket);
/* blocks until the request is done (its transcript in req->proof_out);
 * latency from submit to completion */
int mzk_server_wait(mzk_server *s, uint64_t ticket, double *latency_ms);
int mzk_server_stats(mzk_server *s, uint64_t *waves, uint64_t *proofs, double *busy_ms);
int mzk_server_destroy(mzk_server *s);

/* ---- seeded synthetic inputs (benchmarks and tests) -------------------- */
/* n uniform Fr elements (Montgomery) of stream `seed`, elements first..first+n-1 */
int mzk_gen_rand_fr_device(mzk_ctx *ctx, uint64_t seed, uint64_t first, size_t n, uint64_t *d_out);
/* n affine bases [r_i]G with r_i the Fr elements of stream `seed` */
int mzk_gen_bases_g1_device(mzk_ctx *ctx, uint64_t seed, uint64_t first, size_t n, uint64_t *d_out);
/* A seeded instance of the single-proof configuration's circuit (standard
 * gate over a, b, c, copy cycles, range lookup of a), for benchmarks.
 * gen_config3_fixed: the 7 fixed columns q_l, q_r, q_m, q_o, q_c, table,
 * selector (one DEVICE buffer of 7 x 2^k Fr): the q uniform on the usable rows
 * u = 2^k - blinding_factors - 1 (q_o never zero) and zero after them, the
 * table 0 .. min(table_rows, u) - 1 then zeros, the selector one on the usable
 * rows.  gen_config3_witness: a, b, c (one DEVICE buffer of 3 x 2^k Fr) for
 * those columns: a a table value, b uniform, every cell of one copy cycle the
 * cycle's table value (cycle_of: DEVICE u32 per cell of a then of b, 0xffffffff
 * outside cycles), c solving the gate with inv_qo = 1 / q_o (DEVICE, 2^k Fr);
 * rows from u on are zero.  Element values depend only on (seed, row). */
int mzk_gen_config3_fixed_device(mzk_ctx *ctx, uint32_t k, uint32_t blinding_factors, uint32_t table_rows,
                                 uint64_t seed, uint64_t *d_fixed);
int mzk_gen_config3_witness_device(mzk_ctx *ctx, uint32_t k, uint32_t blinding_factors, uint32_t table_rows,
                                   uint64_t seed, const uint64_t *d_fixed, const uint64_t *d_inv_qo,
                                   const uint32_t *d_cycle_of, uint64_t *d_advice);

#ifdef __cplusplus
}
#endif
#endif
