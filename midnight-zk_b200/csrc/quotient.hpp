// quotient.hpp — kernel parameters of the fused quotient evaluation.
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/mzk.h"
#include "field.cuh"
#include "ntt.hpp"
#include "runtime.hpp"

namespace mzk {

constexpr uint32_t kQMaxAdvice = 16, kQMaxFixed = 16, kQMaxPermCols = 16, kQMaxSets = 8;

// passed by value to the kernel (well under the parameter-space limit)
struct QuotientParams {
    const Fr* advice[kQMaxAdvice];
    const Fr* fixed[kQMaxFixed];
    const Fr* instance[4];  // kQMaxInstance: instance columns a permutation column may name
    const Fr* sigma[kQMaxPermCols];
    const Fr* z[kQMaxSets];
    const Fr *lh, *lz, *lm, *l0, *l_last, *l_active;
    const Fr *tlo, *thi, *tinv;
    Fr* out;
    Fr y, beta, gamma, theta, delta_start, delta;
    uint32_t gate_fixed[5], gate_advice[3];
    uint32_t n_perm_cols, n_sets, chunk_len;
    uint8_t perm_kind[kQMaxPermCols], perm_index[kQMaxPermCols];
    int32_t last_rot;
    int32_t has_lookup, lookup_selector;
    uint32_t lookup_input, lookup_table;
    uint32_t tlen, log_n, log_scale;
    int32_t divide;
    int32_t gate_from_out;  // the custom-gate value of each row is already in out (k_gates_flat)
};

// Flattened programs (mzk_flat_graph: custom gates, lookup helpers,
// trashcans), packed into one device word buffer.  A program's header at word
// h: n_reads, n_ops, static_len, previous_value_idx, result_idx, then the word
// offsets of its reads (4 words each: col_type, col_idx, rot_idx, dst), ops (5
// words: kind, dst, a, b, c), rotation offsets ((rot << log_scale) mod 2^log_n)
// and statics (Fr values [0, static_len): constants and challenge slots,
// 16-byte aligned).
constexpr uint32_t kQMaxInstance = 4, kFlatMaxValues = 256, kFlatMaxRotations = 32;
constexpr uint32_t kQMaxLookups = 8, kQMaxHelpers = 8, kQMaxTrash = 8;
constexpr uint32_t kFlatHeaderWords = 9;
struct FlatCols {
    const Fr* c[3][kQMaxFixed > kQMaxAdvice ? kQMaxFixed : kQMaxAdvice];  // fixed, advice, instance
};
struct GatesParams {  // k_gates_flat: the custom gates
    FlatCols cols;
    const uint32_t* words;
    uint32_t prog, log_n;
    Fr* out;
};
struct TailParams {  // k_tail_flat: lookup and trash terms after the permutations
    FlatCols cols;
    const uint32_t* words;
    const Fr *l0, *l_last, *l_active, *tinv;
    const Fr* agg[kQMaxLookups];
    const Fr* mult[kQMaxLookups];
    const Fr* helper[kQMaxLookups][kQMaxHelpers];
    uint32_t prog[kQMaxLookups][kQMaxHelpers];
    uint32_t outputs[kQMaxLookups][kQMaxHelpers][4];  // sum_partial_products, product, table, selector
    uint32_t n_helpers[kQMaxLookups];
    uint32_t n_lookups;
    const Fr* trash[kQMaxTrash];
    uint32_t trash_sel[kQMaxTrash], trash_prog[kQMaxTrash], n_trash;
    Fr y;
    uint32_t tlen, log_n, log_scale;
    int32_t divide;
    Fr* out;
};

// compute_h_poly (proofs/src/plonk/prover.rs:701-771) without the transcript:
// commitments: quotient_poly_degree x 18 u64 (host); blinds: (limbs - 1) x 4
// u64 (host); d_limbs_out (optional, device): limbs x n Fr
Status compute_h_poly_device(Context* ctx, const Domain* d, const mzk_quotient_desc* desc, const void* d_srs_g,
                             size_t srs_len, const uint64_t* blinds, uint64_t* commitments, void* d_limbs_out,
                             cudaStream_t st);
// the limb stage of compute_h_poly into caller buffers (d_hbuf: 2^ext_k Fr,
// d_blinds: qdeg Fr, both device scratch); blinds on the host
Status compute_h_limbs_device(Context* ctx, const Domain* d, const mzk_quotient_desc* desc, const uint64_t* blinds,
                              void* d_limbs_out, void* d_hbuf, void* d_blinds, cudaStream_t st);
// device part of create_proof for the single-proof circuit (prover.cu)
constexpr int kProofCoreCommitments = 11;  // a, b, c, m, z, Z, h, 4 quotient limbs
// flags: MZK_PROVE_MSM_PER_CALL runs every MSM as its own call (the plain
// one-call-at-a-time form) instead of the two batched MSMs
Status prove_core_device(Context* ctx, const Domain* d, const mzk_proving_key_desc* pk, const mzk_proof_job* jobs,
                         size_t count, uint64_t* out, uint32_t flags, cudaStream_t st);
// jobs of different k: job j uses doms[j] and pks[j] (all keys share one SRS buffer)
Status prove_core_multi(Context* ctx, const Domain* const* doms, const mzk_proving_key_desc* const* pks,
                        const mzk_proof_job* jobs, size_t count, uint64_t* out, uint32_t flags, cudaStream_t st);
// Polynomial::to_delta (order 1) / to_double_delta (order 2) of n device Fr
// (proofs/src/poly/mod.rs:297-336); out must not alias a
Status delta_device(Context* ctx, const void* a, void* out, uint32_t n, int order, cudaStream_t st);
// the MSMs of `items` against the SRS: one batched MSM, or with
// MZK_PROVE_MSM_PER_CALL in flags one call each; with a window table
// (table non-null) the items of at least table->min_n points use it
Status run_msms(Context* ctx, const void* srs, uint64_t srs_len, const std::vector<BatchItem>& items, uint64_t* res,
                uint32_t flags, const MsmTable* table, cudaStream_t st);
// lagrange_to_coeff then coeff_to_extended of `count` polynomials, captured
// once into a CUDA graph per pointer set and replayed when use_graph is set
Status ntt_sequence(Context* ctx, const Domain* d, const void* const* lag, Fr* const* coeff, Fr* const* ext,
                    int count, bool use_graph, cudaStream_t st);
// create_proof with the Fiat-Shamir transcript (plonk.cu)
Status create_proofs(Context* ctx, const mzk_proof_request* reqs, size_t count, uint32_t flags, cudaStream_t st);
uint64_t proof_device_bytes(const mzk_plonk_key* key);
uint64_t proof_rows(const mzk_plonk_key* key);  // 2^k of the key
// one flattened program at every row of the n-point domain over Lagrange
// columns, or (extended) at every row of the extended coset over the
// columns' coset values, a rotation of r rows then 2^(ext_k - k) r rows
Status flat_program_rows(Context* ctx, const Domain* d, const mzk_flat_graph& g, const uint64_t* const* fixed,
                         uint32_t n_fixed, const uint64_t* const* advice, uint32_t n_advice,
                         const uint64_t* const* instance, uint32_t n_instance, const uint64_t beta[4],
                         const uint64_t theta[4], const uint64_t trash[4], const uint64_t y[4], uint64_t* out,
                         cudaStream_t st, bool extended = false);
Status quotient_eval_device(Context* ctx, const Domain* d, const mzk_quotient_desc* desc, int divide, void* d_out,
                            cudaStream_t st);

}  // namespace mzk
