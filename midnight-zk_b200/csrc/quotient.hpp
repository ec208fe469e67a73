// quotient.hpp — kernel parameters of the fused quotient evaluation.
#pragma once
#include <cstdint>

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
};

// compute_h_poly (proofs/src/plonk/prover.rs:701-771) without the transcript:
// commitments: quotient_poly_degree x 18 u64 (host); blinds: (limbs - 1) x 4
// u64 (host); d_limbs_out (optional, device): limbs x n Fr
Status compute_h_poly_device(Context* ctx, const Domain* d, const mzk_quotient_desc* desc, const void* d_srs_g,
                             size_t srs_len, const uint64_t* blinds, uint64_t* commitments, void* d_limbs_out,
                             cudaStream_t st);
Status quotient_eval_device(Context* ctx, const Domain* d, const mzk_quotient_desc* desc, int divide, void* d_out,
                            cudaStream_t st);

}  // namespace mzk
