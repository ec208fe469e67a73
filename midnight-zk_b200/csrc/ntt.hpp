// ntt.hpp — device EvaluationDomain (proofs/src/poly/domain.rs:34-49).
#pragma once
#include <cstdint>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "field.cuh"
#include "host_ec.hpp"
#include "runtime.hpp"

namespace mzk {

// operation codes of mzk_domain_op_device (include/mzk.h)
enum DomainOp : int {
    OP_COEFF_TO_LAGRANGE = 0,
    OP_LAGRANGE_TO_COEFF = 1,
    OP_COEFF_TO_EXTENDED = 2,
    OP_EXTENDED_TO_COEFF = 3,
    OP_EXTENDED_TO_LAGRANGE = 4,
    OP_DIVIDE_BY_VANISHING = 5,
};

// pass split of a multi-pass transform (the autotuner's NTT choice):
// even (larger passes first when uneven), the largest passes (2^11 elements
// per tile) first, or the largest passes last
enum NttSplit : int { kSplitEven = 1, kSplitFront = 2, kSplitBack = 3 };

struct Domain {
    uint32_t k = 0, ext_k = 0;
    uint32_t quotient_poly_degree = 0;  // j - 1
    host::Fr4 omega, omega_inv, ext_omega, ext_omega_inv, zeta, zeta2, ifft_div, ext_ifft_div;
    std::vector<host::Fr4> t_inv;  // 1 / t(zeta * ext_omega^i), i < 2^(ext_k - k)
    // per root (0 omega, 1 omega_inv, 2 ext_omega, 3 ext_omega_inv):
    // lo[r][i] = w^i (i < 4096), hi[r][i] = w^(4096 i)
    Fr* tables[4] = {};
    Fr* lo[4] = {};
    Fr* hi[4] = {};
    void* d_tinv = nullptr;
    // inter-pass twiddles of one non-last DIF pass, laid out as the pass
    // writes its output: tw[(m << (log_s - log_r)) + j] = w^((N/S) j bitrev_r(m))
    // for the pass over segments of S = 2^log_s elements with R = 2^log_r rows
    // (N = 2^log_n of root r).  Keyed by (root, log_s, log_r); built for the
    // split in force when the domain is created, and for another split the
    // first time a transform outside stream capture uses it.
    mutable std::mutex tw_mu;
    mutable std::map<std::tuple<int, uint32_t, uint32_t>, Fr*> pass_tw;
    ~Domain();
};

Status domain_create(Context* ctx, uint32_t j, uint32_t k, Domain** out);
// d_in / d_out device pointers (may alias for the in-place operations)
Status domain_op_device(Context* ctx, const Domain* d, int op, const void* d_in, void* d_out, cudaStream_t st);
// the same operation (C2L, L2C, C2E or E2C) on T inputs of the domain, up to
// 64 transforms per launch of each pass
Status domain_op_batch(Context* ctx, const Domain* d, int op, const void* const* ins, void* const* outs, uint32_t T,
                       cudaStream_t st);
size_t domain_op_in_len(const Domain* d, int op);
size_t domain_op_out_len(const Domain* d, int op);

}  // namespace mzk
