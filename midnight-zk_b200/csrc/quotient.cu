// quotient.cu — fused quotient evaluation over the extended domain.
//
// Replaces Evaluator::evaluate_numerator (proofs/src/plonk/evaluation.rs:818-1114)
// followed by EvaluationDomain::divide_by_vanishing_poly (domain.rs:361-380)
// for the circuit shape of the single-proof configuration: one standard gate
// q_l a + q_r b + q_m a b + q_o c + q_c, permutation sets over advice/fixed
// columns (chunks of cs.degree() - 2 columns), at most one logup lookup with a
// single input column and a single helper, no trashcans.
//
// The reference makes three passes over the 2^extended_k rows (gates, then
// permutations, then lookups) plus one for the division; here one thread per
// row reads every column once (coalesced, rotations are whole-row offsets),
// folds all terms into the y-Horner accumulator in the reference's order and
// multiplies by 1/t(X) before the single store.  The per-row power w^idx of the
// permutation's delta term comes from the domain's split twiddle tables.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mzk.h"
#include "field.cuh"
#include "ntt.hpp"
#include "quotient.hpp"
#include "runtime.hpp"

namespace mzk {

namespace {

__device__ __forceinline__ Fr ldfr(const Fr* p, size_t i) {
    const uint4* s = reinterpret_cast<const uint4*>(p + i);
    const uint4 a = __ldg(s), b = __ldg(s + 1);
    Fr r;
    r.l[0] = a.x; r.l[1] = a.y; r.l[2] = a.z; r.l[3] = a.w;
    r.l[4] = b.x; r.l[5] = b.y; r.l[6] = b.z; r.l[7] = b.w;
    return r;
}

__global__ void __launch_bounds__(256) k_quotient(QuotientParams q) {
    const uint32_t E = 1u << q.log_n;
    const uint32_t mask = E - 1;
    const uint32_t stride = gridDim.x * blockDim.x;
    const Fr one = fr_one();
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < E; idx += stride) {
        const uint32_t r_next = (idx + (1u << q.log_scale)) & mask;
        const uint32_t r_last = (idx + (uint32_t)(q.last_rot * (int32_t)(1u << q.log_scale))) & mask;
        Fr v;
        if (q.gate_from_out) {  // custom gates evaluated by k_gates_flat
            v = q.out[idx];
        } else {  // the standard gate (Horner from zero over its single polynomial)
            const Fr a = ldfr(q.advice[q.gate_advice[0]], idx);
            const Fr b = ldfr(q.advice[q.gate_advice[1]], idx);
            const Fr c = ldfr(q.advice[q.gate_advice[2]], idx);
            v = fr_mul(ldfr(q.fixed[q.gate_fixed[0]], idx), a);
            v = fr_add(v, fr_mul(ldfr(q.fixed[q.gate_fixed[1]], idx), b));
            v = fr_add(v, fr_mul(fr_mul(a, b), ldfr(q.fixed[q.gate_fixed[2]], idx)));
            v = fr_add(v, fr_mul(ldfr(q.fixed[q.gate_fixed[3]], idx), c));
            v = fr_add(v, ldfr(q.fixed[q.gate_fixed[4]], idx));
        }
        Fr l0 = fr_zero(), la = fr_zero();
        if (q.n_sets || q.has_lookup) {
            l0 = ldfr(q.l0, idx);
            la = ldfr(q.l_active, idx);
        }
        if (q.n_sets) {
            const Fr ll = ldfr(q.l_last, idx);
            const Fr z0 = ldfr(q.z[0], idx);
            const Fr zl = ldfr(q.z[q.n_sets - 1], idx);
            v = fr_add(fr_mul(v, q.y), fr_mul(fr_sub(one, z0), l0));
            v = fr_add(fr_mul(v, q.y), fr_mul(fr_sub(fr_mul(zl, zl), zl), ll));
            for (uint32_t s = 1; s < q.n_sets; s++)
                v = fr_add(fr_mul(v, q.y), fr_mul(fr_sub(ldfr(q.z[s], idx), ldfr(q.z[s - 1], r_last)), l0));
            // current_delta = beta * g_coset * w^idx
            Fr ew = q.tlo[idx & 4095u];
            if (idx >> 12) ew = fr_mul(q.thi[idx >> 12], ew);
            Fr cur = fr_mul(q.delta_start, ew);
            uint32_t col = 0;
            for (uint32_t s = 0; s < q.n_sets; s++) {
                Fr left = ldfr(q.z[s], r_next);
                Fr right = ldfr(q.z[s], idx);
                const uint32_t end = min(col + q.chunk_len, q.n_perm_cols);
                for (uint32_t j = col; j < end; j++) {
                    const Fr* colp = q.perm_kind[j] == 0   ? q.advice[q.perm_index[j]]
                                     : q.perm_kind[j] == 1 ? q.fixed[q.perm_index[j]]
                                                           : q.instance[q.perm_index[j]];
                    const Fr val = ldfr(colp, idx);
                    const Fr base = fr_add(val, q.gamma);
                    left = fr_mul(left, fr_add(base, fr_mul(q.beta, ldfr(q.sigma[j], idx))));
                    right = fr_mul(right, fr_add(base, cur));
                    cur = fr_mul(cur, q.delta);
                }
                col = end;
                v = fr_add(fr_mul(v, q.y), fr_mul(fr_sub(left, right), la));
            }
        }
        if (q.has_lookup) {
            const Fr ll = ldfr(q.l_last, idx);
            const Fr Z = ldfr(q.lz, idx);
            const Fr h = ldfr(q.lh, idx);
            v = fr_add(fr_mul(v, q.y), fr_mul(Z, fr_add(l0, ll)));
            // single compressed input (Horner over one expression) + beta
            const Fr f = fr_add(ldfr(q.advice[q.lookup_input], idx), q.beta);
            v = fr_sub(fr_add(fr_mul(v, q.y), fr_mul(h, f)), one);
            const Fr tv = fr_add(ldfr(q.fixed[q.lookup_table], idx), q.beta);
            const Fr sel = q.lookup_selector < 0 ? one : ldfr(q.fixed[q.lookup_selector], idx);
            Fr u = fr_sub(fr_sub(ldfr(q.lz, r_next), Z), fr_mul(sel, h));
            u = fr_add(fr_mul(u, tv), ldfr(q.lm, idx));
            v = fr_add(fr_mul(v, q.y), fr_mul(u, la));
        }
        if (q.divide) v = fr_mul(v, q.tinv[idx & (q.tlen - 1)]);
        q.out[idx] = v;
    }
}

// One row of a packed program, as FlatGraphEvaluator::evaluate
// (evaluation.rs:530-651): statics, the previous value (zero: every program
// here starts from zero), the column reads at their rotations, then the ops.
// Every index was checked on the host against kFlatMaxValues and the column
// counts.
__device__ void run_program(const uint32_t* __restrict__ W, uint32_t h, const FlatCols& cols, uint32_t idx,
                            uint32_t mask, Fr* vals) {
    const uint32_t n_reads = W[h], n_ops = W[h + 1], static_len = W[h + 2], pv = W[h + 3];
    const uint32_t* reads = W + W[h + 5];
    const uint32_t* ops = W + W[h + 6];
    const uint32_t* rot_off = W + W[h + 7];
    const Fr* statics = reinterpret_cast<const Fr*>(W + W[h + 8]);
    for (uint32_t i = 0; i < static_len; i++) vals[i] = statics[i];
    vals[pv] = fr_zero();
    for (uint32_t r = 0; r < n_reads; r++) {
        const uint32_t* rd = reads + 4 * r;
        vals[rd[3]] = ldfr(cols.c[rd[0]][rd[1]], (idx + rot_off[rd[2]]) & mask);
    }
    for (uint32_t o = 0; o < n_ops; o++) {
        const uint32_t* op = ops + 5 * o;
        const Fr& a = vals[op[2]];
        Fr r;
        switch (op[0]) {
            case MZK_FLAT_ADD: r = fr_add(a, vals[op[3]]); break;
            case MZK_FLAT_SUB: r = fr_sub(a, vals[op[3]]); break;
            case MZK_FLAT_MUL: r = fr_mul(a, vals[op[3]]); break;
            case MZK_FLAT_SQUARE: r = fr_mul(a, a); break;
            case MZK_FLAT_DOUBLE: r = fr_add(a, a); break;
            case MZK_FLAT_NEGATE: r = fr_sub(fr_zero(), a); break;
            default: r = fr_add(fr_mul(a, vals[op[3]]), vals[op[4]]); break;  // MZK_FLAT_MULADD
        }
        vals[op[1]] = r;
    }
}

// The custom gates of any circuit, one thread per row (the first pass of
// evaluate_numerator, evaluation.rs:846-856); the values buffer lives in the
// thread's local memory.
__global__ void __launch_bounds__(128) k_gates_flat(GatesParams g) {
    Fr vals[kFlatMaxValues];
    const uint32_t E = 1u << g.log_n, mask = E - 1, stride = gridDim.x * blockDim.x;
    const uint32_t result = g.words[g.prog + 4];
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < E; idx += stride) {
        run_program(g.words, g.prog, g.cols, idx, mask, vals);
        g.out[idx] = vals[result];
    }
}

// The lookup terms (evaluation.rs:1034-1090) and trash terms (:1093-1109) of
// any shape, continuing each row's y-Horner accumulator from out (custom
// gates and permutation terms), then the division by t(X).
__global__ void __launch_bounds__(128) k_tail_flat(TailParams t) {
    Fr vals[kFlatMaxValues];
    const uint32_t E = 1u << t.log_n, mask = E - 1, stride = gridDim.x * blockDim.x;
    const Fr one = fr_one();
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < E; idx += stride) {
        const uint32_t r_next = (idx + (1u << t.log_scale)) & mask;
        Fr v = t.out[idx];
        if (t.n_lookups) {
            const Fr l0 = ldfr(t.l0, idx), ll = ldfr(t.l_last, idx), la = ldfr(t.l_active, idx);
            for (uint32_t n = 0; n < t.n_lookups; n++) {
                const Fr Z = ldfr(t.agg[n], idx);
                v = fr_add(fr_mul(v, t.y), fr_mul(Z, fr_add(l0, ll)));
                Fr sum_h = fr_zero(), table = fr_zero(), sel = fr_zero();
                for (uint32_t fi = 0; fi < t.n_helpers[n]; fi++) {
                    run_program(t.words, t.prog[n][fi], t.cols, idx, mask, vals);
                    const uint32_t* o = t.outputs[n][fi];
                    if (fi == 0) {
                        table = vals[o[2]];
                        sel = vals[o[3]];
                    }
                    const Fr h = ldfr(t.helper[n][fi], idx);
                    v = fr_sub(fr_add(fr_mul(v, t.y), fr_mul(h, vals[o[1]])), vals[o[0]]);
                    sum_h = fr_add(sum_h, h);
                }
                Fr u = fr_sub(fr_sub(ldfr(t.agg[n], r_next), Z), fr_mul(sel, sum_h));
                u = fr_add(fr_mul(u, table), ldfr(t.mult[n], idx));
                v = fr_add(fr_mul(v, t.y), fr_mul(la, u));
            }
        }
        for (uint32_t n = 0; n < t.n_trash; n++) {
            run_program(t.words, t.trash_prog[n], t.cols, idx, mask, vals);
            const Fr q = ldfr(t.cols.c[0][t.trash_sel[n]], idx);
            const Fr compressed = vals[t.words[t.trash_prog[n] + 4]];
            v = fr_add(fr_mul(v, t.y), fr_sub(compressed, fr_mul(fr_sub(one, q), ldfr(t.trash[n], idx))));
        }
        if (t.divide) v = fr_mul(v, t.tinv[idx & (t.tlen - 1)]);
        t.out[idx] = v;
    }
}

Fr fr_from_u64s(const uint64_t* p) {
    Fr r;
    std::memcpy(r.l, p, 32);
    return r;
}


// Appends a flattened program to W after checking every index; returns its
// header offset, or sets `err`.
uint32_t pack_program(std::vector<uint32_t>& W, const mzk_flat_graph& g, const uint32_t n_cols[3],
                      const mzk_quotient_desc* desc, uint32_t log_scale, uint32_t E, std::string& err) {
    if (g.values_len == 0 || g.values_len > kFlatMaxValues) return err = "values_len must be in [1, 256]", 0;
    if (g.n_rotations > kFlatMaxRotations || (g.n_rotations && !g.rotations)) return err = "at most 32 rotations", 0;
    if ((g.n_constants && !g.constants) || (g.n_reads && !g.reads) || (g.n_ops && !g.ops)) return err = "null array", 0;
    const uint32_t slots[6] = {g.beta_idx, g.theta_idx, g.trash_challenge_idx, g.y_idx, g.previous_value_idx,
                               g.result_idx};
    for (uint32_t v : slots)
        if (v >= g.values_len) return err = "slot index past values_len", 0;
    if (g.n_constants > g.values_len) return err = "more constants than values", 0;
    for (uint32_t r = 0; r < g.n_reads; r++) {
        const mzk_column_read& rd = g.reads[r];
        if (rd.col_type > 2 || rd.col_idx >= n_cols[rd.col_type] || rd.rot_idx >= g.n_rotations ||
            rd.dst >= g.values_len)
            return err = "column read " + std::to_string(r) + " out of range", 0;
    }
    for (uint32_t o = 0; o < g.n_ops; o++) {
        const mzk_flat_op& op = g.ops[o];
        const bool uses_b = op.kind == MZK_FLAT_ADD || op.kind == MZK_FLAT_SUB || op.kind == MZK_FLAT_MUL ||
                            op.kind == MZK_FLAT_MULADD;
        if (op.kind > MZK_FLAT_MULADD || op.dst >= g.values_len || op.a >= g.values_len ||
            (uses_b && op.b >= g.values_len) || (op.kind == MZK_FLAT_MULADD && op.c >= g.values_len))
            return err = "op " + std::to_string(o) + " out of range", 0;
    }
    uint32_t static_len = g.n_constants;
    for (int i = 0; i < 4; i++) static_len = std::max(static_len, slots[i] + 1);
    std::vector<Fr> statics(static_len, Fr{});
    for (uint32_t i = 0; i < g.n_constants; i++) statics[i] = fr_from_u64s(g.constants + 4 * i);
    statics[g.beta_idx] = fr_from_u64s(desc->beta);
    statics[g.theta_idx] = fr_from_u64s(desc->theta);
    statics[g.trash_challenge_idx] = fr_from_u64s(desc->trash_challenge);
    statics[g.y_idx] = fr_from_u64s(desc->y);
    const uint32_t h = (uint32_t)W.size();
    W.resize(h + kFlatHeaderWords);
    W[h] = g.n_reads;
    W[h + 1] = g.n_ops;
    W[h + 2] = static_len;
    W[h + 3] = g.previous_value_idx;
    W[h + 4] = g.result_idx;
    W[h + 5] = (uint32_t)W.size();
    for (uint32_t r = 0; r < g.n_reads; r++)
        W.insert(W.end(), {g.reads[r].col_type, g.reads[r].col_idx, g.reads[r].rot_idx, g.reads[r].dst});
    W[h + 6] = (uint32_t)W.size();
    for (uint32_t o = 0; o < g.n_ops; o++)
        W.insert(W.end(), {g.ops[o].kind, g.ops[o].dst, g.ops[o].a, g.ops[o].b, g.ops[o].c});
    W[h + 7] = (uint32_t)W.size();
    for (uint32_t r = 0; r < g.n_rotations; r++)
        W.push_back((uint32_t)(((int64_t)g.rotations[r] << log_scale) & (int64_t)(E - 1)));
    while (W.size() % 4) W.push_back(0);
    W[h + 8] = (uint32_t)W.size();
    const size_t at = W.size();
    W.resize(at + statics.size() * 8);
    std::memcpy(W.data() + at, statics.data(), statics.size() * sizeof(Fr));
    return h;
}

// Checks and packs every program of the descriptor (gates, lookup helpers,
// trashcans) into one device buffer and fills the parameters of the two
// program kernels.
Status pack_programs(Context* ctx, const Domain* d, const mzk_quotient_desc* desc, GatesParams& gp, TailParams& tp,
                     cudaStream_t st) {
    std::string err;
    auto fail = [&](const std::string& m) {
        set_error("quotient programs: " + m);
        return ERR_ARG;
    };
    if (desc->n_instance > kQMaxInstance || (desc->n_instance && !desc->instance))
        return fail("at most 4 instance columns");
    if (desc->n_lookups > kQMaxLookups || (desc->n_lookups && !desc->lookups)) return fail("at most 8 lookups");
    if (desc->n_trash > kQMaxTrash || (desc->n_trash && !desc->trash)) return fail("at most 8 trashcans");
    const uint32_t n_cols[3] = {desc->n_fixed, desc->n_advice, desc->n_instance};
    const uint32_t E = 1u << d->ext_k, log_scale = d->ext_k - d->k;
    FlatCols cols;
    std::memset(&cols, 0, sizeof(cols));
    for (uint32_t i = 0; i < desc->n_fixed; i++) cols.c[0][i] = reinterpret_cast<const Fr*>(desc->fixed[i]);
    for (uint32_t i = 0; i < desc->n_advice; i++) cols.c[1][i] = reinterpret_cast<const Fr*>(desc->advice[i]);
    for (uint32_t i = 0; i < desc->n_instance; i++) cols.c[2][i] = reinterpret_cast<const Fr*>(desc->instance[i]);
    std::vector<uint32_t> W;
    if (desc->gates) {
        gp.prog = pack_program(W, *desc->gates, n_cols, desc, log_scale, E, err);
        if (!err.empty()) return fail("gates: " + err);
    }
    for (uint32_t n = 0; n < desc->n_lookups; n++) {
        const mzk_lookup_arg& L = desc->lookups[n];
        if (L.n_helpers == 0 || L.n_helpers > kQMaxHelpers || !L.programs || !L.outputs || !L.helpers ||
            !L.aggregator || !L.multiplicities)
            return fail("lookup " + std::to_string(n) + ": 1..8 helpers and every column needed");
        tp.agg[n] = reinterpret_cast<const Fr*>(L.aggregator);
        tp.mult[n] = reinterpret_cast<const Fr*>(L.multiplicities);
        tp.n_helpers[n] = L.n_helpers;
        for (uint32_t fi = 0; fi < L.n_helpers; fi++) {
            tp.prog[n][fi] = pack_program(W, L.programs[fi], n_cols, desc, log_scale, E, err);
            if (!err.empty()) return fail("lookup " + std::to_string(n) + " helper " + std::to_string(fi) + ": " + err);
            for (int q = 0; q < 4; q++) {
                if (L.outputs[4 * fi + q] >= L.programs[fi].values_len)
                    return fail("lookup " + std::to_string(n) + ": output index past values_len");
                tp.outputs[n][fi][q] = L.outputs[4 * fi + q];
            }
            tp.helper[n][fi] = reinterpret_cast<const Fr*>(L.helpers[fi]);
        }
    }
    tp.n_lookups = desc->n_lookups;
    for (uint32_t n = 0; n < desc->n_trash; n++) {
        const mzk_trash_arg& T = desc->trash[n];
        if (T.selector_fixed >= desc->n_fixed || !T.trash) return fail("trashcan " + std::to_string(n) + " columns");
        tp.trash_prog[n] = pack_program(W, T.program, n_cols, desc, log_scale, E, err);
        if (!err.empty()) return fail("trashcan " + std::to_string(n) + ": " + err);
        tp.trash_sel[n] = T.selector_fixed;
        tp.trash[n] = reinterpret_cast<const Fr*>(T.trash);
    }
    tp.n_trash = desc->n_trash;
    const size_t bytes = W.size() * 4;
    void *dev, *host;
    MZK_TRY(ctx->ensure("quotient_flat", bytes, &dev));
    MZK_TRY(ctx->ensure_pinned(bytes, &host));
    std::memcpy(host, W.data(), bytes);
    MZK_CUDA_CHECK(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, st));
    // the pinned staging may be reused by the next call: let the copy finish
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    gp.cols = cols;
    tp.cols = cols;
    gp.words = tp.words = static_cast<const uint32_t*>(dev);
    gp.log_n = tp.log_n = d->ext_k;
    tp.log_scale = log_scale;
    return OK;
}

}  // namespace

// One flattened program evaluated at every row of the n-point domain over
// Lagrange columns (rotations are whole rows): the trash argument's
// compressed constraint expressions (trash/prover.rs, `evaluate` over the
// Lagrange values, folded with the trash challenge by the program itself)
// and the lookup input expressions.  extended: at every row of the extended
// coset over coset columns (the lookup input expressions the quotient reads).
Status flat_program_rows(Context* ctx, const Domain* d, const mzk_flat_graph& g, const uint64_t* const* fixed,
                         uint32_t n_fixed, const uint64_t* const* advice, uint32_t n_advice,
                         const uint64_t* const* instance, uint32_t n_instance, const uint64_t beta[4],
                         const uint64_t theta[4], const uint64_t trash[4], const uint64_t y[4], uint64_t* out,
                         cudaStream_t st, bool extended) {
    if (n_fixed > kQMaxFixed || n_advice > kQMaxAdvice || n_instance > kQMaxInstance) {
        set_error("flat program: too many columns");
        return ERR_ARG;
    }
    mzk_quotient_desc desc;  // only the challenge slots are read from it
    std::memset(&desc, 0, sizeof(desc));
    std::memcpy(desc.beta, beta, 32);
    std::memcpy(desc.theta, theta, 32);
    std::memcpy(desc.trash_challenge, trash, 32);
    std::memcpy(desc.y, y, 32);
    const uint32_t n_cols[3] = {n_fixed, n_advice, n_instance};
    const uint32_t log_scale = extended ? d->ext_k - d->k : 0u, n = 1u << (d->k + log_scale);
    std::vector<uint32_t> W;
    std::string err;
    GatesParams gp;
    std::memset(&gp, 0, sizeof(gp));
    gp.prog = pack_program(W, g, n_cols, &desc, log_scale, n, err);
    if (!err.empty()) {
        set_error("flat program: " + err);
        return ERR_ARG;
    }
    for (uint32_t i = 0; i < n_fixed; i++) gp.cols.c[0][i] = reinterpret_cast<const Fr*>(fixed[i]);
    for (uint32_t i = 0; i < n_advice; i++) gp.cols.c[1][i] = reinterpret_cast<const Fr*>(advice[i]);
    for (uint32_t i = 0; i < n_instance; i++) gp.cols.c[2][i] = reinterpret_cast<const Fr*>(instance[i]);
    const size_t bytes = W.size() * 4;
    void *dev, *host;
    MZK_TRY(ctx->ensure("flat_rows", bytes, &dev));
    MZK_TRY(ctx->ensure_pinned(bytes, &host));
    std::memcpy(host, W.data(), bytes);
    MZK_CUDA_CHECK(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, st));
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));  // the pinned staging is reused by the next call
    gp.words = static_cast<const uint32_t*>(dev);
    gp.log_n = d->k + log_scale;
    gp.out = reinterpret_cast<Fr*>(out);
    const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>((n + 127) / 128, (uint32_t)ctx->num_sms * 8));
    k_gates_flat<<<blocks, 128, 0, st>>>(gp);
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

Status quotient_eval_device(Context* ctx, const Domain* d, const mzk_quotient_desc* desc, int divide, void* d_out,
                            cudaStream_t st) {
    if (desc->k != d->k || desc->extended_k != d->ext_k) {
        set_error("quotient: descriptor k / extended_k differ from the domain's");
        return ERR_ARG;
    }
    if (desc->n_advice > kQMaxAdvice || desc->n_fixed > kQMaxFixed || desc->n_perm_cols > kQMaxPermCols ||
        desc->n_perm_sets > kQMaxSets) {
        set_error("quotient: too many columns for the fused kernel");
        return ERR_ARG;
    }
    if (desc->n_perm_sets && (desc->chunk_len == 0 ||
                              (uint64_t)desc->n_perm_sets * desc->chunk_len < desc->n_perm_cols))
    {
        set_error("quotient: permutation sets do not cover the permutation columns");
        return ERR_ARG;
    }
    QuotientParams q;
    std::memset(&q, 0, sizeof(q));
    for (uint32_t i = 0; i < desc->n_advice; i++) q.advice[i] = reinterpret_cast<const Fr*>(desc->advice[i]);
    for (uint32_t i = 0; i < desc->n_fixed; i++) q.fixed[i] = reinterpret_cast<const Fr*>(desc->fixed[i]);
    if (desc->n_instance > kQMaxInstance || (desc->n_instance && !desc->instance)) {
        set_error("quotient: at most 4 instance columns");
        return ERR_ARG;
    }
    for (uint32_t i = 0; i < desc->n_instance; i++) q.instance[i] = reinterpret_cast<const Fr*>(desc->instance[i]);
    const bool tail = desc->n_lookups || desc->n_trash;
    if (tail && desc->has_lookup) {
        set_error("quotient: give either the built-in lookup (has_lookup) or lookup / trash programs");
        return ERR_ARG;
    }
    GatesParams gp;
    TailParams tp;
    std::memset(&gp, 0, sizeof(gp));
    std::memset(&tp, 0, sizeof(tp));
    if (desc->gates || tail) MZK_TRY(pack_programs(ctx, d, desc, gp, tp, st));
    const uint32_t E_rows = 1u << d->ext_k;
    const uint32_t prog_blocks = (uint32_t)std::min<uint64_t>((E_rows + 127) / 128, (uint64_t)ctx->num_sms * 16);
    if (desc->gates) {
        gp.out = static_cast<Fr*>(d_out);
        k_gates_flat<<<prog_blocks, 128, 0, st>>>(gp);
        MZK_LAUNCH_CHECK(ctx);
        q.gate_from_out = 1;
    }
    for (int i = 0; i < 5 && !desc->gates; i++) {
        if (desc->gate_fixed[i] >= desc->n_fixed) {
            set_error("quotient: gate fixed column out of range");
            return ERR_ARG;
        }
        q.gate_fixed[i] = desc->gate_fixed[i];
    }
    for (int i = 0; i < 3 && !desc->gates; i++) {
        if (desc->gate_advice[i] >= desc->n_advice) {
            set_error("quotient: gate advice column out of range");
            return ERR_ARG;
        }
        q.gate_advice[i] = desc->gate_advice[i];
    }
    q.n_perm_cols = desc->n_perm_cols;
    for (uint32_t j = 0; j < desc->n_perm_cols; j++) {
        const uint32_t kind = desc->perm_col_kind[j], idx = desc->perm_col_index[j];
        if (kind > 2 || idx >= (kind == 0 ? desc->n_advice : kind == 1 ? desc->n_fixed : desc->n_instance)) {
            set_error("quotient: permutation column out of range");
            return ERR_ARG;
        }
        q.perm_kind[j] = (uint8_t)kind;
        q.perm_index[j] = (uint8_t)idx;
        q.sigma[j] = reinterpret_cast<const Fr*>(desc->perm_sigma[j]);
    }
    q.n_sets = desc->n_perm_sets;
    for (uint32_t s = 0; s < desc->n_perm_sets; s++) q.z[s] = reinterpret_cast<const Fr*>(desc->perm_z[s]);
    q.chunk_len = desc->chunk_len;
    q.last_rot = -(int32_t)(desc->blinding_factors + 1);
    q.has_lookup = desc->has_lookup ? 1 : 0;
    if (q.has_lookup) {
        if (desc->lookup_input_advice >= desc->n_advice || desc->lookup_table_fixed >= desc->n_fixed ||
            desc->lookup_selector_fixed >= (int32_t)desc->n_fixed) {
            set_error("quotient: lookup column out of range");
            return ERR_ARG;
        }
        q.lookup_input = desc->lookup_input_advice;
        q.lookup_table = desc->lookup_table_fixed;
        q.lookup_selector = desc->lookup_selector_fixed;
        q.lh = reinterpret_cast<const Fr*>(desc->lookup_h);
        q.lz = reinterpret_cast<const Fr*>(desc->lookup_z);
        q.lm = reinterpret_cast<const Fr*>(desc->lookup_m);
    }
    q.l0 = reinterpret_cast<const Fr*>(desc->l0);
    q.l_last = reinterpret_cast<const Fr*>(desc->l_last);
    q.l_active = reinterpret_cast<const Fr*>(desc->l_active);
    q.y = fr_from_u64s(desc->y);
    q.beta = fr_from_u64s(desc->beta);
    q.gamma = fr_from_u64s(desc->gamma);
    q.theta = fr_from_u64s(desc->theta);
    // beta * g_coset computed on the host (domain constants)
    host::Fr4 beta4;
    std::memcpy(beta4.l, desc->beta, 32);
    const host::Fr4 ds = host::fr_mul(beta4, d->zeta);
    std::memcpy(q.delta_start.l, ds.l, 32);
    q.delta = fr_from_u64s(host::FR_DELTA4);
    q.tlo = d->lo[2];
    q.thi = d->hi[2];
    q.tinv = static_cast<const Fr*>(d->d_tinv);
    q.tlen = (uint32_t)d->t_inv.size();
    q.divide = divide ? 1 : 0;
    q.log_n = d->ext_k;
    q.log_scale = d->ext_k - d->k;
    q.out = static_cast<Fr*>(d_out);
    if (tail) q.divide = 0;  // the division comes after the lookup and trash terms
    const uint32_t E = 1u << d->ext_k;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((E + 255) / 256, (uint64_t)ctx->num_sms * 8);
    k_quotient<<<blocks, 256, 0, st>>>(q);
    MZK_LAUNCH_CHECK(ctx);
    if (tail) {
        if (desc->n_lookups && (!desc->l0 || !desc->l_last || !desc->l_active)) {
            set_error("quotient: lookups need l0, l_last and l_active");
            return ERR_ARG;
        }
        tp.l0 = reinterpret_cast<const Fr*>(desc->l0);
        tp.l_last = reinterpret_cast<const Fr*>(desc->l_last);
        tp.l_active = reinterpret_cast<const Fr*>(desc->l_active);
        tp.tinv = static_cast<const Fr*>(d->d_tinv);
        tp.tlen = (uint32_t)d->t_inv.size();
        tp.y = q.y;
        tp.divide = divide ? 1 : 0;
        tp.out = static_cast<Fr*>(d_out);
        k_tail_flat<<<prog_blocks, 128, 0, st>>>(tp);
        MZK_LAUNCH_CHECK(ctx);
    }
    return OK;
}

namespace {

// limb i (length n) = h[i (n-1) .. (i+1)(n-1)) followed by blind[i] (zero for
// the last limb), and limb i's first element minus blind[i-1] for i >= 1
// (blind_quotient_limbs, proofs/src/plonk/prover.rs:774-785)
__global__ void k_split_limbs(const Fr* __restrict__ h, uint32_t n, uint32_t limbs, const Fr* __restrict__ blinds,
                              Fr* __restrict__ out) {
    const uint32_t total = n * limbs;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += stride) {
        const uint32_t i = t / n, j = t % n;
        Fr v;
        if (j < n - 1) v = h[(size_t)i * (n - 1) + j];
        else v = i + 1 < limbs ? blinds[i] : fr_zero();
        if (j == 0 && i > 0) v = fr_sub(v, blinds[i - 1]);
        out[t] = v;
    }
}

}  // namespace

Status compute_h_limbs_device(Context* ctx, const Domain* d, const mzk_quotient_desc* desc, const uint64_t* blinds,
                              void* d_limbs_out, void* d_hbuf, void* d_blinds, cudaStream_t st) {
    const uint32_t n = 1u << d->k, en = 1u << d->ext_k, limbs = d->quotient_poly_degree;
    if (limbs < 2) {
        set_error("compute_h_poly: quotient degree below 2 has no limbs to blind");
        return ERR_ARG;
    }
    if ((uint64_t)(n - 1) * limbs > en) {
        set_error("compute_h_poly: extended domain too small for the quotient degree");
        return ERR_ARG;
    }
    MZK_CUDA_CHECK(cudaMemcpyAsync(d_blinds, blinds, (size_t)(limbs - 1) * sizeof(Fr), cudaMemcpyHostToDevice, st));
    MZK_TRY(quotient_eval_device(ctx, d, desc, 1, d_hbuf, st));
    MZK_TRY(domain_op_device(ctx, d, OP_EXTENDED_TO_COEFF, d_hbuf, d_hbuf, st));
    const uint32_t total = n * limbs;
    k_split_limbs<<<(uint32_t)std::min<uint64_t>((total + 255) / 256, (uint64_t)ctx->num_sms * 8), 256, 0, st>>>(
        static_cast<const Fr*>(d_hbuf), n, limbs, static_cast<const Fr*>(d_blinds), static_cast<Fr*>(d_limbs_out));
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

Status compute_h_poly_device(Context* ctx, const Domain* d, const mzk_quotient_desc* desc, const void* d_srs_g,
                             size_t srs_len, const uint64_t* blinds, uint64_t* commitments, void* d_limbs_out,
                             cudaStream_t st) {
    const uint32_t n = 1u << d->k, en = 1u << d->ext_k, limbs = d->quotient_poly_degree;
    if (srs_len < n) {
        set_error("compute_h_poly: monomial SRS shorter than n");
        return ERR_ARG;
    }
    void *hbuf, *limbs_buf, *dblinds;
    MZK_TRY(ctx->ensure("hpoly_ext", (size_t)en * sizeof(Fr), &hbuf));
    if (d_limbs_out) limbs_buf = d_limbs_out;
    else MZK_TRY(ctx->ensure("hpoly_limbs", (size_t)std::max<uint32_t>(limbs, 1) * n * sizeof(Fr), &limbs_buf));
    MZK_TRY(ctx->ensure("hpoly_blinds", (size_t)std::max<uint32_t>(limbs, 1) * sizeof(Fr), &dblinds));
    MZK_TRY(compute_h_limbs_device(ctx, d, desc, blinds, limbs_buf, hbuf, dblinds, st));
    std::vector<BatchItem> items(limbs);
    for (uint32_t i = 0; i < limbs; i++) {
        items[i].d_scalars = static_cast<const Fr*>(limbs_buf) + (size_t)i * n;
        items[i].base_offset = 0;
        items[i].n = n;
    }
    return msm_g1_batch_device(ctx, d_srs_g, srs_len, items.data(), limbs, commitments, st);
}

}  // namespace mzk
