// prover.cu — the device part of create_proof for the single-proof circuit.
//
// For the circuit shape of the single-proof configuration (three advice
// columns a, b, c under the standard gate, one permutation set over a, b, c,
// one logup lookup of a into a fixed table) this runs every data-parallel step
// of proofs/src/plonk/prover.rs on the GPU, for one or many proofs at once:
//
//   1. witness commitments in the reference's bases (prover.rs:619-623,
//      logup/prover.rs:168, :299, permutation/prover.rs:241): a, b, c and the
//      logup helper h against the Lagrange basis, the multiplicities m and the
//      permutation product z in delta form against the delta basis, the logup
//      aggregator Z in double-delta form against the double-delta basis
//      (Polynomial::to_delta / to_double_delta, proofs/src/poly/mod.rs:297-336);
//   2. lagrange_to_coeff of the seven witness polynomials (prover.rs:231-280);
//   3. coeff_to_extended of the seven (prover.rs:652-659, evaluation.rs:868-960);
//   4. compute_h_poly (prover.rs:701-771): fused quotient, division by t(X),
//      extended_to_coeff, blinded limbs;
//   5. the limb commitments.
// The MSMs of all proofs in a call run as two batched MSMs (step 1 for all
// proofs, step 5 for all proofs), so small proofs share the GPU's chunks; with
// MZK_PROVE_MSM_PER_CALL each MSM is its own call instead (the plain form).
// The permutation product z and the logup helper h and aggregator Z are taken
// from the job or, when it leaves them null, derived on the device first
// (grand.cu).  Witness generation, the lookup multiplicities, the transcript,
// evaluations and the multi-open argument stay with the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mzk.h"
#include "field.cuh"
#include "grand.hpp"
#include "ntt.hpp"
#include "quotient.hpp"
#include "runtime.hpp"

namespace mzk {

namespace {

// order 1: b_0 = a_0, b_i = a_i - a_{i-1}; order 2: c_0 = a_0,
// c_1 = a_1 - 2 a_0, c_i = a_i - 2 a_{i-1} + a_{i-2}
__global__ void k_delta(const Fr* __restrict__ a, Fr* __restrict__ out, uint32_t n, int order) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Fr v = a[i];
        if (i >= 1) {
            const Fr p = a[i - 1];
            v = fr_sub(v, order == 2 ? fr_add(p, p) : p);
        }
        if (order == 2 && i >= 2) v = fr_add(v, a[i - 2]);
        out[i] = v;
    }
}

constexpr int kPolys = 7;  // a, b, c, z, m, h, Z

}  // namespace

Status delta_device(Context* ctx, const void* a, void* out, uint32_t n, int order, cudaStream_t st) {
    const uint32_t grid = (uint32_t)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->num_sms * 8);
    k_delta<<<grid, 256, 0, st>>>(static_cast<const Fr*>(a), static_cast<Fr*>(out), n, order);
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

// the MSMs of `items` against the SRS: one batched MSM, or one call each;
// with a window table (table non-null) the large ones use it either way
Status run_msms(Context* ctx, const void* srs, uint64_t srs_len, const std::vector<BatchItem>& items,
                       uint64_t* res, uint32_t flags, const MsmTable* table, cudaStream_t st) {
    if (!(flags & MZK_PROVE_MSM_PER_CALL))
        return msm_g1_batch_device(ctx, srs, srs_len, items.data(), items.size(), res, st, table);
    for (size_t i = 0; i < items.size(); i++) {
        if (table && items[i].n >= table->min_n) {
            MZK_TRY(msm_g1_batch_device(ctx, srs, srs_len, &items[i], 1, res + i * 18, st, table));
            continue;
        }
        const void* bases = static_cast<const uint8_t*>(srs) + items[i].base_offset * 96;
        MZK_TRY(msm_g1_device(ctx, items[i].d_scalars, bases, items[i].n, res + i * 18, st, nullptr));
    }
    return OK;
}

// One proof's NTT sequence: lagrange_to_coeff then coeff_to_extended of each
// of its `count` polynomials (2-3 pass kernels per transform).  With use_graph
// the sequence is captured once into a CUDA graph per key (the domain, its
// tables, the NTT scratch, the pass splits and the column pointers: all
// that the kernels read) and replayed afterwards; the graph holds the same
// launches with the same arguments, so the results are the same.
Status ntt_sequence(Context* ctx, const Domain* d, const void* const* lag, Fr* const* coeff, Fr* const* ext,
                    int count, bool use_graph, cudaStream_t st) {
    auto eager = [&]() -> Status {
        for (int p = 0; p < count; p++) {
            MZK_TRY(domain_op_device(ctx, d, OP_LAGRANGE_TO_COEFF, lag[p], coeff[p], st));
            MZK_TRY(domain_op_device(ctx, d, OP_COEFF_TO_EXTENDED, coeff[p], ext[p], st));
        }
        return OK;
    };
    if (!use_graph || ctx->profiling || ctx->graphs_unsupported) return eager();
    // the scratch of the largest transform exists before capture: nothing
    // may be allocated while the stream is capturing
    void* tmp;
    MZK_TRY(ctx->ensure("ntt_tmp", ((size_t)1 << d->ext_k) * sizeof(Fr), &tmp));
    std::vector<uintptr_t> key = {(uintptr_t)d, d->k, d->ext_k, (uintptr_t)tmp,
                                  (uintptr_t)ctx->tuned_ntt_split[d->k], (uintptr_t)ctx->tuned_ntt_split[d->ext_k],
                                  (uintptr_t)count};
    for (int r = 0; r < 4; r++) key.push_back((uintptr_t)d->tables[r]);
    for (int p = 0; p < count; p++) {
        key.push_back((uintptr_t)lag[p]);
        key.push_back((uintptr_t)coeff[p]);
        key.push_back((uintptr_t)ext[p]);
    }
    auto& gs = ctx->graphs;
    for (size_t i = 0; i < gs.size();) {  // drop graphs that may hold freed addresses
        if (gs[i].generation != ctx->buf_generation) {
            cudaGraphExecDestroy(gs[i].exec);
            gs.erase(gs.begin() + (ptrdiff_t)i);
        } else {
            i++;
        }
    }
    for (auto& g : gs)
        if (g.key == key) {
            g.last_use = ++ctx->graph_clock;
            MZK_CUDA_CHECK(cudaGraphLaunch(g.exec, st));
            ctx->launches += g.launches;
            ctx->graph_replays++;
            return OK;
        }
    const uint64_t launches0 = ctx->launches, gen0 = ctx->buf_generation;
    MZK_CUDA_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const Status s = eager();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    cudaGraphExec_t exec = nullptr;
    cudaError_t ei = cudaErrorUnknown;
    if (s == OK && e == cudaSuccess && graph && ctx->buf_generation == gen0)
        ei = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {  // not captured: the same launches, issued one by one
        cudaGetLastError();
        ctx->launches = launches0;
        const Status se = eager();
        if (se == OK) ctx->graphs_unsupported = true;  // the capture itself was refused
        return se;
    }
    if (gs.size() >= Context::kMaxGraphs) {  // least recently used out
        size_t lru = 0;
        for (size_t i = 1; i < gs.size(); i++)
            if (gs[i].last_use < gs[lru].last_use) lru = i;
        cudaGraphExecDestroy(gs[lru].exec);
        gs.erase(gs.begin() + (ptrdiff_t)lru);
    }
    gs.push_back({key, exec, ctx->launches - launches0, gen0, ++ctx->graph_clock});
    ctx->graph_captures++;
    MZK_CUDA_CHECK(cudaGraphLaunch(exec, st));
    return OK;
}

Status prove_core_multi(Context* ctx, const Domain* const* doms, const mzk_proving_key_desc* const* pks,
                        const mzk_proof_job* jobs, size_t count, uint64_t* out, uint32_t flags, cudaStream_t st) {
    std::memset(out, 0, count * kProofCoreCommitments * 18 * 8);
    if (count == 0) return OK;
    if (pks[0]->srs == nullptr) {
        set_error("prove_core: null SRS");
        return ERR_ARG;
    }
    const void* srs = pks[0]->srs;
    const uint64_t srs_len = pks[0]->srs_len;
    // a window table over the shared SRS buffer (every key of the call shares it)
    MsmTable table_desc{srs, srs_len, pks[0]->srs_table_c, pks[0]->srs_table_rows, pks[0]->srs_table_min_n};
    const MsmTable* table = pks[0]->srs_table_c > 0 ? &table_desc : nullptr;
    std::vector<BatchItem> items;
    std::vector<Fr*> coeff(count * kPolys), ext(count * kPolys), limbs(count);
    std::vector<const void*> lagrange(count * kPolys);  // a, b, c, z, m, h, Z of every job
    size_t max_en = 0;
    // all per-proof scratch of the call in one buffer, carved in job order, so
    // a call's scratch grows (and is reallocated) only when its total grows
    size_t wave_elems = 0;
    for (size_t j = 0; j < count; j++) {
        const size_t n = (size_t)1 << doms[j]->k, en = (size_t)1 << doms[j]->ext_k;
        // coefficient and extended forms, delta forms, limbs, derived z / h / Z
        wave_elems += kPolys * n + kPolys * en + 3 * n + (size_t)doms[j]->quotient_poly_degree * n + 3 * n;
    }
    void* wave;
    MZK_TRY(ctx->ensure("core_wave", wave_elems * sizeof(Fr), &wave));
    Fr* carve = static_cast<Fr*>(wave);
    for (size_t j = 0; j < count; j++) {
        const Domain* d = doms[j];
        const mzk_proving_key_desc* pk = pks[j];
        const uint32_t n = 1u << d->k, en = 1u << d->ext_k, qdeg = d->quotient_poly_degree;
        const std::string tag = std::to_string(j);
        if (pk->k != d->k || qdeg + 7 != kProofCoreCommitments) {
            set_error("prove_core: job " + tag + ": the key's k must match the domain and the domain must have j = 5");
            return ERR_ARG;
        }
        if (pk->srs != srs || pk->srs_len != srs_len) {
            set_error("prove_core: all keys of one call must share one SRS buffer");
            return ERR_ARG;
        }
        if (pk->off_g + n > srs_len || pk->off_lagrange + n > srs_len || pk->off_lagrange_delta + n > srs_len ||
            pk->off_lagrange_double_delta + n > srs_len) {
            set_error("prove_core: job " + tag + ": SRS bases out of range");
            return ERR_ARG;
        }
        max_en = std::max<size_t>(max_en, en);
        Fr* pc = carve;
        Fr* pe = pc + (size_t)kPolys * n;
        Fr* pd = pe + (size_t)kPolys * en;
        Fr* pl = pd + (size_t)3 * n;
        Fr* pg = pl + (size_t)qdeg * n;  // derived z, h, Z
        carve = pg + (size_t)3 * n;
        for (int p = 0; p < kPolys; p++) {
            coeff[j * kPolys + p] = pc + (size_t)p * n;
            ext[j * kPolys + p] = pe + (size_t)p * en;
        }
        limbs[j] = pl;
        const mzk_proof_job& jb = jobs[j];
        const void** lag = &lagrange[j * kPolys];
        const void* given[kPolys] = {jb.advice[0], jb.advice[1], jb.advice[2], jb.perm_z, jb.lookup_m, jb.lookup_h,
                                     jb.lookup_Z};
        for (int p = 0; p < kPolys; p++) lag[p] = given[p];
        if (pk->blinding_factors > 8 || pk->blinding_factors + 1 >= n) {
            set_error("prove_core: blinding_factors must be at most 8 and below n - 1");
            return ERR_ARG;
        }
        if ((jb.lookup_h == nullptr) != (jb.lookup_Z == nullptr)) {
            set_error("prove_core: job " + tag + ": give both or neither of lookup_h and lookup_Z");
            return ERR_ARG;
        }
        if (!jb.advice[0] || !jb.advice[1] || !jb.advice[2] || !jb.lookup_m) {
            set_error("prove_core: null witness polynomial in job " + tag);
            return ERR_ARG;
        }
        if (!jb.lookup_h) {  // logup helper and aggregator on the device
            if (!pk->table_lagrange || !pk->selector_lagrange) {
                set_error("prove_core: deriving h and Z needs the key's table and selector in Lagrange form");
                return ERR_ARG;
            }
            uint64_t* hz[1] = {reinterpret_cast<uint64_t*>(pg + n)};
            const uint64_t* in[1] = {static_cast<const uint64_t*>(jb.advice[0])};
            const uint32_t cols[1] = {1};
            mzk_logup_desc ld;
            std::memset(&ld, 0, sizeof(ld));
            ld.n_chunks = 1;
            ld.chunk_cols = cols;
            ld.inputs = in;
            ld.table = pk->table_lagrange;
            ld.selector = pk->selector_lagrange;
            ld.multiplicities = jb.lookup_m;
            ld.blinding_factors = pk->blinding_factors;
            ld.blinds = &jb.lookup_blinds[0][0];
            std::memcpy(ld.beta, jb.beta, 32);
            ld.helpers_out = hz;
            ld.aggregator_out = reinterpret_cast<uint64_t*>(pg + 2 * (size_t)n);
            MZK_TRY(logup_device(ctx, d, &ld, st));
            lag[5] = pg + n;
            lag[6] = pg + 2 * (size_t)n;
        }
        if (!jb.perm_z) {  // permutation product on the device
            if (!pk->sigma_lagrange[0] || !pk->sigma_lagrange[1] || !pk->sigma_lagrange[2]) {
                set_error("prove_core: deriving z needs the key's permutation polynomials in Lagrange form");
                return ERR_ARG;
            }
            uint64_t* zo[1] = {reinterpret_cast<uint64_t*>(pg)};
            mzk_permutation_desc pd_;
            std::memset(&pd_, 0, sizeof(pd_));
            pd_.n_cols = 3;
            pd_.values = reinterpret_cast<const uint64_t* const*>(jb.advice);
            pd_.sigmas = pk->sigma_lagrange;
            pd_.chunk_len = 3;  // cs.degree() - 2 with degree 5
            pd_.blinding_factors = pk->blinding_factors;
            pd_.blinds = &jb.perm_blinds[0][0];
            std::memcpy(pd_.beta, jb.beta, 32);
            std::memcpy(pd_.gamma, jb.gamma, 32);
            pd_.z_out = zo;
            MZK_TRY(permutation_z_device(ctx, d, &pd_, st));
            lag[3] = pg;
        }
        const uint32_t grid = (uint32_t)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->num_sms * 8);
        Fr* dm = pd;
        Fr* dz = dm + n;
        Fr* dZ = dz + n;
        k_delta<<<grid, 256, 0, st>>>(reinterpret_cast<const Fr*>(lag[4]), dm, n, 1);
        MZK_LAUNCH_CHECK(ctx);
        k_delta<<<grid, 256, 0, st>>>(reinterpret_cast<const Fr*>(lag[3]), dz, n, 1);
        MZK_LAUNCH_CHECK(ctx);
        k_delta<<<grid, 256, 0, st>>>(reinterpret_cast<const Fr*>(lag[6]), dZ, n, 2);
        MZK_LAUNCH_CHECK(ctx);
        const BatchItem its[7] = {{jb.advice[0], pk->off_lagrange, n},  {jb.advice[1], pk->off_lagrange, n},
                                  {jb.advice[2], pk->off_lagrange, n},  {dm, pk->off_lagrange_delta, n},
                                  {dz, pk->off_lagrange_delta, n},      {dZ, pk->off_lagrange_double_delta, n},
                                  {lag[5], pk->off_lagrange, n}};
        items.insert(items.end(), its, its + 7);
    }
    // 1. witness commitments of every proof in one batch
    std::vector<uint64_t> res1(items.size() * 18);
    MZK_TRY(run_msms(ctx, srs, srs_len, items, res1.data(), flags, table, st));
    for (size_t j = 0; j < count; j++)
        std::memcpy(out + (j * kProofCoreCommitments) * 18, res1.data() + j * 7 * 18, 7 * 18 * 8);
    // 2-4. per proof: coefficient and extended forms, quotient limbs
    void *hbuf, *dbl;
    MZK_TRY(ctx->ensure("core_hbuf", max_en * sizeof(Fr), &hbuf));
    MZK_TRY(ctx->ensure("core_blinds", 8 * sizeof(Fr), &dbl));
    for (size_t j = 0; j < count; j++) {
        const Domain* d = doms[j];
        const mzk_proving_key_desc* pk = pks[j];
        const mzk_proof_job& jb = jobs[j];
        const void* const* lag = &lagrange[j * kPolys];
        MZK_TRY(ntt_sequence(ctx, d, lag, &coeff[j * kPolys], &ext[j * kPolys], kPolys, !(flags & MZK_PROVE_NO_GRAPHS),
                             st));
        Fr* const* e = &ext[j * kPolys];
        const uint64_t* adv[3] = {(const uint64_t*)e[0], (const uint64_t*)e[1], (const uint64_t*)e[2]};
        const uint64_t* sig[3] = {pk->sigma_ext[0], pk->sigma_ext[1], pk->sigma_ext[2]};
        const uint64_t* zs[1] = {(const uint64_t*)e[3]};
        const uint32_t kinds[3] = {0, 0, 0}, idxs[3] = {0, 1, 2};
        mzk_quotient_desc q;
        std::memset(&q, 0, sizeof(q));
        q.k = d->k;
        q.extended_k = d->ext_k;
        q.advice = adv;
        q.n_advice = 3;
        q.fixed = pk->fixed_ext;
        q.n_fixed = 7;
        for (int i = 0; i < 5; i++) q.gate_fixed[i] = (uint32_t)i;
        for (int i = 0; i < 3; i++) q.gate_advice[i] = (uint32_t)i;
        q.n_perm_cols = 3;
        q.perm_col_kind = kinds;
        q.perm_col_index = idxs;
        q.perm_sigma = sig;
        q.n_perm_sets = 1;
        q.perm_z = zs;
        q.chunk_len = 3;  // cs.degree() - 2 with degree 5
        q.blinding_factors = pk->blinding_factors;
        q.has_lookup = 1;
        q.lookup_input_advice = 0;
        q.lookup_table_fixed = 5;
        q.lookup_selector_fixed = 6;
        q.lookup_m = (const uint64_t*)e[4];
        q.lookup_h = (const uint64_t*)e[5];
        q.lookup_z = (const uint64_t*)e[6];
        q.l0 = pk->l0_ext;
        q.l_last = pk->l_last_ext;
        q.l_active = pk->l_active_ext;
        std::memcpy(q.y, jb.y, 32);
        std::memcpy(q.beta, jb.beta, 32);
        std::memcpy(q.gamma, jb.gamma, 32);
        std::memcpy(q.theta, jb.theta, 32);
        MZK_TRY(compute_h_limbs_device(ctx, d, &q, &jb.quotient_blinds[0][0], limbs[j], hbuf, dbl, st));
    }
    // 5. limb commitments of every proof in one batch
    items.clear();
    for (size_t j = 0; j < count; j++) {
        const uint32_t n = 1u << doms[j]->k;
        for (uint32_t i = 0; i < doms[j]->quotient_poly_degree; i++)
            items.push_back({limbs[j] + (size_t)i * n, pks[j]->off_g, n});
    }
    std::vector<uint64_t> res2(items.size() * 18);
    MZK_TRY(run_msms(ctx, srs, srs_len, items, res2.data(), flags, table, st));
    for (size_t j = 0; j < count; j++)
        std::memcpy(out + (j * kProofCoreCommitments + 7) * 18, res2.data() + j * 4 * 18, 4 * 18 * 8);
    return OK;
}

Status prove_core_device(Context* ctx, const Domain* d, const mzk_proving_key_desc* pk, const mzk_proof_job* jobs,
                         size_t count, uint64_t* out, uint32_t flags, cudaStream_t st) {
    std::vector<const Domain*> doms(count, d);
    std::vector<const mzk_proving_key_desc*> pks(count, pk);
    return prove_core_multi(ctx, doms.data(), pks.data(), jobs, count, out, flags, st);
}

}  // namespace mzk
