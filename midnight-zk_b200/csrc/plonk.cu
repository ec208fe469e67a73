// plonk.cu — keygen and create_proof with the Fiat-Shamir transcript.
//
// keygen (proofs/src/plonk/keygen.rs:227-404, permutation/keygen.rs:138-287)
// builds a device-resident proving key: the fixed columns in Lagrange,
// coefficient and extended-coset form, the permutation polynomials from the
// caller's copy mapping in the same three forms, l0 / l_last / l_active_row,
// the VK commitments and the VK's transcript_repr, the lookup table index of
// the multiplicity kernels, and the point-set layout of the multi-open
// argument (which polynomial is opened at which rotations of x).
//
// create_proof (proofs/src/plonk/prover.rs:66-473) runs in the reference's
// Fiat-Shamir order, each phase for every proof of the call before the next,
// so the MSMs of a phase form one batched MSM over the shared SRS:
//   1. advice commitments (Lagrange basis), then theta;
//   2. lookup multiplicities m (logup/prover.rs:95-184, 412-477) committed in
//      delta form, then beta and gamma;
//   3. permutation products z (permutation/prover.rs:81-255, delta form),
//      logup helper h (Lagrange) and aggregator Z (double delta), then the
//      trash challenge and y;
//   4. lagrange_to_coeff / coeff_to_extended of every witness polynomial,
//      the fused quotient, extended_to_coeff and the blinded limbs
//      (compute_h_poly, prover.rs:701-785), the limb commitments, then x;
//   5. the evaluations at x and its rotations (prover.rs:798-868,
//      permutation/prover.rs:270-335, logup/prover.rs:318-352) and the
//      linearization polynomial (linearization/prover.rs:41-86);
//   6-8. multi_open (kzg/mod.rs:110-289): x1, x2, the q polynomials of each
//      point set, f = sum x2^s q_s / prod (X - p), its commitment, x3, the q
//      evaluations at x3, x4, the final polynomial and pi.
// The transcript, the identities at x and the point-set bookkeeping run on
// the host (transcript.hpp); everything proportional to n runs on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/mzk.h"
#include "field.cuh"
#include "grand.hpp"
#include "ntt.hpp"
#include "quotient.hpp"
#include "runtime.hpp"
#include "srs.hpp"
#include "transcript.hpp"

namespace mzk {

Context* context_of(mzk_ctx* ctx);
const Domain* domain_of(mzk_domain* d);

using host::Fr4;

namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kMaxProofLookups = kQMaxLookups;  // lookups of one circuit in create_proof
constexpr uint32_t kMaxProofTrash = kQMaxTrash;      // trashcans of one circuit in create_proof

inline Fr to_dev(const Fr4& a) {
    Fr r;
    std::memcpy(r.l, a.l, 32);
    return r;
}

uint32_t grid_of(const Context* ctx, uint64_t n) {
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((n + kThreads - 1) / kThreads, (uint64_t)ctx->num_sms * 8));
}

// ------------------------------------------------------------- kernels ----
// out[c n + r] = delta^c' omega^r' for (c', r') = mapping of cell (c, r)
// (identity when mapping is null); omega^e = lo[e & 4095] hi[e >> 12]
__global__ void k_perm_values(Fr* __restrict__ out, const uint32_t* __restrict__ mapping, const Fr* __restrict__ deltas,
                              const Fr* __restrict__ wlo, const Fr* __restrict__ whi, uint32_t n, uint32_t cols) {
    const uint64_t total = (uint64_t)n * cols, stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        uint32_t mc = (uint32_t)(i / n), mr = (uint32_t)(i % n);
        if (mapping) {
            mc = mapping[2 * i];
            mr = mapping[2 * i + 1];
        }
        Fr w = wlo[mr & 4095u];
        if (mr >> 12) w = fr_mul(whi[mr >> 12], w);
        out[i] = fr_mul(deltas[mc], w);
    }
}

// out[i] = one for lo <= i < hi, else zero
__global__ void k_unit(Fr* __restrict__ out, uint64_t n, uint64_t lo, uint64_t hi) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = (i >= lo && i < hi) ? fr_one() : fr_zero();
}

// l_active_row = 1 - (l_last + l_blind) (keygen.rs:393-401)
__global__ void k_active(Fr* __restrict__ out, const Fr* __restrict__ l_last, const Fr* __restrict__ l_blind,
                         uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = fr_sub(fr_one(), fr_add(l_last[i], l_blind[i]));
}

__device__ __forceinline__ bool fr_is_zero_dev(const Fr& a) {
    uint32_t acc = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) acc |= a.l[j];
    return acc == 0;
}

// -1, 0, 1 as a < b, a == b, a > b in the order of the table index (the
// four 64-bit words compared from the lowest)
__device__ __forceinline__ int cmp_words(const Fr& a, const Fr& b) {
#pragma unroll
    for (int w = 0; w < 4; w++) {
        const uint64_t x = (uint64_t)a.l[2 * w + 1] << 32 | a.l[2 * w];
        const uint64_t y = (uint64_t)b.l[2 * w + 1] << 32 | b.l[2 * w];
        if (x != y) return x < y ? -1 : 1;
    }
    return 0;
}

// compute_multiplicities, counting half (logup/prover.rs:432-445): every
// selected input row of the usable rows adds one to its table value's count;
// a value not in the table sets *missing (the reference panics)
// A lookup's input columns (a tuple of up to four, compared element by
// element against the tuples of the table index)
struct LookupInputs {
    const Fr* col[4];
    uint32_t width;
};
__device__ __forceinline__ int cmp_tuple(const Fr* __restrict__ uniq, uint32_t t, const LookupInputs& in, uint32_t i) {
    for (uint32_t e = 0; e < in.width; e++)
        if (const int c = cmp_words(uniq[(size_t)t * in.width + e], in.col[e][i])) return c;
    return 0;
}
// (with a tuple, the reference matches the theta-compressed values; the
// tuples match exactly when those do, up to a collision of probability
// ~n^2 / r)
__global__ void k_lookup_count(LookupInputs in, const Fr* __restrict__ selector, uint32_t usable,
                               const Fr* __restrict__ uniq, uint32_t n_uniq, uint32_t* __restrict__ counts,
                               uint32_t* __restrict__ missing) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < usable; i += stride) {
        if (selector && fr_is_zero_dev(selector[i])) continue;
        uint32_t lo = 0, hi = n_uniq;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (cmp_tuple(uniq, mid, in, i) < 0) lo = mid + 1;
            else hi = mid;
        }
        if (lo < n_uniq && cmp_tuple(uniq, lo, in, i) == 0) atomicAdd(&counts[lo], 1u);
        else atomicOr(missing, 1u);
    }
}

// compute_multiplicities, normalising half (:447-476): m_i = count(t_i) /
// (copies of t_i in the table) on the usable rows
__global__ void k_lookup_m(Fr* __restrict__ m, const uint32_t* __restrict__ uid, const uint32_t* __restrict__ counts,
                           const Fr* __restrict__ tinv, uint32_t usable) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < usable; i += stride) {
        const uint32_t u = uid[i];
        Fr c = fr_zero();
        c.l[0] = counts[u];
        m[i] = fr_mul(fr_to_mont(c), tinv[u]);
    }
}

// Batched polynomial evaluation.  A block sums 2048 coefficients of one
// task: each thread runs Horner over 8 consecutive coefficients, then the
// block combines its threads' values pairwise with the powers point^(8 2^l)
// (a tree of 8 levels).  Segment sums land in seg_out; a later level
// evaluates them as a polynomial in point^2048.
struct EvalTask {
    const Fr* poly;
    uint64_t len;
    Fr* seg_out;
    Fr pw[9];  // point, point^8, point^16, ..., point^1024
};
constexpr uint32_t kEvalSeg = 2048;

__global__ void __launch_bounds__(kThreads) k_eval_segments(const EvalTask* __restrict__ tasks) {
    __shared__ Fr part[kThreads];
    const EvalTask& t = tasks[blockIdx.y];
    const uint64_t base = (uint64_t)blockIdx.x * kEvalSeg;
    if (base >= t.len) return;  // uniform across the block
    const uint32_t tid = threadIdx.x;
    const Fr x = t.pw[0];
    Fr acc = fr_zero();
    for (int j = 7; j >= 0; j--) {
        const uint64_t idx = base + 8ull * tid + (uint64_t)j;
        acc = fr_mul(acc, x);
        if (idx < t.len) acc = fr_add(acc, t.poly[idx]);
    }
    part[tid] = acc;
    __syncthreads();
    for (int l = 0; l < 8; l++) {
        const uint32_t s = 1u << l;
        if ((tid & (2 * s - 1)) == 0) part[tid] = fr_add(part[tid], fr_mul(part[tid + s], t.pw[1 + l]));
        __syncthreads();
    }
    if (tid == 0) t.seg_out[blockIdx.x] = part[0];
}

// Batched linear combinations: out_o[i] = sum_t s_t p_t[i] (i < len_t), zero
// past a term's length (poly_inner_product, kzg/mod.rs:125-147)
struct LinTerm {
    const Fr* p;
    uint64_t len;
    Fr s;
};
struct LinOut {
    Fr* out;
    uint64_t len;
    uint32_t t0, nt;
};
__global__ void k_lincomb(const LinOut* __restrict__ outs, const LinTerm* __restrict__ terms) {
    const LinOut o = outs[blockIdx.y];
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < o.len; i += stride) {
        Fr acc = fr_zero();
        for (uint32_t t = o.t0; t < o.t0 + o.nt; t++)
            if (i < terms[t].len) acc = fr_add(acc, fr_mul(terms[t].p[i], terms[t].s));
        o.out[i] = acc;
    }
}

// ------------------------------------------------------- host scalar math --
Fr4 fr_rot(const Domain* d, const Fr4& x, int32_t rot) {
    return rot >= 0 ? host::fr_mul(x, host::fr_pow_u64(d->omega, (uint64_t)rot))
                    : host::fr_mul(x, host::fr_pow_u64(d->omega_inv, (uint64_t)(-(int64_t)rot)));
}

// EvaluationDomain::l_i_range (domain.rs:487-512) at one rotation
Fr4 l_i(const Domain* d, const Fr4& x, const Fr4& xn, int32_t i) {
    const Fr4 wi = fr_rot(d, host::fr_one(), i);
    const Fr4 num = host::fr_mul(host::fr_mul(wi, host::fr_sub(xn, host::fr_one())), d->ifft_div);
    return host::fr_mul(num, host::fr_inv(host::fr_sub(x, wi)));
}

}  // namespace

// ------------------------------------------------------------- the key ----
struct PlonkKey {
    const Domain* dom = nullptr;
    uint32_t k = 0, n = 0, u = 0, bf = 0, degree = 0, qdeg = 0, chunk = 0, n_sets = 0;
    uint32_t n_advice = 0, n_fixed = 0, n_perm = 0, n_instance = 0;
    std::vector<mzk_query> advice_queries, fixed_queries, instance_queries;
    uint32_t gate_fixed[5] = {}, gate_advice[3] = {};
    // custom gates as a flattened program (a validated copy), or the standard gate
    bool has_gates = false;
    std::vector<uint64_t> g_consts;
    std::vector<int32_t> g_rots;
    std::vector<mzk_column_read> g_reads;
    std::vector<mzk_flat_op> g_ops;
    mzk_flat_graph gates = {};
    std::vector<uint32_t> perm_kind, perm_index;
    // lookups, each one advice column into one fixed table column, with the
    // table index of the multiplicity kernels (device)
    struct Lookup {
        mzk_lookup_shape shape = {};
        uint32_t width = 1;                  // the input and table tuples' length
        uint32_t n_inputs = 1;               // parallel input tuples
        uint32_t in[8][4] = {}, tab[4] = {}; // advice input tuples and fixed table columns
        int32_t expr[8][4];                  // input element's program in lk_exprs, or -1: the column in[][]
        uint32_t per_helper = 1;             // inputs per helper chunk (the last may hold fewer)
        uint32_t h0 = 0;                     // the first helper's index among all lookups' helpers
        uint32_t n_helpers() const { return (n_inputs + per_helper - 1) / per_helper; }
        uint32_t chunk_inputs(uint32_t c) const { return std::min(per_helper, n_inputs - c * per_helper); }
        uint32_t n_uniq = 0;
        Fr* uniq = nullptr;       // distinct table tuples of the usable rows, in the index order (width each)
        uint32_t* uid = nullptr;  // per usable row: its value's index in uniq
        Fr* tinv = nullptr;       // per distinct value: 1 / (its copies in the table)
    };
    std::vector<Lookup> lookups;
    uint32_t n_helpers = 0;  // helper polynomials of all lookups
    // a validated copy of a flattened program
    struct Program {
        std::vector<uint64_t> consts;
        std::vector<int32_t> rots;
        std::vector<mzk_column_read> reads;
        std::vector<mzk_flat_op> ops;
        mzk_flat_graph g = {};
        void assign(const mzk_flat_graph& src) {
            consts.assign(src.constants, src.constants + 4 * (size_t)src.n_constants);
            rots.assign(src.rotations, src.rotations + src.n_rotations);
            reads.assign(src.reads, src.reads + src.n_reads);
            ops.assign(src.ops, src.ops + src.n_ops);
            g = src;
            g.constants = consts.data();
            g.rotations = rots.data();
            g.reads = reads.data();
            g.ops = ops.data();
        }
    };
    // lookup input expressions that are not plain advice columns; the proof
    // evaluates each over the Lagrange rows (multiplicities, helpers) and over
    // the extended coset, where the lookup programs read it as advice column
    // n_advice + its index
    std::vector<Program> lk_exprs;
    // with more than one lookup the quotient takes them as helper programs
    // (one per helper chunk, indexed like the helpers; the single one-column
    // lookup uses the fused built-in term)
    std::vector<uint64_t> lk_consts;
    std::vector<int32_t> lk_rots;
    std::vector<mzk_column_read> lk_reads;
    std::vector<mzk_flat_op> lk_ops;
    std::vector<mzk_flat_graph> lk_programs;
    std::vector<uint32_t> lk_outputs;
    // trashcans (trash/prover.rs): a validated copy of each program and its selector
    struct Trash {
        std::vector<uint64_t> consts;
        std::vector<int32_t> rots;
        std::vector<mzk_column_read> reads;
        std::vector<mzk_flat_op> ops;
        mzk_flat_graph program = {};
        uint32_t selector = 0;
    };
    std::vector<Trash> trash;
    // simple selectors: the gates program's slot of each gate polynomial, its
    // selector's fixed column (-1: none), and which fixed columns are simple
    std::vector<uint32_t> gate_poly_values;
    std::vector<int32_t> gate_poly_selector;
    std::vector<uint8_t> simple_col;
    bool is_simple(uint32_t fixed_col) const { return fixed_col < simple_col.size() && simple_col[fixed_col]; }
    // device
    void* mem = nullptr;
    std::vector<Fr*> fixed_lag, fixed_coeff, fixed_ext, perm_lag, perm_coeff, perm_ext;
    Fr *l0 = nullptr, *l_last = nullptr, *l_active = nullptr, *ones = nullptr;
    mzk_srs_desc srs = {};
    // verifying key
    std::vector<std::array<uint64_t, 18>> fixed_coms, perm_coms;
    Fr4 repr = {};
    // multi-open layout: polynomials (kind, index) and point sets sorted by
    // (size, first appearance), each with its polynomials and rotations
    enum PolyKind { P_ADVICE = 0, P_PERM_Z, P_M, P_H, P_AGG, P_FIXED, P_PERM_FIXED, P_LIN, P_TRASH };
    struct OpenSet {
        std::vector<std::pair<int, uint32_t>> polys;
        std::vector<int32_t> rots;
    };
    std::vector<OpenSet> open_sets;
    size_t proof_len = 0, n_blinds = 0;
    int32_t last_rot() const { return -(int32_t)(bf + 1); }
    ~PlonkKey() {
        if (mem) cudaFree(mem);
    }
};

namespace {

// a program that only reads one advice column at rotation 0 into its result:
// that column (else -1)
int plain_advice(const mzk_flat_graph& g) {
    if (g.n_ops || g.n_reads != 1) return -1;
    const mzk_column_read& r = g.reads[0];
    if (r.col_type != 1 || g.rotations[r.rot_idx] != 0 || r.dst != g.result_idx) return -1;
    return (int)r.col_idx;
}

// Expression::degree (circuit.rs:1074-1086) of a program's result: a column
// read has degree 1, a constant or challenge slot 0, a product the sum of
// its factors' degrees, a sum the larger one
uint32_t program_degree(const mzk_flat_graph& g) {
    std::vector<uint32_t> deg(g.values_len, 0);
    for (uint32_t i = 0; i < g.n_reads; i++) deg[g.reads[i].dst] = 1;
    for (uint32_t i = 0; i < g.n_ops; i++) {
        const mzk_flat_op& o = g.ops[i];
        switch (o.kind) {
            case MZK_FLAT_MUL: deg[o.dst] = deg[o.a] + deg[o.b]; break;
            case MZK_FLAT_SQUARE: deg[o.dst] = 2 * deg[o.a]; break;
            case MZK_FLAT_DOUBLE:
            case MZK_FLAT_NEGATE: deg[o.dst] = deg[o.a]; break;
            case MZK_FLAT_MULADD: deg[o.dst] = std::max(deg[o.a] + deg[o.b], deg[o.c]); break;
            default: deg[o.dst] = std::max(deg[o.a], deg[o.b]); break;  // add, sub
        }
    }
    return deg[g.result_idx];
}

// parallel lookup inputs per helper polynomial (nb_parallel_lookups_per_chunk,
// logup.rs:168-183): next_pow2(cs.degree() - 1) / the inputs' largest degree
uint32_t lookup_per_helper(uint32_t degree, uint32_t input_degree) {
    uint32_t p = 1;
    while (p < degree - 1) p <<= 1;
    return p / std::max(1u, input_degree);
}

// the largest degree of lookup l's input expressions (1 for columns)
uint32_t lookup_input_degree(const mzk_circuit_desc* cs, uint32_t l) {
    if (!cs->lookup_input_programs) return 1;
    uint32_t at = 0;
    for (uint32_t i = 0; i < l; i++) at += cs->lookup_tuples ? cs->lookup_tuples[i].n_inputs * cs->lookup_tuples[i].width : 1;
    const uint32_t m = cs->lookup_tuples ? cs->lookup_tuples[l].n_inputs * cs->lookup_tuples[l].width : 1;
    uint32_t d = 0;
    for (uint32_t e = 0; e < m; e++) d = std::max(d, program_degree(cs->lookup_input_programs[at + e]));
    return d;
}

Status check_circuit(const Domain* d, const mzk_circuit_desc* cs) {
    auto fail = [](const std::string& m) {
        set_error("keygen: " + m);
        return ERR_ARG;
    };
    if (cs->degree < 3 || cs->degree > 9) return fail("degree must be in 3..9");
    if (d->quotient_poly_degree != cs->degree - 1) return fail("the domain must be created with j = degree");
    const uint64_t n = 1ull << d->k;
    if ((uint64_t)cs->blinding_factors + 2 >= n) return fail("blinding_factors too large for the domain");
    if (cs->n_advice == 0 || cs->n_advice > kQMaxAdvice || cs->n_fixed > kQMaxFixed)
        return fail("1..16 advice and at most 16 fixed columns");
    if (cs->n_perm_cols > kQMaxPermCols || (cs->n_perm_cols + cs->degree - 3) / (cs->degree - 2) > kQMaxSets)
        return fail("at most 16 permutation columns in at most 8 sets");
    if (cs->n_lookups > kMaxProofLookups) return fail("at most 8 lookups");
    if ((cs->n_advice_queries && !cs->advice_queries) || (cs->n_fixed_queries && !cs->fixed_queries) ||
        (cs->n_instance_queries && !cs->instance_queries))
        return fail("null query list");
    if (cs->n_instance > kQMaxInstance) return fail("at most 4 instance columns");
    if ((cs->n_perm_cols && (!cs->perm_col_kind || !cs->perm_col_index)) || (cs->n_lookups && !cs->lookups))
        return fail("null column list");
    auto queried = [&](const mzk_query* q, uint32_t nq, uint32_t col) {
        for (uint32_t i = 0; i < nq; i++)
            if (q[i].column == col && q[i].rotation == 0) return true;
        return false;
    };
    for (uint32_t i = 0; i < cs->n_advice_queries; i++) {
        const mzk_query q = cs->advice_queries[i];
        if (q.column >= cs->n_advice) return fail("advice query column out of range");
        if (q.rotation <= -(int32_t)n || q.rotation >= (int32_t)n) return fail("rotation out of range");
        for (uint32_t j = 0; j < i; j++)
            if (cs->advice_queries[j].column == q.column && cs->advice_queries[j].rotation == q.rotation)
                return fail("duplicated advice query");
    }
    for (uint32_t i = 0; i < cs->n_fixed_queries; i++) {
        const mzk_query q = cs->fixed_queries[i];
        if (q.column >= cs->n_fixed) return fail("fixed query column out of range");
        if (q.rotation <= -(int32_t)n || q.rotation >= (int32_t)n) return fail("rotation out of range");
        for (uint32_t j = 0; j < i; j++)
            if (cs->fixed_queries[j].column == q.column && cs->fixed_queries[j].rotation == q.rotation)
                return fail("duplicated fixed query");
    }
    for (uint32_t i = 0; i < cs->n_instance_queries; i++) {
        const mzk_query q = cs->instance_queries[i];
        if (q.column >= cs->n_instance) return fail("instance query column out of range");
        if (q.rotation <= -(int32_t)n || q.rotation >= (int32_t)n) return fail("rotation out of range");
        for (uint32_t j = 0; j < i; j++)
            if (cs->instance_queries[j].column == q.column && cs->instance_queries[j].rotation == q.rotation)
                return fail("duplicated instance query");
    }
    // every index the host evaluation of a program at x uses is checked here;
    // the quotient checks the program again when it packs it
    auto check_program = [&](const mzk_flat_graph* g, const std::string& what) -> Status {
        const uint32_t V = g->values_len;
        if (V == 0 || V > kFlatMaxValues || g->n_constants > V || g->n_rotations > kFlatMaxRotations)
            return fail(what + ": bad values_len, constant count or rotation count");
        if ((g->n_constants && !g->constants) || (g->n_rotations && !g->rotations) || (g->n_reads && !g->reads) ||
            (g->n_ops && !g->ops))
            return fail(what + ": null array");
        for (uint32_t idx : {g->beta_idx, g->theta_idx, g->trash_challenge_idx, g->y_idx, g->previous_value_idx,
                             g->result_idx})
            if (idx >= V) return fail(what + ": slot index out of range");
        for (uint32_t i = 0; i < g->n_reads; i++) {
            const mzk_column_read& r = g->reads[i];
            if (r.dst >= V || r.rot_idx >= g->n_rotations) return fail(what + ": read index out of range");
            const int32_t rot = g->rotations[r.rot_idx];
            bool ok = false;
            if (r.col_type <= 2) {
                const mzk_query* q = r.col_type == 0   ? cs->fixed_queries
                                     : r.col_type == 1 ? cs->advice_queries
                                                       : cs->instance_queries;
                const uint32_t nq = r.col_type == 0   ? cs->n_fixed_queries
                                    : r.col_type == 1 ? cs->n_advice_queries
                                                      : cs->n_instance_queries;
                for (uint32_t j = 0; j < nq; j++) ok = ok || (q[j].column == r.col_idx && q[j].rotation == rot);
            }
            if (!ok) return fail(what + ": a read is not a fixed, advice or instance query of the circuit");
        }
        for (uint32_t i = 0; i < g->n_ops; i++) {
            const mzk_flat_op& o = g->ops[i];
            if (o.kind > MZK_FLAT_MULADD || o.dst >= V || o.a >= V || o.b >= V || o.c >= V)
                return fail(what + ": op out of range");
        }
        return OK;
    };
    if (cs->n_trash > kMaxProofTrash || (cs->n_trash && !cs->trash)) return fail("at most 8 trashcans");
    for (uint32_t t = 0; t < cs->n_trash; t++) {
        MZK_TRY(check_program(&cs->trash[t].program, "trashcan " + std::to_string(t)));
        if (!queried(cs->fixed_queries, cs->n_fixed_queries, cs->trash[t].selector_fixed))
            return fail("a trashcan selector is not a fixed column queried at rotation 0");
    }
    if (cs->n_gate_polys) {
        if (!cs->gates || !cs->gate_poly_values || !cs->gate_poly_selector)
            return fail("gate polynomials need the gates program and both arrays");
        for (uint32_t i = 0; i < cs->n_gate_polys; i++) {
            if (cs->gate_poly_values[i] >= cs->gates->values_len) return fail("gate polynomial slot out of range");
            const int32_t sel = cs->gate_poly_selector[i];
            if (sel >= 0 && !queried(cs->fixed_queries, cs->n_fixed_queries, (uint32_t)sel))
                return fail("a simple selector is not a fixed column queried at rotation 0");
        }
    }
    if (const mzk_flat_graph* g = cs->gates) {
        MZK_TRY(check_program(g, "gates"));
    } else {
        for (int i = 0; i < 5; i++)
            if (!queried(cs->fixed_queries, cs->n_fixed_queries, cs->gate_fixed[i]))
                return fail("a gate fixed column is not queried at rotation 0");
        for (int i = 0; i < 3; i++)
            if (!queried(cs->advice_queries, cs->n_advice_queries, cs->gate_advice[i]))
                return fail("a gate advice column is not queried at rotation 0");
    }
    for (uint32_t i = 0; i < cs->n_perm_cols; i++) {
        const uint32_t kind = cs->perm_col_kind[i], col = cs->perm_col_index[i];
        if (kind > 2) return fail("permutation column kind must be 0 (advice), 1 (fixed) or 2 (instance)");
        if (kind == 0   ? !queried(cs->advice_queries, cs->n_advice_queries, col)
            : kind == 1 ? !queried(cs->fixed_queries, cs->n_fixed_queries, col)
                        : !queried(cs->instance_queries, cs->n_instance_queries, col))
            return fail("a permutation column is not queried at rotation 0");
    }
    for (uint32_t i = 0; i < cs->n_lookups && cs->lookup_tuples; i++) {
        const mzk_lookup_tuple& t = cs->lookup_tuples[i];
        if (t.width < 1 || t.width > 4) return fail("a lookup tuple has 1..4 columns");
        if (t.n_inputs < 1 || t.n_inputs > 8) return fail("a lookup has 1..8 input tuples");
        // the helper constraint of a chunk has degree 1 + its inputs, at most
        // next_pow2(degree - 1) inputs (nb_parallel_lookups_per_chunk,
        // logup.rs:168-183), within cs.degree() as the reference's degree()
        // makes it (circuit.rs:2174-2199, logup.rs:186-212)

        for (uint32_t e = 0; e < t.width; e++) {
            if (!queried(cs->fixed_queries, cs->n_fixed_queries, t.table_fixed[e]))
                return fail("a lookup column is not queried at rotation 0");
            for (uint32_t j = 0; j < t.n_inputs && !cs->lookup_input_programs; j++)
                if (!queried(cs->advice_queries, cs->n_advice_queries, t.input_advice[j][e]))
                    return fail("a lookup column is not queried at rotation 0");
        }
    }
    if (cs->lookup_input_programs) {
        for (uint32_t i = 0, at = 0; i < cs->n_lookups; i++) {
            const uint32_t m = cs->lookup_tuples ? cs->lookup_tuples[i].n_inputs * cs->lookup_tuples[i].width : 1;
            for (uint32_t e = 0; e < m; e++, at++)
                MZK_TRY(check_program(&cs->lookup_input_programs[at],
                                      "lookup " + std::to_string(i) + " input " + std::to_string(e)));
        }
    }
    // each helper constraint h prod_j (f_j + beta) = sum_j prod_(k != j) (f_k + beta)
    // has degree 1 + (inputs of its chunk) x (input degree), within cs.degree()
    // as the reference's degree() makes it (circuit.rs:2174-2199, logup.rs:186-212)
    for (uint32_t i = 0; i < cs->n_lookups; i++) {
        const uint32_t n_in = cs->lookup_tuples ? cs->lookup_tuples[i].n_inputs : 1;
        const uint32_t d_in = lookup_input_degree(cs, i), per = lookup_per_helper(cs->degree, d_in);
        if (per == 0 || std::min(per, n_in) * d_in + 1 > cs->degree)
            return fail("lookup " + std::to_string(i) + ": its helper constraints exceed cs.degree()");
    }
    for (uint32_t i = 0; i < cs->n_lookups; i++) {
        const mzk_lookup_shape& l = cs->lookups[i];
        if ((!cs->lookup_input_programs && !queried(cs->advice_queries, cs->n_advice_queries, l.input_advice)) ||
            !queried(cs->fixed_queries, cs->n_fixed_queries, l.table_fixed) ||
            (l.selector_fixed >= 0 && !queried(cs->fixed_queries, cs->n_fixed_queries, (uint32_t)l.selector_fixed)))
            return fail("a lookup column is not queried at rotation 0");
    }
    return OK;
}

// construct_intermediate_sets (kzg/utils.rs:46-140) over the symbolic
// queries (polynomial, rotation of x), then the sort by (size, index) of
// multi_open (kzg/mod.rs:207-221).  Distinct rotations are distinct points
// for any x outside the n-th roots of unity.
void build_open_sets(PlonkKey* key, const std::vector<std::pair<std::pair<int, uint32_t>, int32_t>>& queries) {
    std::map<int32_t, uint32_t> point_index;
    std::vector<std::pair<std::pair<int, uint32_t>, std::vector<uint32_t>>> com;
    for (const auto& q : queries) {
        auto it = point_index.find(q.second);
        if (it == point_index.end()) it = point_index.emplace(q.second, (uint32_t)point_index.size()).first;
        bool found = false;
        for (auto& c : com)
            if (c.first == q.first) {
                c.second.push_back(it->second);
                found = true;
                break;
            }
        if (!found) com.push_back({q.first, {it->second}});
    }
    std::map<std::vector<uint32_t>, uint32_t> set_index;
    std::vector<std::pair<std::pair<int, uint32_t>, uint32_t>> labels;
    for (auto& c : com) {
        std::vector<uint32_t> s = c.second;
        std::sort(s.begin(), s.end());
        auto it = set_index.find(s);
        if (it == set_index.end()) it = set_index.emplace(s, (uint32_t)set_index.size()).first;
        labels.push_back({c.first, it->second});
    }
    std::vector<int32_t> rot_of(point_index.size());
    for (auto& kv : point_index) rot_of[kv.second] = kv.first;
    std::vector<PlonkKey::OpenSet> sets(set_index.size());
    for (auto& kv : set_index)
        for (uint32_t pi : kv.first) sets[kv.second].rots.push_back(rot_of[pi]);
    for (auto& l : labels) sets[l.second].polys.push_back(l.first);
    std::vector<uint32_t> order(sets.size());
    for (uint32_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return sets[a].rots.size() < sets[b].rots.size(); });
    key->open_sets.clear();
    for (uint32_t i : order) key->open_sets.push_back(sets[i]);
}

// the fixed evaluations a proof writes: every fixed query but those of simple
// selectors (write_evals_to_transcript, prover.rs:857-862)
size_t fixed_written(const PlonkKey& k) {
    size_t m = 0;
    for (auto& q : k.fixed_queries) m += k.is_simple(q.column) ? 0 : 1;
    return m;
}

// The helper program of each lookup chunk for the quotient
// (Evaluator::lookups_flat, evaluation.rs:691-770): every input tuple of the
// chunk theta-compressed (Horner in the tuple's order) plus beta, f_j; their
// product; the sum of partial products sum_j prod_{k!=j} f_k (one input: the
// constant one); for the first chunk also the compressed table plus beta and
// the selector (the quotient reads those from the first chunk only, as
// evaluation.rs:1066-1069 does).  The partial products come from prefix and
// suffix products: the same field values as the reference's per-j loops.
// An input expression that is not a plain advice column is read as the
// extra advice column n_advice + its index (its values on the extended coset,
// which the proof evaluates before the quotient).  Values: 0, 1 (constants),
// beta, theta, trash challenge, y, the previous value, then the reads and
// the ops.
void build_lookup_programs(PlonkKey* key) {
    const Fr4 zero = host::fr_zero(), one = host::fr_one();
    key->lk_consts.assign(zero.l, zero.l + 4);
    key->lk_consts.insert(key->lk_consts.end(), one.l, one.l + 4);
    key->lk_rots = {0};
    key->lk_reads.clear();
    key->lk_ops.clear();
    key->lk_outputs.clear();
    const uint32_t H = key->n_helpers;
    std::vector<uint32_t> n_reads(H), n_ops(H), vlen(H), result(H);
    for (const PlonkKey::Lookup& lk : key->lookups) {
        for (uint32_t c = 0; c < lk.n_helpers(); c++) {
            const uint32_t h = lk.h0 + c, w = lk.width, m = lk.chunk_inputs(c), i0 = c * lk.per_helper;
            const size_t r_start = key->lk_reads.size(), o_start = key->lk_ops.size();
            uint32_t slot = 7;
            auto op = [&](uint32_t kind, uint32_t a, uint32_t b, uint32_t cc) {
                key->lk_ops.push_back({kind, slot, a, b, cc});
                return slot++;
            };
            // reads: the chunk's input tuples, then (first chunk) the table and selector
            std::vector<uint32_t> in_at(m * w), tab_at(w);
            for (uint32_t j = 0; j < m; j++)
                for (uint32_t e = 0; e < w; e++) {
                    const int32_t x = lk.expr[i0 + j][e];
                    key->lk_reads.push_back({1, x >= 0 ? key->n_advice + (uint32_t)x : lk.in[i0 + j][e], 0, slot});
                    in_at[j * w + e] = slot++;
                }
            uint32_t sel = 1;
            if (c == 0) {
                for (uint32_t e = 0; e < w; e++) {
                    key->lk_reads.push_back({0, lk.tab[e], 0, slot});
                    tab_at[e] = slot++;
                }
                if (lk.shape.selector_fixed >= 0) {
                    key->lk_reads.push_back({0, (uint32_t)lk.shape.selector_fixed, 0, slot});
                    sel = slot++;
                }
            }
            // f_j = Horner_theta(tuple j) + beta
            std::vector<uint32_t> f(m);
            for (uint32_t j = 0; j < m; j++) {
                uint32_t acc = 0;
                for (uint32_t e = 0; e < w; e++) acc = op(MZK_FLAT_MULADD, acc, 3, in_at[j * w + e]);
                f[j] = op(MZK_FLAT_ADD, acc, 2, 0);
            }
            uint32_t table = 1;
            if (c == 0) {
                uint32_t acc = 0;
                for (uint32_t e = 0; e < w; e++) acc = op(MZK_FLAT_MULADD, acc, 3, tab_at[e]);
                table = op(MZK_FLAT_ADD, acc, 2, 0);
            }
            uint32_t product = f[0], spp = 1;
            if (m > 1) {
                // pre[j] = f_0 .. f_(j-1), suf[j] = f_(j+1) .. f_(m-1)
                std::vector<uint32_t> pre(m), suf(m);
                pre[1] = f[0];
                for (uint32_t j = 2; j < m; j++) pre[j] = op(MZK_FLAT_MUL, pre[j - 1], f[j - 1], 0);
                product = op(MZK_FLAT_MUL, pre[m - 1], f[m - 1], 0);
                suf[m - 2] = f[m - 1];
                for (uint32_t j = m - 2; j-- > 0;) suf[j] = op(MZK_FLAT_MUL, f[j + 1], suf[j + 1], 0);
                spp = suf[0];
                for (uint32_t j = 1; j + 1 < m; j++) spp = op(MZK_FLAT_ADD, spp, op(MZK_FLAT_MUL, pre[j], suf[j], 0), 0);
                spp = op(MZK_FLAT_ADD, spp, pre[m - 1], 0);
            }
            n_reads[h] = (uint32_t)(key->lk_reads.size() - r_start);
            n_ops[h] = (uint32_t)(key->lk_ops.size() - o_start);
            vlen[h] = slot;
            result[h] = spp;
            for (uint32_t o : {spp, product, table, sel}) key->lk_outputs.push_back(o);
        }
    }
    key->lk_programs.assign(H, mzk_flat_graph{});
    size_t r0 = 0, o0 = 0;
    for (uint32_t h = 0; h < H; h++) {
        mzk_flat_graph& g = key->lk_programs[h];
        g.constants = key->lk_consts.data();
        g.n_constants = 2;
        g.rotations = key->lk_rots.data();
        g.n_rotations = 1;
        g.reads = key->lk_reads.data() + r0;
        g.n_reads = n_reads[h];
        g.ops = key->lk_ops.data() + o0;
        g.n_ops = n_ops[h];
        g.values_len = vlen[h];
        g.beta_idx = 2;
        g.theta_idx = 3;
        g.trash_challenge_idx = 4;
        g.y_idx = 5;
        g.previous_value_idx = 6;
        g.result_idx = result[h];
        r0 += n_reads[h];
        o0 += n_ops[h];
    }
}

}  // namespace

Status vk_transcript_repr(uint32_t k, const uint64_t* fixed, size_t n_fixed, const uint64_t* perm, size_t n_perm,
                          const uint8_t* pinned, size_t pinned_len, Fr4* out) {
    static const char kPersonal[] = "Halo2-Verify-Key";
    host::Blake2b h(64, nullptr, 0, reinterpret_cast<const uint8_t*>(kPersonal), 16);
    uint8_t head[6] = {0x03, (uint8_t)k, 0, 0, 0, 0};  // VERSION (plonk/mod.rs:74), k, u32 count
    for (int b = 0; b < 4; b++) head[2 + b] = (uint8_t)(n_fixed >> (8 * b));
    h.update(head, 6);
    uint8_t enc[96];
    for (size_t i = 0; i < n_fixed; i++) {
        host::g1_uncompressed(fixed + 18 * i, enc);
        h.update(enc, 96);
    }
    uint8_t cnt[4];
    for (int b = 0; b < 4; b++) cnt[b] = (uint8_t)(n_perm >> (8 * b));
    h.update(cnt, 4);
    for (size_t i = 0; i < n_perm; i++) {
        host::g1_uncompressed(perm + 18 * i, enc);
        h.update(enc, 96);
    }
    if (pinned_len) h.update(pinned, pinned_len);
    uint8_t d[64];
    h.digest(d);
    *out = host::fr_from_uniform(d);
    return OK;
}

// perm_values (host, n_perm_cols columns of n Fr): the permutation
// polynomials' Lagrange values as given (ProvingKey::read, permutation.rs:
// 153-166); otherwise they are built from `mapping` (or the identity)
// given_coms (optional, host): the fixed then permutation commitments in the
// 18-u64 layout, as a key file holds them; otherwise they are computed
Status keygen(Context* ctx, const Domain* d, const mzk_circuit_desc* cs, const mzk_srs_desc* srs,
              const uint64_t* const* fixed_values, const uint32_t* mapping, const uint64_t* const* perm_values,
              const uint8_t* pinned, size_t pinned_len, PlonkKey** out, const uint64_t* given_coms = nullptr) {
    MZK_TRY(check_circuit(d, cs));
    const uint32_t n = 1u << d->k, E = 1u << d->ext_k;
    if (!srs || !srs->srs) {
        set_error("keygen: null SRS");
        return ERR_ARG;
    }
    for (uint64_t off : {srs->off_g, srs->off_lagrange, srs->off_lagrange_delta, srs->off_lagrange_double_delta})
        if (off + n > srs->srs_len) {
            set_error("keygen: SRS bases out of range");
            return ERR_ARG;
        }
    if (cs->n_fixed && !fixed_values) {
        set_error("keygen: null fixed columns");
        return ERR_ARG;
    }
    for (uint32_t i = 0; i < cs->n_fixed; i++)
        if (!fixed_values[i]) {
            set_error("keygen: null fixed column");
            return ERR_ARG;
        }
    const uint32_t P = cs->n_perm_cols;
    if (mapping)
        for (uint64_t i = 0; i < (uint64_t)P * n; i++)
            if (mapping[2 * i] >= P || mapping[2 * i + 1] >= n) {
                set_error("keygen: permutation mapping out of range");
                return ERR_ARG;
            }
    auto key = std::unique_ptr<PlonkKey>(new PlonkKey);
    key->dom = d;
    key->k = d->k;
    key->n = n;
    key->bf = cs->blinding_factors;
    key->u = n - cs->blinding_factors - 1;
    key->degree = cs->degree;
    key->qdeg = cs->degree - 1;
    key->chunk = cs->degree - 2;
    key->n_perm = P;
    key->n_sets = (P + key->chunk - 1) / key->chunk;
    key->n_advice = cs->n_advice;
    key->n_fixed = cs->n_fixed;
    key->advice_queries.assign(cs->advice_queries, cs->advice_queries + cs->n_advice_queries);
    key->fixed_queries.assign(cs->fixed_queries, cs->fixed_queries + cs->n_fixed_queries);
    key->n_instance = cs->n_instance;
    key->instance_queries.assign(cs->instance_queries, cs->instance_queries + cs->n_instance_queries);
    key->trash.resize(cs->n_trash);
    for (uint32_t t = 0; t < cs->n_trash; t++) {
        const mzk_flat_graph& g = cs->trash[t].program;
        PlonkKey::Trash& tr = key->trash[t];
        tr.consts.assign(g.constants, g.constants + 4 * (size_t)g.n_constants);
        tr.rots.assign(g.rotations, g.rotations + g.n_rotations);
        tr.reads.assign(g.reads, g.reads + g.n_reads);
        tr.ops.assign(g.ops, g.ops + g.n_ops);
        tr.program = g;
        tr.program.constants = tr.consts.data();
        tr.program.rotations = tr.rots.data();
        tr.program.reads = tr.reads.data();
        tr.program.ops = tr.ops.data();
        tr.selector = cs->trash[t].selector_fixed;
    }
    key->simple_col.assign(cs->n_fixed, 0);
    for (uint32_t i = 0; i < cs->n_gate_polys; i++) {
        key->gate_poly_values.push_back(cs->gate_poly_values[i]);
        key->gate_poly_selector.push_back(cs->gate_poly_selector[i]);
        if (cs->gate_poly_selector[i] >= 0) key->simple_col[cs->gate_poly_selector[i]] = 1;
    }
    std::memcpy(key->gate_fixed, cs->gate_fixed, sizeof(key->gate_fixed));
    std::memcpy(key->gate_advice, cs->gate_advice, sizeof(key->gate_advice));
    if (const mzk_flat_graph* g = cs->gates) {
        key->has_gates = true;
        key->g_consts.assign(g->constants, g->constants + 4 * (size_t)g->n_constants);
        key->g_rots.assign(g->rotations, g->rotations + g->n_rotations);
        key->g_reads.assign(g->reads, g->reads + g->n_reads);
        key->g_ops.assign(g->ops, g->ops + g->n_ops);
        key->gates = *g;
        key->gates.constants = key->g_consts.data();
        key->gates.rotations = key->g_rots.data();
        key->gates.reads = key->g_reads.data();
        key->gates.ops = key->g_ops.data();
    }
    key->perm_kind.assign(cs->perm_col_kind, cs->perm_col_kind + P);
    key->perm_index.assign(cs->perm_col_index, cs->perm_col_index + P);
    const uint32_t L = cs->n_lookups;
    key->lookups.resize(L);
    size_t n_programs = 0;  // lookup input programs given
    for (uint32_t l = 0; l < L && cs->lookup_input_programs; l++)
        n_programs += cs->lookup_tuples ? cs->lookup_tuples[l].n_inputs * cs->lookup_tuples[l].width : 1;
    key->lk_exprs.reserve(n_programs);  // no reallocation: each Program's graph points into itself
    for (uint32_t l = 0, at = 0; l < L; l++) {
        PlonkKey::Lookup& lk = key->lookups[l];
        lk.shape = cs->lookups[l];
        if (cs->lookup_tuples) {
            const mzk_lookup_tuple& t = cs->lookup_tuples[l];
            lk.width = t.width;
            lk.n_inputs = t.n_inputs;
            for (uint32_t e = 0; e < lk.width; e++) {
                for (uint32_t j = 0; j < lk.n_inputs; j++) lk.in[j][e] = t.input_advice[j][e];
                lk.tab[e] = t.table_fixed[e];
            }
        } else {
            lk.width = 1;
            lk.in[0][0] = lk.shape.input_advice;
            lk.tab[0] = lk.shape.table_fixed;
        }
        for (uint32_t j = 0; j < 8; j++)
            for (uint32_t e = 0; e < 4; e++) lk.expr[j][e] = -1;
        for (uint32_t j = 0; j < lk.n_inputs && cs->lookup_input_programs; j++)
            for (uint32_t e = 0; e < lk.width; e++) {
                const mzk_flat_graph& g = cs->lookup_input_programs[at++];
                const int col = plain_advice(g);
                if (col >= 0) {
                    lk.in[j][e] = (uint32_t)col;
                } else {
                    lk.expr[j][e] = (int32_t)key->lk_exprs.size();
                    key->lk_exprs.emplace_back();
                    key->lk_exprs.back().assign(g);
                }
            }
        lk.per_helper = lookup_per_helper(cs->degree, lookup_input_degree(cs, l));
        lk.h0 = key->n_helpers;
        key->n_helpers += lk.n_helpers();
    }
    if (cs->n_advice + key->lk_exprs.size() > kQMaxAdvice) {
        set_error("keygen: advice columns and lookup input expressions exceed 16 quotient columns");
        return ERR_ARG;
    }
    key->srs = *srs;
    const uint32_t F = cs->n_fixed, u = key->u;
    // lookup table indexes (host): the distinct table tuples of the usable
    // rows in the order of the device search (element by element, each from
    // its lowest 64-bit word: the map's order), each row's index, 1 / copies
    std::vector<std::vector<uint64_t>> uniq(L);
    std::vector<std::vector<uint32_t>> uid(L);
    std::vector<std::vector<Fr4>> tinv(L);
    bool need_ones = false;
    size_t uniq_total = 0;
    for (uint32_t l = 0; l < L; l++) {
        const PlonkKey::Lookup& lk = key->lookups[l];
        auto row_key = [&](uint32_t i) {
            std::vector<uint64_t> kv(4 * lk.width);
            for (uint32_t e = 0; e < lk.width; e++) std::memcpy(&kv[4 * e], fixed_values[lk.tab[e]] + 4 * (size_t)i, 32);
            return kv;
        };
        std::map<std::vector<uint64_t>, uint32_t> count;
        for (uint32_t i = 0; i < u; i++) count[row_key(i)]++;
        std::map<std::vector<uint64_t>, uint32_t> index;
        for (auto& kv : count) {
            index[kv.first] = (uint32_t)(uniq[l].size() / (4 * lk.width));
            uniq[l].insert(uniq[l].end(), kv.first.begin(), kv.first.end());
            tinv[l].push_back(host::fr_inv(host::fr_from_u64(kv.second)));
        }
        uid[l].resize(u);
        for (uint32_t i = 0; i < u; i++) uid[l][i] = index[row_key(i)];
        key->lookups[l].n_uniq = (uint32_t)count.size();
        uniq_total += (size_t)count.size() * (lk.width + 1);
        need_ones = need_ones || lk.shape.selector_fixed < 0;
    }
    // one device allocation for the whole key
    const size_t fr_elems = (size_t)F * (2 * n + E) + (size_t)P * (2 * n + E) + 3 * (size_t)E + (need_ones ? n : 0) +
                            uniq_total;
    const size_t bytes = fr_elems * sizeof(Fr) + (size_t)u * 4 * L + 256;
    cudaError_t e = cudaMalloc(&key->mem, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("keygen: device allocation of " + std::to_string(bytes) + " bytes failed");
        return ERR_OOM;
    }
    cudaStream_t st = ctx->stream;
    Fr* carve = static_cast<Fr*>(key->mem);
    auto take = [&](size_t elems) {
        Fr* p = carve;
        carve += elems;
        return p;
    };
    for (uint32_t i = 0; i < F; i++) {
        key->fixed_lag.push_back(take(n));
        key->fixed_coeff.push_back(take(n));
        key->fixed_ext.push_back(take(E));
    }
    // the permutation columns' Lagrange forms are contiguous: k_perm_values
    // writes them as one P x n array
    for (uint32_t i = 0; i < P; i++) key->perm_lag.push_back(take(n));
    for (uint32_t i = 0; i < P; i++) {
        key->perm_coeff.push_back(take(n));
        key->perm_ext.push_back(take(E));
    }
    key->l0 = take(E);
    key->l_last = take(E);
    key->l_active = take(E);
    if (need_ones) key->ones = take(n);
    for (auto& lk : key->lookups) {
        lk.uniq = take((size_t)lk.n_uniq * lk.width);
        lk.tinv = take(lk.n_uniq);
    }
    for (uint32_t l = 0; l < L; l++) key->lookups[l].uid = reinterpret_cast<uint32_t*>(carve) + (size_t)l * u;
    // fixed columns
    for (uint32_t i = 0; i < F; i++) {
        MZK_CUDA_CHECK(cudaMemcpyAsync(key->fixed_lag[i], fixed_values[i], (size_t)n * sizeof(Fr),
                                       cudaMemcpyHostToDevice, st));
        MZK_TRY(domain_op_device(ctx, d, OP_LAGRANGE_TO_COEFF, key->fixed_lag[i], key->fixed_coeff[i], st));
        MZK_TRY(domain_op_device(ctx, d, OP_COEFF_TO_EXTENDED, key->fixed_coeff[i], key->fixed_ext[i], st));
    }
    // permutation polynomials (build_pk)
    if (P) {
        std::vector<Fr4> deltas(P);
        Fr4 delta;
        std::memcpy(delta.l, host::FR_DELTA4, 32);
        deltas[0] = host::fr_one();
        for (uint32_t c = 1; c < P; c++) deltas[c] = host::fr_mul(deltas[c - 1], delta);
        void *d_tab, *d_map = nullptr;
        MZK_TRY(ctx->ensure("kg_deltas", (size_t)P * sizeof(Fr), &d_tab));
        MZK_CUDA_CHECK(cudaMemcpyAsync(d_tab, deltas.data(), (size_t)P * 32, cudaMemcpyHostToDevice, st));
        if (mapping) {
            MZK_TRY(ctx->ensure("kg_mapping", (size_t)P * n * 8, &d_map));
            MZK_CUDA_CHECK(cudaMemcpyAsync(d_map, mapping, (size_t)P * n * 8, cudaMemcpyHostToDevice, st));
        }
        if (perm_values) {
            for (uint32_t i = 0; i < P; i++) {
                if (!perm_values[i]) {
                    set_error("keygen: null permutation column");
                    return ERR_ARG;
                }
                MZK_CUDA_CHECK(cudaMemcpyAsync(key->perm_lag[i], perm_values[i], (size_t)n * sizeof(Fr),
                                               cudaMemcpyHostToDevice, st));
            }
        } else {
            k_perm_values<<<grid_of(ctx, (uint64_t)P * n), kThreads, 0, st>>>(
                key->perm_lag[0], static_cast<const uint32_t*>(d_map), static_cast<const Fr*>(d_tab), d->lo[0],
                d->hi[0], n, P);
            MZK_LAUNCH_CHECK(ctx);
        }
        for (uint32_t i = 0; i < P; i++) {
            MZK_TRY(domain_op_device(ctx, d, OP_LAGRANGE_TO_COEFF, key->perm_lag[i], key->perm_coeff[i], st));
            MZK_TRY(domain_op_device(ctx, d, OP_COEFF_TO_EXTENDED, key->perm_coeff[i], key->perm_ext[i], st));
        }
    }
    // l0, l_last, l_active_row (compute_lagrange_polys)
    {
        void* tmp;
        MZK_TRY(ctx->ensure("kg_lagrange", (size_t)(2 * n + E) * sizeof(Fr), &tmp));
        Fr* lag = static_cast<Fr*>(tmp);
        Fr* coeff = lag + n;
        Fr* blind_ext = coeff + n;
        const uint64_t bf = key->bf;
        struct {
            uint64_t lo, hi;
            Fr* ext;
        } polys[3] = {{0, 1, key->l0}, {n - bf - 1, n - bf, key->l_last}, {n - bf, n, blind_ext}};
        for (auto& p : polys) {
            k_unit<<<grid_of(ctx, n), kThreads, 0, st>>>(lag, n, p.lo, p.hi);
            MZK_LAUNCH_CHECK(ctx);
            MZK_TRY(domain_op_device(ctx, d, OP_LAGRANGE_TO_COEFF, lag, coeff, st));
            MZK_TRY(domain_op_device(ctx, d, OP_COEFF_TO_EXTENDED, coeff, p.ext, st));
        }
        k_active<<<grid_of(ctx, E), kThreads, 0, st>>>(key->l_active, key->l_last, blind_ext, E);
        MZK_LAUNCH_CHECK(ctx);
    }
    if (need_ones) {
        k_unit<<<grid_of(ctx, n), kThreads, 0, st>>>(key->ones, n, 0, n);
        MZK_LAUNCH_CHECK(ctx);
    }
    for (uint32_t l = 0; l < L; l++) {
        PlonkKey::Lookup& lk = key->lookups[l];
        MZK_CUDA_CHECK(cudaMemcpyAsync(lk.uniq, uniq[l].data(), uniq[l].size() * 8, cudaMemcpyHostToDevice, st));
        MZK_CUDA_CHECK(cudaMemcpyAsync(lk.tinv, tinv[l].data(), tinv[l].size() * 32, cudaMemcpyHostToDevice, st));
        MZK_CUDA_CHECK(cudaMemcpyAsync(lk.uid, uid[l].data(), uid[l].size() * 4, cudaMemcpyHostToDevice, st));
    }
    // the quotient's built-in lookup term serves a single one-column lookup
    // without trashcans; otherwise every lookup goes to it as helper programs
    bool tuples = !key->lk_exprs.empty();
    for (auto& lk : key->lookups) tuples = tuples || lk.width > 1 || lk.n_inputs > 1;
    if (L > 1 || (L && (cs->n_trash || tuples))) build_lookup_programs(key.get());
    // VK commitments (Lagrange basis) as one batch
    std::vector<BatchItem> items;
    for (uint32_t i = 0; i < F; i++) items.push_back({key->fixed_lag[i], srs->off_lagrange, n});
    for (uint32_t i = 0; i < P; i++) items.push_back({key->perm_lag[i], srs->off_lagrange, n});
    std::vector<uint64_t> res(items.size() * 18);
    MsmTable table{srs->srs, srs->srs_len, srs->table_c, srs->table_rows, srs->table_min_n};
    if (given_coms) std::memcpy(res.data(), given_coms, res.size() * 8);
    else if (!items.empty())
        MZK_TRY(run_msms(ctx, srs->srs, srs->srs_len, items, res.data(), 0, srs->table_c > 0 ? &table : nullptr, st));
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    key->fixed_coms.resize(F);
    key->perm_coms.resize(P);
    for (uint32_t i = 0; i < F; i++) std::memcpy(key->fixed_coms[i].data(), &res[18 * i], 144);
    for (uint32_t i = 0; i < P; i++) std::memcpy(key->perm_coms[i].data(), &res[18 * (F + i)], 144);
    MZK_TRY(vk_transcript_repr(d->k, F ? key->fixed_coms[0].data() : nullptr, F,
                               P ? key->perm_coms[0].data() : nullptr, P, pinned, pinned_len, &key->repr));
    // the multi-open layout (prover.rs:871-933 query order)
    std::vector<std::pair<std::pair<int, uint32_t>, int32_t>> qs;
    for (auto& q : key->advice_queries) qs.push_back({{PlonkKey::P_ADVICE, q.column}, q.rotation});
    for (uint32_t s = 0; s < key->n_sets; s++) {
        qs.push_back({{PlonkKey::P_PERM_Z, s}, 0});
        qs.push_back({{PlonkKey::P_PERM_Z, s}, 1});
    }
    for (uint32_t s = key->n_sets; s-- > 1;) qs.push_back({{PlonkKey::P_PERM_Z, s - 1}, key->last_rot()});
    for (uint32_t l = 0; l < L; l++) {  // logup Evaluated::open per lookup (logup/prover.rs:357-392)
        qs.push_back({{PlonkKey::P_M, l}, 0});
        for (uint32_t c = 0; c < key->lookups[l].n_helpers(); c++)
            qs.push_back({{PlonkKey::P_H, key->lookups[l].h0 + c}, 0});
        qs.push_back({{PlonkKey::P_AGG, l}, 0});
        qs.push_back({{PlonkKey::P_AGG, l}, 1});
    }
    for (uint32_t t = 0; t < cs->n_trash; t++) qs.push_back({{PlonkKey::P_TRASH, t}, 0});  // trash Evaluated::open
    for (auto& q : key->fixed_queries)  // a simple selector is not opened (prover.rs:913-918)
        if (!key->is_simple(q.column)) qs.push_back({{PlonkKey::P_FIXED, q.column}, q.rotation});
    for (uint32_t i = 0; i < P; i++) qs.push_back({{PlonkKey::P_PERM_FIXED, i}, 0});
    qs.push_back({{PlonkKey::P_LIN, 0}, 0});
    build_open_sets(key.get(), qs);
    const uint32_t S = key->n_sets;
    const size_t T = cs->n_trash;
    const size_t H = key->n_helpers;
    const size_t points = cs->n_advice + L + S + H + L + T + key->qdeg + 2;
    const size_t scalars = key->advice_queries.size() + fixed_written(*key) + P + (S ? 3 * S - 1 : 0) + 3 * L + H + T +
                           key->open_sets.size();
    key->proof_len = 48 * points + 32 * scalars;
    key->n_blinds = (size_t)cs->n_advice * (key->bf + 1) + L * (key->bf + 1) + (size_t)S * key->bf + L * key->bf +
                    (key->qdeg - 1);
    *out = key.release();
    return OK;
}

// ------------------------------------------------------ key file formats ----
// VerifyingKey::write / ProvingKey::write (plonk/mod.rs:95-113, 391-399) and
// their readers (:120-196, :418-453).  SerdeFormat: Processed writes points
// compressed (48 bytes); RawBytes and RawBytesUnchecked write them
// uncompressed (96 bytes, G1Affine::to_uncompressed); field elements of the
// polynomial slices are always the raw Montgomery limbs (Fq::write_raw,
// fq.rs:912-917), each slice a u32 big-endian count of polynomials, each
// polynomial a u32 big-endian length (helpers.rs:150-160, poly/mod.rs:544-550).
namespace {

void put_u32_le(std::vector<uint8_t>& v, uint32_t x) {
    for (int b = 0; b < 4; b++) v.push_back((uint8_t)(x >> (8 * b)));
}
void put_u32_be(std::vector<uint8_t>& v, uint32_t x) {
    for (int b = 3; b >= 0; b--) v.push_back((uint8_t)(x >> (8 * b)));
}
void put_point(std::vector<uint8_t>& v, const uint64_t* p18, int format) {
    uint8_t enc[96];
    if (format == MZK_SERDE_PROCESSED) {
        host::g1_compress(p18, enc);
        v.insert(v.end(), enc, enc + 48);
    } else {
        host::g1_uncompressed(p18, enc);
        v.insert(v.end(), enc, enc + 96);
    }
}

struct Reader {
    const uint8_t* p;
    size_t len, pos = 0;
    bool take(size_t m, const uint8_t** out) {
        if (len - pos < m) return false;
        *out = p + pos;
        pos += m;
        return true;
    }
};

// points of a key file into the 18-u64 layout.  Compressed encodings go
// through the device decompression (flags, x < p, square root, subgroup);
// uncompressed ones are recompressed and decompressed the same way, and the
// decoded y must equal the given one (RawBytes), or are taken as they are
// (RawBytesUnchecked)
Status decode_points(Context* ctx, const std::vector<const uint8_t*>& enc, int format,
                     std::vector<std::array<uint64_t, 18>>& pts, cudaStream_t st) {
    const size_t m = enc.size();
    pts.assign(m, {});
    if (m == 0) return OK;
    host::Fp6 r2;
    static const uint64_t kR2[6] = {0xf4df1f341c341746ULL, 0x0a76e6a609d104f1ULL, 0x8de5476c4c95b6d5ULL,
                                    0x67eb88a9939d83c0ULL, 0x9a793e85b519952dULL, 0x11988fe592cae3aaULL};
    std::memcpy(r2.l, kR2, 48);
    auto be48 = [](const uint8_t* b, uint64_t out[6]) {
        for (int i = 0; i < 6; i++) {
            uint64_t w = 0;
            for (int k = 0; k < 8; k++) w = (w << 8) | b[47 - (8 * i + 7 - k)];
            out[i] = w;
        }
    };
    std::vector<uint8_t> comp(m * 48);
    std::vector<std::array<uint64_t, 6>> ys(m);
    for (size_t i = 0; i < m; i++) {
        const uint8_t* e = enc[i];
        if (format == MZK_SERDE_PROCESSED) {
            std::memcpy(&comp[48 * i], e, 48);
            continue;
        }
        // uncompressed: flags 0x80 (compressed) and 0x20 (sort) must be clear
        if (e[0] & 0xa0) {
            set_error("key file: bad uncompressed point encoding");
            return ERR_ARG;
        }
        if (e[0] & 0x40) {  // identity: every other bit zero
            for (int b = 1; b < 96; b++)
                if (e[b]) {
                    set_error("key file: bad identity encoding");
                    return ERR_ARG;
                }
            if (e[0] != 0x40) {
                set_error("key file: bad identity encoding");
                return ERR_ARG;
            }
            std::memset(&comp[48 * i], 0, 48);
            comp[48 * i] = 0xc0;
            ys[i].fill(0);
            continue;
        }
        uint64_t x[6], y[6];
        be48(e, x);
        be48(e + 48, y);
        if (host::geq6(x, host::P6) || host::geq6(y, host::P6)) {
            set_error("key file: coordinate not below p");
            return ERR_ARG;
        }
        host::Fp6 xc, yc;
        std::memcpy(xc.l, x, 48);
        std::memcpy(yc.l, y, 48);
        const host::Fp6 xm = host::canon(host::mul(xc, r2)), ym = host::canon(host::mul(yc, r2));
        if (format == MZK_SERDE_RAW_UNCHECKED) {
            std::memcpy(pts[i].data(), xm.l, 48);
            std::memcpy(pts[i].data() + 6, ym.l, 48);
            std::memcpy(pts[i].data() + 12, host::ONE6, 48);
            continue;
        }
        std::memcpy(ys[i].data(), ym.l, 48);
        uint64_t p18[18];
        std::memcpy(p18, xm.l, 48);
        std::memcpy(p18 + 6, ym.l, 48);
        std::memcpy(p18 + 12, host::ONE6, 48);
        host::g1_compress(p18, &comp[48 * i]);
    }
    if (format == MZK_SERDE_RAW_UNCHECKED) return OK;
    void *d_in, *d_out, *d_st;
    MZK_TRY(ctx->ensure("kf_enc", m * 48, &d_in));
    MZK_TRY(ctx->ensure("kf_aff", m * 96, &d_out));
    MZK_TRY(ctx->ensure("kf_status", m, &d_st));
    MZK_CUDA_CHECK(cudaMemcpyAsync(d_in, comp.data(), m * 48, cudaMemcpyHostToDevice, st));
    uint64_t invalid = 0;
    MZK_TRY(g1_decompress_device(ctx, d_in, m, 1, d_out, static_cast<uint8_t*>(d_st), &invalid, st));
    std::vector<uint64_t> aff(m * 12);
    MZK_CUDA_CHECK(cudaMemcpyAsync(aff.data(), d_out, m * 96, cudaMemcpyDeviceToHost, st));
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    if (invalid) {
        set_error("key file: " + std::to_string(invalid) + " invalid point(s) (encoding, curve or subgroup)");
        return ERR_ARG;
    }
    for (size_t i = 0; i < m; i++) {
        const uint64_t* a = &aff[12 * i];
        bool zero = true;
        for (int j = 0; j < 12; j++) zero = zero && a[j] == 0;
        std::memcpy(pts[i].data(), a, 96);
        if (!zero) std::memcpy(pts[i].data() + 12, host::ONE6, 48);
        if (format == MZK_SERDE_RAW && !zero && std::memcmp(a + 6, ys[i].data(), 48) != 0) {
            set_error("key file: point not on the curve");
            return ERR_ARG;
        }
    }
    return OK;
}

}  // namespace

Status vk_serialize(const PlonkKey* k, int format, std::vector<uint8_t>& out) {
    out.clear();
    out.push_back(0x03);
    out.push_back((uint8_t)k->k);
    put_u32_le(out, (uint32_t)k->fixed_coms.size());
    for (auto& c : k->fixed_coms) put_point(out, c.data(), format);
    for (auto& c : k->perm_coms) put_point(out, c.data(), format);
    return OK;
}

Status pk_serialize(Context* ctx, const PlonkKey* k, int format, std::vector<uint8_t>& out, cudaStream_t st) {
    MZK_TRY(vk_serialize(k, format, out));
    std::vector<uint8_t> vals((size_t)k->n * 32);
    auto slice = [&](const std::vector<Fr*>& cols) -> Status {
        put_u32_be(out, (uint32_t)cols.size());
        for (Fr* c : cols) {
            put_u32_be(out, k->n);
            MZK_CUDA_CHECK(cudaMemcpyAsync(vals.data(), c, vals.size(), cudaMemcpyDeviceToHost, st));
            MZK_CUDA_CHECK(cudaStreamSynchronize(st));
            out.insert(out.end(), vals.begin(), vals.end());  // raw Montgomery limbs, little-endian
        }
        return OK;
    };
    MZK_TRY(slice(k->fixed_lag));
    MZK_TRY(slice(k->perm_lag));
    return OK;
}

Status pk_read(Context* ctx, const Domain* d, const mzk_circuit_desc* cs, const mzk_srs_desc* srs,
               const uint8_t* bytes, size_t len, int format, const uint8_t* pinned, size_t pinned_len,
               PlonkKey** out, cudaStream_t st) {
    auto fail = [](const std::string& m) {
        set_error("pk_read: " + m);
        return ERR_ARG;
    };
    Reader r{bytes, len};
    const uint8_t* p;
    if (!r.take(2, &p)) return fail("short file");
    if (p[0] != 0x03) return fail("unexpected version byte");
    if (p[1] != d->k) return fail("k of the file differs from the domain's");
    if (!r.take(4, &p)) return fail("short file");
    const uint32_t nf = (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24;
    if (nf != cs->n_fixed) return fail("fixed column count differs from the constraint system's");
    const size_t psz = format == MZK_SERDE_PROCESSED ? 48 : 96;
    std::vector<const uint8_t*> enc;
    for (uint32_t i = 0; i < nf + cs->n_perm_cols; i++) {
        if (!r.take(psz, &p)) return fail("short file");
        enc.push_back(p);
    }
    std::vector<std::array<uint64_t, 18>> pts;
    MZK_TRY(decode_points(ctx, enc, format, pts, st));
    std::vector<uint64_t> coms(pts.size() * 18);
    for (size_t i = 0; i < pts.size(); i++) std::memcpy(&coms[18 * i], pts[i].data(), 144);
    const uint32_t n = 1u << d->k;
    auto read_slice = [&](uint32_t expect, std::vector<const uint64_t*>& cols) -> Status {
        if (!r.take(4, &p)) return fail("short file");
        const uint32_t cnt = (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3];
        if (cnt != expect) return fail("polynomial count differs from the constraint system's");
        for (uint32_t c = 0; c < cnt; c++) {
            if (!r.take(4, &p)) return fail("short file");
            const uint32_t pl = (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3];
            if (pl != n) return fail("polynomial length differs from the domain's");
            if (!r.take((size_t)n * 32, &p)) return fail("short file");
            const uint64_t* v = reinterpret_cast<const uint64_t*>(p);  // raw little-endian limbs
            if (format != MZK_SERDE_RAW_UNCHECKED)
                for (uint32_t i = 0; i < n; i++)
                    if (host::fr_geq(v + 4 * (size_t)i, host::R4)) return fail("field element not below r");
            cols.push_back(v);
        }
        return OK;
    };
    std::vector<const uint64_t*> fixed, perm;
    MZK_TRY(read_slice(cs->n_fixed, fixed));
    MZK_TRY(read_slice(cs->n_perm_cols, perm));
    if (r.pos != len) return fail("trailing bytes");
    // the limbs are read in place: copy them to aligned host columns
    std::vector<std::vector<uint64_t>> fcols(fixed.size()), pcols(perm.size());
    std::vector<const uint64_t*> fptr, pptr;
    for (size_t i = 0; i < fixed.size(); i++) {
        fcols[i].resize((size_t)4 * n);
        std::memcpy(fcols[i].data(), fixed[i], (size_t)n * 32);
        fptr.push_back(fcols[i].data());
    }
    for (size_t i = 0; i < perm.size(); i++) {
        pcols[i].resize((size_t)4 * n);
        std::memcpy(pcols[i].data(), perm[i], (size_t)n * 32);
        pptr.push_back(pcols[i].data());
    }
    return keygen(ctx, d, cs, srs, fptr.data(), nullptr, pptr.data(), pinned, pinned_len, out, coms.data());
}

// --------------------------------------------------------------- prover ----
namespace {

struct FsProof {
    const PlonkKey* key = nullptr;
    const mzk_proof_request* req = nullptr;
    host::Transcript tr;
    Fr4 theta, beta, gamma, trash, y, x, xn, x1, x2, x3, x4;
    std::vector<Fr*> adv_lag, adv_coeff, adv_ext, z_lag, z_delta, z_coeff, z_ext, q, fdiv;
    std::vector<Fr*> qt;  // per point set: the intermediate quotient of its divisions
    std::vector<Fr*> inst_lag, inst_coeff, inst_ext;  // instance columns (zero past their values)
    std::vector<Fr*> trash_lag, trash_coeff, trash_ext;  // trash columns
    // per lookup: multiplicities and aggregator; per helper (Lookup::h0 + chunk): helper
    std::vector<Fr*> m_lag, m_delta, m_coeff, m_ext, h_lag, h_coeff, h_ext, Z_lag, Z_dd, Z_coeff, Z_ext;
    // theta-compressed inputs (per input tuple) and table of a tuple lookup (else empty / null)
    std::vector<std::vector<Fr*>> f_lag;
    std::vector<Fr*> t_lag;
    // the key's lookup input expressions over the Lagrange rows and the extended coset
    std::vector<Fr*> e_lag, e_ext;
    std::vector<uint32_t*> counts;
    Fr *limbs = nullptr, *lin = nullptr, *f = nullptr, *fin = nullptr, *pi = nullptr;
    Fr* d_blinds = nullptr;
    uint64_t f_len = 0;
    Fr4 lin_c = {};  // the linearization's constant term C (when the identities were evaluated)
    // blinding offsets (elements of req->blinds)
    size_t off_mult = 0, off_perm = 0, off_logup = 0, off_quot = 0;
    // evaluations
    std::vector<Fr4> ev_adv, ev_fix, ev_pc, ev_sets, ev_lk, ev_inst, ev_trash, q_x3;
};

// input element e of lookup input tuple i over the Lagrange rows: its
// expression's values, or its advice column
const Fr* lookup_input_lag(const FsProof& p, const PlonkKey::Lookup& lk, uint32_t i, uint32_t e) {
    return lk.expr[i][e] >= 0 ? p.e_lag[lk.expr[i][e]] : p.adv_lag[lk.in[i][e]];
}

size_t proof_scratch_elems(const PlonkKey* k) {
    const size_t n = k->n, E = (size_t)1 << k->dom->ext_k, A = k->n_advice, S = k->n_sets;
    const size_t L = k->lookups.size(), O = k->open_sets.size();
    size_t counts = 0;
    for (const auto& lk : k->lookups) counts += (lk.n_uniq + 7) / 8 + (lk.width > 1 ? (lk.n_inputs + 1) * n : 0);
    return (A + k->n_instance + k->trash.size()) * (2 * n + E) + S * (3 * n + E) +
           L * ((3 * n + E) + (3 * n + E)) + k->n_helpers * (2 * n + E) + k->lk_exprs.size() * (n + E) +
           k->qdeg * n + (4 + 3 * O) * n + k->n_blinds + counts;
}

Status eval_many(Context* ctx, const std::vector<EvalTask>& in, std::vector<Fr4>& results, cudaStream_t st) {
    results.assign(in.size(), host::fr_zero());
    if (in.empty()) return OK;
    // level sizes: level l of task t has ceil(len / 2048^l) values; the last
    // level with more than one value writes into the results slot
    std::vector<uint64_t> cur_len(in.size());
    std::vector<Fr4> point(in.size());
    size_t scratch = 0;
    for (size_t t = 0; t < in.size(); t++) {
        cur_len[t] = in[t].len;
        std::memcpy(point[t].l, in[t].pw[0].l, 32);
        uint64_t len = in[t].len;
        while (len > kEvalSeg) {
            len = (len + kEvalSeg - 1) / kEvalSeg;
            scratch += len;
        }
    }
    void *d_res, *d_seg, *d_tab;
    MZK_TRY(ctx->ensure("fs_eval_res", in.size() * sizeof(Fr), &d_res));
    MZK_TRY(ctx->ensure("fs_eval_seg", std::max<size_t>(scratch, 1) * sizeof(Fr), &d_seg));
    MZK_TRY(ctx->ensure("fs_eval_tab", in.size() * sizeof(EvalTask), &d_tab));
    MZK_CUDA_CHECK(cudaMemsetAsync(d_res, 0, in.size() * sizeof(Fr), st));
    Fr* seg = static_cast<Fr*>(d_seg);
    std::vector<const Fr*> src(in.size());
    for (size_t t = 0; t < in.size(); t++) src[t] = in[t].poly;
    for (;;) {
        std::vector<EvalTask> lvl;
        uint32_t max_blocks = 0;
        for (size_t t = 0; t < in.size(); t++) {
            if (cur_len[t] == 0) continue;
            EvalTask e{};
            e.poly = src[t];
            e.len = cur_len[t];
            const uint64_t blocks = (cur_len[t] + kEvalSeg - 1) / kEvalSeg;
            Fr* dst = blocks == 1 ? static_cast<Fr*>(d_res) + t : seg;
            if (blocks > 1) seg += blocks;
            e.seg_out = dst;
            Fr4 p = point[t];
            e.pw[0] = to_dev(p);
            Fr4 p8 = host::fr_pow_u64(p, 8);
            for (int l = 0; l < 8; l++) {
                e.pw[1 + l] = to_dev(p8);
                p8 = host::fr_mul(p8, p8);
            }
            lvl.push_back(e);
            max_blocks = std::max<uint32_t>(max_blocks, (uint32_t)blocks);
            // the next level evaluates the segment sums at point^2048
            src[t] = dst;
            point[t] = host::fr_pow_u64(p, kEvalSeg);
            cur_len[t] = blocks == 1 ? 0 : blocks;
        }
        if (lvl.empty()) break;
        MZK_TRY(ctx->ensure("fs_eval_tab", lvl.size() * sizeof(EvalTask), &d_tab));
        MZK_CUDA_CHECK(cudaMemcpyAsync(d_tab, lvl.data(), lvl.size() * sizeof(EvalTask), cudaMemcpyHostToDevice, st));
        k_eval_segments<<<dim3(max_blocks, (uint32_t)lvl.size()), kThreads, 0, st>>>(
            static_cast<const EvalTask*>(d_tab));
        MZK_LAUNCH_CHECK(ctx);
        // the task table is read by the kernel: the next level's upload waits for it
        MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    }
    MZK_CUDA_CHECK(cudaMemcpyAsync(results.data(), d_res, in.size() * 32, cudaMemcpyDeviceToHost, st));
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    return OK;
}

EvalTask eval_task(const Fr* p, uint64_t len, const Fr4& point) {
    EvalTask e{};
    e.poly = p;
    e.len = len;
    e.pw[0] = to_dev(point);
    return e;
}

struct LinSpec {
    Fr* out;
    uint64_t len;
    std::vector<LinTerm> terms;
};

Status lincomb_many(Context* ctx, const std::vector<LinSpec>& specs, cudaStream_t st) {
    if (specs.empty()) return OK;
    std::vector<LinOut> outs;
    std::vector<LinTerm> terms;
    uint64_t max_len = 0;
    for (auto& s : specs) {
        outs.push_back({s.out, s.len, (uint32_t)terms.size(), (uint32_t)s.terms.size()});
        terms.insert(terms.end(), s.terms.begin(), s.terms.end());
        max_len = std::max(max_len, s.len);
    }
    void* d_tab;
    const size_t ob = outs.size() * sizeof(LinOut), tb = terms.size() * sizeof(LinTerm);
    MZK_TRY(ctx->ensure("fs_lin_tab", ob + tb + 16, &d_tab));
    std::vector<uint8_t> h(ob + tb);
    std::memcpy(h.data(), outs.data(), ob);
    std::memcpy(h.data() + ob, terms.data(), tb);
    MZK_CUDA_CHECK(cudaMemcpyAsync(d_tab, h.data(), h.size(), cudaMemcpyHostToDevice, st));
    const uint32_t gx = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>((max_len + kThreads - 1) / kThreads, (uint64_t)ctx->num_sms * 4));
    k_lincomb<<<dim3(gx, (uint32_t)outs.size()), kThreads, 0, st>>>(
        static_cast<const LinOut*>(d_tab), reinterpret_cast<const LinTerm*>(static_cast<uint8_t*>(d_tab) + ob));
    MZK_LAUNCH_CHECK(ctx);
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));  // the table buffer is reused by the next call
    return OK;
}

// the identities of partially_evaluate_identities (plonk/mod.rs:502-608) in
// order, each with the fixed column of its simple selector (-1: none, the
// identity is fully evaluated); a simple selector's evaluation is one here
// (ev_fix holds one for its queries)
std::vector<std::pair<int32_t, Fr4>> identities_at_x(const FsProof& p) {
    using namespace host;
    const PlonkKey* k = p.key;
    const Domain* d = k->dom;
    const Fr4 one = host::fr_one();
    auto adv = [&](uint32_t col) {
        for (size_t i = 0; i < k->advice_queries.size(); i++)
            if (k->advice_queries[i].column == col && k->advice_queries[i].rotation == 0) return p.ev_adv[i];
        return host::fr_zero();
    };
    auto fix = [&](uint32_t col) {
        for (size_t i = 0; i < k->fixed_queries.size(); i++)
            if (k->fixed_queries[i].column == col && k->fixed_queries[i].rotation == 0) return p.ev_fix[i];
        return host::fr_zero();
    };
    auto ins = [&](uint32_t col) {
        for (size_t i = 0; i < k->instance_queries.size(); i++)
            if (k->instance_queries[i].column == col && k->instance_queries[i].rotation == 0) return p.ev_inst[i];
        return host::fr_zero();
    };
    std::vector<std::pair<int32_t, Fr4>> ids;
    // a flattened program at x: each read is the evaluation of its query
    // (partially_evaluate_identities evaluates the same expressions)
    auto program_at_x = [&](const mzk_flat_graph& g) {
        std::vector<Fr4> val(g.values_len, host::fr_zero());
        for (uint32_t i = 0; i < g.n_constants; i++) std::memcpy(val[i].l, g.constants + 4 * (size_t)i, 32);
        val[g.beta_idx] = p.beta;
        val[g.theta_idx] = p.theta;
        val[g.trash_challenge_idx] = p.trash;
        val[g.y_idx] = p.y;
        val[g.previous_value_idx] = host::fr_zero();
        for (uint32_t i = 0; i < g.n_reads; i++) {
            const mzk_column_read& r = g.reads[i];
            const auto& qs = r.col_type == 0 ? k->fixed_queries : r.col_type == 1 ? k->advice_queries
                                                                                   : k->instance_queries;
            const auto& ev = r.col_type == 0 ? p.ev_fix : r.col_type == 1 ? p.ev_adv : p.ev_inst;
            for (size_t j = 0; j < qs.size(); j++)
                if (qs[j].column == r.col_idx && qs[j].rotation == g.rotations[r.rot_idx]) val[r.dst] = ev[j];
        }
        for (uint32_t i = 0; i < g.n_ops; i++) {
            const mzk_flat_op& o = g.ops[i];
            const Fr4 &x = val[o.a], &y2 = val[o.b], &z = val[o.c];
            switch (o.kind) {
                case MZK_FLAT_ADD: val[o.dst] = fr_add(x, y2); break;
                case MZK_FLAT_SUB: val[o.dst] = fr_sub(x, y2); break;
                case MZK_FLAT_MUL: val[o.dst] = fr_mul(x, y2); break;
                case MZK_FLAT_SQUARE: val[o.dst] = fr_mul(x, x); break;
                case MZK_FLAT_DOUBLE: val[o.dst] = fr_add(x, x); break;
                case MZK_FLAT_NEGATE: val[o.dst] = fr_neg(x); break;
                default: val[o.dst] = fr_add(fr_mul(x, y2), z); break;
            }
        }
        return val;
    };
    if (k->has_gates) {
        const std::vector<Fr4> val = program_at_x(k->gates);
        if (k->gate_poly_values.empty()) {
            ids.push_back({-1, val[k->gates.result_idx]});  // all gate polynomials, already folded in y
        } else {
            for (size_t i = 0; i < k->gate_poly_values.size(); i++)
                ids.push_back({k->gate_poly_selector[i], val[k->gate_poly_values[i]]});
        }
    } else {
        // the standard gate
        const Fr4 a = adv(k->gate_advice[0]), b = adv(k->gate_advice[1]), c = adv(k->gate_advice[2]);
        Fr4 g = fr_mul(fix(k->gate_fixed[0]), a);
        g = fr_add(g, fr_mul(fix(k->gate_fixed[1]), b));
        g = fr_add(g, fr_mul(fr_mul(fix(k->gate_fixed[2]), a), b));
        g = fr_add(g, fr_mul(fix(k->gate_fixed[3]), c));
        g = fr_add(g, fix(k->gate_fixed[4]));
        ids.push_back({-1, g});
    }
    // l_last, l_blind, l_0 (l_i_range over -(bf + 1) ..= 0)
    const int32_t bf = (int32_t)k->bf;
    const Fr4 l_last = l_i(d, p.x, p.xn, -(bf + 1));
    Fr4 l_blind = host::fr_zero();
    for (int32_t i = -bf; i <= -1; i++) l_blind = fr_add(l_blind, l_i(d, p.x, p.xn, i));
    const Fr4 l_0 = l_i(d, p.x, p.xn, 0);
    const Fr4 active = fr_sub(one, fr_add(l_last, l_blind));
    // permutation (permutation.rs:195-290)
    const uint32_t S = k->n_sets;
    if (S) {
        auto z = [&](uint32_t s, int which) { return p.ev_sets[3 * s + which]; };
        ids.push_back({-1, fr_mul(l_0, fr_sub(one, z(0, 0)))});
        ids.push_back({-1, fr_mul(fr_sub(fr_mul(z(S - 1, 0), z(S - 1, 0)), z(S - 1, 0)), l_last)});
        for (uint32_t s = 1; s < S; s++) ids.push_back({-1, fr_mul(fr_sub(z(s, 0), z(s - 1, 2)), l_0)});
        Fr4 delta;
        std::memcpy(delta.l, host::FR_DELTA4, 32);
        for (uint32_t s = 0; s < S; s++) {
            const uint32_t c0 = s * k->chunk, c1 = std::min(k->n_perm, c0 + k->chunk);
            Fr4 left = z(s, 1), right = z(s, 0);
            Fr4 cur = fr_mul(fr_mul(p.beta, p.x), fr_pow_u64(delta, c0));
            for (uint32_t ci = c0; ci < c1; ci++) {
                const uint32_t kind = k->perm_kind[ci], col = k->perm_index[ci];
                const Fr4 e = kind == 0 ? adv(col) : kind == 1 ? fix(col) : ins(col);
                left = fr_mul(left, fr_add(fr_add(e, fr_mul(p.beta, p.ev_pc[ci])), p.gamma));
                right = fr_mul(right, fr_add(fr_add(e, cur), p.gamma));
                cur = fr_mul(cur, delta);
            }
            ids.push_back({-1, fr_mul(fr_sub(left, right), active)});
        }
    }
    // the lookups (Evaluated::expressions, logup.rs:405-485): the boundary,
    // one helper constraint per chunk of input tuples (each a column or a
    // theta-compressed tuple of columns), the accumulator
    for (size_t l = 0, e0 = 0; l < k->lookups.size(); l++) {
        const PlonkKey::Lookup& lk = k->lookups[l];
        const mzk_lookup_shape& sh = lk.shape;
        const uint32_t H = lk.n_helpers();
        const Fr4 m = p.ev_lk[e0], Z = p.ev_lk[e0 + 1 + H], Zn = p.ev_lk[e0 + 2 + H];
        Fr4 t = host::fr_zero();
        for (uint32_t e = 0; e < lk.width; e++) t = fr_add(fr_mul(t, p.theta), fix(lk.tab[e]));
        const Fr4 sel = sh.selector_fixed >= 0 ? fix((uint32_t)sh.selector_fixed) : one;
        ids.push_back({-1, fr_mul(fr_add(l_0, l_last), Z)});
        Fr4 sum_h = host::fr_zero();
        for (uint32_t c = 0; c < H; c++) {
            const Fr4 h = p.ev_lk[e0 + 1 + c];
            std::vector<Fr4> fb;
            for (uint32_t j = c * lk.per_helper; j < c * lk.per_helper + lk.chunk_inputs(c); j++) {
                Fr4 f = host::fr_zero();
                for (uint32_t e = 0; e < lk.width; e++) {
                    const int32_t x = lk.expr[j][e];
                    const Fr4 v = x >= 0 ? program_at_x(k->lk_exprs[x].g)[k->lk_exprs[x].g.result_idx] : adv(lk.in[j][e]);
                    f = fr_add(fr_mul(f, p.theta), v);
                }
                fb.push_back(fr_add(f, p.beta));
            }
            Fr4 product = one, spp = host::fr_zero();
            for (size_t j = 0; j < fb.size(); j++) {
                Fr4 partial = one;
                for (size_t i = 0; i < fb.size(); i++)
                    if (i != j) partial = fr_mul(partial, fb[i]);
                spp = fr_add(spp, partial);
                product = fr_mul(product, fb[j]);
            }
            ids.push_back({-1, fr_sub(fr_mul(h, product), spp)});
            sum_h = fr_add(sum_h, h);
        }
        Fr4 acc = fr_sub(fr_sub(Zn, Z), fr_mul(sel, sum_h));
        acc = fr_add(fr_mul(acc, fr_add(t, p.beta)), m);
        ids.push_back({-1, fr_mul(acc, active)});
        e0 += 3 + H;
    }
    // the trashcans (trash.rs:60-86): compressed - (1 - q) trash
    for (size_t t = 0; t < k->trash.size(); t++) {
        const Fr4 compressed = program_at_x(k->trash[t].program)[k->trash[t].program.result_idx];
        const Fr4 q = fix(k->trash[t].selector);
        ids.push_back({-1, fr_sub(compressed, fr_mul(fr_sub(one, q), p.ev_trash[t]))});
    }
    return ids;
}

// compute_linearization_poly's split (linearization/prover.rs:41-86): the
// identity j of M gets y^(M-1-j); fully evaluated identities add up to the
// constant C, the others scale their selector's fixed polynomial in L'(X)
Fr4 linearization_split(const std::vector<std::pair<int32_t, Fr4>>& ids, const Fr4& y,
                        std::vector<std::pair<uint32_t, Fr4>>* selector_terms) {
    using namespace host;
    Fr4 c = host::fr_zero(), pw = host::fr_one();
    for (size_t j = ids.size(); j-- > 0;) {
        const Fr4 v = fr_mul(pw, ids[j].second);
        if (ids[j].first < 0) c = fr_add(c, v);
        else if (selector_terms) selector_terms->push_back({(uint32_t)ids[j].first, v});
        pw = fr_mul(pw, y);
    }
    return c;
}

const Fr* open_poly(const FsProof& p, std::pair<int, uint32_t> id) {
    const PlonkKey* k = p.key;
    switch (id.first) {
        case PlonkKey::P_ADVICE: return p.adv_coeff[id.second];
        case PlonkKey::P_PERM_Z: return p.z_coeff[id.second];
        case PlonkKey::P_M: return p.m_coeff[id.second];
        case PlonkKey::P_H: return p.h_coeff[id.second];
        case PlonkKey::P_AGG: return p.Z_coeff[id.second];
        case PlonkKey::P_FIXED: return k->fixed_coeff[id.second];
        case PlonkKey::P_PERM_FIXED: return k->perm_coeff[id.second];
        case PlonkKey::P_TRASH: return p.trash_coeff[id.second];
        default: return p.lin;
    }
}

}  // namespace

// device bytes one proof of `key` takes in a call: its carved buffers plus
// the sorted MSM entries it adds to the largest batched MSM of a phase
uint64_t proof_device_bytes(const mzk_plonk_key* key) {
    const PlonkKey* k = reinterpret_cast<const PlonkKey*>(key);
    const uint64_t msm_entries = (uint64_t)std::max<uint32_t>(k->n_advice, k->qdeg) * k->n * 20;
    return (proof_scratch_elems(k) + 8) * sizeof(Fr) + msm_entries * 4;
}

uint64_t proof_rows(const mzk_plonk_key* key) { return reinterpret_cast<const PlonkKey*>(key)->n; }

Status create_proofs(Context* ctx, const mzk_proof_request* reqs, size_t count, uint32_t flags, cudaStream_t st) {
    using namespace host;
    if (count == 0) return OK;
    const PlonkKey* k0 = reinterpret_cast<const PlonkKey*>(reqs[0].key);
    if (!k0) {
        set_error("create_proof: null key");
        return ERR_ARG;
    }
    const mzk_srs_desc srs = k0->srs;
    for (size_t j = 0; j < count; j++) {
        const PlonkKey* k = reinterpret_cast<const PlonkKey*>(reqs[j].key);
        if (!k || !reqs[j].advice || !reqs[j].blinds || !reqs[j].proof_out) {
            set_error("create_proof: null argument in request " + std::to_string(j));
            return ERR_ARG;
        }
        if (k->srs.srs != srs.srs || k->srs.srs_len != srs.srs_len || k->srs.table_c != srs.table_c) {
            set_error("create_proof: all keys of one call must share one SRS buffer");
            return ERR_ARG;
        }
        for (uint32_t i = 0; i < k->n_advice; i++)
            if (!reqs[j].advice[i]) {
                set_error("create_proof: null advice column in request " + std::to_string(j));
                return ERR_ARG;
            }
        if (k->n_instance && (!reqs[j].instance || !reqs[j].instance_len)) {
            set_error("create_proof: request " + std::to_string(j) + " has no instance columns");
            return ERR_ARG;
        }
        for (uint32_t i = 0; i < k->n_instance; i++) {
            if (reqs[j].instance_len[i] > k->u) {  // Error::InstanceTooLarge (prover.rs:500-502)
                set_error("create_proof: request " + std::to_string(j) + ": instance column " + std::to_string(i) +
                          " has more values than usable rows");
                return ERR_ARG;
            }
            if (reqs[j].instance_len[i] && !reqs[j].instance[i]) {
                set_error("create_proof: null instance column in request " + std::to_string(j));
                return ERR_ARG;
            }
        }
    }
    MsmTable table{srs.srs, srs.srs_len, srs.table_c, srs.table_rows, srs.table_min_n};
    const MsmTable* tab = srs.table_c > 0 ? &table : nullptr;
    // wall time per phase (each ends with a stream sync)
    using clock = std::chrono::steady_clock;
    auto t_phase = clock::now();
    auto phase_done = [&](int ph) {
        const auto t = clock::now();
        ctx->prove_ms[ph] += std::chrono::duration<double, std::milli>(t - t_phase).count();
        t_phase = t;
    };
    ctx->prove_calls++;
    // scratch: every proof's buffers carved from one device buffer
    size_t total = 0, max_E = 0;
    for (size_t j = 0; j < count; j++) {
        const PlonkKey* k = reinterpret_cast<const PlonkKey*>(reqs[j].key);
        total += proof_scratch_elems(k) + 8;
        max_E = std::max<size_t>(max_E, (size_t)1 << k->dom->ext_k);
    }
    void *wave, *hbuf, *dbl, *dmiss;
    MZK_TRY(ctx->ensure("fs_wave", total * sizeof(Fr), &wave));
    MZK_TRY(ctx->ensure("fs_hbuf", max_E * sizeof(Fr), &hbuf));
    MZK_TRY(ctx->ensure("fs_qblinds", 16 * sizeof(Fr), &dbl));
    MZK_TRY(ctx->ensure("fs_missing", count * 4, &dmiss));
    std::vector<FsProof> ps(count);
    Fr* carve = static_cast<Fr*>(wave);
    auto take = [&](size_t elems) {
        Fr* p = carve;
        carve += elems;
        return p;
    };
    for (size_t j = 0; j < count; j++) {
        FsProof& p = ps[j];
        p.req = &reqs[j];
        p.key = reinterpret_cast<const PlonkKey*>(reqs[j].key);
        const PlonkKey* k = p.key;
        const size_t n = k->n, E = (size_t)1 << k->dom->ext_k;
        Fr* start = carve;
        for (uint32_t i = 0; i < k->n_advice; i++) {
            p.adv_lag.push_back(take(n));
            p.adv_coeff.push_back(take(n));
            p.adv_ext.push_back(take(E));
        }
        for (uint32_t i = 0; i < k->n_instance; i++) {
            p.inst_lag.push_back(take(n));
            p.inst_coeff.push_back(take(n));
            p.inst_ext.push_back(take(E));
        }
        for (size_t t = 0; t < k->trash.size(); t++) {
            p.trash_lag.push_back(take(n));
            p.trash_coeff.push_back(take(n));
            p.trash_ext.push_back(take(E));
        }
        for (uint32_t s = 0; s < k->n_sets; s++) {
            p.z_lag.push_back(take(n));
            p.z_delta.push_back(take(n));
            p.z_coeff.push_back(take(n));
            p.z_ext.push_back(take(E));
        }
        for (size_t l = 0; l < k->lookups.size(); l++) {
            p.m_lag.push_back(take(n)), p.m_delta.push_back(take(n)), p.m_coeff.push_back(take(n));
            p.m_ext.push_back(take(E));
            p.Z_lag.push_back(take(n)), p.Z_dd.push_back(take(n)), p.Z_coeff.push_back(take(n));
            p.Z_ext.push_back(take(E));
            const PlonkKey::Lookup& lk = k->lookups[l];
            p.f_lag.emplace_back();
            for (uint32_t j = 0; lk.width > 1 && j < lk.n_inputs; j++) p.f_lag.back().push_back(take(n));
            p.t_lag.push_back(lk.width > 1 ? take(n) : nullptr);
        }
        for (uint32_t h = 0; h < k->n_helpers; h++)
            p.h_lag.push_back(take(n)), p.h_coeff.push_back(take(n)), p.h_ext.push_back(take(E));
        for (size_t x = 0; x < k->lk_exprs.size(); x++) p.e_lag.push_back(take(n)), p.e_ext.push_back(take(E));
        p.limbs = take((size_t)k->qdeg * n);
        p.lin = take(n), p.f = take(n), p.fin = take(n), p.pi = take(n);
        for (size_t s = 0; s < k->open_sets.size(); s++) {
            p.q.push_back(take(n));
            p.fdiv.push_back(take(n));
            p.qt.push_back(take(n));
        }
        p.d_blinds = take(k->n_blinds);
        for (const auto& lk : k->lookups) p.counts.push_back(reinterpret_cast<uint32_t*>(take((lk.n_uniq + 7) / 8)));
        carve = start + proof_scratch_elems(k) + 8;
        const size_t A = k->n_advice, L = k->lookups.size();
        p.off_mult = A * (k->bf + 1);
        p.off_perm = p.off_mult + L * (k->bf + 1);
        p.off_logup = p.off_perm + (size_t)k->n_sets * k->bf;
        p.off_quot = p.off_logup + L * k->bf;
        MZK_CUDA_CHECK(cudaMemcpyAsync(p.d_blinds, reqs[j].blinds, k->n_blinds * sizeof(Fr), cudaMemcpyHostToDevice,
                                       st));
        p.tr.common_fr(k->repr);  // vk.hash_into (prover.rs:101)
        // compute_instances (prover.rs:475-539): each instance column's length
        // and values go into the transcript; its Lagrange form is the values
        // padded with zeros
        for (uint32_t i = 0; i < k->n_instance; i++) {
            const uint64_t len = reqs[j].instance_len[i];
            p.tr.common_fr(fr_from_u64(len));
            for (uint64_t v = 0; v < len; v++) {
                Fr4 x;
                std::memcpy(x.l, reqs[j].instance[i] + 4 * v, 32);
                p.tr.common_fr(x);
            }
            MZK_CUDA_CHECK(cudaMemsetAsync(p.inst_lag[i], 0, n * sizeof(Fr), st));
            if (len)
                MZK_CUDA_CHECK(cudaMemcpyAsync(p.inst_lag[i], reqs[j].instance[i], len * sizeof(Fr),
                                               cudaMemcpyHostToDevice, st));
        }
    }
    auto write_points = [&](FsProof& p, const uint64_t* res, size_t m) {
        for (size_t i = 0; i < m; i++) p.tr.write_point(res + 18 * i);
    };
    std::vector<BatchItem> items;
    std::vector<uint64_t> res;
    auto msm = [&]() -> Status {
        res.assign(items.size() * 18, 0);
        MZK_CUDA_CHECK(cudaStreamSynchronize(st));  // the MSM time below is the MSMs' own
        const auto t0 = clock::now();
        if (!items.empty()) MZK_TRY(run_msms(ctx, srs.srs, srs.srs_len, items, res.data(), flags, tab, st));
        MZK_CUDA_CHECK(cudaStreamSynchronize(st));
        ctx->prove_ms[9] += std::chrono::duration<double, std::milli>(clock::now() - t0).count();
        return OK;
    };
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    phase_done(0);
    // ---- 1. advice (parse_advices, prover.rs:604-627), theta -------------
    items.clear();
    for (auto& p : ps) {
        const PlonkKey* k = p.key;
        const size_t n = k->n, u = k->u;
        for (uint32_t i = 0; i < k->n_advice; i++) {
            MZK_CUDA_CHECK(cudaMemcpyAsync(p.adv_lag[i], p.req->advice[i], u * sizeof(Fr),
                                           p.req->advice_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                           st));
            MZK_CUDA_CHECK(cudaMemcpyAsync(p.adv_lag[i] + u, p.d_blinds + (size_t)i * (k->bf + 1),
                                           (n - u) * sizeof(Fr), cudaMemcpyDeviceToDevice, st));
            items.push_back({p.adv_lag[i], k->srs.off_lagrange, n});
        }
    }
    MZK_TRY(msm());
    for (size_t j = 0, at = 0; j < count; j++) {
        write_points(ps[j], &res[18 * at], ps[j].key->n_advice);
        at += ps[j].key->n_advice;
        ps[j].theta = ps[j].tr.squeeze();
    }
    phase_done(1);
    // ---- 2. multiplicities, beta, gamma ---------------------------------
    items.clear();
    MZK_CUDA_CHECK(cudaMemsetAsync(dmiss, 0, count * 4, st));
    static const uint64_t kZero4[4] = {0, 0, 0, 0};
    for (size_t j = 0; j < count; j++) {
        FsProof& p = ps[j];
        const PlonkKey* k = p.key;
        const uint32_t n = k->n, u = k->u;
        // the lookup input expressions at every row (evaluate over n rows,
        // rotations wrapping, as compute_multiplicities_parallel does)
        if (!k->lk_exprs.empty()) {
            std::vector<const uint64_t*> fl(k->n_fixed), al(k->n_advice), il(k->n_instance);
            for (uint32_t i = 0; i < k->n_fixed; i++) fl[i] = reinterpret_cast<const uint64_t*>(k->fixed_lag[i]);
            for (uint32_t i = 0; i < k->n_advice; i++) al[i] = reinterpret_cast<const uint64_t*>(p.adv_lag[i]);
            for (uint32_t i = 0; i < k->n_instance; i++) il[i] = reinterpret_cast<const uint64_t*>(p.inst_lag[i]);
            for (size_t x = 0; x < k->lk_exprs.size(); x++)
                MZK_TRY(flat_program_rows(ctx, k->dom, k->lk_exprs[x].g, fl.data(), k->n_fixed, al.data(), k->n_advice,
                                          il.data(), k->n_instance, kZero4, p.theta.l, kZero4, kZero4,
                                          reinterpret_cast<uint64_t*>(p.e_lag[x]), st));
        }
        for (size_t l = 0; l < k->lookups.size(); l++) {
            const PlonkKey::Lookup& lk = k->lookups[l];
            const Fr* sel = lk.shape.selector_fixed >= 0 ? k->fixed_lag[lk.shape.selector_fixed] : nullptr;
            MZK_CUDA_CHECK(cudaMemsetAsync(p.counts[l], 0, (size_t)lk.n_uniq * 4, st));
            for (uint32_t i = 0; i < lk.n_inputs; i++) {  // every input tuple counts into one m
                LookupInputs li{};
                li.width = lk.width;
                for (uint32_t e = 0; e < lk.width; e++) li.col[e] = lookup_input_lag(p, lk, i, e);
                k_lookup_count<<<grid_of(ctx, u), kThreads, 0, st>>>(li, sel, u, lk.uniq, lk.n_uniq, p.counts[l],
                                                                     static_cast<uint32_t*>(dmiss) + j);
                MZK_LAUNCH_CHECK(ctx);
            }
            k_lookup_m<<<grid_of(ctx, u), kThreads, 0, st>>>(p.m_lag[l], lk.uid, p.counts[l], lk.tinv, u);
            MZK_LAUNCH_CHECK(ctx);
            MZK_CUDA_CHECK(cudaMemcpyAsync(p.m_lag[l] + u, p.d_blinds + p.off_mult + l * (k->bf + 1),
                                           (size_t)(n - u) * sizeof(Fr), cudaMemcpyDeviceToDevice, st));
            MZK_TRY(delta_device(ctx, p.m_lag[l], p.m_delta[l], n, 1, st));
            items.push_back({p.m_delta[l], k->srs.off_lagrange_delta, n});
        }
    }
    MZK_TRY(msm());
    {
        std::vector<uint32_t> miss(count);
        MZK_CUDA_CHECK(cudaMemcpy(miss.data(), dmiss, count * 4, cudaMemcpyDeviceToHost));
        for (size_t j = 0; j < count; j++)
            if (miss[j]) {
                set_error("create_proof: request " + std::to_string(j) + ": a lookup input value is not in the table");
                return ERR_ARG;
            }
    }
    for (size_t j = 0, at = 0; j < count; j++) {
        FsProof& p = ps[j];
        write_points(p, &res[18 * at], p.key->lookups.size());
        at += p.key->lookups.size();
        p.beta = p.tr.squeeze();
        p.gamma = p.tr.squeeze();
    }
    phase_done(2);
    // ---- 3. permutation products, logup helper and aggregator, trash, y --
    // a tuple lookup's input tuples and table, compressed with theta (Horner
    // in the tuple's order: the first column gets theta^(w-1)), in the
    // Lagrange basis
    {
        std::vector<LinSpec> comp;
        for (auto& p : ps) {
            const PlonkKey* k = p.key;
            for (size_t l = 0; l < k->lookups.size(); l++) {
                const PlonkKey::Lookup& lk = k->lookups[l];
                if (lk.width < 2) continue;
                std::vector<Fr> pw(lk.width);
                Fr4 w = host::fr_one();
                for (uint32_t e = lk.width; e-- > 0;) pw[e] = to_dev(w), w = fr_mul(w, p.theta);
                LinSpec ts{p.t_lag[l], k->n, {}};
                for (uint32_t e = 0; e < lk.width; e++) ts.terms.push_back({k->fixed_lag[lk.tab[e]], k->n, pw[e]});
                comp.push_back(ts);
                for (uint32_t i = 0; i < lk.n_inputs; i++) {
                    LinSpec fs{p.f_lag[l][i], k->n, {}};
                    for (uint32_t e = 0; e < lk.width; e++) fs.terms.push_back({lookup_input_lag(p, lk, i, e), k->n, pw[e]});
                    comp.push_back(fs);
                }
            }
        }
        MZK_TRY(lincomb_many(ctx, comp, st));
    }
    items.clear();
    for (auto& p : ps) {
        const PlonkKey* k = p.key;
        const uint32_t n = k->n;
        if (k->n_sets) {
            std::vector<const uint64_t*> vals(k->n_perm), sig(k->n_perm);
            for (uint32_t c = 0; c < k->n_perm; c++) {
                const uint32_t kind = k->perm_kind[c], col = k->perm_index[c];
                vals[c] = reinterpret_cast<const uint64_t*>(kind == 0   ? p.adv_lag[col]
                                                            : kind == 1 ? k->fixed_lag[col]
                                                                        : p.inst_lag[col]);
                sig[c] = reinterpret_cast<const uint64_t*>(k->perm_lag[c]);
            }
            std::vector<uint64_t*> zo(k->n_sets);
            for (uint32_t s = 0; s < k->n_sets; s++) zo[s] = reinterpret_cast<uint64_t*>(p.z_lag[s]);
            mzk_permutation_desc pd;
            std::memset(&pd, 0, sizeof(pd));
            pd.n_cols = k->n_perm;
            pd.values = vals.data();
            pd.sigmas = sig.data();
            pd.chunk_len = k->chunk;
            pd.blinding_factors = k->bf;
            pd.blinds = p.req->blinds + 4 * p.off_perm;
            std::memcpy(pd.beta, p.beta.l, 32);
            std::memcpy(pd.gamma, p.gamma.l, 32);
            pd.z_out = zo.data();
            MZK_TRY(permutation_z_device(ctx, k->dom, &pd, st));
            for (uint32_t s = 0; s < k->n_sets; s++) {
                MZK_TRY(delta_device(ctx, p.z_lag[s], p.z_delta[s], n, 1, st));
                items.push_back({p.z_delta[s], k->srs.off_lagrange_delta, n});
            }
        }
        for (size_t l = 0; l < k->lookups.size(); l++) {
            const PlonkKey::Lookup& lk = k->lookups[l];
            const mzk_lookup_shape& sh = lk.shape;
            const bool tuple = lk.width > 1;
            const uint32_t H = lk.n_helpers();
            std::vector<const uint64_t*> in(lk.n_inputs);
            for (uint32_t i = 0; i < lk.n_inputs; i++)
                in[i] = reinterpret_cast<const uint64_t*>(tuple ? p.f_lag[l][i] : lookup_input_lag(p, lk, i, 0));
            std::vector<uint64_t*> ho(H);
            std::vector<uint32_t> cols(H);
            for (uint32_t c = 0; c < H; c++) {
                ho[c] = reinterpret_cast<uint64_t*>(p.h_lag[lk.h0 + c]);
                cols[c] = lk.chunk_inputs(c);
            }
            mzk_logup_desc ld;
            std::memset(&ld, 0, sizeof(ld));
            ld.n_chunks = H;
            ld.chunk_cols = cols.data();
            ld.inputs = in.data();
            ld.table = reinterpret_cast<const uint64_t*>(tuple ? p.t_lag[l] : k->fixed_lag[sh.table_fixed]);
            ld.selector = reinterpret_cast<const uint64_t*>(sh.selector_fixed >= 0 ? k->fixed_lag[sh.selector_fixed]
                                                                                     : k->ones);
            ld.multiplicities = reinterpret_cast<const uint64_t*>(p.m_lag[l]);
            ld.blinding_factors = k->bf;
            ld.blinds = p.req->blinds + 4 * (p.off_logup + l * k->bf);
            std::memcpy(ld.beta, p.beta.l, 32);
            ld.helpers_out = ho.data();
            ld.aggregator_out = reinterpret_cast<uint64_t*>(p.Z_lag[l]);
            MZK_TRY(logup_device(ctx, k->dom, &ld, st));
            MZK_TRY(delta_device(ctx, p.Z_lag[l], p.Z_dd[l], n, 2, st));
            // per lookup its helpers, then its aggregator (prover.rs:221-227)
            for (uint32_t c = 0; c < H; c++) items.push_back({p.h_lag[lk.h0 + c], k->srs.off_lagrange, n});
            items.push_back({p.Z_dd[l], k->srs.off_lagrange_double_delta, n});
        }
    }
    MZK_TRY(msm());
    for (size_t j = 0, at = 0; j < count; j++) {
        FsProof& p = ps[j];
        const size_t m = p.key->n_sets + p.key->n_helpers + p.key->lookups.size();
        write_points(p, &res[18 * at], m);
        at += m;
        p.trash = p.tr.squeeze();
    }
    // y is not drawn yet: a trash program reads no y slot (its slot is zero)
    static const uint64_t kNoY[4] = {0, 0, 0, 0};
    // the trash columns (trash/prover.rs:29-77): each trashcan's constraint
    // expressions over the Lagrange columns, compressed with the trash
    // challenge, committed in the Lagrange basis; then y
    items.clear();
    for (auto& p : ps) {
        const PlonkKey* k = p.key;
        if (k->trash.empty()) continue;
        std::vector<const uint64_t*> fl(k->n_fixed), al(k->n_advice), il(k->n_instance);
        for (uint32_t i = 0; i < k->n_fixed; i++) fl[i] = reinterpret_cast<const uint64_t*>(k->fixed_lag[i]);
        for (uint32_t i = 0; i < k->n_advice; i++) al[i] = reinterpret_cast<const uint64_t*>(p.adv_lag[i]);
        for (uint32_t i = 0; i < k->n_instance; i++) il[i] = reinterpret_cast<const uint64_t*>(p.inst_lag[i]);
        for (size_t t = 0; t < k->trash.size(); t++) {
            MZK_TRY(flat_program_rows(ctx, k->dom, k->trash[t].program, fl.data(), k->n_fixed, al.data(), k->n_advice,
                                      il.data(), k->n_instance, p.beta.l, p.theta.l, p.trash.l, kNoY,
                                      reinterpret_cast<uint64_t*>(p.trash_lag[t]), st));
            items.push_back({p.trash_lag[t], k->srs.off_lagrange, k->n});
        }
    }
    if (!items.empty()) MZK_TRY(msm());
    for (size_t j = 0, at = 0; j < count; j++) {
        FsProof& p = ps[j];
        write_points(p, &res[18 * at], p.key->trash.size());
        at += p.key->trash.size();
        p.y = p.tr.squeeze();
    }
    phase_done(3);
    // ---- 4. cosets, quotient limbs, x -------------------------------------
    items.clear();
    // every polynomial of a proof that the quotient reads on the extended
    // coset: Lagrange -> coefficients -> coset
    auto ntt_lists = [](const FsProof& p, std::vector<const void*>& lag, std::vector<Fr*>& co,
                        std::vector<Fr*>& ex) {
        const PlonkKey* k = p.key;
        for (uint32_t i = 0; i < k->n_advice; i++) {
            lag.push_back(p.adv_lag[i]);
            co.push_back(p.adv_coeff[i]);
            ex.push_back(p.adv_ext[i]);
        }
        for (uint32_t i = 0; i < k->n_instance; i++) {
            lag.push_back(p.inst_lag[i]);
            co.push_back(p.inst_coeff[i]);
            ex.push_back(p.inst_ext[i]);
        }
        for (size_t t = 0; t < k->trash.size(); t++) {
            lag.push_back(p.trash_lag[t]);
            co.push_back(p.trash_coeff[t]);
            ex.push_back(p.trash_ext[t]);
        }
        for (uint32_t s = 0; s < k->n_sets; s++) {
            lag.push_back(p.z_lag[s]);
            co.push_back(p.z_coeff[s]);
            ex.push_back(p.z_ext[s]);
        }
        for (size_t l = 0; l < k->lookups.size(); l++) {
            lag.insert(lag.end(), {p.m_lag[l], p.Z_lag[l]});
            co.insert(co.end(), {p.m_coeff[l], p.Z_coeff[l]});
            ex.insert(ex.end(), {p.m_ext[l], p.Z_ext[l]});
        }
        for (uint32_t h = 0; h < k->n_helpers; h++) {
            lag.push_back(p.h_lag[h]);
            co.push_back(p.h_coeff[h]);
            ex.push_back(p.h_ext[h]);
        }
    };
    // the transforms of all proofs of one domain together, one launch per
    // pass for up to 64 polynomials (MZK_PROVE_NO_GRAPHS: proof by proof,
    // kernel by kernel, the plain form)
    const bool batched_ntt = !(flags & MZK_PROVE_NO_GRAPHS);
    if (batched_ntt) {
        std::map<const Domain*, std::array<std::vector<void*>, 3>> by_dom;
        for (auto& p : ps) {
            std::vector<const void*> lag;
            std::vector<Fr*> co, ex;
            ntt_lists(p, lag, co, ex);
            auto& g = by_dom[p.key->dom];
            for (size_t i = 0; i < lag.size(); i++) {
                g[0].push_back(const_cast<void*>(lag[i]));
                g[1].push_back(co[i]);
                g[2].push_back(ex[i]);
            }
        }
        for (auto& kv : by_dom) {
            auto& g = kv.second;
            MZK_TRY(domain_op_batch(ctx, kv.first, OP_LAGRANGE_TO_COEFF, const_cast<const void* const*>(g[0].data()),
                                    g[1].data(), (uint32_t)g[0].size(), st));
            MZK_TRY(domain_op_batch(ctx, kv.first, OP_COEFF_TO_EXTENDED, const_cast<const void* const*>(g[1].data()),
                                    g[2].data(), (uint32_t)g[1].size(), st));
        }
    }
    for (auto& p : ps) {
        const PlonkKey* k = p.key;
        const Domain* d = k->dom;
        if (!batched_ntt) {
            std::vector<const void*> lag;
            std::vector<Fr*> co, ex;
            ntt_lists(p, lag, co, ex);
            MZK_TRY(ntt_sequence(ctx, d, lag.data(), co.data(), ex.data(), (int)lag.size(), false, st));
        }
        std::vector<const uint64_t*> adv(k->n_advice), fixed(k->n_fixed), sig(k->n_perm), zs(k->n_sets),
            inst(k->n_instance);
        for (uint32_t i = 0; i < k->n_instance; i++) inst[i] = reinterpret_cast<const uint64_t*>(p.inst_ext[i]);
        for (uint32_t i = 0; i < k->n_advice; i++) adv[i] = reinterpret_cast<const uint64_t*>(p.adv_ext[i]);
        for (uint32_t i = 0; i < k->n_fixed; i++) fixed[i] = reinterpret_cast<const uint64_t*>(k->fixed_ext[i]);
        for (uint32_t i = 0; i < k->n_perm; i++) sig[i] = reinterpret_cast<const uint64_t*>(k->perm_ext[i]);
        for (uint32_t s = 0; s < k->n_sets; s++) zs[s] = reinterpret_cast<const uint64_t*>(p.z_ext[s]);
        // the lookup input expressions on the extended coset, read by the
        // lookup programs as the advice columns after the circuit's
        for (size_t x = 0; x < k->lk_exprs.size(); x++)
            MZK_TRY(flat_program_rows(ctx, d, k->lk_exprs[x].g, fixed.data(), k->n_fixed, adv.data(), k->n_advice,
                                      inst.data(), k->n_instance, kZero4, p.theta.l, kZero4, kZero4,
                                      reinterpret_cast<uint64_t*>(p.e_ext[x]), st, true));
        for (size_t x = 0; x < k->lk_exprs.size(); x++) adv.push_back(reinterpret_cast<const uint64_t*>(p.e_ext[x]));
        mzk_quotient_desc q;
        std::memset(&q, 0, sizeof(q));
        q.k = d->k;
        q.extended_k = d->ext_k;
        q.advice = adv.data();
        q.n_advice = (uint32_t)adv.size();
        q.fixed = fixed.data();
        q.n_fixed = k->n_fixed;
        std::memcpy(q.gate_fixed, k->gate_fixed, sizeof(q.gate_fixed));
        std::memcpy(q.gate_advice, k->gate_advice, sizeof(q.gate_advice));
        q.gates = k->has_gates ? &k->gates : nullptr;
        q.instance = inst.data();
        q.n_instance = k->n_instance;
        q.n_perm_cols = k->n_perm;
        q.perm_col_kind = k->perm_kind.data();
        q.perm_col_index = k->perm_index.data();
        q.perm_sigma = sig.data();
        q.n_perm_sets = k->n_sets;
        q.perm_z = zs.data();
        q.chunk_len = k->chunk;
        q.blinding_factors = k->bf;
        const size_t L = k->lookups.size();
        std::vector<const uint64_t*> hext(k->n_helpers);
        for (uint32_t h = 0; h < k->n_helpers; h++) hext[h] = reinterpret_cast<const uint64_t*>(p.h_ext[h]);
        std::vector<mzk_lookup_arg> largs(L);
        std::vector<mzk_trash_arg> targs(k->trash.size());
        for (size_t t = 0; t < k->trash.size(); t++) {
            targs[t].program = k->trash[t].program;
            targs[t].selector_fixed = k->trash[t].selector;
            targs[t].trash = reinterpret_cast<const uint64_t*>(p.trash_ext[t]);
        }
        if (!targs.empty()) {
            q.n_trash = (uint32_t)targs.size();
            q.trash = targs.data();
        }
        if (L == 1 && k->lk_programs.empty()) {  // the fused built-in term (one column, no trashcans)
            const mzk_lookup_shape& sh = k->lookups[0].shape;
            q.has_lookup = 1;
            q.lookup_input_advice = sh.input_advice;
            q.lookup_table_fixed = sh.table_fixed;
            q.lookup_selector_fixed = sh.selector_fixed;
            q.lookup_h = reinterpret_cast<const uint64_t*>(p.h_ext[0]);
            q.lookup_z = reinterpret_cast<const uint64_t*>(p.Z_ext[0]);
            q.lookup_m = reinterpret_cast<const uint64_t*>(p.m_ext[0]);
        } else if (L >= 1) {  // one helper program per chunk
            for (size_t l = 0; l < L; l++) {
                const PlonkKey::Lookup& lk = k->lookups[l];
                largs[l].n_helpers = lk.n_helpers();
                largs[l].programs = &k->lk_programs[lk.h0];
                largs[l].outputs = &k->lk_outputs[4 * (size_t)lk.h0];
                largs[l].helpers = &hext[lk.h0];
                largs[l].aggregator = reinterpret_cast<const uint64_t*>(p.Z_ext[l]);
                largs[l].multiplicities = reinterpret_cast<const uint64_t*>(p.m_ext[l]);
            }
            q.n_lookups = (uint32_t)L;
            q.lookups = largs.data();
        }
        q.l0 = reinterpret_cast<const uint64_t*>(k->l0);
        q.l_last = reinterpret_cast<const uint64_t*>(k->l_last);
        q.l_active = reinterpret_cast<const uint64_t*>(k->l_active);
        std::memcpy(q.y, p.y.l, 32);
        std::memcpy(q.beta, p.beta.l, 32);
        std::memcpy(q.gamma, p.gamma.l, 32);
        std::memcpy(q.theta, p.theta.l, 32);
        std::memcpy(q.trash_challenge, p.trash.l, 32);
        MZK_TRY(compute_h_limbs_device(ctx, d, &q, p.req->blinds + 4 * p.off_quot, p.limbs, hbuf, dbl, st));
        for (uint32_t i = 0; i < k->qdeg; i++) items.push_back({p.limbs + (size_t)i * k->n, k->srs.off_g, k->n});
    }
    MZK_TRY(msm());
    for (size_t j = 0, at = 0; j < count; j++) {
        FsProof& p = ps[j];
        write_points(p, &res[18 * at], p.key->qdeg);
        at += p.key->qdeg;
        p.x = p.tr.squeeze();
        p.xn = fr_pow_u64(p.x, p.key->n);
    }
    phase_done(4);
    // ---- 5. evaluations, linearization, x1, x2 ----------------------------
    {
        // the identities at x are evaluated for the self-check, and for keys
        // with simple selectors, whose linearization polynomial needs them;
        // instance evaluations (not in the transcript: no committed
        // instances) only for those
        const bool check = (flags & MZK_PROVE_SELF_CHECK) != 0;
        auto need_ids = [&](const PlonkKey* k) { return check || !k->gate_poly_values.empty(); };
        std::vector<EvalTask> tasks;
        for (auto& p : ps) {
            const PlonkKey* k = p.key;
            const Domain* d = k->dom;
            const uint64_t n = k->n;
            for (auto& q : k->advice_queries) tasks.push_back(eval_task(p.adv_coeff[q.column], n, fr_rot(d, p.x, q.rotation)));
            for (auto& q : k->fixed_queries)  // a simple selector's evaluation is one, not computed
                if (!k->is_simple(q.column))
                    tasks.push_back(eval_task(k->fixed_coeff[q.column], n, fr_rot(d, p.x, q.rotation)));
            for (uint32_t i = 0; i < k->n_perm; i++) tasks.push_back(eval_task(k->perm_coeff[i], n, p.x));
            for (uint32_t s = 0; s < k->n_sets; s++) {
                tasks.push_back(eval_task(p.z_coeff[s], n, p.x));
                tasks.push_back(eval_task(p.z_coeff[s], n, fr_rot(d, p.x, 1)));
                tasks.push_back(eval_task(p.z_coeff[s], n, fr_rot(d, p.x, k->last_rot())));
            }
            for (size_t l = 0; l < k->lookups.size(); l++) {  // Committed::evaluate (logup/prover.rs:318-355)
                tasks.push_back(eval_task(p.m_coeff[l], n, p.x));
                for (uint32_t c = 0; c < k->lookups[l].n_helpers(); c++)
                    tasks.push_back(eval_task(p.h_coeff[k->lookups[l].h0 + c], n, p.x));
                tasks.push_back(eval_task(p.Z_coeff[l], n, p.x));
                tasks.push_back(eval_task(p.Z_coeff[l], n, fr_rot(d, p.x, 1)));
            }
            for (size_t t = 0; t < k->trash.size(); t++) tasks.push_back(eval_task(p.trash_coeff[t], n, p.x));
            if (need_ids(k))
                for (auto& q : k->instance_queries)
                    tasks.push_back(eval_task(p.inst_coeff[q.column], n, fr_rot(d, p.x, q.rotation)));
        }
        std::vector<Fr4> ev;
        MZK_TRY(eval_many(ctx, tasks, ev, st));
        size_t at = 0;
        std::vector<LinSpec> lins;
        for (auto& p : ps) {
            const PlonkKey* k = p.key;
            auto grab = [&](std::vector<Fr4>& dst, size_t m) {
                dst.assign(ev.begin() + at, ev.begin() + at + m);
                at += m;
            };
            grab(p.ev_adv, k->advice_queries.size());
            std::vector<Fr4> fix_written;
            grab(fix_written, fixed_written(*k));
            p.ev_fix.clear();
            for (size_t i = 0, w = 0; i < k->fixed_queries.size(); i++)
                p.ev_fix.push_back(k->is_simple(k->fixed_queries[i].column) ? host::fr_one() : fix_written[w++]);
            grab(p.ev_pc, k->n_perm);
            grab(p.ev_sets, 3 * (size_t)k->n_sets);
            grab(p.ev_lk, 3 * k->lookups.size() + k->n_helpers);
            grab(p.ev_trash, k->trash.size());
            grab(p.ev_inst, need_ids(k) ? k->instance_queries.size() : 0);
            // transcript order (write_evals_to_transcript, permutation / logup evaluate)
            for (auto& v : p.ev_adv) p.tr.write_fr(v);
            for (auto& v : fix_written) p.tr.write_fr(v);
            for (auto& v : p.ev_pc) p.tr.write_fr(v);
            for (uint32_t s = 0; s < k->n_sets; s++) {
                p.tr.write_fr(p.ev_sets[3 * s]);
                p.tr.write_fr(p.ev_sets[3 * s + 1]);
                if (s + 1 < k->n_sets) p.tr.write_fr(p.ev_sets[3 * s + 2]);
            }
            for (auto& v : p.ev_lk) p.tr.write_fr(v);
            for (auto& v : p.ev_trash) p.tr.write_fr(v);
            // L'(X) = -sum_i (x^n - 1) (x^(n-1))^i h_i(X): the identities are
            // all constants here (no simple selectors)
            const Fr4 sf = fr_pow_u64(p.x, k->n - 1);
            Fr4 s = fr_neg(fr_sub(p.xn, host::fr_one()));
            LinSpec ls{p.lin, k->n, {}};
            for (uint32_t i = 0; i < k->qdeg; i++) {
                ls.terms.push_back({p.limbs + (size_t)i * k->n, k->n, to_dev(s)});
                s = fr_mul(s, sf);
            }
            if (need_ids(k)) {  // + sum of simple selectors' fixed polynomials times their identities
                std::vector<std::pair<uint32_t, Fr4>> sel_terms;
                p.lin_c = linearization_split(identities_at_x(p), p.y, &sel_terms);
                for (auto& t : sel_terms) ls.terms.push_back({k->fixed_coeff[t.first], k->n, to_dev(t.second)});
            }
            lins.push_back(ls);
            p.x1 = p.tr.squeeze();
            p.x2 = p.tr.squeeze();
        }
        MZK_TRY(lincomb_many(ctx, lins, st));
    }
    phase_done(5);
    // ---- 6. q polynomials, f = sum x2^s q_s / prod (X - p), its commitment, x3
    {
        std::vector<LinSpec> qs;
        for (auto& p : ps) {
            const PlonkKey* k = p.key;
            for (size_t s = 0; s < k->open_sets.size(); s++) {
                LinSpec ls{p.q[s], k->n, {}};
                Fr4 pw = host::fr_one();
                for (auto& id : k->open_sets[s].polys) {
                    ls.terms.push_back({open_poly(p, id), k->n, to_dev(pw)});
                    pw = fr_mul(pw, p.x1);
                }
                qs.push_back(ls);
            }
        }
        MZK_TRY(lincomb_many(ctx, qs, st));
        // each set's q divided by (X - x_r) for its points in turn
        // (kzg/mod.rs:219-240): stage r of every set of every proof at once,
        // grouped by length n - r; the divisions of a set alternate between
        // its fdiv and qt so that the last one lands in fdiv
        size_t max_rots = 0;
        for (auto& p : ps)
            for (auto& os : p.key->open_sets) max_rots = std::max(max_rots, os.rots.size());
        auto div_out = [](FsProof& p, size_t s, size_t r) {
            const size_t R = p.key->open_sets[s].rots.size();
            return (R - 1 - r) % 2 == 0 ? p.fdiv[s] : p.qt[s];
        };
        for (size_t r = 0; r < max_rots; r++) {
            std::map<uint64_t, std::tuple<std::vector<const void*>, std::vector<void*>, std::vector<Fr4>>> by_len;
            for (auto& p : ps) {
                const PlonkKey* k = p.key;
                for (size_t s = 0; s < k->open_sets.size(); s++) {
                    const auto& rots = k->open_sets[s].rots;
                    if (r >= rots.size()) continue;
                    auto& g = by_len[(uint64_t)k->n - r];
                    std::get<0>(g).push_back(r == 0 ? p.q[s] : div_out(p, s, r - 1));
                    std::get<1>(g).push_back(div_out(p, s, r));
                    std::get<2>(g).push_back(fr_rot(k->dom, p.x, rots[r]));
                }
            }
            for (auto& kv : by_len) {
                auto& g = kv.second;
                MZK_TRY(kate_division_batch(ctx, std::get<0>(g).data(), std::get<1>(g).data(), std::get<2>(g).data(),
                                            (uint32_t)std::get<0>(g).size(), kv.first, st));
            }
        }
        std::vector<LinSpec> fs;
        items.clear();
        for (auto& p : ps) {
            const PlonkKey* k = p.key;
            LinSpec ls{p.f, 0, {}};
            Fr4 pw = host::fr_one();
            for (size_t s = 0; s < k->open_sets.size(); s++) {
                const uint64_t len = k->n - k->open_sets[s].rots.size();
                ls.terms.push_back({p.fdiv[s], len, to_dev(pw)});
                ls.len = std::max<uint64_t>(ls.len, len);
                pw = fr_mul(pw, p.x2);
            }
            p.f_len = ls.len;
            fs.push_back(ls);
            items.push_back({p.f, k->srs.off_g, p.f_len});
        }
        MZK_TRY(lincomb_many(ctx, fs, st));
        MZK_TRY(msm());
        for (size_t j = 0; j < count; j++) {
            write_points(ps[j], &res[18 * j], 1);
            ps[j].x3 = ps[j].tr.squeeze();
        }
    }
    phase_done(6);
    // ---- 7. q evaluations at x3, x4 ---------------------------------------
    {
        const bool check = (flags & MZK_PROVE_SELF_CHECK) != 0;
        std::vector<EvalTask> tasks;
        for (auto& p : ps) {
            for (size_t s = 0; s < p.key->open_sets.size(); s++) tasks.push_back(eval_task(p.q[s], p.key->n, p.x3));
            if (check) tasks.push_back(eval_task(p.lin, p.key->n, p.x));
        }
        std::vector<Fr4> ev;
        MZK_TRY(eval_many(ctx, tasks, ev, st));
        size_t at = 0;
        for (size_t j = 0; j < count; j++) {
            FsProof& p = ps[j];
            for (size_t s = 0; s < p.key->open_sets.size(); s++) p.tr.write_fr(ev[at++]);
            if (check) {
                // L'(x) = -C holds iff the witness satisfies every identity
                // (the reference's debug assertion, prover.rs:404-408)
                const Fr4 lin_x = ev[at++];
                if (!fr_eq(lin_x, fr_neg(p.lin_c))) {
                    set_error("create_proof: request " + std::to_string(j) +
                              ": the witness does not satisfy the circuit (L'(x) != -C)");
                    return ERR_ARG;
                }
            }
            p.x4 = p.tr.squeeze();
        }
    }
    phase_done(7);
    // ---- 8. final polynomial and pi ---------------------------------------
    // pi = (final - v) / (X - x3) with v = final(x3); kate_division drops the
    // remainder, so the quotient of final itself is the same polynomial
    {
        std::vector<LinSpec> fins;
        for (auto& p : ps) {
            const PlonkKey* k = p.key;
            LinSpec ls{p.fin, k->n, {}};
            Fr4 pw = host::fr_one();
            for (size_t s = 0; s < k->open_sets.size(); s++) {
                ls.terms.push_back({p.q[s], k->n, to_dev(pw)});
                pw = fr_mul(pw, p.x4);
            }
            ls.terms.push_back({p.f, p.f_len, to_dev(pw)});
            fins.push_back(ls);
        }
        MZK_TRY(lincomb_many(ctx, fins, st));
        items.clear();
        std::map<uint64_t, std::tuple<std::vector<const void*>, std::vector<void*>, std::vector<Fr4>>> by_len;
        for (auto& p : ps) {
            auto& g = by_len[p.key->n];
            std::get<0>(g).push_back(p.fin);
            std::get<1>(g).push_back(p.pi);
            std::get<2>(g).push_back(p.x3);
            items.push_back({p.pi, p.key->srs.off_g, (uint64_t)p.key->n - 1});
        }
        for (auto& kv : by_len) {
            auto& g = kv.second;
            MZK_TRY(kate_division_batch(ctx, std::get<0>(g).data(), std::get<1>(g).data(), std::get<2>(g).data(),
                                        (uint32_t)std::get<0>(g).size(), kv.first, st));
        }
        MZK_TRY(msm());
        for (size_t j = 0; j < count; j++) {
            write_points(ps[j], &res[18 * j], 1);
            const auto& pr = ps[j].tr.proof();
            if (pr.size() != ps[j].key->proof_len) {
                set_error("create_proof: internal proof length mismatch");
                return ERR_STATE;
            }
            std::memcpy(reqs[j].proof_out, pr.data(), pr.size());
        }
    }
    phase_done(8);
    return OK;
}

}  // namespace mzk

// ------------------------------------------------------------ the C ABI ----
struct mzk_transcript {
    mzk::host::Transcript t;
};

using mzk::Status;

extern "C" {

int mzk_transcript_create(mzk_transcript** out) {
    if (!out) {
        mzk::set_error("null out pointer");
        return mzk::ERR_ARG;
    }
    *out = new (std::nothrow) mzk_transcript;
    return *out ? mzk::OK : mzk::ERR_OOM;
}
int mzk_transcript_destroy(mzk_transcript* t) {
    delete t;
    return mzk::OK;
}
int mzk_transcript_common_fr(mzk_transcript* t, const uint64_t v[4]) {
    if (!t || !v) return mzk::ERR_ARG;
    mzk::host::Fr4 a;
    std::memcpy(a.l, v, 32);
    t->t.common_fr(a);
    return mzk::OK;
}
int mzk_transcript_write_fr(mzk_transcript* t, const uint64_t v[4]) {
    if (!t || !v) return mzk::ERR_ARG;
    mzk::host::Fr4 a;
    std::memcpy(a.l, v, 32);
    t->t.write_fr(a);
    return mzk::OK;
}
int mzk_transcript_write_point(mzk_transcript* t, const uint64_t p[18]) {
    if (!t || !p) return mzk::ERR_ARG;
    t->t.write_point(p);
    return mzk::OK;
}
int mzk_transcript_squeeze(mzk_transcript* t, uint64_t out[4]) {
    if (!t || !out) return mzk::ERR_ARG;
    const mzk::host::Fr4 c = t->t.squeeze();
    std::memcpy(out, c.l, 32);
    return mzk::OK;
}
int mzk_transcript_proof(const mzk_transcript* t, uint8_t* out, size_t cap, size_t* len) {
    if (!t || !len) return mzk::ERR_ARG;
    const auto& p = t->t.proof();
    *len = p.size();
    if (out) {
        if (cap < p.size()) {
            mzk::set_error("transcript: output buffer too small");
            return mzk::ERR_ARG;
        }
        std::memcpy(out, p.data(), p.size());
    }
    return mzk::OK;
}
int mzk_vk_transcript_repr(uint32_t k, const uint64_t* fixed_coms, size_t n_fixed, const uint64_t* perm_coms,
                           size_t n_perm, const uint8_t* pinned, size_t pinned_len, uint64_t out[4]) {
    if (!out || (n_fixed && !fixed_coms) || (n_perm && !perm_coms) || (pinned_len && !pinned) || k > 255) {
        mzk::set_error("vk_transcript_repr: bad argument");
        return mzk::ERR_ARG;
    }
    mzk::host::Fr4 r;
    MZK_TRY(mzk::vk_transcript_repr(k, fixed_coms, n_fixed, perm_coms, n_perm, pinned, pinned_len, &r));
    std::memcpy(out, r.l, 32);
    return mzk::OK;
}

int mzk_keygen(mzk_ctx* ctx, mzk_domain* d, const mzk_circuit_desc* cs, const mzk_srs_desc* srs,
               const uint64_t* const* fixed_values, const uint32_t* perm_mapping, const uint8_t* pinned,
               size_t pinned_len, mzk_plonk_key** out) {
    if (!ctx || !d || !cs || !out || (pinned_len && !pinned)) {
        mzk::set_error("keygen: null argument");
        return mzk::ERR_ARG;
    }
    *out = nullptr;
    mzk::Context* c = mzk::context_of(ctx);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    mzk::PlonkKey* key = nullptr;
    MZK_TRY(mzk::keygen(c, mzk::domain_of(d), cs, srs, fixed_values, perm_mapping, nullptr, pinned, pinned_len,
                        &key));
    *out = reinterpret_cast<mzk_plonk_key*>(key);
    return mzk::OK;
}

int mzk_keygen_from_values(mzk_ctx* ctx, mzk_domain* d, const mzk_circuit_desc* cs, const mzk_srs_desc* srs,
                           const uint64_t* const* fixed_values, const uint64_t* const* perm_values,
                           const uint8_t* pinned, size_t pinned_len, mzk_plonk_key** out) {
    if (!ctx || !d || !cs || !out || (pinned_len && !pinned) || (cs->n_perm_cols && !perm_values)) {
        mzk::set_error("keygen: null argument");
        return mzk::ERR_ARG;
    }
    *out = nullptr;
    mzk::Context* c = mzk::context_of(ctx);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    mzk::PlonkKey* key = nullptr;
    MZK_TRY(mzk::keygen(c, mzk::domain_of(d), cs, srs, fixed_values, nullptr, perm_values, pinned, pinned_len,
                        &key));
    *out = reinterpret_cast<mzk_plonk_key*>(key);
    return mzk::OK;
}

int mzk_vk_write(const mzk_plonk_key* key, int format, uint8_t* out, size_t cap, size_t* len) {
    if (!key || !len || format < 0 || format > 2) return mzk::ERR_ARG;
    std::vector<uint8_t> v;
    MZK_TRY(mzk::vk_serialize(reinterpret_cast<const mzk::PlonkKey*>(key), format, v));
    *len = v.size();
    if (out) {
        if (cap < v.size()) {
            mzk::set_error("vk_write: output buffer too small");
            return mzk::ERR_ARG;
        }
        std::memcpy(out, v.data(), v.size());
    }
    return mzk::OK;
}

int mzk_pk_write(mzk_ctx* ctx, const mzk_plonk_key* key, int format, uint8_t* out, size_t cap, size_t* len) {
    if (!ctx || !key || !len || format < 0 || format > 2) return mzk::ERR_ARG;
    mzk::Context* c = mzk::context_of(ctx);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    const mzk::PlonkKey* k = reinterpret_cast<const mzk::PlonkKey*>(key);
    const size_t psz = format == MZK_SERDE_PROCESSED ? 48 : 96;
    const size_t need = 6 + psz * (k->fixed_coms.size() + k->perm_coms.size()) + 8 +
                        (k->fixed_coms.size() + k->perm_coms.size()) * (4 + (size_t)k->n * 32);
    *len = need;
    if (!out) return mzk::OK;
    if (cap < need) {
        mzk::set_error("pk_write: output buffer too small");
        return mzk::ERR_ARG;
    }
    std::vector<uint8_t> v;
    MZK_TRY(mzk::pk_serialize(c, k, format, v, c->stream));
    if (v.size() != need) {
        mzk::set_error("pk_write: internal size mismatch");
        return mzk::ERR_STATE;
    }
    std::memcpy(out, v.data(), v.size());
    return mzk::OK;
}

int mzk_pk_read(mzk_ctx* ctx, mzk_domain* d, const mzk_circuit_desc* cs, const mzk_srs_desc* srs,
                const uint8_t* bytes, size_t len, int format, const uint8_t* pinned, size_t pinned_len,
                mzk_plonk_key** out) {
    if (!ctx || !d || !cs || !out || !bytes || format < 0 || format > 2 || (pinned_len && !pinned)) {
        mzk::set_error("pk_read: bad argument");
        return mzk::ERR_ARG;
    }
    *out = nullptr;
    mzk::Context* c = mzk::context_of(ctx);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    mzk::PlonkKey* key = nullptr;
    MZK_TRY(mzk::pk_read(c, mzk::domain_of(d), cs, srs, bytes, len, format, pinned, pinned_len, &key, c->stream));
    *out = reinterpret_cast<mzk_plonk_key*>(key);
    return mzk::OK;
}

int mzk_plonk_key_transcript_layout(const mzk_plonk_key* key, uint8_t* ops, size_t cap, size_t* len) {
    if (!key || !len) return mzk::ERR_ARG;
    const mzk::PlonkKey* k = reinterpret_cast<const mzk::PlonkKey*>(key);
    std::vector<uint8_t> v;
    auto put = [&](uint8_t op, size_t times) { v.insert(v.end(), times, op); };
    const size_t L = k->lookups.size(), S = k->n_sets;
    put(MZK_TR_COMMON_FR, 1);                  // vk.hash_into
    put(MZK_TR_WRITE_POINT, k->n_advice);      // advice commitments
    put(MZK_TR_SQUEEZE, 1);                    // theta
    put(MZK_TR_WRITE_POINT, L);                // multiplicities
    put(MZK_TR_SQUEEZE, 2);                    // beta, gamma
    put(MZK_TR_WRITE_POINT, S + k->n_helpers + L);  // permutation products, logup helpers and aggregators
    put(MZK_TR_SQUEEZE, 1);                    // trash challenge
    put(MZK_TR_WRITE_POINT, k->trash.size());  // trash columns
    put(MZK_TR_SQUEEZE, 1);                    // y
    put(MZK_TR_WRITE_POINT, k->qdeg);          // quotient limbs
    put(MZK_TR_SQUEEZE, 1);                    // x
    put(MZK_TR_WRITE_FR, k->advice_queries.size() + mzk::fixed_written(*k) + k->n_perm + (S ? 3 * S - 1 : 0) +
                             3 * L + k->n_helpers + k->trash.size());  // evaluations
    put(MZK_TR_SQUEEZE, 2);                    // x1, x2
    put(MZK_TR_WRITE_POINT, 1);                // f
    put(MZK_TR_SQUEEZE, 1);                    // x3
    put(MZK_TR_WRITE_FR, k->open_sets.size()); // q evaluations
    put(MZK_TR_SQUEEZE, 1);                    // x4
    put(MZK_TR_WRITE_POINT, 1);                // pi
    *len = v.size();
    if (ops) {
        if (cap < v.size()) {
            mzk::set_error("transcript layout: output buffer too small");
            return mzk::ERR_ARG;
        }
        std::memcpy(ops, v.data(), v.size());
    }
    return mzk::OK;
}

int mzk_plonk_key_destroy(mzk_plonk_key* key) {
    delete reinterpret_cast<mzk::PlonkKey*>(key);
    return mzk::OK;
}

int mzk_plonk_key_info(const mzk_plonk_key* key, uint64_t repr[4], size_t* proof_len, size_t* n_blinds) {
    if (!key) return mzk::ERR_ARG;
    const mzk::PlonkKey* k = reinterpret_cast<const mzk::PlonkKey*>(key);
    if (repr) std::memcpy(repr, k->repr.l, 32);
    if (proof_len) *proof_len = k->proof_len;
    if (n_blinds) *n_blinds = k->n_blinds;
    return mzk::OK;
}

int mzk_plonk_key_commitments(const mzk_plonk_key* key, uint64_t* fixed, uint64_t* perm) {
    if (!key) return mzk::ERR_ARG;
    const mzk::PlonkKey* k = reinterpret_cast<const mzk::PlonkKey*>(key);
    if (fixed)
        for (size_t i = 0; i < k->fixed_coms.size(); i++) std::memcpy(fixed + 18 * i, k->fixed_coms[i].data(), 144);
    if (perm)
        for (size_t i = 0; i < k->perm_coms.size(); i++) std::memcpy(perm + 18 * i, k->perm_coms[i].data(), 144);
    return mzk::OK;
}

int mzk_plonk_key_srs(const mzk_plonk_key* key, mzk_srs_desc* out) {
    if (!key || !out) return mzk::ERR_ARG;
    *out = reinterpret_cast<const mzk::PlonkKey*>(key)->srs;
    return mzk::OK;
}

int mzk_create_proofs(mzk_ctx* ctx, const mzk_proof_request* reqs, size_t count, uint32_t flags) {
    if (!ctx || (count && !reqs)) {
        mzk::set_error("create_proof: null argument");
        return mzk::ERR_ARG;
    }
    mzk::Context* c = mzk::context_of(ctx);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    cudaSetDevice(c->device);
    const Status s = mzk::create_proofs(c, reqs, count, flags, c->stream);
    if (s != mzk::OK) cudaStreamSynchronize(c->stream);
    return s;
}

}  // extern "C"
