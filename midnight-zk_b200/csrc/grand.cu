// grand.cu — the prover stages around the commitments that are scans over a
// column rather than MSMs or NTTs:
//
//   * batch inversion with ff 0.13 BatchInvert semantics (zeros stay zero),
//     used by both arguments below;
//   * the permutation argument's grand products z of every set
//     (proofs/src/plonk/permutation/prover.rs:81-255);
//   * the logup argument's helper polynomials and running-sum aggregator
//     (proofs/src/plonk/logup/prover.rs:195-300);
//   * eval_polynomial (proofs/src/utils/arithmetic.rs:59-87) and
//     kate_division (arithmetic.rs:106-125), both first-order linear
//     recurrences y_i = c_i + k y_{i+1} solved by one chunked primitive.
//
// Every result is an exact field value, so the parallel orders here give the
// reference's bytes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mzk.h"
#include "field.cuh"
#include "host_ec.hpp"
#include "grand.hpp"
#include "ntt.hpp"
#include "runtime.hpp"

namespace mzk {

namespace {

constexpr int kThreads = 256;
// elements per thread of a linear recurrence: up to 64, fewer when n is too
// small to give every SM work (each thread's chunk is a serial chain)
constexpr uint32_t kRecChunkMax = 64, kRecChunkMin = 4;
constexpr uint32_t kScanItems = 8;  // elements per thread of a block scan
constexpr uint32_t kMaxPermSetCols = 8;
constexpr uint32_t kMaxLogupChunks = 8;

__device__ __forceinline__ bool fr_is_zero(const Fr& a) {
    uint32_t acc = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) acc |= a.l[j];
    return acc == 0;
}

// 1/a for a non-zero a (zero gives zero): the binary extended Euclidean
// algorithm (inv_binary_raw) on the stored Montgomery limbs A = a R yields
// A^-1 = a^-1 R^-1, and one Montgomery product with R^3 gives a^-1 R, the
// Montgomery form of 1/a.  A block's single inversion is a serial chain on
// one thread, and this finishes it several times sooner than a Fermat
// power.  Variable time in the value.
__device__ __noinline__ Fr fr_inv(const Fr& a) {
    Fr x, r2;
    if (!inv_binary_raw<8>(x.l, a.l, FrMod())) return fr_zero();
#pragma unroll
    for (int j = 0; j < 8; j++) r2.l[j] = FrP::r2(j);
    return fr_mul(x, fr_mul(r2, r2));  // x R^3 R^-1 = a^-1 R
}

Fr to_dev(const host::Fr4& h) {
    Fr r;
    std::memcpy(r.l, h.l, 32);
    return r;
}
host::Fr4 to_host(const uint64_t* p) {
    host::Fr4 r;
    std::memcpy(r.l, p, 32);
    return r;
}

uint32_t grid_for(const Context* ctx, uint64_t items, uint32_t threads) {
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((items + threads - 1) / threads, (uint64_t)ctx->num_sms * 16));
}

// ---- exclusive scans (product or sum) of Fr values ----
template <bool kMul>
__device__ __forceinline__ Fr op(const Fr& a, const Fr& b) {
    return kMul ? fr_mul(a, b) : fr_add(a, b);
}
template <bool kMul>
__device__ __forceinline__ Fr identity() {
    return kMul ? fr_one() : fr_zero();
}

// block-wide exclusive scan of one value per thread (Hillis-Steele in shared
// memory); returns the exclusive prefix, *total the block's total
template <bool kMul>
__device__ Fr block_exclusive(Fr v, Fr* sm, Fr* total) {
    sm[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t off = 1; off < blockDim.x; off <<= 1) {
        Fr o = identity<kMul>();
        if (threadIdx.x >= off) o = sm[threadIdx.x - off];
        __syncthreads();
        if (threadIdx.x >= off) sm[threadIdx.x] = op<kMul>(o, sm[threadIdx.x]);
        __syncthreads();
    }
    *total = sm[blockDim.x - 1];
    const Fr ex = threadIdx.x ? sm[threadIdx.x - 1] : identity<kMul>();
    __syncthreads();
    return ex;
}

// block-wide exclusive suffix product of one value per thread: the product of
// the values of the threads above this one
__device__ Fr block_exclusive_suffix_product(Fr v, Fr* sm) {
    sm[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t off = 1; off < blockDim.x; off <<= 1) {
        Fr o = fr_one();
        if (threadIdx.x + off < blockDim.x) o = sm[threadIdx.x + off];
        __syncthreads();
        if (threadIdx.x + off < blockDim.x) sm[threadIdx.x] = fr_mul(o, sm[threadIdx.x]);
        __syncthreads();
    }
    const Fr ex = threadIdx.x + 1 < blockDim.x ? sm[threadIdx.x + 1] : fr_one();
    __syncthreads();
    return ex;
}

// ---- batch inversion (ff BatchInvert: zeros stay zero): a block takes
// kThreads x C consecutive elements (thread t the elements t, t + kThreads,
// ... of the block's range, so loads and stores are coalesced), each thread
// multiplies its C non-zero elements in registers, the block combines the
// threads' products by a prefix and a suffix scan in shared memory, and the
// inverse of the block's total gives every thread the inverse of its product
// (prefix x suffix x 1/total); the backward pass then inverts each element.
// The inverse of the total is one Fermat inversion in the block when the
// blocks fit one wave on the GPU; otherwise the totals are batch-inverted
// first (k_invert_totals, then this function on the totals), since a serial
// inversion per block would leave the SMs idle wave after wave.
constexpr int kInvPerThread = 4;

template <int C>
__global__ void __launch_bounds__(kThreads) k_invert_totals(const Fr* __restrict__ a, uint64_t n, Fr* __restrict__ tot) {
    __shared__ Fr sm[kThreads];
    const uint64_t base = (uint64_t)blockIdx.x * kThreads * C + threadIdx.x;
    Fr acc = fr_one();
#pragma unroll
    for (int k = 0; k < C; k++) {
        const uint64_t i = base + (uint64_t)k * kThreads;
        if (i < n) {
            const Fr v = a[i];
            if (!fr_is_zero(v)) acc = fr_mul(acc, v);
        }
    }
    Fr total;
    block_exclusive<true>(acc, sm, &total);
    if (threadIdx.x == 0) tot[blockIdx.x] = total;  // non-zero: a product of non-zero elements (or one)
}

template <int C, bool kGivenInverse>
__global__ void __launch_bounds__(kThreads) k_batch_invert(Fr* __restrict__ a, uint64_t n,
                                                           const Fr* __restrict__ tot_inv) {
    __shared__ Fr sm[kThreads];
    __shared__ Fr total_inv;
    const uint64_t base = (uint64_t)blockIdx.x * kThreads * C + threadIdx.x;
    Fr v[C], pre[C];
#pragma unroll
    for (int k = 0; k < C; k++) {
        const uint64_t i = base + (uint64_t)k * kThreads;
        v[k] = i < n ? a[i] : fr_zero();
    }
    Fr acc = fr_one();
#pragma unroll
    for (int k = 0; k < C; k++) {
        pre[k] = acc;
        if (!fr_is_zero(v[k])) acc = fr_mul(acc, v[k]);
    }
    Fr total;
    const Fr below = block_exclusive<true>(acc, sm, &total);
    const Fr above = block_exclusive_suffix_product(acc, sm);
    if (threadIdx.x == 0) total_inv = kGivenInverse ? tot_inv[blockIdx.x] : fr_inv(total);
    __syncthreads();
    Fr inv = fr_mul(fr_mul(total_inv, below), above);  // 1 / acc
#pragma unroll
    for (int k = C - 1; k >= 0; k--) {
        const uint64_t i = base + (uint64_t)k * kThreads;
        if (!fr_is_zero(v[k])) {
            if (i < n) a[i] = fr_mul(pre[k], inv);
            inv = fr_mul(inv, v[k]);
        }
    }
}

Status batch_invert_level(Context* ctx, Fr* a, uint64_t n, cudaStream_t st, int level) {
    if (n == 0) return OK;
    const uint64_t per = (uint64_t)kThreads * kInvPerThread;
    const uint64_t blocks = (n + per - 1) / per;
    if (blocks <= (uint64_t)ctx->num_sms * 2) {  // one wave at 2 blocks per SM
        k_batch_invert<kInvPerThread, false><<<(uint32_t)blocks, kThreads, 0, st>>>(a, n, nullptr);
        MZK_LAUNCH_CHECK(ctx);
        return OK;
    }
    if (level >= 4) {
        set_error("batch_invert: too many elements");
        return ERR_ARG;
    }
    static const char* const kTotNames[4] = {"grand_inv_tot0", "grand_inv_tot1", "grand_inv_tot2", "grand_inv_tot3"};
    void* buf;
    MZK_TRY(ctx->ensure(kTotNames[level], blocks * sizeof(Fr), &buf));
    Fr* tot = static_cast<Fr*>(buf);
    k_invert_totals<kInvPerThread><<<(uint32_t)blocks, kThreads, 0, st>>>(a, n, tot);
    MZK_LAUNCH_CHECK(ctx);
    MZK_TRY(batch_invert_level(ctx, tot, blocks, st, level + 1));
    k_batch_invert<kInvPerThread, true><<<(uint32_t)blocks, kThreads, 0, st>>>(a, n, tot);
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

Status batch_invert(Context* ctx, Fr* a, uint64_t n, cudaStream_t st) { return batch_invert_level(ctx, a, n, st, 0); }

// pass 1: out = exclusive scan within each tile of kThreads * kScanItems, sums[tile] = tile total
template <bool kMul>
__global__ void __launch_bounds__(kThreads) k_scan_tile(const Fr* in, Fr* out, uint64_t n, Fr* __restrict__ sums) {
    __shared__ Fr sm[kThreads];
    const uint64_t base = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) * kScanItems;
    Fr v[kScanItems];
    Fr acc = identity<kMul>();
#pragma unroll
    for (uint32_t j = 0; j < kScanItems; j++) {
        v[j] = base + j < n ? in[base + j] : identity<kMul>();
        acc = op<kMul>(acc, v[j]);
    }
    Fr total;
    Fr pre = block_exclusive<kMul>(acc, sm, &total);
#pragma unroll
    for (uint32_t j = 0; j < kScanItems; j++) {
        if (base + j < n) out[base + j] = pre;
        pre = op<kMul>(pre, v[j]);
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// pass 3: out[i] = prefix[tile] (op) out[i]
template <bool kMul>
__global__ void k_scan_apply(Fr* __restrict__ out, uint64_t n, const Fr* __restrict__ prefix) {
    const uint64_t tile = (uint64_t)kThreads * kScanItems;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t t = i / tile;
        if (t) out[i] = op<kMul>(prefix[t], out[i]);
    }
}

// out[i] = in[0] (op) ... (op) in[i-1] (the identity for i = 0); in and out may alias
template <bool kMul>
Status scan_exclusive(Context* ctx, const Fr* in, Fr* out, uint64_t n, cudaStream_t st, int depth = 0) {
    if (n == 0) return OK;
    const uint64_t tile = (uint64_t)kThreads * kScanItems;
    const uint64_t tiles = (n + tile - 1) / tile;
    void* sums;
    MZK_TRY(ctx->ensure(("grand_scan_" + std::to_string(depth)).c_str(), (tiles + 1) * sizeof(Fr), &sums));
    k_scan_tile<kMul><<<(uint32_t)tiles, kThreads, 0, st>>>(in, out, n, (Fr*)sums);
    MZK_LAUNCH_CHECK(ctx);
    if (tiles > 1) {
        // exclusive scan of the tile totals (recursively), then fold it in
        MZK_TRY(scan_exclusive<kMul>(ctx, (const Fr*)sums, (Fr*)sums, tiles, st, depth + 1));
        k_scan_apply<kMul><<<grid_for(ctx, n, kThreads), kThreads, 0, st>>>(out, n, (const Fr*)sums);
        MZK_LAUNCH_CHECK(ctx);
    }
    return OK;
}

// ---- first-order linear recurrence from the top: y_i = c_i + k y_{i+1},
// y_n = 0.  Thread t solves its chunk [tK, tK+K) with a zero carry-in and
// records L_t = its local y at tK; the true values at the chunk starts solve
// the same recurrence over the L_t with k^K; a last pass adds k^(hi-i) Y_{t+1}.
__global__ void __launch_bounds__(kThreads) k_rec_local(const Fr* __restrict__ c, Fr* __restrict__ y, uint64_t n,
                                                        Fr k, Fr* __restrict__ lows, uint32_t K) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t lo = t * K;
    if (lo >= n) return;
    const uint64_t hi = min(n, lo + K);
    Fr acc = fr_zero();
    for (uint64_t i = hi; i-- > lo;) {
        acc = fr_add(c[i], fr_mul(k, acc));
        y[i] = acc;
    }
    lows[t] = acc;
}
__global__ void __launch_bounds__(kThreads) k_rec_fix(Fr* __restrict__ y, uint64_t n, Fr k,
                                                      const Fr* __restrict__ starts, uint64_t chunks, uint32_t K) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t + 1 >= chunks) return;  // the top chunk has a zero carry-in
    const uint64_t lo = t * K, hi = lo + K;
    const Fr carry = starts[t + 1];
    Fr pw = k;  // k^(hi - i) for i = hi - 1
    for (uint64_t i = hi; i-- > lo;) {
        y[i] = fr_add(y[i], fr_mul(pw, carry));
        pw = fr_mul(pw, k);
    }
}

// y (n) from c (n), in and out may not alias
Status linrec_suffix(Context* ctx, const Fr* c, Fr* y, uint64_t n, const host::Fr4& k, cudaStream_t st, int depth = 0) {
    if (n == 0) return OK;
    // the chunk length: 64 while that leaves at least 2 threads of 256 per SM
    // per warp slot, down to 4 for smaller n; small recursion levels keep 64
    uint32_t K = kRecChunkMax;
    const uint64_t want_threads = (uint64_t)ctx->num_sms * kThreads * 2;
    while (K > kRecChunkMin && n / K < want_threads && n > (uint64_t)kRecChunkMax * kRecChunkMax) K >>= 1;
    const uint64_t chunks = (n + K - 1) / K;
    void* lows;
    MZK_TRY(ctx->ensure(("grand_rec_" + std::to_string(depth)).c_str(), 2 * chunks * sizeof(Fr), &lows));
    Fr* L = (Fr*)lows;
    Fr* Y = L + chunks;
    k_rec_local<<<(uint32_t)((chunks + kThreads - 1) / kThreads), kThreads, 0, st>>>(c, y, n, to_dev(k), L, K);
    MZK_LAUNCH_CHECK(ctx);
    if (chunks > 1) {
        host::Fr4 kk = k;  // k^K
        for (uint32_t b = 1; b < K; b <<= 1) kk = host::fr_mul(kk, kk);
        MZK_TRY(linrec_suffix(ctx, L, Y, chunks, kk, st, depth + 1));
        k_rec_fix<<<(uint32_t)((chunks + kThreads - 1) / kThreads), kThreads, 0, st>>>(y, n, to_dev(k), Y, chunks, K);
        MZK_LAUNCH_CHECK(ctx);
    }
    return OK;
}

// The same recurrences for T tasks of one length n, blockIdx.y picking the
// task: its input, output and factor, and its slice of the chunk values.
constexpr uint32_t kRecBatch = 32;
struct RecTasks {
    const Fr* c[kRecBatch];
    Fr* y[kRecBatch];
    Fr k[kRecBatch];
};
__global__ void __launch_bounds__(kThreads) k_rec_local_batch(const RecTasks t, uint64_t n, Fr* __restrict__ lows,
                                                              uint64_t chunks, uint32_t K) {
    const uint32_t j = blockIdx.y;
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t lo = c * K;
    if (lo >= n) return;
    const uint64_t hi = min(n, lo + K);
    const Fr k = t.k[j];
    const Fr* __restrict__ in = t.c[j];
    Fr* __restrict__ y = t.y[j];
    Fr acc = fr_zero();
    for (uint64_t i = hi; i-- > lo;) {
        acc = fr_add(in[i], fr_mul(k, acc));
        y[i] = acc;
    }
    lows[2 * chunks * j + c] = acc;
}
__global__ void __launch_bounds__(kThreads) k_rec_fix_batch(const RecTasks t, uint64_t n, const Fr* __restrict__ lows,
                                                            uint64_t chunks, uint32_t K) {
    const uint32_t j = blockIdx.y;
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c + 1 >= chunks) return;  // the top chunk has a zero carry-in
    const uint64_t lo = c * K, hi = lo + K;
    const Fr k = t.k[j];
    const Fr carry = lows[2 * chunks * j + chunks + c + 1];  // Y of the chunk above
    Fr* __restrict__ y = t.y[j];
    Fr pw = k;
    for (uint64_t i = hi; i-- > lo;) {
        y[i] = fr_add(y[i], fr_mul(pw, carry));
        pw = fr_mul(pw, k);
    }
}

// linrec_suffix for T tasks of one length: y[j] (n) from c[j] (n) with
// factor k[j]; the chunk values of every level sit in one buffer per level
// (task j: its lows L_j then its starts Y_j)
Status linrec_suffix_batch(Context* ctx, const Fr* const* c, Fr* const* y, const host::Fr4* k, uint32_t T, uint64_t n,
                           cudaStream_t st, int depth = 0) {
    if (n == 0 || T == 0) return OK;
    uint32_t K = kRecChunkMax;
    const uint64_t want_threads = (uint64_t)ctx->num_sms * kThreads * 2;
    while (K > kRecChunkMin && n * T / K < want_threads && n > (uint64_t)kRecChunkMax * kRecChunkMax) K >>= 1;
    const uint64_t chunks = (n + K - 1) / K;
    for (uint32_t j0 = 0; j0 < T; j0 += kRecBatch) {
        const uint32_t tb = std::min(kRecBatch, T - j0);
        void* lows;
        MZK_TRY(ctx->ensure(("grand_recb_" + std::to_string(depth)).c_str(), 2 * chunks * tb * sizeof(Fr), &lows));
        Fr* L = (Fr*)lows;
        RecTasks t;
        for (uint32_t j = 0; j < tb; j++) {
            t.c[j] = c[j0 + j];
            t.y[j] = y[j0 + j];
            t.k[j] = to_dev(k[j0 + j]);
        }
        const dim3 grid((uint32_t)((chunks + kThreads - 1) / kThreads), tb);
        k_rec_local_batch<<<grid, kThreads, 0, st>>>(t, n, L, chunks, K);
        MZK_LAUNCH_CHECK(ctx);
        if (chunks > 1) {
            // the chunk starts: the same recurrence over the lows with k^K
            std::vector<const Fr*> lc(tb);
            std::vector<Fr*> ly(tb);
            std::vector<host::Fr4> kk(tb);
            for (uint32_t j = 0; j < tb; j++) {
                lc[j] = L + 2 * chunks * j;
                ly[j] = L + 2 * chunks * j + chunks;
                kk[j] = k[j0 + j];
                for (uint32_t b = 1; b < K; b <<= 1) kk[j] = host::fr_mul(kk[j], kk[j]);
            }
            MZK_TRY(linrec_suffix_batch(ctx, lc.data(), ly.data(), kk.data(), tb, chunks, st, depth + 1));
            k_rec_fix_batch<<<grid, kThreads, 0, st>>>(t, n, L, chunks, K);
            MZK_LAUNCH_CHECK(ctx);
        }
    }
    return OK;
}

// ---- permutation argument ----
struct PermCols {
    const Fr* values[kMaxPermSetCols];
    const Fr* sigmas[kMaxPermSetCols];
    Fr delta_pow[kMaxPermSetCols];  // delta^(set chunk_len + j)
    uint32_t cols;
};

// den[i] = prod_j (beta s_j[i] + gamma + p_j[i])
__global__ void k_perm_den(PermCols pc, Fr beta, Fr gamma, Fr* __restrict__ den, uint32_t n) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Fr acc = fr_one();
        for (uint32_t j = 0; j < pc.cols; j++)
            acc = fr_mul(acc, fr_add(fr_add(fr_mul(beta, pc.sigmas[j][i]), gamma), pc.values[j][i]));
        den[i] = acc;
    }
}
// mv[i] *= prod_j (delta^(..+j) w^i beta + gamma + p_j[i]); w^i from the split tables
__global__ void k_perm_num(PermCols pc, Fr beta, Fr gamma, const Fr* __restrict__ wlo, const Fr* __restrict__ whi,
                           Fr* __restrict__ mv, uint32_t n) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const Fr wb = fr_mul(fr_mul(wlo[i & 4095u], whi[i >> 12]), beta);
        Fr acc = mv[i];
        for (uint32_t j = 0; j < pc.cols; j++)
            acc = fr_mul(acc, fr_add(fr_add(fr_mul(pc.delta_pow[j], wb), gamma), pc.values[j][i]));
        mv[i] = acc;
    }
}
constexpr uint32_t kMaxPermSets = 16;
struct SetPtrs {
    Fr* z[kMaxPermSets];
};
// corr[0] = 1, corr[s] = corr[s-1] * z_{s-1}[n - bf - 1] (the uncorrected last
// products, read before any set is corrected); one thread, sets in order
__global__ void k_perm_corrections(SetPtrs sp, uint32_t sets, uint32_t last, Fr* __restrict__ corr) {
    Fr c = fr_one();
    for (uint32_t s = 0; s < sets; s++) {
        corr[s] = c;
        c = fr_mul(c, sp.z[s][last]);
    }
}
// z[i] = (i < n - bf ? z[i] : blinds[i - (n - bf)]) * corr (multiplying by
// one where the reference skips the product leaves the value unchanged)
__global__ void k_perm_finish(Fr* __restrict__ z, uint32_t n, uint32_t bf, const Fr* __restrict__ blinds,
                              const Fr* __restrict__ corr) {
    const Fr c = *corr;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const Fr v = i < n - bf ? z[i] : blinds[i - (n - bf)];
        z[i] = fr_mul(v, c);
    }
}

// ---- logup argument ----
// out[i] = beta + v[i]
__global__ void k_add_const(const Fr* __restrict__ v, Fr beta, Fr* __restrict__ out, uint32_t n) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = fr_add(beta, v[i]);
}
// h[i] = sum of the chunk's inverted columns (cols consecutive arrays of n)
__global__ void k_sum_cols(const Fr* __restrict__ inv, uint32_t cols, Fr* __restrict__ h, uint32_t n) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Fr acc = fr_zero();
        for (uint32_t j = 0; j < cols; j++) acc = fr_add(acc, inv[(size_t)j * n + i]);
        h[i] = acc;
    }
}
// ld[i] = sel[i] * sum_c h_c[i] - m[i] * tden[i]
struct HelperPtrs {
    Fr* h[kMaxLogupChunks];
    uint32_t chunks;
};
__global__ void k_logderivative(HelperPtrs hp, const Fr* __restrict__ sel, const Fr* __restrict__ m,
                                const Fr* __restrict__ tden, Fr* __restrict__ ld, uint32_t n) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Fr s = fr_zero();
        for (uint32_t c = 0; c < hp.chunks; c++) s = fr_add(s, hp.h[c][i]);
        ld[i] = fr_sub(fr_mul(sel[i], s), fr_mul(m[i], tden[i]));
    }
}
// z[n - bf + b] = blinds[b]
__global__ void k_set_tail(Fr* __restrict__ z, uint32_t n, uint32_t bf, const Fr* __restrict__ blinds) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < bf) z[n - bf + b] = blinds[b];
}

}  // namespace

Status permutation_z_device(Context* ctx, const Domain* d, const mzk_permutation_desc* desc, cudaStream_t st) {
    const uint32_t n = 1u << d->k, bf = desc->blinding_factors;
    if (desc->chunk_len == 0 || desc->chunk_len > kMaxPermSetCols || bf + 1 >= n || desc->n_cols == 0 ||
        !desc->values || !desc->sigmas || !desc->z_out || (bf && !desc->blinds)) {
        set_error("permutation_z: need 1..8 columns per set, blinding_factors < n - 1 and non-null arrays");
        return ERR_ARG;
    }
    const uint32_t sets = (desc->n_cols + desc->chunk_len - 1) / desc->chunk_len;
    if (sets > kMaxPermSets) {
        set_error("permutation_z: at most 16 sets");
        return ERR_ARG;
    }
    void *mv_buf, *dbl, *corr;
    MZK_TRY(ctx->ensure("perm_mv", (size_t)n * sizeof(Fr), &mv_buf));
    MZK_TRY(ctx->ensure("perm_blinds", ((size_t)sets * bf + 1) * sizeof(Fr), &dbl));
    MZK_TRY(ctx->ensure("perm_corr", (size_t)sets * sizeof(Fr), &corr));
    if (bf)
        MZK_CUDA_CHECK(cudaMemcpyAsync(dbl, desc->blinds, (size_t)sets * bf * sizeof(Fr), cudaMemcpyHostToDevice, st));
    Fr* mv = (Fr*)mv_buf;
    const Fr beta = to_dev(to_host(desc->beta)), gamma = to_dev(to_host(desc->gamma));
    const host::Fr4 delta = to_host(host::FR_DELTA4);
    const uint32_t grid = grid_for(ctx, n, kThreads);
    for (uint32_t s = 0; s < sets; s++) {
        PermCols pc;
        pc.cols = std::min(desc->chunk_len, desc->n_cols - s * desc->chunk_len);
        const uint64_t e0 = (uint64_t)s * desc->chunk_len;
        host::Fr4 dp = host::fr_pow(delta, &e0, 1);
        for (uint32_t j = 0; j < pc.cols; j++) {
            const uint32_t c = s * desc->chunk_len + j;
            if (!desc->values[c] || !desc->sigmas[c] || !desc->z_out[s]) {
                set_error("permutation_z: null column");
                return ERR_ARG;
            }
            pc.values[j] = reinterpret_cast<const Fr*>(desc->values[c]);
            pc.sigmas[j] = reinterpret_cast<const Fr*>(desc->sigmas[c]);
            pc.delta_pow[j] = to_dev(dp);
            dp = host::fr_mul(dp, delta);
        }
        k_perm_den<<<grid, kThreads, 0, st>>>(pc, beta, gamma, mv, n);
        MZK_LAUNCH_CHECK(ctx);
        MZK_TRY(batch_invert(ctx, mv, n, st));
        k_perm_num<<<grid, kThreads, 0, st>>>(pc, beta, gamma, d->lo[0], d->hi[0], mv, n);
        MZK_LAUNCH_CHECK(ctx);
        Fr* z = reinterpret_cast<Fr*>(desc->z_out[s]);
        MZK_TRY(scan_exclusive<true>(ctx, mv, z, n, st));
    }
    // corrections from the uncorrected last products z_s[n - bf - 1], on the
    // device (no host round trip), then blinds and corrections per set
    SetPtrs sp;
    for (uint32_t s = 0; s < sets; s++) sp.z[s] = reinterpret_cast<Fr*>(desc->z_out[s]);
    k_perm_corrections<<<1, 1, 0, st>>>(sp, sets, n - bf - 1, (Fr*)corr);
    MZK_LAUNCH_CHECK(ctx);
    for (uint32_t s = 0; s < sets; s++) {
        k_perm_finish<<<grid, kThreads, 0, st>>>(sp.z[s], n, bf, (const Fr*)dbl + (size_t)s * bf, (const Fr*)corr + s);
        MZK_LAUNCH_CHECK(ctx);
    }
    return OK;
}

Status logup_device(Context* ctx, const Domain* d, const mzk_logup_desc* desc, cudaStream_t st) {
    const uint32_t n = 1u << d->k, bf = desc->blinding_factors;
    if (desc->n_chunks == 0 || desc->n_chunks > kMaxLogupChunks || bf + 1 >= n || !desc->chunk_cols ||
        !desc->inputs || !desc->table || !desc->selector || !desc->multiplicities || !desc->helpers_out ||
        !desc->aggregator_out || (bf && !desc->blinds)) {
        set_error("logup: need 1..8 chunks, blinding_factors < n - 1 and non-null arrays");
        return ERR_ARG;
    }
    uint32_t total_cols = 0;
    for (uint32_t c = 0; c < desc->n_chunks; c++) total_cols += desc->chunk_cols[c];
    void *tden_buf, *cols_buf, *ld_buf, *dbl;
    MZK_TRY(ctx->ensure("logup_tden", (size_t)n * sizeof(Fr), &tden_buf));
    MZK_TRY(ctx->ensure("logup_cols", (size_t)std::max(1u, total_cols) * n * sizeof(Fr), &cols_buf));
    MZK_TRY(ctx->ensure("logup_ld", (size_t)n * sizeof(Fr), &ld_buf));
    MZK_TRY(ctx->ensure("logup_blinds", ((size_t)bf + 1) * sizeof(Fr), &dbl));
    if (bf) MZK_CUDA_CHECK(cudaMemcpyAsync(dbl, desc->blinds, (size_t)bf * sizeof(Fr), cudaMemcpyHostToDevice, st));
    Fr *tden = (Fr*)tden_buf, *cols = (Fr*)cols_buf, *ld = (Fr*)ld_buf;
    const Fr beta = to_dev(to_host(desc->beta));
    const uint32_t grid = grid_for(ctx, n, kThreads);
    // T = 1 / (t + beta)
    k_add_const<<<grid, kThreads, 0, st>>>(reinterpret_cast<const Fr*>(desc->table), beta, tden, n);
    MZK_LAUNCH_CHECK(ctx);
    MZK_TRY(batch_invert(ctx, tden, n, st));
    // every input column: 1 / (f + beta) (inverting them together gives the same field values)
    for (uint32_t j = 0; j < total_cols; j++) {
        if (!desc->inputs[j]) {
            set_error("logup: null input column");
            return ERR_ARG;
        }
        k_add_const<<<grid, kThreads, 0, st>>>(reinterpret_cast<const Fr*>(desc->inputs[j]), beta,
                                               cols + (size_t)j * n, n);
        MZK_LAUNCH_CHECK(ctx);
    }
    MZK_TRY(batch_invert(ctx, cols, (uint64_t)total_cols * n, st));
    HelperPtrs hp;
    hp.chunks = desc->n_chunks;
    for (uint32_t c = 0, j = 0; c < desc->n_chunks; j += desc->chunk_cols[c], c++) {
        if (!desc->helpers_out[c]) {
            set_error("logup: null helper output");
            return ERR_ARG;
        }
        hp.h[c] = reinterpret_cast<Fr*>(desc->helpers_out[c]);
        k_sum_cols<<<grid, kThreads, 0, st>>>(cols + (size_t)j * n, desc->chunk_cols[c], hp.h[c], n);
        MZK_LAUNCH_CHECK(ctx);
    }
    k_logderivative<<<grid, kThreads, 0, st>>>(hp, reinterpret_cast<const Fr*>(desc->selector),
                                               reinterpret_cast<const Fr*>(desc->multiplicities), tden, ld, n);
    MZK_LAUNCH_CHECK(ctx);
    // aggregator: exclusive running sum over the first n - bf rows, then the blinds
    Fr* agg = reinterpret_cast<Fr*>(desc->aggregator_out);
    MZK_TRY(scan_exclusive<false>(ctx, ld, agg, n - bf, st));
    if (bf) {
        k_set_tail<<<1, 64, 0, st>>>(agg, n, bf, (const Fr*)dbl);
        MZK_LAUNCH_CHECK(ctx);
    }
    return OK;
}

namespace {
// out[i] = sum_p s_p polys[p][i] (i < len_p), polys and lengths in device tables
__global__ void k_inner_product(const Fr* const* __restrict__ polys, const uint64_t* __restrict__ lens,
                                const Fr* __restrict__ scalars, uint32_t m, Fr* __restrict__ out, uint64_t out_len) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < out_len; i += stride) {
        Fr acc = fr_zero();
        for (uint32_t p = 0; p < m; p++)
            if (i < lens[p]) acc = fr_add(acc, fr_mul(polys[p][i], scalars[p]));
        out[i] = acc;
    }
}
}  // namespace

Status poly_inner_product_device(Context* ctx, const uint64_t* const* polys, const uint64_t* lens, uint32_t m,
                                 const uint64_t* scalars, void* out, uint64_t out_len, cudaStream_t st) {
    if (out_len == 0) return OK;
    // one device table: m pointers, m lengths, m scalars (staged through pinned memory)
    const size_t bytes = (size_t)m * (8 + 8 + 32);
    void *d_tab, *h_tab;
    MZK_TRY(ctx->ensure("grand_ip_tab", bytes + 64, &d_tab));
    MZK_TRY(ctx->ensure_pinned(bytes + 64, &h_tab));
    char* h = static_cast<char*>(h_tab);
    std::memcpy(h, polys, (size_t)m * 8);
    std::memcpy(h + (size_t)m * 8, lens, (size_t)m * 8);
    std::memcpy(h + (size_t)m * 16, scalars, (size_t)m * 32);
    MZK_CUDA_CHECK(cudaMemcpyAsync(d_tab, h_tab, bytes, cudaMemcpyHostToDevice, st));
    const char* d = static_cast<const char*>(d_tab);
    k_inner_product<<<grid_for(ctx, out_len, kThreads), kThreads, 0, st>>>(
        reinterpret_cast<const Fr* const*>(d), reinterpret_cast<const uint64_t*>(d + (size_t)m * 8),
        reinterpret_cast<const Fr*>(d + (size_t)m * 16), m, static_cast<Fr*>(out), out_len);
    MZK_LAUNCH_CHECK(ctx);
    // the pinned table is reused by the next call: finish this one first
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    return OK;
}

namespace {
__global__ void k_fill(Fr* __restrict__ out, uint64_t n, Fr v) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = v;
}
}  // namespace

Status fr_powers_device(Context* ctx, const uint64_t s[4], uint64_t n, void* out, cudaStream_t st) {
    if (n == 0) return OK;
    k_fill<<<grid_for(ctx, n, kThreads), kThreads, 0, st>>>(static_cast<Fr*>(out), n, to_dev(to_host(s)));
    MZK_LAUNCH_CHECK(ctx);
    return scan_exclusive<true>(ctx, static_cast<const Fr*>(out), static_cast<Fr*>(out), n, st);
}

Status batch_invert_device(Context* ctx, void* a, uint64_t n, cudaStream_t st) {
    return batch_invert(ctx, static_cast<Fr*>(a), n, st);
}

Status eval_polynomial_device(Context* ctx, const void* poly, uint64_t n, const uint64_t point[4], uint64_t out[4],
                              cudaStream_t st) {
    std::memset(out, 0, 32);
    if (n == 0) return OK;
    void* y;
    MZK_TRY(ctx->ensure("grand_eval", n * sizeof(Fr), &y));
    MZK_TRY(linrec_suffix(ctx, static_cast<const Fr*>(poly), (Fr*)y, n, to_host(point), st));
    MZK_CUDA_CHECK(cudaMemcpyAsync(out, y, 32, cudaMemcpyDeviceToHost, st));
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    return OK;
}

Status kate_division_device(Context* ctx, const void* a, uint64_t n, const uint64_t b[4], void* q, cudaStream_t st) {
    if (n < 2) return OK;
    // q_i = a_{i+1} + b q_{i+1}, q_{n-1} = 0
    return linrec_suffix(ctx, static_cast<const Fr*>(a) + 1, static_cast<Fr*>(q), n - 1, to_host(b), st);
}

Status kate_division_batch(Context* ctx, const void* const* a, void* const* q, const host::Fr4* b, uint32_t T,
                           uint64_t n, cudaStream_t st) {
    if (n < 2 || T == 0) return OK;
    std::vector<const Fr*> c(T);
    for (uint32_t j = 0; j < T; j++) c[j] = static_cast<const Fr*>(a[j]) + 1;
    return linrec_suffix_batch(ctx, c.data(), reinterpret_cast<Fr* const*>(q), b, T, n - 1, st);
}

}  // namespace mzk
