// ntt.cu — the Fr NTTs of EvaluationDomain on the device.
//
// Replaces EvaluationDomain::{coeff_to_lagrange, lagrange_to_coeff,
// coeff_to_extended, extended_to_coeff, extended_to_lagrange,
// divide_by_vanishing_poly} (proofs/src/poly/domain.rs:249-380) and the FFTs
// under them (curves/src/fft.rs:56-198).  Outputs are the same field elements
// (an NTT has exactly one result), computed by a different schedule:
//
//  * passes of radix 2^r (r <= 11) decimation-in-frequency: a block loads a
//    tile of 2048 elements = 2^r rows x (2048 / 2^r) columns, runs r radix-2
//    Gentleman-Sande stages in shared memory, multiplies row k1 of column j by
//    the inter-pass twiddle w_S^(j*k1) and stores in place.  log2 n = 24 takes
//    three passes (8 + 8 + 8), 2^26 three (9 + 9 + 8).  Natural order in,
//    bit-reversed order out.
//  * one in-place bit-reversal pass restores natural order and applies the
//    output scaling of the inverse transforms (n^-1, and the coset factors of
//    extended_to_coeff) in the same sweep.
//  * coeff_to_extended's coset scaling (a_i *= zeta^(i mod 3),
//    distribute_powers_zeta, domain.rs:398-414) and zero padding from n to 4n
//    are applied while the first pass loads its tile (indices >= n are never
//    read), so the padded vector is never materialised.
//  * twiddles w^e come from two small tables per root (w^i and w^(4096 i)),
//    one multiplication per lookup, instead of an n/2-entry table.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "field.cuh"
#include "host_ec.hpp"
#include "ntt.hpp"
#include "runtime.hpp"

namespace mzk {

namespace {

constexpr uint32_t kTileLog = 11;
constexpr uint32_t kTile = 1u << kTileLog;  // elements per block
constexpr int kNttThreads = 256;
static_assert(kTile % kNttThreads == 0, "a tile is a whole number of elements per thread");
constexpr uint32_t kLoBits = 12;            // low table: w^i for i < 4096

// w^e from the split tables (e < N)
__device__ __forceinline__ Fr root_pow(const Fr* __restrict__ tlo, const Fr* __restrict__ thi, uint32_t e) {
    const Fr lo = tlo[e & ((1u << kLoBits) - 1)];
    if ((e >> kLoBits) == 0) return lo;
    return fr_mul(thi[e >> kLoBits], lo);
}

// transforms of one batched launch (blockIdx.y picks one)
constexpr uint32_t kNttBatch = 64;

struct PassArgs {
    const Fr* in[kNttBatch];
    Fr* out[kNttBatch];
    const Fr* tlo;
    const Fr* thi;
    const Fr* ptw;  // the pass's twiddle table (Domain::pass_tw), or null: formed from tlo x thi
    uint32_t log_n, log_s, log_r;
    uint32_t n_real;   // elements present in `in`; larger indices read as zero
    int use_pre;       // multiply input element i by pre[i % 3] (coset scaling)
    int twiddle_after; // inter-pass twiddle (all passes but the last)
    Fr pre[3];
    // last pass only: write element idx to out[bitrev(idx)] (natural order),
    // times post[bitrev(idx) % 3] when use_post, and only when bitrev(idx) < m_out
    int bitrev_out;
    int use_post;
    uint32_t m_out;
    Fr post[3];
};

// Shared-memory tiles hold Fr elements as two planes of 16-byte halves, so a
// warp's element accesses are contiguous 128-bit loads without bank conflicts
// (a 32-byte element read word by word at a 32-byte stride conflicts 8-way).
struct FrPlanes {
    uint4* lo;
    uint4* hi;
    __device__ __forceinline__ Fr get(uint32_t i) const {
        const uint4 a = lo[i], b = hi[i];
        Fr r;
        r.l[0] = a.x; r.l[1] = a.y; r.l[2] = a.z; r.l[3] = a.w;
        r.l[4] = b.x; r.l[5] = b.y; r.l[6] = b.z; r.l[7] = b.w;
        return r;
    }
    __device__ __forceinline__ void set(uint32_t i, const Fr& v) const {
        lo[i] = make_uint4(v.l[0], v.l[1], v.l[2], v.l[3]);
        hi[i] = make_uint4(v.l[4], v.l[5], v.l[6], v.l[7]);
    }
};

// Shared-memory slot of tile element e: the low 3 bits XORed with bits 3..5.
// A quarter-warp's 16-byte accesses then hit 8 different 16-byte bank
// groups for the strided patterns of the last rounds (row strides of 8, 16
// and 32 elements) as well as for contiguous runs.
__device__ __forceinline__ uint32_t swz(uint32_t e) { return e ^ ((e >> 3) & 7u); }

// Shared-memory slot of twiddle w_R^u (u < 1024): the low 3 bits XORed with
// the XOR of the 3-bit chunks above them.  A stage reads u = j << sigma for
// consecutive j (sigma = 0..9); for every sigma the 8 lanes of a
// quarter-warp then land in 8 different 16-byte bank groups.
__device__ __forceinline__ uint32_t tw_swz(uint32_t u) { return u ^ (((u >> 3) ^ (u >> 6) ^ (u >> 9)) & 7u); }

// K consecutive DIF stages s .. s+K-1 of the tile in registers: each thread
// takes groups of 2^K elements of one column at rows m0 + i q (q = 2^log_q,
// the last stage's half-size), runs the K radix-2 stages on them and stores
// them back.  Stage s+t pairs rows r and r + q 2^(K-1-t); its twiddle is
// w_R^(pos << (s+t)) with pos = r mod (q 2^(K-t)).
// Every product of a stage is issued unconditionally, so the stage is one
// basic block whose independent carry chains the scheduler interleaves: a
// butterfly with pos = 0 multiplies by w^0 = 1 (Montgomery one; the product
// is the same canonical value).  In the pass's last round (kLast: q = 1,
// j = 0) the pos = 0 butterflies are known at compile time and skipped.
template <int K, bool kLast>
__device__ __forceinline__ void dif_round(const FrPlanes& sx, const FrPlanes& sw, uint32_t s, uint32_t log_r,
                                          uint32_t log_b, uint32_t tile) {
    const uint32_t log_q = kLast ? 0u : log_r - s - K;
    const uint32_t B = 1u << log_b;
    for (uint32_t g = threadIdx.x; g < (tile >> K); g += blockDim.x) {
        const uint32_t b = g & (B - 1);
        const uint32_t rest = g >> log_b;
        const uint32_t j = kLast ? 0u : rest & ((1u << log_q) - 1);
        const uint32_t m0 = ((rest >> log_q) << (log_q + K)) + j;
        Fr x[1 << K];
#pragma unroll
        for (int i = 0; i < (1 << K); i++) x[i] = sx.get(swz(((m0 + ((uint32_t)i << log_q)) << log_b) + b));
#pragma unroll
        for (int t = 0; t < K; t++) {
            const int d = 1 << (K - 1 - t);
#pragma unroll
            for (int i = 0; i < (1 << K); i++) {
                const int off = i & (2 * d - 1);
                if (off < d) {
                    const Fr x0 = x[i], x1 = x[i + d];
                    x[i] = fr_add(x0, x1);
                    const Fr v = fr_sub(x0, x1);
                    if (kLast && off == 0) {
                        x[i + d] = v;
                    } else {
                        const uint32_t pos = j + ((uint32_t)off << log_q);
                        x[i + d] = fr_mul(v, sw.get(tw_swz(pos << (s + (uint32_t)t))));
                    }
                }
            }
        }
#pragma unroll
        for (int i = 0; i < (1 << K); i++) sx.set(swz(((m0 + ((uint32_t)i << log_q)) << log_b) + b), x[i]);
    }
}

__global__ void __launch_bounds__(kNttThreads, 2) k_ntt_dif_pass(PassArgs a) {
    extern __shared__ uint4 smem_raw[];
    const uint32_t N = 1u << a.log_n;
    const uint32_t R = 1u << a.log_r;
    const uint32_t log_m = a.log_s - a.log_r;  // columns per segment = 2^log_m
    const uint32_t tile = min(kTile, N);
    const uint32_t log_b = (31 - __clz(tile)) - a.log_r;  // columns per block = 2^log_b
    const uint32_t B = 1u << log_b;
    const FrPlanes sx{smem_raw, smem_raw + tile};
    const FrPlanes sw{smem_raw + 2 * tile, smem_raw + 2 * tile + R / 2};  // w_R^u for u < R/2
    // columns of this block: B consecutive columns, or, in the last pass, the
    // columns blockIdx.x + b * 2^(log_ncol - log_b), whose bit-reversed
    // output positions are B consecutive elements (256-byte runs for B = 8)
    const uint32_t log_ncol = a.log_n - a.log_r;
    const uint32_t c0 = a.bitrev_out ? blockIdx.x : blockIdx.x << log_b;
    const uint32_t cstep_log = a.bitrev_out ? log_ncol - log_b : 0u;

    for (uint32_t u = threadIdx.x; u < R / 2; u += blockDim.x)
        sw.set(tw_swz(u), root_pow(a.tlo, a.thi, u << (a.log_n - a.log_r)));
    // all of a thread's global loads are issued before the first is used
    constexpr int kPer = kTile / kNttThreads;
    Fr v[kPer];
    uint32_t vidx[kPer];
#pragma unroll
    for (int q = 0; q < kPer; q++) {
        const uint32_t e = threadIdx.x + (uint32_t)q * kNttThreads;
        const uint32_t m = e >> log_b, b = e & (B - 1);
        const uint32_t c = c0 + (b << cstep_log);
        vidx[q] = ((c >> log_m) << a.log_s) + (m << log_m) + (c & ((1u << log_m) - 1));
        v[q] = fr_zero();
        if (e < tile && vidx[q] < a.n_real) v[q] = a.in[blockIdx.y][vidx[q]];
    }
#pragma unroll
    for (int q = 0; q < kPer; q++) {
        const uint32_t e = threadIdx.x + (uint32_t)q * kNttThreads;
        if (e >= tile) continue;
        if (a.use_pre && vidx[q] < a.n_real) {
            const uint32_t r3 = vidx[q] % 3;
            if (r3) v[q] = fr_mul(v[q], a.pre[r3]);
        }
        sx.set(swz(e), v[q]);
    }
    __syncthreads();
    // stages in rounds of three (radix 8), the last round of one or two
    for (uint32_t s = 0; s < a.log_r;) {
        const uint32_t k = min(3u, a.log_r - s);
        const bool last = s + k == a.log_r;
        if (k == 3) {
            if (last) dif_round<3, true>(sx, sw, s, a.log_r, log_b, tile);
            else dif_round<3, false>(sx, sw, s, a.log_r, log_b, tile);
        } else if (k == 2) {
            if (last) dif_round<2, true>(sx, sw, s, a.log_r, log_b, tile);
            else dif_round<2, false>(sx, sw, s, a.log_r, log_b, tile);
        } else {
            if (last) dif_round<1, true>(sx, sw, s, a.log_r, log_b, tile);
            else dif_round<1, false>(sx, sw, s, a.log_r, log_b, tile);
        }
        __syncthreads();
        s += k;
    }
    // unrolled so that the twiddle-table loads of several elements are in flight
#pragma unroll 4
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) {
        const uint32_t m = e >> log_b, b = e & (B - 1);
        const uint32_t c = c0 + (b << cstep_log);
        const uint32_t j = c & ((1u << log_m) - 1);
        const uint32_t idx = ((c >> log_m) << a.log_s) + (m << log_m) + j;
        Fr v = sx.get(swz(e));
        if (a.twiddle_after) {  // uniform; j k1 = 0 multiplies by w^0 = 1 (branch-free)
            Fr w;
            if (a.ptw) {  // uniform: one coalesced load at the element's offset in its segment
                w = a.ptw[(m << log_m) + j];
            } else {
                const uint32_t k1 = __brev(m) >> (32 - a.log_r);
                const uint32_t ex = ((j * k1) << (a.log_n - a.log_s)) & (N - 1);  // (N/S) j k1 < N
                w = fr_mul(a.thi[ex >> kLoBits], a.tlo[ex & ((1u << kLoBits) - 1)]);
            }
            v = fr_mul(v, w);
        }
        if (a.bitrev_out) {
            const uint32_t o = a.log_n ? (__brev(idx) >> (32 - a.log_n)) : 0u;
            if (o < a.m_out) {
                if (a.use_post) {
                    const uint32_t r = o % 3;
                    v = fr_mul(v, a.post[r]);
                }
                a.out[blockIdx.y][o] = v;
            }
        } else {
            a.out[blockIdx.y][idx] = v;
        }
    }
}

// a[i] *= f[i & (len - 1)]
__global__ void k_scale_periodic(Fr* __restrict__ a, uint32_t n, const Fr* __restrict__ f, uint32_t len) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) a[i] = fr_mul(a[i], f[i & (len - 1)]);
}

// out[i] = base^(i * step) for i < count (table construction)
__global__ void k_pow_table(Fr base, uint32_t count, Fr* __restrict__ out) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        Fr acc = fr_one(), b = base;
        for (uint32_t e = i; e; e >>= 1) {
            if (e & 1u) acc = fr_mul(acc, b);
            b = fr_mul(b, b);
        }
        out[i] = acc;
    }
}

// tw[i] = w^((N/S) j bitrev_r(m)) for i = (m << (log_s - log_r)) + j < S: the
// inter-pass twiddle of the element a pass writes at offset i of its segment
__global__ void k_pass_twiddles(const Fr* __restrict__ tlo, const Fr* __restrict__ thi, uint32_t log_n,
                                uint32_t log_s, uint32_t log_r, Fr* __restrict__ tw) {
    const uint32_t S = 1u << log_s, N = 1u << log_n, log_m = log_s - log_r;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < S; i += stride) {
        const uint32_t m = i >> log_m, j = i & ((1u << log_m) - 1);
        const uint32_t k1 = __brev(m) >> (32 - log_r);
        const uint32_t ex = ((j * k1) << (log_n - log_s)) & (N - 1);
        tw[i] = fr_mul(thi[ex >> kLoBits], tlo[ex & ((1u << kLoBits) - 1)]);
    }
}

Fr to_dev(const host::Fr4& x) {
    Fr r;
    std::memcpy(r.l, x.l, 32);
    return r;
}

// ROOT_OF_UNITY (2^32-th root, Montgomery) and ZETA (cube root), fq.rs:70-77, :702-710
const uint64_t kRootOfUnity[4] = {0xb9b58d8c5f0e466aULL, 0x5b1b4c801819d7ecULL, 0x0af53ae352a31e64ULL,
                                  0x5bf3adda19e9b27bULL};
const uint64_t kZeta[4] = {0x92d9090b093011d2ULL, 0xfc9cbd719d6aa073ULL, 0xc1f14ef0cd65a1a6ULL,
                           0x017f6d35e72fcdebULL};

uint32_t grid_for(Context* ctx, uint32_t n, uint32_t threads) {
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(((uint64_t)n + threads - 1) / threads,
                                                               (uint64_t)ctx->num_sms * 16));
}

}  // namespace

// log2 of the rows of each pass of a transform of 2^log_n elements under a
// split mode: every pass keeps at least one stage and at most the tile's;
// the remaining passes can always take what is left
static std::vector<uint32_t> pass_logs(uint32_t log_n, int split) {
    const uint32_t tile_log = std::min(kTileLog, log_n);
    const uint32_t passes = (log_n + tile_log - 1) / tile_log;
    std::vector<uint32_t> logs;
    uint32_t log_s = log_n;
    for (uint32_t p = 0; p < passes; p++) {
        const uint32_t rem = passes - p;
        uint32_t log_r = (log_s + rem - 1) / rem;  // even split, larger passes first
        if (split == kSplitFront) log_r = std::min(tile_log, log_s - (rem - 1));
        if (split == kSplitBack) log_r = std::max(1u, log_s - (rem - 1) * tile_log);
        logs.push_back(log_r);
        log_s -= log_r;
    }
    return logs;
}

static int split_of(const Context* ctx, uint32_t log_n) {
    return log_n < (uint32_t)kTuneSlots ? ctx->tuned_ntt_split[log_n] : 0;
}

// The twiddle table of a non-last pass (Domain::pass_tw), built when missing.
// Building allocates and synchronises `st` (so that other streams may read
// the table at once), so it is skipped while `st` is being captured, and a
// failed allocation is not an error: either way the pass forms its twiddles
// from the split tables instead (the same values).
static const Fr* pass_twiddles(Context* ctx, const Domain* d, int root, uint32_t log_n, uint32_t log_s,
                               uint32_t log_r, cudaStream_t st) {
    std::lock_guard<std::mutex> g(d->tw_mu);
    const auto key = std::make_tuple(root, log_s, log_r);
    const auto it = d->pass_tw.find(key);
    if (it != d->pass_tw.end()) return it->second;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return nullptr;
    Fr* p = nullptr;
    if (cudaMalloc(&p, ((size_t)1 << log_s) * sizeof(Fr)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    k_pass_twiddles<<<grid_for(ctx, 1u << log_s, 256), 256, 0, st>>>(d->lo[root], d->hi[root], log_n, log_s, log_r, p);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
        cudaFree(p);
        return nullptr;
    }
    ctx->launches++;
    d->pass_tw[key] = p;
    return p;
}

Domain::~Domain() {
    for (auto& t : tables)
        if (t) cudaFree(t);
    for (auto& kv : pass_tw) cudaFree(kv.second);
    if (d_tinv) cudaFree(d_tinv);
}

// EvaluationDomain::new (proofs/src/poly/domain.rs:54-167)
Status domain_create(Context* ctx, uint32_t j, uint32_t k, Domain** out) {
    // the pass kernel's shared memory limit, set here once rather than per
    // transform: transforms may be captured into CUDA graphs
    MZK_CUDA_CHECK(cudaFuncSetAttribute(k_ntt_dif_pass, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(kTile * sizeof(Fr) + kTile / 2 * sizeof(Fr))));
    *out = nullptr;
    if (j < 2 || k < 1 || k > 28) {
        set_error("domain: need j >= 2 and 1 <= k <= 28");
        return ERR_ARG;
    }
    const uint64_t qdeg = j - 1, n = 1ull << k;
    uint32_t ext_k = k;
    while ((1ull << ext_k) < n * qdeg) ext_k++;
    if (ext_k > 28) {
        set_error("domain: extended domain above 2^28");
        return ERR_ARG;
    }
    Domain* d = new Domain();
    d->k = k;
    d->ext_k = ext_k;
    d->quotient_poly_degree = (uint32_t)qdeg;
    host::Fr4 ext_omega;
    std::memcpy(ext_omega.l, kRootOfUnity, 32);
    for (uint32_t i = ext_k; i < 32; i++) ext_omega = host::fr_mul(ext_omega, ext_omega);
    host::Fr4 omega = ext_omega;
    for (uint32_t i = k; i < ext_k; i++) omega = host::fr_mul(omega, omega);
    std::memcpy(d->zeta.l, kZeta, 32);
    d->zeta2 = host::fr_mul(d->zeta, d->zeta);
    d->omega = omega;
    d->ext_omega = ext_omega;
    d->omega_inv = host::fr_inv(omega);
    d->ext_omega_inv = host::fr_inv(ext_omega);
    d->ifft_div = host::fr_inv(host::fr_from_u64(n));
    d->ext_ifft_div = host::fr_inv(host::fr_from_u64(1ull << ext_k));
    // t(X) = X^n - 1 on the coset zeta * ext_omega^i, inverted
    uint64_t ne[1] = {n};
    const host::Fr4 orig = host::fr_pow(d->zeta, ne, 1), step = host::fr_pow(ext_omega, ne, 1);
    host::Fr4 cur = orig;
    const uint32_t tlen = 1u << (ext_k - k);
    for (uint32_t i = 0; i < tlen; i++) {
        d->t_inv.push_back(host::fr_inv(host::fr_sub(cur, host::fr_one())));
        cur = host::fr_mul(cur, step);
    }
    // device tables: for each root w of order N: w^i (i < 4096) and w^(4096 i)
    const host::Fr4 roots[4] = {d->omega, d->omega_inv, d->ext_omega, d->ext_omega_inv};
    const uint32_t logs[4] = {k, k, ext_k, ext_k};
    for (int r = 0; r < 4; r++) {
        const uint32_t N = 1u << logs[r];
        const uint32_t lo = std::min<uint32_t>(N, 1u << kLoBits);
        const uint32_t hi = std::max<uint32_t>(1, N >> kLoBits);
        Fr* p = nullptr;
        cudaError_t e = cudaMalloc(&p, (size_t)(lo + hi) * sizeof(Fr));
        if (e != cudaSuccess) {
            delete d;
            set_error(std::string("domain tables: ") + cudaGetErrorString(e));
            return ERR_OOM;
        }
        d->tables[r] = p;
        d->lo[r] = p;
        d->hi[r] = p + lo;
        uint64_t e4096[1] = {1ull << kLoBits};
        const host::Fr4 w4096 = host::fr_pow(roots[r], e4096, 1);
        k_pow_table<<<grid_for(ctx, lo, 128), 128, 0, ctx->stream>>>(to_dev(roots[r]), lo, d->lo[r]);
        MZK_LAUNCH_CHECK(ctx);
        k_pow_table<<<grid_for(ctx, hi, 128), 128, 0, ctx->stream>>>(to_dev(w4096), hi, d->hi[r]);
        MZK_LAUNCH_CHECK(ctx);
    }
    {
        cudaError_t e = cudaMalloc(&d->d_tinv, (size_t)tlen * sizeof(Fr));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d->d_tinv, d->t_inv.data(), (size_t)tlen * 32, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            delete d;
            set_error(std::string("domain set-up: ") + cudaGetErrorString(e));
            return ERR_CUDA;
        }
    }
    // the pass twiddle tables of the split in force for each root's size
    for (int r = 0; r < 4; r++) {
        const uint32_t log_n = logs[r];
        const std::vector<uint32_t> pl = pass_logs(log_n, split_of(ctx, log_n));
        uint32_t log_s = log_n;
        for (size_t p = 0; p + 1 < pl.size(); p++) {
            pass_twiddles(ctx, d, r, log_n, log_s, pl[p], ctx->stream);
            log_s -= pl[p];
        }
    }
    *out = d;
    return OK;
}

// The DIF passes of T transforms over 2^log_n elements each with root table
// `root` (0..3), ending in natural order, up to kNttBatch transforms per
// launch (blockIdx.y: the transform; every transform has its own slice of
// the scratch).  The first pass reads in[t] (n_real elements, optional coset
// scaling).  The last pass writes every element to its bit-reversed position
// (times post[i % 3] when post is given, only positions < m_out).  Since
// that pass's writes cross blocks, it reads from the scratch the earlier
// passes wrote, so in[t] and out[t] may be the same buffer.  A transform of
// one tile (log_n <= 11) is one block, which reads all before it writes.
static Status dif_passes(Context* ctx, const Domain* d, int root, uint32_t log_n, const Fr* const* in,
                         Fr* const* out, uint32_t T, uint32_t n_real, bool coset, const host::Fr4* post,
                         uint32_t m_out, cudaStream_t st) {
    const uint32_t N = 1u << log_n;
    const uint32_t tile = std::min(kTile, N);
    const std::vector<uint32_t> logs = pass_logs(log_n, split_of(ctx, log_n));
    const uint32_t passes = (uint32_t)logs.size();
    // transforms per launch: at most kNttBatch and 2^25 elements of scratch
    // (large transforms fill the GPU alone)
    const uint32_t TB = std::min({T, kNttBatch, std::max(1u, (1u << 25) >> log_n)});
    Fr* tmp = nullptr;
    if (passes > 1) {
        void* p;
        MZK_TRY(ctx->ensure("ntt_tmp", (size_t)TB * N * sizeof(Fr), &p));
        tmp = static_cast<Fr*>(p);
    }
    for (uint32_t t0 = 0; t0 < T; t0 += TB) {
        const uint32_t tb = std::min(TB, T - t0);
        uint32_t log_s = log_n;
        for (uint32_t p = 0; p < passes; p++) {
            const uint32_t log_r = logs[p];
            const bool last = p + 1 == passes;
            PassArgs a;
            for (uint32_t t = 0; t < tb; t++) {
                a.in[t] = p == 0 ? in[t0 + t] : tmp + (size_t)t * N;
                a.out[t] = last ? out[t0 + t] : tmp + (size_t)t * N;
            }
            a.tlo = d->lo[root];
            a.thi = d->hi[root];
            a.ptw = last ? nullptr : pass_twiddles(ctx, d, root, log_n, log_s, log_r, st);
            a.log_n = log_n;
            a.log_s = log_s;
            a.log_r = log_r;
            a.n_real = p == 0 ? n_real : N;
            a.use_pre = (p == 0 && coset) ? 1 : 0;
            a.twiddle_after = last ? 0 : 1;
            a.pre[0] = to_dev(host::fr_one());
            a.pre[1] = to_dev(d->zeta);
            a.pre[2] = to_dev(d->zeta2);
            a.bitrev_out = last ? 1 : 0;
            a.use_post = post ? 1 : 0;
            a.m_out = m_out;
            for (int i = 0; i < 3; i++) a.post[i] = to_dev(post ? post[i] : host::fr_one());
            const size_t smem = (size_t)tile * sizeof(Fr) + (size_t)(1u << log_r) / 2 * sizeof(Fr);
            k_ntt_dif_pass<<<dim3(N / tile, tb), kNttThreads, smem, st>>>(a);
            MZK_LAUNCH_CHECK(ctx);
            log_s -= log_r;
        }
    }
    return OK;
}

static Status dif_passes(Context* ctx, const Domain* d, int root, uint32_t log_n, const Fr* in, Fr* out,
                         uint32_t n_real, bool coset, const host::Fr4* post, uint32_t m_out, cudaStream_t st) {
    return dif_passes(ctx, d, root, log_n, &in, &out, 1, n_real, coset, post, m_out, st);
}

// The same domain operation on T inputs of equal size, their passes
// launched together (the transforms of many polynomials of one domain).
Status domain_op_batch(Context* ctx, const Domain* d, int op, const void* const* ins, void* const* outs, uint32_t T,
                       cudaStream_t st) {
    if (T == 0) return OK;
    const uint32_t k = d->k, ek = d->ext_k;
    const uint32_t n = 1u << k, en = 1u << ek;
    const Fr* const* in = reinterpret_cast<const Fr* const*>(ins);
    Fr* const* out = reinterpret_cast<Fr* const*>(outs);
    switch (op) {
        case OP_COEFF_TO_LAGRANGE:
            return dif_passes(ctx, d, 0, k, in, out, T, n, false, nullptr, n, st);
        case OP_LAGRANGE_TO_COEFF: {
            const host::Fr4 post[3] = {d->ifft_div, d->ifft_div, d->ifft_div};
            return dif_passes(ctx, d, 1, k, in, out, T, n, false, post, n, st);
        }
        case OP_COEFF_TO_EXTENDED:
            return dif_passes(ctx, d, 2, ek, in, out, T, n, true, nullptr, en, st);
        case OP_EXTENDED_TO_COEFF: {
            const host::Fr4 post[3] = {d->ext_ifft_div, host::fr_mul(d->ext_ifft_div, d->zeta2),
                                       host::fr_mul(d->ext_ifft_div, d->zeta)};
            return dif_passes(ctx, d, 3, ek, in, out, T, en, false, post, en, st);
        }
        default:
            set_error("domain: batched operation must be C2L, L2C, C2E or E2C");
            return ERR_ARG;
    }
}

Status domain_op_device(Context* ctx, const Domain* d, int op, const void* d_in, void* d_out, cudaStream_t st) {
    const uint32_t k = d->k, ek = d->ext_k;
    const uint32_t n = 1u << k, en = 1u << ek;
    const host::Fr4 one = host::fr_one();
    Fr* out = static_cast<Fr*>(d_out);
    const Fr* in = static_cast<const Fr*>(d_in);
    switch (op) {
        case OP_COEFF_TO_LAGRANGE:  // best_fft(a, omega)
            return dif_passes(ctx, d, 0, k, in, out, n, false, nullptr, n, st);
        case OP_LAGRANGE_TO_COEFF: {  // ifft: best_fft(a, omega_inv), * n^-1
            const host::Fr4 post[3] = {d->ifft_div, d->ifft_div, d->ifft_div};
            return dif_passes(ctx, d, 1, k, in, out, n, false, post, n, st);
        }
        case OP_COEFF_TO_EXTENDED:  // zeta^(i mod 3) scaling, pad to 2^ext_k, fft(ext_omega)
            return dif_passes(ctx, d, 2, ek, in, out, n, true, nullptr, en, st);
        case OP_EXTENDED_TO_COEFF: {  // ifft(ext_omega_inv), * (2^ext_k)^-1, zeta unscaling
            const host::Fr4 post[3] = {d->ext_ifft_div, host::fr_mul(d->ext_ifft_div, d->zeta2),
                                       host::fr_mul(d->ext_ifft_div, d->zeta)};
            return dif_passes(ctx, d, 3, ek, in, out, en, false, post, en, st);
        }
        case OP_EXTENDED_TO_LAGRANGE: {  // in (2^ext_k) -> out (n): E2C truncated to n, then C2L
            const host::Fr4 post[3] = {d->ext_ifft_div, host::fr_mul(d->ext_ifft_div, d->zeta2),
                                       host::fr_mul(d->ext_ifft_div, d->zeta)};
            MZK_TRY(dif_passes(ctx, d, 3, ek, in, out, en, false, post, n, st));
            return dif_passes(ctx, d, 0, k, out, out, n, false, nullptr, n, st);
        }
        case OP_DIVIDE_BY_VANISHING: {
            if (in != out) MZK_CUDA_CHECK(cudaMemcpyAsync(out, in, (size_t)en * sizeof(Fr), cudaMemcpyDeviceToDevice, st));
            k_scale_periodic<<<grid_for(ctx, en, 256), 256, 0, st>>>(out, en, static_cast<const Fr*>(d->d_tinv),
                                                                   (uint32_t)d->t_inv.size());
            MZK_LAUNCH_CHECK(ctx);
            return OK;
        }
        default:
            set_error("domain: unknown operation");
            return ERR_ARG;
    }
}

size_t domain_op_in_len(const Domain* d, int op) {
    const size_t n = 1ull << d->k, en = 1ull << d->ext_k;
    switch (op) {
        case OP_COEFF_TO_LAGRANGE:
        case OP_LAGRANGE_TO_COEFF:
        case OP_COEFF_TO_EXTENDED:
            return n;
        default:
            return en;
    }
}

size_t domain_op_out_len(const Domain* d, int op) {
    const size_t n = 1ull << d->k, en = 1ull << d->ext_k;
    switch (op) {
        case OP_COEFF_TO_LAGRANGE:
        case OP_LAGRANGE_TO_COEFF:
        case OP_EXTENDED_TO_LAGRANGE:
            return n;
        default:
            return en;
    }
}

}  // namespace mzk
