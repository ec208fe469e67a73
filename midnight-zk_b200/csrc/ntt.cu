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
constexpr uint32_t kLoBits = 12;            // low table: w^i for i < 4096

// w^e from the split tables (e < N)
__device__ __forceinline__ Fr root_pow(const Fr* __restrict__ tlo, const Fr* __restrict__ thi, uint32_t e) {
    const Fr lo = tlo[e & ((1u << kLoBits) - 1)];
    if ((e >> kLoBits) == 0) return lo;
    return fr_mul(thi[e >> kLoBits], lo);
}

struct PassArgs {
    const Fr* in;
    Fr* out;
    const Fr* tlo;
    const Fr* thi;
    uint32_t log_n, log_s, log_r;
    uint32_t n_real;   // elements present in `in`; larger indices read as zero
    int use_pre;       // multiply input element i by pre[i % 3] (coset scaling)
    int twiddle_after; // inter-pass twiddle (all passes but the last)
    Fr pre[3];
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

__global__ void __launch_bounds__(kNttThreads) k_ntt_dif_pass(PassArgs a) {
    extern __shared__ uint4 smem_raw[];
    const uint32_t N = 1u << a.log_n;
    const uint32_t R = 1u << a.log_r;
    const uint32_t log_m = a.log_s - a.log_r;  // columns per segment = 2^log_m
    const uint32_t tile = min(kTile, N);
    const uint32_t log_b = (31 - __clz(tile)) - a.log_r;  // columns per block = 2^log_b
    const uint32_t B = 1u << log_b;
    const FrPlanes sx{smem_raw, smem_raw + tile};
    const FrPlanes sw{smem_raw + 2 * tile, smem_raw + 2 * tile + R / 2};  // w_R^u for u < R/2
    const uint32_t c0 = blockIdx.x << log_b;

    for (uint32_t u = threadIdx.x; u < R / 2; u += blockDim.x) sw.set(u, root_pow(a.tlo, a.thi, u << (a.log_n - a.log_r)));
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) {
        const uint32_t m = e >> log_b, b = e & (B - 1);
        const uint32_t c = c0 + b;
        const uint32_t idx = ((c >> log_m) << a.log_s) + (m << log_m) + (c & ((1u << log_m) - 1));
        Fr v = fr_zero();
        if (idx < a.n_real) {
            v = a.in[idx];
            if (a.use_pre) {
                const uint32_t r3 = idx % 3;
                if (r3) v = fr_mul(v, a.pre[r3]);
            }
        }
        sx.set(e, v);
    }
    __syncthreads();
    for (uint32_t s = 0; s < a.log_r; s++) {
        const uint32_t log_h = a.log_r - 1 - s;
        const uint32_t h = 1u << log_h;
        for (uint32_t q = threadIdx.x; q < tile / 2; q += blockDim.x) {
            const uint32_t b = q & (B - 1), p = q >> log_b;
            const uint32_t pos = p & (h - 1);
            const uint32_t m0 = ((p >> log_h) << (log_h + 1)) + pos;
            const uint32_t i0 = (m0 << log_b) + b, i1 = ((m0 + h) << log_b) + b;
            const Fr x0 = sx.get(i0), x1 = sx.get(i1);
            sx.set(i0, fr_add(x0, x1));
            Fr v = fr_sub(x0, x1);
            if (pos) v = fr_mul(v, sw.get(pos << s));
            sx.set(i1, v);
        }
        __syncthreads();
    }
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) {
        const uint32_t m = e >> log_b, b = e & (B - 1);
        const uint32_t c = c0 + b;
        const uint32_t j = c & ((1u << log_m) - 1);
        const uint32_t idx = ((c >> log_m) << a.log_s) + (m << log_m) + j;
        Fr v = sx.get(e);
        if (a.twiddle_after && j) {
            const uint32_t k1 = __brev(m) >> (32 - a.log_r);
            const uint32_t ex = (j * k1) << (a.log_n - a.log_s);  // (N/S) j k1 < N
            v = fr_mul(v, root_pow(a.tlo, a.thi, ex & (N - 1)));
        }
        a.out[idx] = v;
    }
}

// in place: a[i] <-> a[bitrev(i)], each output multiplied by scale[i % 3]
__global__ void k_bitrev_scale(Fr* __restrict__ a, uint32_t log_n, int use_scale, Fr s0, Fr s1, Fr s2) {
    const uint32_t N = 1u << log_n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
        const uint32_t j = log_n ? (__brev(i) >> (32 - log_n)) : 0u;
        if (j < i) continue;
        const Fr x = a[i];
        const Fr y = a[j];
        Fr oi = y, oj = x;
        if (use_scale) {
            const uint32_t ri = i % 3, rj = j % 3;
            oi = fr_mul(oi, ri == 0 ? s0 : (ri == 1 ? s1 : s2));
            oj = fr_mul(oj, rj == 0 ? s0 : (rj == 1 ? s1 : s2));
        }
        a[i] = oi;
        if (j != i) a[j] = oj;
    }
}

// out[i] = in[bitrev(i)] * scale[i % 3] for i < m (gathers a prefix of the
// natural-order result out of a bit-reversed vector of length 2^log_n)
__global__ void k_bitrev_gather(const Fr* __restrict__ in, Fr* __restrict__ out, uint32_t log_n, uint32_t m, Fr s0,
                                Fr s1, Fr s2) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const uint32_t j = log_n ? (__brev(i) >> (32 - log_n)) : 0u;
        const uint32_t r = i % 3;
        out[i] = fr_mul(in[j], r == 0 ? s0 : (r == 1 ? s1 : s2));
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

Domain::~Domain() {
    for (auto& t : tables)
        if (t) cudaFree(t);
    if (d_tinv) cudaFree(d_tinv);
}

// EvaluationDomain::new (proofs/src/poly/domain.rs:54-167)
Status domain_create(Context* ctx, uint32_t j, uint32_t k, Domain** out) {
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
    *out = d;
    return OK;
}

// Forward DIF passes over 2^log_n elements with root table `root` (0..3),
// first pass reading `in` (n_real elements, optional coset scaling) and
// writing `out`; later passes in place on `out`.  Output bit-reversed.
static Status dif_passes(Context* ctx, const Domain* d, int root, uint32_t log_n, const Fr* in, Fr* out,
                         uint32_t n_real, bool coset, cudaStream_t st) {
    const uint32_t N = 1u << log_n;
    const uint32_t tile = std::min(kTile, N);
    const uint32_t tile_log = std::min(kTileLog, log_n);
    const uint32_t passes = (log_n + tile_log - 1) / tile_log;
    MZK_CUDA_CHECK(cudaFuncSetAttribute(k_ntt_dif_pass, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(kTile * sizeof(Fr) + kTile / 2 * sizeof(Fr))));
    uint32_t log_s = log_n;
    for (uint32_t p = 0; p < passes; p++) {
        const uint32_t rem = passes - p;
        const uint32_t log_r = (log_s + rem - 1) / rem;  // even split, larger passes first
        PassArgs a;
        a.in = p == 0 ? in : out;
        a.out = out;
        a.tlo = d->lo[root];
        a.thi = d->hi[root];
        a.log_n = log_n;
        a.log_s = log_s;
        a.log_r = log_r;
        a.n_real = p == 0 ? n_real : N;
        a.use_pre = (p == 0 && coset) ? 1 : 0;
        a.twiddle_after = p + 1 < passes ? 1 : 0;
        a.pre[0] = to_dev(host::fr_one());
        a.pre[1] = to_dev(d->zeta);
        a.pre[2] = to_dev(d->zeta2);
        const size_t smem = (size_t)tile * sizeof(Fr) + (size_t)(1u << log_r) / 2 * sizeof(Fr);
        k_ntt_dif_pass<<<N / tile, kNttThreads, smem, st>>>(a);
        MZK_LAUNCH_CHECK(ctx);
        log_s -= log_r;
    }
    return OK;
}

static Status bitrev(Context* ctx, Fr* a, uint32_t log_n, bool scale, const host::Fr4& s0, const host::Fr4& s1,
                     const host::Fr4& s2, cudaStream_t st) {
    const uint32_t N = 1u << log_n;
    k_bitrev_scale<<<grid_for(ctx, N, 256), 256, 0, st>>>(a, log_n, scale ? 1 : 0, to_dev(s0), to_dev(s1), to_dev(s2));
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

Status domain_op_device(Context* ctx, const Domain* d, int op, const void* d_in, void* d_out, cudaStream_t st) {
    const uint32_t k = d->k, ek = d->ext_k;
    const uint32_t n = 1u << k, en = 1u << ek;
    const host::Fr4 one = host::fr_one();
    Fr* out = static_cast<Fr*>(d_out);
    const Fr* in = static_cast<const Fr*>(d_in);
    switch (op) {
        case OP_COEFF_TO_LAGRANGE:  // best_fft(a, omega)
            MZK_TRY(dif_passes(ctx, d, 0, k, in, out, n, false, st));
            return bitrev(ctx, out, k, false, one, one, one, st);
        case OP_LAGRANGE_TO_COEFF:  // ifft: best_fft(a, omega_inv), * n^-1
            MZK_TRY(dif_passes(ctx, d, 1, k, in, out, n, false, st));
            return bitrev(ctx, out, k, true, d->ifft_div, d->ifft_div, d->ifft_div, st);
        case OP_COEFF_TO_EXTENDED:  // zeta^(i mod 3) scaling, pad to 2^ext_k, fft(ext_omega)
            MZK_TRY(dif_passes(ctx, d, 2, ek, in, out, n, true, st));
            return bitrev(ctx, out, ek, false, one, one, one, st);
        case OP_EXTENDED_TO_COEFF: {  // ifft(ext_omega_inv), * (2^ext_k)^-1, zeta unscaling
            MZK_TRY(dif_passes(ctx, d, 3, ek, in, out, en, false, st));
            const host::Fr4 s1 = host::fr_mul(d->ext_ifft_div, d->zeta2), s2 = host::fr_mul(d->ext_ifft_div, d->zeta);
            return bitrev(ctx, out, ek, true, d->ext_ifft_div, s1, s2, st);
        }
        case OP_EXTENDED_TO_LAGRANGE: {  // in (2^ext_k, consumed) -> out (n)
            Fr* work = const_cast<Fr*>(in);
            MZK_TRY(dif_passes(ctx, d, 3, ek, in, work, en, false, st));
            const host::Fr4 s1 = host::fr_mul(d->ext_ifft_div, d->zeta2), s2 = host::fr_mul(d->ext_ifft_div, d->zeta);
            k_bitrev_gather<<<grid_for(ctx, n, 256), 256, 0, st>>>(work, out, ek, n, to_dev(d->ext_ifft_div), to_dev(s1),
                                                                 to_dev(s2));
            MZK_LAUNCH_CHECK(ctx);
            MZK_TRY(dif_passes(ctx, d, 0, k, out, out, n, false, st));
            return bitrev(ctx, out, k, false, one, one, one, st);
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
