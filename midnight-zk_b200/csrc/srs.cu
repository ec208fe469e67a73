// srs.cu — the G1 part of the KZG test setup on the device
// (ParamsKZG::unsafe_setup, proofs/src/poly/kzg/params.rs:160-209):
//
//   g[i]                    = [s^i] G
//   g_lagrange[i]           = [L_i(s)] G,  L_i(s) = (s^n - 1) / n * w^i / (s - w^i)
//   g_lagrange_delta        = suffix_sum(g_lagrange)        (params.rs:47-57)
//   g_lagrange_double_delta = suffix_sum(g_lagrange_delta)
//
// Scalars come from device scans (powers of s, one batch inversion), the
// points from the fixed-base table of G, the suffix sums from a chunked
// point scan in XYZZ coordinates, normalised to affine at the end.  Affine
// points are unique, so the results equal the reference's batch-normalised
// Jacobian sums.  The G2 part (g2, [s]g2) is not built here.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>
#include <string>

#include "../../include/mzk.h"
#include "ec.cuh"
#include "grand.hpp"
#include "host_ec.hpp"
#include "ntt.hpp"
#include "runtime.hpp"
#include "srs.hpp"

namespace mzk {

namespace {

constexpr int kThreads = 128;
constexpr uint32_t kSufChunk = 32;  // points per thread of a suffix scan

__device__ __forceinline__ Xyzz ld_point(const Affine* p) { return xyzz_from_affine(*p); }
__device__ __forceinline__ Xyzz ld_point(const Xyzz* p) { return *p; }

// local suffix sums of each chunk (zero carry-in) and the chunk totals
template <class In>
__global__ void __launch_bounds__(kThreads) k_suf_local(const In* __restrict__ in, uint64_t n, Xyzz* __restrict__ out,
                                                        Xyzz* __restrict__ totals) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t lo = t * kSufChunk;
    if (lo >= n) return;
    const uint64_t hi = min(n, lo + kSufChunk);
    Xyzz acc;
    xyzz_set_inf(acc);
    for (uint64_t i = hi; i-- > lo;) {
        acc = xyzz_add(acc, ld_point(in + i));
        out[i] = acc;
    }
    totals[t] = acc;
}
// out[i] += carry of the chunks above (their suffix-scanned totals)
__global__ void __launch_bounds__(kThreads) k_suf_apply(Xyzz* __restrict__ out, uint64_t n,
                                                        const Xyzz* __restrict__ scanned, uint64_t chunks) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t + 1 >= chunks) return;
    const Xyzz carry = scanned[t + 1];
    const uint64_t lo = t * kSufChunk, hi = lo + kSufChunk;
    for (uint64_t i = lo; i < hi; i++) out[i] = xyzz_add(out[i], carry);
}
__global__ void __launch_bounds__(kThreads) k_to_affine(const Xyzz* __restrict__ in, uint64_t n,
                                                        Affine* __restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = xyzz_to_affine(in[i]);
}

uint32_t blocks_for(const Context* ctx, uint64_t items) {
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((items + kThreads - 1) / kThreads, (uint64_t)ctx->num_sms * 16));
}

// suffix sums (XYZZ) of n points of type In into out (n), recursively over the chunk totals
template <class In>
Status suffix_scan(Context* ctx, const In* in, Xyzz* out, uint64_t n, cudaStream_t st, int depth = 0) {
    const uint64_t chunks = (n + kSufChunk - 1) / kSufChunk;
    void* tot;
    MZK_TRY(ctx->ensure(("srs_suf_" + std::to_string(depth)).c_str(), 2 * chunks * sizeof(Xyzz), &tot));
    Xyzz* totals = static_cast<Xyzz*>(tot);
    Xyzz* scanned = totals + chunks;
    k_suf_local<In><<<(uint32_t)((chunks + kThreads - 1) / kThreads), kThreads, 0, st>>>(in, n, out, totals);
    MZK_LAUNCH_CHECK(ctx);
    if (chunks > 1) {
        MZK_TRY(suffix_scan<Xyzz>(ctx, totals, scanned, chunks, st, depth + 1));
        k_suf_apply<<<(uint32_t)((chunks + kThreads - 1) / kThreads), kThreads, 0, st>>>(out, n, scanned, chunks);
        MZK_LAUNCH_CHECK(ctx);
    }
    return OK;
}

// den[i] = s - w^i
__global__ void k_lag_den(const Fr* __restrict__ wlo, const Fr* __restrict__ whi, Fr s, uint32_t n,
                          Fr* __restrict__ den) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        den[i] = fr_sub(s, fr_mul(wlo[i & 4095u], whi[i >> 12]));
}
// scal[i] = mult * w^i * inv[i]
__global__ void k_lag_scal(const Fr* __restrict__ wlo, const Fr* __restrict__ whi, Fr mult, uint32_t n,
                           Fr* __restrict__ scal) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        scal[i] = fr_mul(fr_mul(mult, fr_mul(wlo[i & 4095u], whi[i >> 12])), scal[i]);
}

// ---- compressed G1 points (ZCash format, G1Affine::from_compressed,
// curves/src/bls12_381/g1.rs:367-376) ----
struct Exp12 {
    uint32_t l[12];
};

// (p + 1) / 4 and the group order r as 32-bit limbs, from the moduli
Exp12 sqrt_exponent() {
    Exp12 e;
    uint64_t carry = 1;
    for (int i = 0; i < 12; i++) {
        const uint64_t v = (uint64_t)FpP::mod(i) + carry;
        e.l[i] = (uint32_t)v;
        carry = v >> 32;
    }
    for (int i = 0; i < 12; i++) e.l[i] = (e.l[i] >> 2) | (i < 11 ? e.l[i + 1] << 30 : 0u);
    return e;
}
// The G1 membership test of Scott (ePrint 2021/1130, section 6; its proof
// for BLS12-381 completed in ePrint 2022/352): a point P of E(Fp) lies in G1
// iff phi(P) = -[u^2] P, where u = 0xd201000000010000 is |x| of the curve
// parameter x = -u and phi(x, y) = (beta x, y) with beta the cube root of
// unity on which phi acts on G1 as -u^2 (the other root acts as u^2 - 1).
// Same decision as [r] P = O (blst_p1_affine_in_g1, which G1Affine::
// is_torsion_free calls, g1.rs:398-400) for ~1/3 of the group operations.
// beta in Montgomery form (beta * 2^384 mod p); beta = 0x5f19672fdf76ce51
// ba69c6076a0f77eaddb3a93be6f89688de17d813620a00022e01fffffffefffe.
__device__ __forceinline__ uint32_t g1_beta_mont(int i) {
    return i == 0 ? 0x798a64e8u : i == 1 ? 0x30f1361bu : i == 2 ? 0x7ece5a2au : i == 3 ? 0xf3b8ddabu
         : i == 4 ? 0xc61577f7u : i == 5 ? 0x16a8ca3au : i == 6 ? 0x74fd029bu : i == 7 ? 0xc26a2ff8u
         : i == 8 ? 0x60701c6eu : i == 9 ? 0x3636b766u : i == 10 ? 0x241b6160u : 0x051ba4abu;
}
// [u] q, MSB-first double-and-add over the 64-bit u (63 doublings, 5 additions)
__device__ Xyzz xyzz_mul_bls_u(const Xyzz& q) {
    constexpr uint64_t kU = 0xd201000000010000ull;
    Xyzz acc = q;
#pragma unroll 1
    for (int bit = 62; bit >= 0; bit--) {
        acc = xyzz_dbl(acc);
        if ((kU >> bit) & 1u) acc = xyzz_add(acc, q);
    }
    return acc;
}
__device__ bool g1_in_subgroup(const Affine& p) {
    const Xyzz q = xyzz_mul_bls_u(xyzz_mul_bls_u(xyzz_from_affine(p)));
    if (xyzz_is_inf(q)) return false;  // p is not the identity, so phi(p) is not either
    Fp beta;
#pragma unroll
    for (int k = 0; k < 12; k++) beta.l[k] = g1_beta_mont(k);
    // phi(p) = -q  <=>  beta x ZZ = X  and  y ZZZ = -Y
    const Fp bx = fp_mul(beta, p.x);
    return fp_is_zero(fp_sub(q.x, fp_mul(bx, q.zz))) && fp_is_zero(fp_add(q.y, fp_mul(p.y, q.zzz)));
}

__device__ __forceinline__ Fp fp_pow_limbs(const Fp& a, const uint32_t* e, int limbs) {
    Fp acc = fp_one();
    // kept rolled: a full unroll of 384 square-and-multiply steps only
    // inflates the code and the compile time
#pragma unroll 1
    for (int i = limbs - 1; i >= 0; i--)
#pragma unroll 1
        for (int bit = 31; bit >= 0; bit--) {
            acc = fp_sqr(acc);
            if ((e[i] >> bit) & 1u) acc = fp_mul(acc, a);
        }
    return acc;
}

// status: 0 ok, 1 bad encoding, 2 not on the curve, 3 not in G1
__global__ void __launch_bounds__(kThreads) k_g1_decompress(const uint8_t* __restrict__ in, uint64_t n, int check,
                                                            Exp12 sqrt_e, Affine* __restrict__ out,
                                                            uint8_t* __restrict__ status,
                                                            unsigned long long* __restrict__ invalid) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint8_t* b = in + 48 * i;
        uint32_t w[12];
#pragma unroll
        for (int k = 0; k < 12; k++) {  // limb k little-endian from big-endian bytes
            const uint8_t* q = b + 44 - 4 * k;
            w[k] = ((uint32_t)q[0] << 24) | ((uint32_t)q[1] << 16) | ((uint32_t)q[2] << 8) | q[3];
        }
        const uint32_t flags = b[0] & 0xe0u;
        w[11] &= 0x1fffffffu;
        uint8_t st = 0;
        Affine p;
        p.x = fp_zero();
        p.y = fp_zero();
        if (!(flags & 0x80u)) {
            st = 1;
        } else if (flags & 0x40u) {
            uint32_t rest = b[0] & 0x3fu;
#pragma unroll
            for (int k = 0; k < 11; k++) rest |= w[k];
            rest |= w[11];
            if (rest) st = 1;
        } else {
            // x < p
            bool less = false, decided = false;
            for (int k = 11; k >= 0 && !decided; k--)
                if (w[k] != FpP::mod(k)) {
                    less = w[k] < FpP::mod(k);
                    decided = true;
                }
            if (!less) {
                st = 1;
            } else {
                Fp x, r2;
#pragma unroll
                for (int k = 0; k < 12; k++) {
                    x.l[k] = w[k];
                    r2.l[k] = FpP::r2(k);
                }
                x = fp_canonical(fp_mul(x, r2));
                Fp four_m = fp_add(fp_add(fp_one(), fp_one()), fp_add(fp_one(), fp_one()));
                const Fp rhs = fp_add(fp_mul(fp_sqr(x), x), four_m);
                Fp y = fp_canonical(fp_pow_limbs(rhs, sqrt_e.l, 12));
                if (!fp_is_zero(fp_sub(fp_sqr(y), rhs))) {
                    st = 2;
                } else {
                    // the sign flag marks the larger root: y > p - y as integers,
                    // so compare the canonical (non-Montgomery) values
                    const Fp ny = fp_canonical(fp_sub(fp_zero(), y));
                    Fp one_raw;
#pragma unroll
                    for (int k = 0; k < 12; k++) one_raw.l[k] = k == 0 ? 1u : 0u;
                    const Fp yi = fp_canonical(fp_mul(y, one_raw)), nyi = fp_canonical(fp_mul(ny, one_raw));
                    bool y_larger = false;
                    decided = false;
                    for (int k = 11; k >= 0 && !decided; k--)
                        if (yi.l[k] != nyi.l[k]) {
                            y_larger = yi.l[k] > nyi.l[k];
                            decided = true;
                        }
                    if (y_larger != ((flags & 0x20u) != 0)) y = ny;
                    p.x = x;
                    p.y = y;
                    if (check && !g1_in_subgroup(p)) st = 3;
                }
            }
        }
        if (st) {
            p.x = fp_zero();
            p.y = fp_zero();
            atomicAdd(invalid, 1ull);
        }
        out[i] = p;
        if (status) status[i] = st;
    }
}

// ZCash-format compression (G1Affine::to_compressed, g1.rs:326-334, blst's
// p1_affine_compress): x as 48 big-endian bytes of its canonical value,
// flags in the top bits of byte 0: 0x80 compressed, 0x40 the identity (every
// other bit zero), 0x20 y is the larger of y and p - y.
__global__ void __launch_bounds__(kThreads) k_g1_compress(const Affine* __restrict__ in, uint64_t n,
                                                          uint8_t* __restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const Affine p = in[i];
        uint8_t* o = out + 48 * i;
        if (aff_is_inf(p)) {
            o[0] = 0xc0u;
            for (int k = 1; k < 48; k++) o[k] = 0;
            continue;
        }
        Fp one_raw;
#pragma unroll
        for (int k = 0; k < 12; k++) one_raw.l[k] = k == 0 ? 1u : 0u;
        const Fp x = fp_canonical(fp_mul(p.x, one_raw));
        const Fp y = fp_canonical(fp_mul(p.y, one_raw));
        const Fp ny = fp_canonical(fp_sub(fp_zero(), y));  // p - y (0 when y = 0)
        bool y_larger = false, decided = false;
        for (int k = 11; k >= 0 && !decided; k--)
            if (y.l[k] != ny.l[k]) {
                y_larger = y.l[k] > ny.l[k];
                decided = true;
            }
#pragma unroll
        for (int k = 0; k < 12; k++) {  // limb k little-endian -> bytes 44 - 4k .. 47 - 4k big-endian
            const uint32_t w = x.l[k];
            o[44 - 4 * k] = (uint8_t)(w >> 24);
            o[45 - 4 * k] = (uint8_t)(w >> 16);
            o[46 - 4 * k] = (uint8_t)(w >> 8);
            o[47 - 4 * k] = (uint8_t)w;
        }
        o[0] |= 0x80u | (y_larger ? 0x20u : 0u);
    }
}

// ---- g_to_lagrange (proofs/src/utils/arithmetic.rs:34-54): inverse FFT over
// G1 points.  Decimation-in-frequency radix-2 stages in global memory (the
// butterflies are compute-bound: one variable-base scalar multiplication
// each), then bit reversal, the 1/n scaling and normalisation in one pass.

__device__ __forceinline__ Xyzz xyzz_neg(const Xyzz& p) {
    Xyzz r = p;
    r.y = fp_sub(fp_zero(), p.y);
    return r;
}

// [k] P through the endomorphism (GLV): k = a0 + a1 u + a2 u^2 + a3 u^3 in
// base u = 0xd201000000010000 (k < r < u^4), k1 = a0 + a1 u, k2 = a2 + a3 u,
// both below 2^128, and u^2 = -lambda (mod r) where phi(P) = [lambda] P (the
// endomorphism of the subgroup check), so [k] P = [k1] P + [k2] (-phi(P)).
// One joint double-and-add over 128 bits instead of 255.
struct Glv {
    uint64_t k1[2], k2[2];
};
__device__ Xyzz xyzz_mul_glv(const Xyzz& p, const Glv& s) {
    Xyzz psi = p;  // -phi(P) = (beta X, -Y, ZZ, ZZZ)
    Fp beta;
#pragma unroll
    for (int k = 0; k < 12; k++) beta.l[k] = g1_beta_mont(k);
    psi.x = fp_mul(p.x, beta);
    psi.y = fp_sub(fp_zero(), p.y);
    const Xyzz both = xyzz_add(p, psi);
    Xyzz acc;
    xyzz_set_inf(acc);
    int top = 127;
    while (top >= 0 && !(((s.k1[top >> 6] | s.k2[top >> 6]) >> (top & 63)) & 1u)) top--;
#pragma unroll 1
    for (int bit = top; bit >= 0; bit--) {
        acc = xyzz_dbl(acc);
        const uint32_t b1 = (uint32_t)(s.k1[bit >> 6] >> (bit & 63)) & 1u;
        const uint32_t b2 = (uint32_t)(s.k2[bit >> 6] >> (bit & 63)) & 1u;
        if (b1 | b2) acc = xyzz_add(acc, (b1 & b2) ? both : (b1 ? p : psi));
    }
    return acc;
}

__global__ void __launch_bounds__(kThreads) k_aff_to_xyzz(const Affine* __restrict__ in, uint64_t n,
                                                          Xyzz* __restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = xyzz_from_affine(in[i]);
}
// one DIF stage of half-size h = 2^log_h: (a, b) -> (a + b, (a - b) w^(pos n / 2h))
// glv[e]: the decomposition of w^e (w = omega^-1) for e < n/2
__global__ void __launch_bounds__(kThreads) k_ec_dif_stage(Xyzz* __restrict__ a, uint32_t log_n, uint32_t log_h,
                                                           const Glv* __restrict__ glv) {
    const uint32_t half = 1u << (log_n - 1);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < half; q += stride) {
        const uint32_t pos = q & ((1u << log_h) - 1);
        const uint32_t i0 = ((q >> log_h) << (log_h + 1)) + pos, i1 = i0 + (1u << log_h);
        const Xyzz x0 = a[i0], x1 = a[i1];
        a[i0] = xyzz_add(x0, x1);
        Xyzz d = xyzz_add(x0, xyzz_neg(x1));
        if (pos) {
            const uint32_t e = pos << (log_n - 1 - log_h);  // w_n^(pos n / 2h)
            d = xyzz_mul_glv(d, glv[e]);
        }
        a[i1] = d;
    }
}
// out[bitrev(i)] = affine([n_inv] a[i])
__global__ void __launch_bounds__(kThreads) k_ec_finish(const Xyzz* __restrict__ a, uint32_t log_n, Glv n_inv,
                                                        Affine* __restrict__ out) {
    const uint32_t n = 1u << log_n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t o = log_n ? (__brev(i) >> (32 - log_n)) : 0u;
        out[o] = xyzz_to_affine(xyzz_mul_glv(a[i], n_inv));
    }
}

Fr to_dev_fr(const host::Fr4& h) {
    Fr r;
    std::memcpy(r.l, h.l, 32);
    return r;
}

}  // namespace

Status g1_suffix_sum_device(Context* ctx, const void* in, uint64_t n, void* out, cudaStream_t st) {
    if (n == 0) return OK;
    void* x;
    MZK_TRY(ctx->ensure("srs_xyzz", n * sizeof(Xyzz), &x));
    MZK_TRY(suffix_scan<Affine>(ctx, static_cast<const Affine*>(in), static_cast<Xyzz*>(x), n, st));
    k_to_affine<<<blocks_for(ctx, n), kThreads, 0, st>>>(static_cast<const Xyzz*>(x), n, static_cast<Affine*>(out));
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

Status g1_decompress_device(Context* ctx, const void* in, uint64_t n, int check_subgroup, void* out,
                            uint8_t* status, uint64_t* invalid, cudaStream_t st) {
    if (invalid) *invalid = 0;
    if (n == 0) return OK;
    void* cnt;
    MZK_TRY(ctx->ensure("srs_invalid", 16, &cnt));
    MZK_CUDA_CHECK(cudaMemsetAsync(cnt, 0, 8, st));
    k_g1_decompress<<<blocks_for(ctx, n), kThreads, 0, st>>>(static_cast<const uint8_t*>(in), n, check_subgroup,
                                                             sqrt_exponent(), static_cast<Affine*>(out),
                                                             status, static_cast<unsigned long long*>(cnt));
    MZK_LAUNCH_CHECK(ctx);
    if (invalid) {
        void* h;
        MZK_TRY(ctx->ensure_pinned(16, &h));
        MZK_CUDA_CHECK(cudaMemcpyAsync(h, cnt, 8, cudaMemcpyDeviceToHost, st));
        MZK_CUDA_CHECK(cudaStreamSynchronize(st));
        *invalid = *static_cast<const uint64_t*>(h);
    }
    return OK;
}

Status g1_compress_device(Context* ctx, const void* in, uint64_t n, void* out, cudaStream_t st) {
    if (n == 0) return OK;
    k_g1_compress<<<blocks_for(ctx, n), kThreads, 0, st>>>(static_cast<const Affine*>(in), n,
                                                           static_cast<uint8_t*>(out));
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

// ParamsKZG::write_custom(.., SerdeFormat::Processed) (params.rs:260-281), G1
// part: k as u32 little-endian, then g and g_lagrange compressed.
Status srs_write_processed(Context* ctx, const void* g, const void* lag, uint64_t n, uint8_t* out, size_t out_len,
                           cudaStream_t st) {
    if (n == 0 || (n & (n - 1)) || n > (1ull << 31)) {
        set_error("srs_write: n must be a power of two (2^k points)");
        return ERR_ARG;
    }
    if (out_len < 4 + 2 * n * 48) {
        set_error("srs_write: output shorter than 4 + 96 n bytes");
        return ERR_ARG;
    }
    const uint32_t k = (uint32_t)__builtin_ctzll(n);
    std::memcpy(out, &k, 4);
    void* comp;
    MZK_TRY(ctx->ensure("srs_comp", 2 * n * 48, &comp));
    MZK_TRY(g1_compress_device(ctx, g, n, comp, st));
    MZK_TRY(g1_compress_device(ctx, lag, n, static_cast<uint8_t*>(comp) + n * 48, st));
    MZK_CUDA_CHECK(cudaMemcpyAsync(out + 4, comp, 2 * n * 48, cudaMemcpyDeviceToHost, st));
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    return OK;
}

Status srs_read_processed(Context* ctx, const uint8_t* bytes, size_t len, uint64_t capacity, uint32_t* k_out,
                          void* g, void* lag, void* delta, void* ddelta, cudaStream_t st) {
    if (len < 4) {
        set_error("srs_read: buffer shorter than the k field");
        return ERR_ARG;
    }
    uint32_t k;
    std::memcpy(&k, bytes, 4);  // u32 little-endian (params.rs:265)
    if (k > 31 || (1ull << k) > capacity) {
        set_error("srs_read: k = " + std::to_string(k) + " exceeds the output capacity");
        return ERR_ARG;
    }
    const uint64_t n = 1ull << k;
    if (len < 4 + 2 * n * 48) {
        set_error("srs_read: buffer shorter than 2^k compressed g and g_lagrange points");
        return ERR_ARG;
    }
    *k_out = k;
    void* comp;
    MZK_TRY(ctx->ensure("srs_comp", 2 * n * 48, &comp));
    MZK_CUDA_CHECK(cudaMemcpyAsync(comp, bytes + 4, 2 * n * 48, cudaMemcpyHostToDevice, st));
    void* lag_out = lag;
    if (!lag_out) MZK_TRY(ctx->ensure("srs_lag", n * sizeof(Affine), &lag_out));
    uint64_t bad_g = 0, bad_l = 0;
    if (g) MZK_TRY(g1_decompress_device(ctx, comp, n, 1, g, nullptr, &bad_g, st));
    MZK_TRY(g1_decompress_device(ctx, static_cast<const uint8_t*>(comp) + n * 48, n, 1, lag_out, nullptr, &bad_l, st));
    if (bad_g || bad_l) {
        set_error("srs_read: invalid point encoding (" + std::to_string(bad_g + bad_l) + " points)");
        return ERR_ARG;
    }
    // the delta bases are derived after reading (params.rs:340-341)
    if (!delta && !ddelta) return OK;
    void* delta_out = delta;
    if (!delta_out) MZK_TRY(ctx->ensure("srs_delta", n * sizeof(Affine), &delta_out));
    MZK_TRY(g1_suffix_sum_device(ctx, lag_out, n, delta_out, st));
    if (ddelta) MZK_TRY(g1_suffix_sum_device(ctx, delta_out, n, ddelta, st));
    return OK;
}

namespace {
// the GLV decomposition of a Montgomery-form scalar (see xyzz_mul_glv)
Glv glv_split(const host::Fr4& mont) {
    host::Fr4 one_raw = {};
    one_raw.l[0] = 1;
    const host::Fr4 c = host::fr_mul(mont, one_raw);  // canonical
    uint64_t q[4] = {c.l[0], c.l[1], c.l[2], c.l[3]}, digit[4];
    constexpr uint64_t kU = 0xd201000000010000ull;
    for (int d = 0; d < 4; d++) {  // base-u digits, least significant first
        unsigned __int128 rem = 0;
        for (int i = 3; i >= 0; i--) {
            const unsigned __int128 cur = (rem << 64) | q[i];
            q[i] = (uint64_t)(cur / kU);
            rem = cur % kU;
        }
        digit[d] = (uint64_t)rem;
    }
    Glv g;
    const unsigned __int128 k1 = (unsigned __int128)digit[1] * kU + digit[0];
    const unsigned __int128 k2 = (unsigned __int128)digit[3] * kU + digit[2];
    g.k1[0] = (uint64_t)k1;
    g.k1[1] = (uint64_t)(k1 >> 64);
    g.k2[0] = (uint64_t)k2;
    g.k2[1] = (uint64_t)(k2 >> 64);
    return g;
}
}  // namespace

Status g1_to_lagrange_device(Context* ctx, const Domain* d, const void* g, void* out, cudaStream_t st) {
    const uint32_t k = d->k, n = 1u << k;
    void* x;
    MZK_TRY(ctx->ensure("srs_ecfft", (size_t)n * sizeof(Xyzz), &x));
    Xyzz* a = static_cast<Xyzz*>(x);
    // the decompositions of every twiddle w^e (w = omega^-1, e < n/2): the
    // last stage uses all of them, earlier stages every 2^s-th
    const uint32_t half = std::max(1u, n / 2);
    std::vector<Glv> glv(half);
    host::Fr4 w = host::fr_one();
    for (uint32_t e = 0; e < half; e++) {
        glv[e] = glv_split(w);
        w = host::fr_mul(w, d->omega_inv);
    }
    void* dg;
    MZK_TRY(ctx->ensure("srs_glv", (size_t)half * sizeof(Glv), &dg));
    MZK_CUDA_CHECK(cudaMemcpyAsync(dg, glv.data(), (size_t)half * sizeof(Glv), cudaMemcpyHostToDevice, st));
    k_aff_to_xyzz<<<blocks_for(ctx, n), kThreads, 0, st>>>(static_cast<const Affine*>(g), n, a);
    MZK_LAUNCH_CHECK(ctx);
    for (int log_h = (int)k - 1; log_h >= 0; log_h--) {
        k_ec_dif_stage<<<blocks_for(ctx, n / 2), kThreads, 0, st>>>(a, k, (uint32_t)log_h,
                                                                      static_cast<const Glv*>(dg));
        MZK_LAUNCH_CHECK(ctx);
    }
    // 1/n (the domain's ifft divisor, Montgomery form)
    k_ec_finish<<<blocks_for(ctx, n), kThreads, 0, st>>>(a, k, glv_split(d->ifft_div), static_cast<Affine*>(out));
    MZK_LAUNCH_CHECK(ctx);
    // the host table must outlive the copy
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    return OK;
}

Status srs_downsize_device(Context* ctx, const Domain* d, const void* g, void* lag, void* delta, void* ddelta,
                           cudaStream_t st) {
    const uint64_t n = 1ull << d->k;
    void* lag_out = lag;
    if (!lag_out) MZK_TRY(ctx->ensure("srs_lag", n * sizeof(Affine), &lag_out));
    MZK_TRY(g1_to_lagrange_device(ctx, d, g, lag_out, st));
    if (!delta && !ddelta) return OK;
    void* delta_out = delta;
    if (!delta_out) MZK_TRY(ctx->ensure("srs_delta", n * sizeof(Affine), &delta_out));
    MZK_TRY(g1_suffix_sum_device(ctx, lag_out, n, delta_out, st));
    if (ddelta) MZK_TRY(g1_suffix_sum_device(ctx, delta_out, n, ddelta, st));
    return OK;
}

Status srs_setup_device(Context* ctx, const Domain* d, const uint64_t s[4], void* g, void* lag, void* delta,
                        void* ddelta, cudaStream_t st) {
    const uint32_t n = 1u << d->k;
    void* scal;
    MZK_TRY(ctx->ensure("srs_scal", (size_t)n * sizeof(Fr), &scal));
    if (g) {  // g[i] = [s^i] G
        MZK_TRY(fr_powers_device(ctx, s, n, scal, st));
        MZK_TRY(fixed_base_g1(ctx, scal, n, g, st));
    }
    if (!lag && !delta && !ddelta) return OK;
    host::Fr4 sh;
    std::memcpy(sh.l, s, 32);
    const uint64_t en[1] = {n};
    // (s^n - 1) * n^-1
    const host::Fr4 mult = host::fr_mul(host::fr_sub(host::fr_pow(sh, en, 1), host::fr_one()), d->ifft_div);
    const uint32_t grid = blocks_for(ctx, n);
    k_lag_den<<<grid, kThreads, 0, st>>>(d->lo[0], d->hi[0], to_dev_fr(sh), n, static_cast<Fr*>(scal));
    MZK_LAUNCH_CHECK(ctx);
    MZK_TRY(batch_invert_device(ctx, scal, n, st));
    k_lag_scal<<<grid, kThreads, 0, st>>>(d->lo[0], d->hi[0], to_dev_fr(mult), n, static_cast<Fr*>(scal));
    MZK_LAUNCH_CHECK(ctx);
    void* lag_out = lag;
    if (!lag_out) MZK_TRY(ctx->ensure("srs_lag", (size_t)n * sizeof(Affine), &lag_out));
    MZK_TRY(fixed_base_g1(ctx, scal, n, lag_out, st));
    if (!delta && !ddelta) return OK;
    void* delta_out = delta;
    if (!delta_out) MZK_TRY(ctx->ensure("srs_delta", (size_t)n * sizeof(Affine), &delta_out));
    MZK_TRY(g1_suffix_sum_device(ctx, lag_out, n, delta_out, st));
    if (ddelta) MZK_TRY(g1_suffix_sum_device(ctx, delta_out, n, ddelta, st));
    return OK;
}

}  // namespace mzk
