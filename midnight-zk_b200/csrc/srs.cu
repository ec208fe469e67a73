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
