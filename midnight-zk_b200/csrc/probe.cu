// probe.cu — microbenchmarks for the roofline denominators of the integer
// kernels: the integer multiply-add issue rate of the GPU, and the rate the
// 12-limb Montgomery multiplication of field.cuh reaches on it.
#include <cuda_runtime.h>

#include <algorithm>

#include "ec.cuh"
#include "field.cuh"
#include "runtime.hpp"

namespace mzk {

namespace {

constexpr int kProbeIters = 4096;

// 16 independent 32-bit multiply-adds per iteration (8 low halves, 8 high
// halves), enough independent chains per warp to saturate the pipe.
__global__ void k_probe_imad(uint32_t seed, uint32_t* sink) {
    uint32_t a[8], b[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        a[k] = seed + threadIdx.x * 7u + (uint32_t)k;
        b[k] = seed ^ (threadIdx.x + 13u * (uint32_t)k);
    }
    const uint32_t x = seed | 1u, y = 0x9e3779b9u;
    for (int it = 0; it < kProbeIters; it++) {
#pragma unroll
        for (int k = 0; k < 8; k++) {
            asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(x), "r"(y));
            asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(b[k]) : "r"(x), "r"(y));
        }
    }
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) acc ^= a[k] ^ b[k];
    if (acc == 0x12345678u) sink[0] = acc;
}

// The forms the field code issues: carry-chained low/high multiply-adds.
// Eight independent two-limb chains per iteration (each chain restarts with
// mad.lo.cc, so chains only share the carry flag by renaming).
__global__ void k_probe_imad_cc(uint32_t seed, uint32_t* sink) {
    uint32_t a[8], b[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        a[k] = seed + threadIdx.x * 7u + (uint32_t)k;
        b[k] = seed ^ (threadIdx.x + 13u * (uint32_t)k);
    }
    const uint32_t x = seed | 1u;
    for (int it = 0; it < kProbeIters; it++) {
#pragma unroll
        for (int k = 0; k < 8; k++)
            asm volatile("mad.lo.cc.u32 %0, %0, %2, %1;\n\tmadc.hi.u32 %1, %1, %2, %0;" : "+r"(a[k]), "+r"(b[k]) : "r"(x));
    }
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) acc ^= a[k] ^ b[k];
    if (acc == 0x12345678u) sink[0] = acc;
}

// 16 independent mad.lo.u32 per iteration (low halves only)
__global__ void k_probe_imad_lo(uint32_t seed, uint32_t* sink) {
    uint32_t a[16];
#pragma unroll
    for (int k = 0; k < 16; k++) a[k] = seed + threadIdx.x * 7u + (uint32_t)k;
    const uint32_t x = seed | 1u, y = 0x9e3779b9u;
    for (int it = 0; it < kProbeIters; it++) {
#pragma unroll
        for (int k = 0; k < 16; k++) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(x), "r"(y));
    }
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) acc ^= a[k];
    if (acc == 0x12345678u) sink[0] = acc;
}

constexpr int kProbeMulIters = 256;

// Every operand depends on the thread index: a product whose operands are all
// warp-uniform is computed once per warp on the uniform datapath, next to the
// per-thread pipes, and would inflate the rate (measured: 53 vs 30.6 G/s).
__global__ void __launch_bounds__(128) k_probe_fp_mul(uint32_t seed, uint32_t* sink) {
    Fp a, b, c;
#pragma unroll
    for (int j = 0; j < 12; j++) {
        a.l[j] = (seed * (j + 1) + threadIdx.x) & 0x0fffffffu;
        b.l[j] = (seed ^ (j * 977u + threadIdx.x * 3u)) & 0x0fffffffu;
        c.l[j] = (seed + j * 31u + threadIdx.x * 5u) & 0x0fffffffu;
    }
    for (int it = 0; it < kProbeMulIters; it++) {
        a = fp_mul(a, b);
        c = fp_mul(c, b);
    }
    uint32_t acc = 0;
#pragma unroll
    for (int j = 0; j < 12; j++) acc ^= a.l[j] ^ c.l[j];
    if (acc == 0x12345678u) sink[0] = acc;
}

// The bucket-accumulation inner step alone: mixed XYZZ additions of a point
// held in registers, no memory traffic; isolates the cost of the addition code.
constexpr int kProbeMaddIters = 64;

__global__ void __launch_bounds__(128, 1) k_probe_madd(uint32_t seed, uint32_t* sink) {
    Affine p;
    Xyzz acc;
#pragma unroll
    for (int j = 0; j < 12; j++) {
        p.x.l[j] = (seed * (j + 3) + threadIdx.x) & 0x0fffffffu;
        p.y.l[j] = (seed ^ (j * 131u + threadIdx.x)) & 0x0fffffffu;
        acc.x.l[j] = (seed + j * 17u) & 0x0fffffffu;
        acc.y.l[j] = (seed * 7u + j) & 0x0fffffffu;
        acc.zz.l[j] = (seed ^ (j * 5u)) & 0x0fffffffu;
        acc.zzz.l[j] = (seed + 99u * j) & 0x0fffffffu;
    }
    for (int it = 0; it < kProbeMaddIters; it++) xyzz_add_affine_fast(acc, p);
    uint32_t r = 0;
#pragma unroll
    for (int j = 0; j < 12; j++) r ^= acc.x.l[j] ^ acc.y.l[j] ^ acc.zz.l[j] ^ acc.zzz.l[j];
    if (r == 0x12345678u) sink[0] = r;
}

// Batch-affine addition (the accumulation scheme of the reference's
// batch_add / Schedule, curves/src/msm.rs:58-144): each thread holds B affine
// accumulators P_i and adds to each a point Q from shared memory, all B
// additions sharing one field inversion by Montgomery's trick:
//   forward  c_i = prod_{j<i} (x_Q - x_Pj)                     1 mul
//   one inversion of the full product
//   backward 1/(x_Q - x_Pi) = inv c_i, inv *= (x_Q - x_Pi)     2 mul
//   lambda = (y_Q - y_Pi) / (x_Q - x_Pi), x3 = lambda^2 - x_P - x_Q,
//   y3 = lambda (x_P - x3) - y_P                               2 mul + 1 sqr
// = 6 products per addition plus the inversion's share, against the 10 of
// the mixed XYZZ addition.  The accumulators and prefix products live in the
// thread's local memory (3 x 48 bytes per addition in flight), as a real
// batch-affine accumulation must hold them somewhere.  No gathers, no bucket
// bookkeeping: an upper bound on what the scheme can reach here.  Operands
// are arbitrary field elements (the formulas do not check the curve); a zero
// denominator (probability ~B / p) would only zero one accumulator.
constexpr int kProbeAffineRounds = 4;

template <int B, bool kBinaryInverse>
__global__ void __launch_bounds__(128) k_probe_batch_affine(uint32_t seed, uint32_t* sink) {
    __shared__ Fp qx[64], qy[64];
    for (int i = threadIdx.x; i < 64; i += blockDim.x) {
#pragma unroll
        for (int j = 0; j < 12; j++) {
            qx[i].l[j] = (seed * (j + 5) + i * 977u) & 0x0fffffffu;
            qy[i].l[j] = (seed ^ (j * 313u + i * 31u)) & 0x0fffffffu;
        }
    }
    __syncthreads();
    Fp px[B], py[B], c[B];
    for (int i = 0; i < B; i++) {
#pragma unroll
        for (int j = 0; j < 12; j++) {
            px[i].l[j] = (seed * (j + 3) + threadIdx.x * 7u + i * 131u) & 0x0fffffffu;
            py[i].l[j] = (seed ^ (j * 131u + threadIdx.x + i * 17u)) & 0x0fffffffu;
        }
    }
    for (int r = 0; r < kProbeAffineRounds; r++) {
        Fp acc = fp_one();
        for (int i = 0; i < B; i++) {
            const int q = (i + threadIdx.x + r) & 63;
            c[i] = acc;
            acc = fp_mul(acc, fp_sub(qx[q], px[i]));
        }
        Fp inv;
        if (kBinaryInverse) {
            Fp x, r2;
            const Fp a = fp_canonical(acc);
            if (!inv_binary_raw<12>(x.l, a.l, FpMod())) x = fp_zero();
#pragma unroll
            for (int j = 0; j < 12; j++) r2.l[j] = FpP::r2(j);
            inv = fp_mul(x, fp_mul(r2, r2));  // (a R)^-1 R^3 R^-1 = a^-1 R
        } else {
            inv = fp_inv(acc);
        }
        for (int i = B - 1; i >= 0; i--) {
            const int q = (i + threadIdx.x + r) & 63;
            const Fp d = fp_sub(qx[q], px[i]);
            const Fp di = fp_mul(inv, c[i]);
            inv = fp_mul(inv, d);
            const Fp lam = fp_mul(fp_sub(qy[q], py[i]), di);
            const Fp x3 = fp_sub(fp_sub(fp_sqr(lam), px[i]), qx[q]);
            py[i] = fp_sub(fp_mul(lam, fp_sub(px[i], x3)), py[i]);
            px[i] = x3;
        }
    }
    uint32_t acc = 0;
    for (int i = 0; i < B; i++)
#pragma unroll
        for (int j = 0; j < 12; j++) acc ^= px[i].l[j] ^ py[i].l[j];
    if (acc == 0x12345678u) sink[0] = acc;
}

// Self-check of the binary inversion: a^-1 a = 1 for every input (the
// Montgomery one), and the inverse equals the Fermat power's.
__global__ void k_check_fp_inv(const Fp* __restrict__ in, size_t n, unsigned long long* __restrict__ mismatches) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const Fp a = fp_canonical(in[i]);
        if (fp_is_zero_raw(a)) continue;
        Fp x, r2;
        if (!inv_binary_raw<12>(x.l, a.l, FpMod())) {
            atomicAdd(mismatches, 1ull);
            continue;
        }
#pragma unroll
        for (int j = 0; j < 12; j++) r2.l[j] = FpP::r2(j);
        const Fp inv = fp_canonical(fp_mul(x, fp_mul(r2, r2)));
        const Fp ferm = fp_canonical(fp_inv(a));
        const Fp one = fp_canonical(fp_mul(inv, a));
        uint32_t diff = 0;
#pragma unroll
        for (int j = 0; j < 12; j++) diff |= (inv.l[j] ^ ferm.l[j]) | (one.l[j] ^ FpP::one(j));
        if (diff) atomicAdd(mismatches, 1ull);
    }
}

// Self-check of the dedicated squaring: fp_sqr(a) and fp_mul(a, a) must agree
// limb for limb (both are (a^2 + M p) / R with the same unique M).
__global__ void k_check_fp_sqr(const Fp* __restrict__ in, size_t n, unsigned long long* __restrict__ mismatches) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const Fp a = in[i];
        const Fp s = fp_sqr(a), m = fp_mul(a, a);
        uint32_t diff = 0;
#pragma unroll
        for (int j = 0; j < 12; j++) diff |= s.l[j] ^ m.l[j];
        if (diff) atomicAdd(mismatches, 1ull);
    }
}

}  // namespace

Status check_fp_sqr(Context* ctx, const void* d_values, size_t n, uint64_t* mismatches) {
    void* cnt;
    MZK_TRY(ctx->ensure("probe_count", 64, &cnt));
    MZK_CUDA_CHECK(cudaMemsetAsync(cnt, 0, 8, ctx->stream));
    if (n) {
        const uint32_t blocks = (uint32_t)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 8);
        k_check_fp_sqr<<<blocks, 256, 0, ctx->stream>>>(static_cast<const Fp*>(d_values), n,
                                                        static_cast<unsigned long long*>(cnt));
        MZK_LAUNCH_CHECK(ctx);
    }
    MZK_CUDA_CHECK(cudaMemcpyAsync(mismatches, cnt, 8, cudaMemcpyDeviceToHost, ctx->stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    return OK;
}

Status check_fp_inv(Context* ctx, const void* d_values, size_t n, uint64_t* mismatches) {
    void* cnt;
    MZK_TRY(ctx->ensure("probe_count", 64, &cnt));
    MZK_CUDA_CHECK(cudaMemsetAsync(cnt, 0, 8, ctx->stream));
    if (n) {
        const uint32_t blocks = (uint32_t)std::min<size_t>((n + 127) / 128, (size_t)ctx->num_sms * 8);
        k_check_fp_inv<<<blocks, 128, 0, ctx->stream>>>(static_cast<const Fp*>(d_values), n,
                                                        static_cast<unsigned long long*>(cnt));
        MZK_LAUNCH_CHECK(ctx);
    }
    MZK_CUDA_CHECK(cudaMemcpyAsync(mismatches, cnt, 8, cudaMemcpyDeviceToHost, ctx->stream));
    MZK_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));
    return OK;
}

template <int B, bool kBin>
Status time_batch_affine(Context* ctx, void* sink, uint32_t blocks, double* adds_per_s) {
    cudaEvent_t e0, e1;
    MZK_CUDA_CHECK(cudaEventCreate(&e0));
    MZK_CUDA_CHECK(cudaEventCreate(&e1));
    cudaStream_t st = ctx->stream;
    float best = 1e30f;
    for (int rep = 0; rep < 3; rep++) {
        MZK_CUDA_CHECK(cudaEventRecord(e0, st));
        k_probe_batch_affine<B, kBin><<<blocks, 128, 0, st>>>(0x4242u + rep, (uint32_t*)sink);
        MZK_LAUNCH_CHECK(ctx);
        MZK_CUDA_CHECK(cudaEventRecord(e1, st));
        MZK_CUDA_CHECK(cudaEventSynchronize(e1));
        float ms;
        MZK_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *adds_per_s = (double)blocks * 128 * B * kProbeAffineRounds / (best * 1e-3);
    return OK;
}

// batch-affine additions per second for batches of 16, 32, 64 and 128 per
// thread, with the Fermat inversion (out[0..3]) and the binary one (out[4..7])
Status probe_batch_affine(Context* ctx, double* out) {
    void* sink;
    MZK_TRY(ctx->ensure("probe_sink", 64, &sink));
    const uint32_t blocks = (uint32_t)ctx->num_sms * 4;
    MZK_TRY((time_batch_affine<16, false>(ctx, sink, blocks, out + 0)));
    MZK_TRY((time_batch_affine<32, false>(ctx, sink, blocks, out + 1)));
    MZK_TRY((time_batch_affine<64, false>(ctx, sink, blocks, out + 2)));
    MZK_TRY((time_batch_affine<128, false>(ctx, sink, blocks, out + 3)));
    MZK_TRY((time_batch_affine<16, true>(ctx, sink, blocks, out + 4)));
    MZK_TRY((time_batch_affine<32, true>(ctx, sink, blocks, out + 5)));
    MZK_TRY((time_batch_affine<64, true>(ctx, sink, blocks, out + 6)));
    MZK_TRY((time_batch_affine<128, true>(ctx, sink, blocks, out + 7)));
    return OK;
}

Status probe_imad(Context* ctx, double* imad_per_s, double* fp_mul_per_s, double* variants) {
    void* sink;
    MZK_TRY(ctx->ensure("probe_sink", 64, &sink));
    cudaEvent_t e0, e1;
    MZK_CUDA_CHECK(cudaEventCreate(&e0));
    MZK_CUDA_CHECK(cudaEventCreate(&e1));
    cudaStream_t st = ctx->stream;
    const uint32_t blocks = (uint32_t)ctx->num_sms * 8, threads = 256;
    double rates[3];
    for (int v = 0; v < 3; v++) {
        float best = 1e30f;
        for (int rep = 0; rep < 3; rep++) {
            MZK_CUDA_CHECK(cudaEventRecord(e0, st));
            if (v == 0) k_probe_imad<<<blocks, threads, 0, st>>>(0x1234u + rep, (uint32_t*)sink);
            else if (v == 1) k_probe_imad_cc<<<blocks, threads, 0, st>>>(0x1234u + rep, (uint32_t*)sink);
            else k_probe_imad_lo<<<blocks, threads, 0, st>>>(0x1234u + rep, (uint32_t*)sink);
            MZK_LAUNCH_CHECK(ctx);
            MZK_CUDA_CHECK(cudaEventRecord(e1, st));
            MZK_CUDA_CHECK(cudaEventSynchronize(e1));
            float ms;
            MZK_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0 && ms < best) best = ms;
        }
        rates[v] = (double)blocks * threads * kProbeIters * 16.0 / (best * 1e-3);
        if (variants) variants[v] = rates[v];
    }
    // the carry-chained form is what the field arithmetic issues
    *imad_per_s = rates[1];
    float best;
    int per_sm = 0;
    MZK_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_probe_fp_mul, 128, 0));
    const uint32_t mblocks = (uint32_t)ctx->num_sms * (uint32_t)(per_sm > 0 ? per_sm : 1) * 4;
    best = 1e30f;
    for (int rep = 0; rep < 3; rep++) {
        MZK_CUDA_CHECK(cudaEventRecord(e0, st));
        k_probe_fp_mul<<<mblocks, 128, 0, st>>>(0x777u + rep, (uint32_t*)sink);
        MZK_LAUNCH_CHECK(ctx);
        MZK_CUDA_CHECK(cudaEventRecord(e1, st));
        MZK_CUDA_CHECK(cudaEventSynchronize(e1));
        float ms;
        MZK_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0 && ms < best) best = ms;
    }
    *fp_mul_per_s = (double)mblocks * 128 * kProbeMulIters * 2.0 / (best * 1e-3);
    if (variants) {
        // variants[3]: mixed additions per second of the accumulation step in registers
        const uint32_t ablocks = (uint32_t)ctx->num_sms * 2 * 8;
        best = 1e30f;
        for (int rep = 0; rep < 3; rep++) {
            MZK_CUDA_CHECK(cudaEventRecord(e0, st));
            k_probe_madd<<<ablocks, 128, 0, st>>>(0x999u + rep, (uint32_t*)sink);
            MZK_LAUNCH_CHECK(ctx);
            MZK_CUDA_CHECK(cudaEventRecord(e1, st));
            MZK_CUDA_CHECK(cudaEventSynchronize(e1));
            float ms;
            MZK_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0 && ms < best) best = ms;
        }
        variants[3] = (double)ablocks * 128 * kProbeMaddIters / (best * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return OK;
}

}  // namespace mzk
