// gen.cu — seeded synthetic inputs generated on the device.
//
// Benchmarks and tests need 2^24 uniform scalars and bases [r_i]G; building
// them on the host would take minutes.  Element i depends only on (seed, i),
// so any slice can be regenerated anywhere (the C oracle implements the same
// generator for the parity checks):
//   word ctr of stream `seed` = SplitMix64 finaliser of seed + (ctr+1)*golden
//   uniform Fr: rejection sampling as Fq::random (curves/src/bls12_381/
//               fq.rs:382-396), attempt a of element i uses words (i*64+a)*4..+3
//   bases: [r_i]G by an 8-bit fixed-base table of the generator G
//          (curves/README.md:96-101), normalised to affine per point;
//   the fixed columns and witnesses of the single-proof configuration's
//          circuit (standard gate, copy cycles, range lookup).
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "ec.cuh"
#include "host_ec.hpp"
#include "runtime.hpp"

namespace mzk {

namespace {

__device__ __forceinline__ uint64_t rand64(uint64_t seed, uint64_t ctr) {
    uint64_t z = seed + (ctr + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// canonical uniform element of [0, r)
__device__ Fr rand_fr_canonical(uint64_t seed, uint64_t i) {
    Fr out = fr_zero();
    for (uint64_t a = 0; a < 64; a++) {
        uint32_t w[8];
        for (int k = 0; k < 4; k++) {
            uint64_t v = rand64(seed, (i * 64 + a) * 4 + (uint64_t)k);
            if (k == 3) v &= 0x7fffffffffffffffull;
            w[2 * k] = (uint32_t)v;
            w[2 * k + 1] = (uint32_t)(v >> 32);
        }
        // accept if w < r
        bool less = false, decided = false;
        for (int k = 7; k >= 0 && !decided; k--) {
            if (w[k] != FrP::mod(k)) {
                less = w[k] < FrP::mod(k);
                decided = true;
            }
        }
        if (decided && less) {
            for (int k = 0; k < 8; k++) out.l[k] = w[k];
            return out;
        }
    }
    return out;
}

__global__ void k_rand_fr(uint64_t seed, uint64_t first, size_t n, Fr* __restrict__ out) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = fr_to_mont(rand_fr_canonical(seed, first + i));
}

__global__ void __launch_bounds__(128) k_gen_bases(uint64_t seed, uint64_t first, size_t n,
                                                   const Affine* __restrict__ table, Affine* __restrict__ out) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Fr r = rand_fr_canonical(seed, first + i);
        Xyzz acc;
        xyzz_set_inf(acc);
        for (int j = 0; j < 32; j++) {
            const uint32_t v = (r.l[j >> 2] >> (8 * (j & 3))) & 0xffu;
            if (v) xyzz_add_affine(acc, load_affine(table, (uint32_t)(j * 256) + v));
        }
        out[i] = xyzz_to_affine(acc);
    }
}

// [s_i]G for scalars s_i (Montgomery) by the same fixed-base table
__global__ void __launch_bounds__(128) k_fixed_base(const Fr* __restrict__ scalars, size_t n,
                                                    const Affine* __restrict__ table, Affine* __restrict__ out) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const Fr r = fr_from_mont(scalars[i]);
        Xyzz acc;
        xyzz_set_inf(acc);
        for (int j = 0; j < 32; j++) {
            const uint32_t v = (r.l[j >> 2] >> (8 * (j & 3))) & 0xffu;
            if (v) xyzz_add_affine(acc, load_affine(table, (uint32_t)(j * 256) + v));
        }
        out[i] = xyzz_to_affine(acc);
    }
}

// G1 generator, canonical coordinates (curves/README.md:96-101)
const uint64_t kGenX[6] = {0xfb3af00adb22c6bbULL, 0x6c55e83ff97a1aefULL, 0xa14e3a3f171bac58ULL,
                           0xc3688c4f9774b905ULL, 0x2695638c4fa9ac0fULL, 0x17f1d3a73197d794ULL};
const uint64_t kGenY[6] = {0x0caa232946c5e7e1ULL, 0xd03cc744a2888ae4ULL, 0x00db18cb2c04b3edULL,
                           0xfcf5e095d5d00af6ULL, 0xa09e30ed741d8ae4ULL, 0x08b3f481e3aaa0f1ULL};
const uint64_t kFpR2[6] = {0xf4df1f341c341746ULL, 0x0a76e6a609d104f1ULL, 0x8de5476c4c95b6d5ULL,
                           0x67eb88a9939d83c0ULL, 0x9a793e85b519952dULL, 0x11988fe592cae3aaULL};

Status ensure_gen_table(Context* ctx) {
    if (ctx->gen_table) return OK;
    host::Fp6 r2, gx, gy;
    std::memcpy(r2.l, kFpR2, 48);
    std::memcpy(gx.l, kGenX, 48);
    std::memcpy(gy.l, kGenY, 48);
    host::Xyzz6 base{host::mul(gx, r2), host::mul(gy, r2), host::one(), host::one()};
    std::vector<uint64_t> table((size_t)32 * 256 * 12, 0);
    for (int j = 0; j < 32; j++) {
        host::Xyzz6 acc = host::infinity();
        for (int v = 1; v < 256; v++) {
            acc = host::add(acc, base);
            uint64_t jac[18];
            host::to_jacobian_normalised(acc, jac);
            std::memcpy(&table[((size_t)j * 256 + v) * 12], jac, 96);
        }
        for (int b = 0; b < 8; b++) base = host::dbl(base);
    }
    void* d;
    MZK_CUDA_CHECK(cudaMalloc(&d, table.size() * 8));
    MZK_CUDA_CHECK(cudaMemcpy(d, table.data(), table.size() * 8, cudaMemcpyHostToDevice));
    ctx->gen_table = d;
    return OK;
}

// small integer v < 2^32 in Montgomery form
__device__ __forceinline__ Fr fr_small(uint32_t v) {
    Fr r = fr_zero();
    r.l[0] = v;
    return fr_to_mont(r);
}

// fixed columns of the single-proof configuration's circuit (one buffer of
// 7 x n): q_l, q_r, q_m, q_o, q_c uniform on the usable rows (q_o never zero)
// and zero after, the table 0 .. table_rows - 1 then zeros, the lookup
// selector one on the usable rows
__global__ void k_cfg3_fixed(uint64_t seed, uint32_t n, uint32_t u, uint32_t table_rows, Fr* __restrict__ f) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        for (uint32_t j = 0; j < 5; j++) {
            Fr v = fr_zero();
            if (i < u) {
                v = fr_to_mont(rand_fr_canonical(seed + j, i));
                if (j == 3) {
                    uint32_t acc = 0;
                    for (int w = 0; w < 8; w++) acc |= v.l[w];
                    if (acc == 0) v = fr_one();
                }
            }
            f[(size_t)j * n + i] = v;
        }
        f[(size_t)5 * n + i] = i < table_rows ? fr_small(i) : fr_zero();
        f[(size_t)6 * n + i] = i < u ? fr_one() : fr_zero();
    }
}

// a witness of that circuit: a a table value, b uniform, every cell of one
// copy cycle the cycle's table value, c = -(q_l a + q_r b + q_m a b + q_c) / q_o
__global__ void k_cfg3_witness(uint64_t seed, uint32_t n, uint32_t u, uint32_t table_rows, const Fr* __restrict__ f,
                               const Fr* __restrict__ inv_qo, const uint32_t* __restrict__ cycle_of,
                               Fr* __restrict__ adv) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t kNone = 0xffffffffu;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Fr a = fr_zero(), b = fr_zero(), c = fr_zero();
        if (i < u) {
            const uint32_t ca = cycle_of[i], cb = cycle_of[(size_t)n + i];
            const uint64_t ra = ca != kNone ? rand64(seed, (1ull << 40) + ca) : rand64(seed, i);
            a = fr_small((uint32_t)(ra % table_rows));
            b = cb != kNone ? fr_small((uint32_t)(rand64(seed, (1ull << 40) + cb) % table_rows))
                            : fr_to_mont(rand_fr_canonical(seed ^ 0xB0B0B0B0ull, i));
            Fr t = fr_mul(f[i], a);
            t = fr_add(t, fr_mul(f[(size_t)n + i], b));
            t = fr_add(t, fr_mul(fr_mul(f[(size_t)2 * n + i], a), b));
            t = fr_add(t, f[(size_t)4 * n + i]);
            c = fr_sub(fr_zero(), fr_mul(t, inv_qo[i]));
        }
        adv[i] = a;
        adv[(size_t)n + i] = b;
        adv[(size_t)2 * n + i] = c;
    }
}

}  // namespace

Status gen_config3_fixed(Context* ctx, uint32_t k, uint32_t bf, uint32_t table_rows, uint64_t seed, void* d_fixed,
                         cudaStream_t st) {
    const uint32_t n = 1u << k, u = n - bf - 1;
    const uint32_t blocks = (uint32_t)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 32);
    k_cfg3_fixed<<<blocks, 256, 0, st>>>(seed, n, u, std::min(table_rows, u), static_cast<Fr*>(d_fixed));
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

Status gen_config3_witness(Context* ctx, uint32_t k, uint32_t bf, uint32_t table_rows, uint64_t seed,
                           const void* d_fixed, const void* d_inv_qo, const uint32_t* d_cycle_of, void* d_advice,
                           cudaStream_t st) {
    const uint32_t n = 1u << k, u = n - bf - 1;
    const uint32_t blocks = (uint32_t)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 32);
    k_cfg3_witness<<<blocks, 256, 0, st>>>(seed, n, u, std::min(table_rows, u), static_cast<const Fr*>(d_fixed),
                                           static_cast<const Fr*>(d_inv_qo), d_cycle_of, static_cast<Fr*>(d_advice));
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

Status gen_rand_fr(Context* ctx, uint64_t seed, uint64_t first, size_t n, void* d_out, cudaStream_t st) {
    if (n == 0) return OK;
    const uint32_t blocks = (uint32_t)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 32);
    k_rand_fr<<<blocks, 256, 0, st>>>(seed, first, n, static_cast<Fr*>(d_out));
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

Status fixed_base_g1(Context* ctx, const void* d_scalars, size_t n, void* d_out, cudaStream_t st) {
    if (n == 0) return OK;
    MZK_TRY(ensure_gen_table(ctx));
    const uint32_t blocks = (uint32_t)std::min<size_t>((n + 127) / 128, (size_t)ctx->num_sms * 16);
    k_fixed_base<<<blocks, 128, 0, st>>>(static_cast<const Fr*>(d_scalars), n,
                                         static_cast<const Affine*>(ctx->gen_table), static_cast<Affine*>(d_out));
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

Status gen_bases_g1(Context* ctx, uint64_t seed, uint64_t first, size_t n, void* d_out, cudaStream_t st) {
    if (n == 0) return OK;
    MZK_TRY(ensure_gen_table(ctx));
    const uint32_t blocks = (uint32_t)std::min<size_t>((n + 127) / 128, (size_t)ctx->num_sms * 16);
    k_gen_bases<<<blocks, 128, 0, st>>>(seed, first, n, static_cast<const Affine*>(ctx->gen_table),
                                        static_cast<Affine*>(d_out));
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

}  // namespace mzk
