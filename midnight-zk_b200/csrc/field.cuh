// field.cuh — BLS12-381 Fp (base field) and Fr (scalar field) on sm_100a.
//
// Elements are little-endian 32-bit limbs in Montgomery form with the same R
// as the reference (Fp: R = 2^384, 12 limbs; Fr: R = 2^256, 8 limbs), so the
// device bytes are exactly the bytes of the reference's `blst_fp` / `blst_fr`
// (curves/src/bls12_381/fp.rs:96-98, fq.rs:25-29) and no conversion happens
// at the C ABI.
//
// Multiplication is word-serial Montgomery (CIOS) written for the integer
// multiply-add pipe: every 32x32 partial product is one `mad.lo`/`mad.hi`
// inside a PTX carry chain.  The products of one row a*b_i are split by the
// parity of the limb index of `a`: even-index products land on the word pairs
// (0,1),(2,3),... and odd-index products on (1,2),(3,4),... so each parity is
// one unbroken carry chain.  Two accumulators hold the running value
// T = X + 2^32 * Y (X aligned at word 0, Y at word 1); after the reduction
// zeroes X's low word, dividing by 2^32 is a relabelling: the next X is
// Y + X[1] and the next Y is X shifted down two words, and that shift is folded
// into the next row's odd chain.  This column-parity technique is the one
// published for modular multiplication on NVIDIA GPUs by Emmart and Weems.
//
// Fp values are kept lazily reduced in [0, 2p): with 4p < 2^384 the
// Montgomery product of two such values is again < 2p, so the multiply has no
// final subtraction and add/sub fold into [0, 2p) with one conditional 2p.
// `fp_canonical` brings a value to [0, p) for output and comparisons.
// Fr values are always fully reduced in [0, r) (4r > 2^256 rules out laziness).
#pragma once
#include <cstdint>

namespace mzk {

// ---------------------------------------------------------------- params ----
// Moduli: p from curves/src/bls12_381/fp.rs:20-27, r from fq.rs:43-48.
// N0 = -m^{-1} mod 2^32, ONE = 2^(32N) mod m, R2 = 2^(64N) mod m.
struct FpP {
    static constexpr int N = 12;
    static constexpr uint32_t N0 = 0xfffcfffdu;
    __host__ __device__ static constexpr uint32_t mod(int i) {
        return i == 0 ? 0xffffaaabu : i == 1 ? 0xb9feffffu : i == 2 ? 0xb153ffffu : i == 3 ? 0x1eabfffeu
             : i == 4 ? 0xf6b0f624u : i == 5 ? 0x6730d2a0u : i == 6 ? 0xf38512bfu : i == 7 ? 0x64774b84u
             : i == 8 ? 0x434bacd7u : i == 9 ? 0x4b1ba7b6u : i == 10 ? 0x397fe69au : 0x1a0111eau;
    }
    __host__ __device__ static constexpr uint32_t mod2(int i) {
        return i == 0 ? 0xffff5556u : i == 1 ? 0x73fdffffu : i == 2 ? 0x62a7ffffu : i == 3 ? 0x3d57fffdu
             : i == 4 ? 0xed61ec48u : i == 5 ? 0xce61a541u : i == 6 ? 0xe70a257eu : i == 7 ? 0xc8ee9709u
             : i == 8 ? 0x869759aeu : i == 9 ? 0x96374f6cu : i == 10 ? 0x72ffcd34u : 0x340223d4u;
    }
    __host__ __device__ static constexpr uint32_t one(int i) {
        return i == 0 ? 0x0002fffdu : i == 1 ? 0x76090000u : i == 2 ? 0xc40c0002u : i == 3 ? 0xebf4000bu
             : i == 4 ? 0x53c758bau : i == 5 ? 0x5f489857u : i == 6 ? 0x70525745u : i == 7 ? 0x77ce5853u
             : i == 8 ? 0xa256ec6du : i == 9 ? 0x5c071a97u : i == 10 ? 0xfa80e493u : 0x15f65ec3u;
    }
    // R^2 mod p (R = 2^384): canonical -> Montgomery by one multiplication
    __host__ __device__ static constexpr uint32_t r2(int i) {
        return i == 0 ? 0x1c341746u : i == 1 ? 0xf4df1f34u : i == 2 ? 0x09d104f1u : i == 3 ? 0x0a76e6a6u
             : i == 4 ? 0x4c95b6d5u : i == 5 ? 0x8de5476cu : i == 6 ? 0x939d83c0u : i == 7 ? 0x67eb88a9u
             : i == 8 ? 0xb519952du : i == 9 ? 0x9a793e85u : i == 10 ? 0x92cae3aau : 0x11988fe5u;
    }
};

struct FrP {
    static constexpr int N = 8;
    static constexpr uint32_t N0 = 0xffffffffu;
    __host__ __device__ static constexpr uint32_t mod(int i) {
        return i == 0 ? 0x00000001u : i == 1 ? 0xffffffffu : i == 2 ? 0xfffe5bfeu : i == 3 ? 0x53bda402u
             : i == 4 ? 0x09a1d805u : i == 5 ? 0x3339d808u : i == 6 ? 0x299d7d48u : 0x73eda753u;
    }
    __host__ __device__ static constexpr uint32_t one(int i) {
        return i == 0 ? 0xfffffffeu : i == 1 ? 0x00000001u : i == 2 ? 0x00034802u : i == 3 ? 0x5884b7fau
             : i == 4 ? 0xecbc4ff5u : i == 5 ? 0x998c4fefu : i == 6 ? 0xacc5056fu : 0x1824b159u;
    }
    __host__ __device__ static constexpr uint32_t r2(int i) {
        return i == 0 ? 0xf3f29c6du : i == 1 ? 0xc999e990u : i == 2 ? 0x87925c23u : i == 3 ? 0x2b6cedcbu
             : i == 4 ? 0x7254398fu : i == 5 ? 0x05d31496u : i == 6 ? 0x9f59ff11u : 0x0748d9d9u;
    }
};

struct Fp { uint32_t l[12]; };
struct Fr { uint32_t l[8]; };

// ------------------------------------------------------------ PTX pieces ----
#define MZK_ASM asm volatile

// Montgomery product r = a*b*2^(-32N) mod m for N-limb operands, result in
// [0, 2m) when a, b < 2m and 4m < 2^(32N) (or a, b < m otherwise).
template <class P>
__device__ __forceinline__ void mont_mul_raw(uint32_t* r, const uint32_t* a, const uint32_t* b) {
    constexpr int N = P::N;
    uint32_t x[N + 1];  // aligned at word 0, x[N] = overflow word
    uint32_t y[N];      // aligned at word 1
    // row 0: plain products, even-index limbs of a into x, odd-index into y
#pragma unroll
    for (int j = 0; j < N; j += 2) {
        MZK_ASM("mul.lo.u32 %0, %2, %3;\n\tmul.hi.u32 %1, %2, %3;" : "=r"(x[j]), "=r"(x[j + 1]) : "r"(a[j]), "r"(b[0]));
        MZK_ASM("mul.lo.u32 %0, %2, %3;\n\tmul.hi.u32 %1, %2, %3;" : "=r"(y[j]), "=r"(y[j + 1]) : "r"(a[j + 1]), "r"(b[0]));
    }
    x[N] = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        if (i > 0) {
            // divide the previous row by 2^32 while adding a*b_i:
            //   new x = y + x[1] + even products, new y = x>>64 + odd products
            uint32_t nx[N + 1], ny[N];
            const uint32_t bi = b[i];
            MZK_ASM("add.cc.u32 %0, %1, %2;" : "=r"(nx[0]) : "r"(y[0]), "r"(x[1]));
#pragma unroll
            for (int k = 0; k < N - 2; k += 2) {
                MZK_ASM("madc.lo.cc.u32 %0, %2, %3, %4;\n\tmadc.hi.cc.u32 %1, %2, %3, %5;"
                        : "=r"(ny[k]), "=r"(ny[k + 1]) : "r"(a[k + 1]), "r"(bi), "r"(x[k + 2]), "r"(x[k + 3]));
            }
            MZK_ASM("madc.lo.cc.u32 %0, %2, %3, %4;\n\tmadc.hi.u32 %1, %2, %3, 0;"
                    : "=r"(ny[N - 2]), "=r"(ny[N - 1]) : "r"(a[N - 1]), "r"(bi), "r"(x[N]));
            MZK_ASM("mad.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %4;"
                    : "+r"(nx[0]), "=r"(nx[1]) : "r"(a[0]), "r"(bi), "r"(y[1]));
#pragma unroll
            for (int j = 2; j < N; j += 2) {
                MZK_ASM("madc.lo.cc.u32 %0, %2, %3, %4;\n\tmadc.hi.cc.u32 %1, %2, %3, %5;"
                        : "=r"(nx[j]), "=r"(nx[j + 1]) : "r"(a[j]), "r"(bi), "r"(y[j]), "r"(j + 1 < N ? y[j + 1] : 0u));
            }
            MZK_ASM("addc.u32 %0, 0, 0;" : "=r"(nx[N]));
#pragma unroll
            for (int j = 0; j <= N; j++) x[j] = nx[j];
#pragma unroll
            for (int j = 0; j < N; j++) y[j] = ny[j];
        }
        // reduction: m zeroes word 0 of x
        const uint32_t m = x[0] * P::N0;
        MZK_ASM("mad.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                : "+r"(x[0]), "+r"(x[1]) : "r"(m), "r"(P::mod(0)));
#pragma unroll
        for (int j = 2; j < N; j += 2) {
            MZK_ASM("madc.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                    : "+r"(x[j]), "+r"(x[j + 1]) : "r"(m), "r"(P::mod(j)));
        }
        MZK_ASM("addc.u32 %0, %0, 0;" : "+r"(x[N]));
        MZK_ASM("mad.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                : "+r"(y[0]), "+r"(y[1]) : "r"(m), "r"(P::mod(1)));
#pragma unroll
        for (int j = 3; j < N - 1; j += 2) {
            MZK_ASM("madc.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                    : "+r"(y[j - 1]), "+r"(y[j]) : "r"(m), "r"(P::mod(j)));
        }
        MZK_ASM("madc.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.u32 %1, %2, %3, %1;"
                : "+r"(y[N - 2]), "+r"(y[N - 1]) : "r"(m), "r"(P::mod(N - 1)));
    }
    // final division by 2^32: r = y + (x >> 32)
    MZK_ASM("add.cc.u32 %0, %1, %2;" : "=r"(r[0]) : "r"(y[0]), "r"(x[1]));
#pragma unroll
    for (int j = 1; j < N - 1; j++) MZK_ASM("addc.cc.u32 %0, %1, %2;" : "=r"(r[j]) : "r"(y[j]), "r"(x[j + 1]));
    MZK_ASM("addc.u32 %0, %1, %2;" : "=r"(r[N - 1]) : "r"(y[N - 1]), "r"(x[N]));
}

// r = a + b (N limbs), returns nothing; caller guarantees no overflow
template <int N>
__device__ __forceinline__ void add_n(uint32_t* r, const uint32_t* a, const uint32_t* b) {
    MZK_ASM("add.cc.u32 %0, %1, %2;" : "=r"(r[0]) : "r"(a[0]), "r"(b[0]));
#pragma unroll
    for (int j = 1; j < N - 1; j++) MZK_ASM("addc.cc.u32 %0, %1, %2;" : "=r"(r[j]) : "r"(a[j]), "r"(b[j]));
    MZK_ASM("addc.u32 %0, %1, %2;" : "=r"(r[N - 1]) : "r"(a[N - 1]), "r"(b[N - 1]));
}
// r = a - b, returns borrow mask (0 or 0xffffffff)
template <int N>
__device__ __forceinline__ uint32_t sub_n(uint32_t* r, const uint32_t* a, const uint32_t* b) {
    uint32_t bw;
    MZK_ASM("sub.cc.u32 %0, %1, %2;" : "=r"(r[0]) : "r"(a[0]), "r"(b[0]));
#pragma unroll
    for (int j = 1; j < N; j++) MZK_ASM("subc.cc.u32 %0, %1, %2;" : "=r"(r[j]) : "r"(a[j]), "r"(b[j]));
    MZK_ASM("subc.u32 %0, 0, 0;" : "=r"(bw));
    return bw;
}
// r = t - M if t >= M else t, with M given limb-wise by the functor
template <int N, class ModF>
__device__ __forceinline__ void cond_sub(uint32_t* r, const uint32_t* t, ModF modf) {
    uint32_t s[N], bw;
    MZK_ASM("sub.cc.u32 %0, %1, %2;" : "=r"(s[0]) : "r"(t[0]), "r"(modf(0)));
#pragma unroll
    for (int j = 1; j < N; j++) MZK_ASM("subc.cc.u32 %0, %1, %2;" : "=r"(s[j]) : "r"(t[j]), "r"(modf(j)));
    MZK_ASM("subc.u32 %0, 0, 0;" : "=r"(bw));
#pragma unroll
    for (int j = 0; j < N; j++) r[j] = (t[j] & bw) | (s[j] & ~bw);
}
// r = t + (M & mask)
template <int N, class ModF>
__device__ __forceinline__ void add_masked(uint32_t* r, const uint32_t* t, uint32_t mask, ModF modf) {
    MZK_ASM("add.cc.u32 %0, %1, %2;" : "=r"(r[0]) : "r"(t[0]), "r"(modf(0) & mask));
#pragma unroll
    for (int j = 1; j < N - 1; j++) MZK_ASM("addc.cc.u32 %0, %1, %2;" : "=r"(r[j]) : "r"(t[j]), "r"(modf(j) & mask));
    MZK_ASM("addc.u32 %0, %1, %2;" : "=r"(r[N - 1]) : "r"(t[N - 1]), "r"(modf(N - 1) & mask));
}

// Montgomery square r = a^2 * 2^(-32N) mod m, the same value as
// mont_mul_raw(r, a, a) with ~N^2/2 fewer wide multiply-adds:
//  1. T = sum_{i<j} a_i a_j 2^(32(i+j)) (2N words).  Row i's products are
//     split by the parity of j - i into two chains of aligned word pairs; the
//     chain reaching word i+N runs first, and the row's last carries land in
//     word i+N+1, which no earlier row has reached.
//  2. T = 2T + sum_i a_i^2 2^(64i): a funnel shift, then one chain of the
//     diagonal products.
//  3. Montgomery reduction of the low half on an N+1-word window X (N rows
//     of X = (X + m m_mod) / 2^32, X < R throughout), then + the high half:
//     (T_lo + M m_mod)/R + T_hi = (T + M m_mod)/R, where M = -T m_mod^-1 mod R
//     is the unique multiplier word-serial Montgomery uses as well.  With
//     a < 2m and 4m < R the result is < m + 1 + m/2 < 2m.
template <class P>
__device__ __forceinline__ void mont_sqr_raw(uint32_t* r, const uint32_t* a) {
    constexpr int N = P::N;
    uint32_t t[2 * N];
#pragma unroll
    for (int k = 0; k < 2 * N; k++) t[k] = 0;
#pragma unroll
    for (int i = 0; i < N - 1; i++) {
        // chain reaching the top product a_i a_{N-1}: j = N-1, N-3, ... > i
        const int j_top0 = ((N - 1 - i) & 1) ? i + 1 : i + 2;  // first j of that parity
        MZK_ASM("mad.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                : "+r"(t[i + j_top0]), "+r"(t[i + j_top0 + 1]) : "r"(a[i]), "r"(a[j_top0]));
#pragma unroll
        for (int j = j_top0 + 2; j < N; j += 2)
            MZK_ASM("madc.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                    : "+r"(t[i + j]), "+r"(t[i + j + 1]) : "r"(a[i]), "r"(a[j]));
        MZK_ASM("addc.u32 %0, 0, 0;" : "=r"(t[i + N + 1]));
        // the other parity: j = N-2, N-4, ... > i, ending at word i+N-1
        const int j_oth0 = j_top0 == i + 1 ? i + 2 : i + 1;
        if (j_oth0 <= N - 2) {
            MZK_ASM("mad.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                    : "+r"(t[i + j_oth0]), "+r"(t[i + j_oth0 + 1]) : "r"(a[i]), "r"(a[j_oth0]));
#pragma unroll
            for (int j = j_oth0 + 2; j < N - 1; j += 2)
                MZK_ASM("madc.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                        : "+r"(t[i + j]), "+r"(t[i + j + 1]) : "r"(a[i]), "r"(a[j]));
            MZK_ASM("addc.cc.u32 %0, %0, 0;\n\taddc.u32 %1, %1, 0;" : "+r"(t[i + N]), "+r"(t[i + N + 1]));
        }
    }
    // doubling (the off-diagonal sum is < 2^(64N-1)), then the diagonal
#pragma unroll
    for (int k = 2 * N - 1; k > 0; k--)
        MZK_ASM("shf.l.clamp.b32 %0, %1, %0, 1;" : "+r"(t[k]) : "r"(t[k - 1]));
    t[0] <<= 1;
    MZK_ASM("mad.lo.cc.u32 %0, %2, %2, %0;\n\tmadc.hi.cc.u32 %1, %2, %2, %1;" : "+r"(t[0]), "+r"(t[1]) : "r"(a[0]));
#pragma unroll
    for (int i = 1; i < N - 1; i++)
        MZK_ASM("madc.lo.cc.u32 %0, %2, %2, %0;\n\tmadc.hi.cc.u32 %1, %2, %2, %1;"
                : "+r"(t[2 * i]), "+r"(t[2 * i + 1]) : "r"(a[i]));
    MZK_ASM("madc.lo.cc.u32 %0, %2, %2, %0;\n\tmadc.hi.u32 %1, %2, %2, %1;"
            : "+r"(t[2 * N - 2]), "+r"(t[2 * N - 1]) : "r"(a[N - 1]));
    // reduction of the low half
    uint32_t x[N + 1];
#pragma unroll
    for (int k = 0; k < N; k++) x[k] = t[k];
    x[N] = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        const uint32_t m = x[0] * P::N0;
        MZK_ASM("mad.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                : "+r"(x[0]), "+r"(x[1]) : "r"(m), "r"(P::mod(0)));
#pragma unroll
        for (int j = 2; j < N; j += 2)
            MZK_ASM("madc.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                    : "+r"(x[j]), "+r"(x[j + 1]) : "r"(m), "r"(P::mod(j)));
        MZK_ASM("addc.u32 %0, %0, 0;" : "+r"(x[N]));
        MZK_ASM("mad.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                : "+r"(x[1]), "+r"(x[2]) : "r"(m), "r"(P::mod(1)));
#pragma unroll
        for (int j = 3; j < N - 1; j += 2)
            MZK_ASM("madc.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.cc.u32 %1, %2, %3, %1;"
                    : "+r"(x[j]), "+r"(x[j + 1]) : "r"(m), "r"(P::mod(j)));
        MZK_ASM("madc.lo.cc.u32 %0, %2, %3, %0;\n\tmadc.hi.u32 %1, %2, %3, %1;"
                : "+r"(x[N - 1]), "+r"(x[N]) : "r"(m), "r"(P::mod(N - 1)));
        // x[0] is zero: divide by 2^32
#pragma unroll
        for (int k = 0; k < N; k++) x[k] = x[k + 1];
        x[N] = 0;
    }
    add_n<N>(r, x, t + N);
}

// -------------------------------------------------------------------- Fp ----
struct FpMod { __device__ __forceinline__ uint32_t operator()(int i) const { return FpP::mod(i); } };
struct FpMod2 { __device__ __forceinline__ uint32_t operator()(int i) const { return FpP::mod2(i); } };

__device__ __forceinline__ Fp fp_mul(const Fp& a, const Fp& b) {
    Fp r;
    mont_mul_raw<FpP>(r.l, a.l, b.l);
    return r;
}
// two independent products in one basic block, so their carry chains can be
// scheduled side by side
__device__ __forceinline__ void fp_mul2(Fp& r1, const Fp& a1, const Fp& b1, Fp& r2, const Fp& a2, const Fp& b2) {
    Fp t1, t2;
    mont_mul_raw<FpP>(t1.l, a1.l, b1.l);
    mont_mul_raw<FpP>(t2.l, a2.l, b2.l);
    r1 = t1;
    r2 = t2;
}
__device__ __forceinline__ Fp fp_sqr(const Fp& a) {
    Fp r;
    mont_sqr_raw<FpP>(r.l, a.l);
    return r;
}
__device__ __forceinline__ Fp fp_add(const Fp& a, const Fp& b) {
    Fp t, r;
    add_n<12>(t.l, a.l, b.l);
    cond_sub<12>(r.l, t.l, FpMod2());
    return r;
}
__device__ __forceinline__ Fp fp_sub(const Fp& a, const Fp& b) {
    Fp t, r;
    uint32_t bw = sub_n<12>(t.l, a.l, b.l);
    add_masked<12>(r.l, t.l, bw, FpMod2());
    return r;
}
__device__ __forceinline__ Fp fp_dbl(const Fp& a) { return fp_add(a, a); }
__device__ __forceinline__ Fp fp_neg(const Fp& a) {
    Fp z;
#pragma unroll
    for (int j = 0; j < 12; j++) z.l[j] = 0;
    return fp_sub(z, a);
}
// [0, 2p) -> [0, p)
__device__ __forceinline__ Fp fp_canonical(const Fp& a) {
    Fp r;
    cond_sub<12>(r.l, a.l, FpMod());
    return r;
}
__device__ __forceinline__ bool fp_is_zero_raw(const Fp& a) {
    uint32_t acc = 0;
#pragma unroll
    for (int j = 0; j < 12; j++) acc |= a.l[j];
    return acc == 0;
}
// zero modulo p for a lazily reduced value
__device__ __forceinline__ bool fp_is_zero(const Fp& a) { return fp_is_zero_raw(fp_canonical(a)); }
__device__ __forceinline__ Fp fp_zero() {
    Fp r;
#pragma unroll
    for (int j = 0; j < 12; j++) r.l[j] = 0;
    return r;
}
__device__ __forceinline__ Fp fp_one() {
    Fp r;
#pragma unroll
    for (int j = 0; j < 12; j++) r.l[j] = FpP::one(j);
    return r;
}
// out = a^-1 mod m for plain N-limb integers, a in [1, m), m odd and m < 2^(32N-1)
// (so x + m never overflows): the binary extended Euclidean algorithm
// (Hankerson, Menezes and Vanstone, Guide to Elliptic Curve Cryptography,
// Algorithm 2.22).  u = a, v = m, x1 = 1, x2 = 0 with a x1 = u and a x2 = v
// (mod m) throughout; halve the even one of u, v (and its x modulo m),
// subtract the smaller from the larger, until u or v is 1.  Every outer step
// ends with an even value to halve, so the bit lengths of u and v shrink by
// at least one per step: at most 64 N steps.  Returns false for a = 0 (no
// inverse) or if that bound were ever passed.  Shifts and subtractions on the
// ALU pipe instead of the multiplications of a Fermat inversion: a single
// thread finishes several times sooner.  Variable time in the value.
template <int N>
__device__ __forceinline__ bool u_is_one(const uint32_t* a) {
    uint32_t acc = a[0] ^ 1u;
#pragma unroll
    for (int j = 1; j < N; j++) acc |= a[j];
    return acc == 0;
}
template <int N>
__device__ __forceinline__ void u_shr1(uint32_t* a) {
#pragma unroll
    for (int j = 0; j < N - 1; j++) a[j] = __funnelshift_r(a[j], a[j + 1], 1);
    a[N - 1] >>= 1;
}
template <int N, class ModF>
__device__ __noinline__ bool inv_binary_raw(uint32_t* out, const uint32_t* a, ModF modf) {
    uint32_t u[N], v[N], x1[N], x2[N], t[N];
    uint32_t nz = 0;
#pragma unroll
    for (int j = 0; j < N; j++) {
        u[j] = a[j];
        v[j] = modf(j);
        x1[j] = j == 0 ? 1u : 0u;
        x2[j] = 0u;
        nz |= a[j];
    }
    if (!nz) return false;
    for (int step = 0; step <= 64 * N; step++) {
        if (u_is_one<N>(u)) {
#pragma unroll
            for (int j = 0; j < N; j++) out[j] = x1[j];
            return true;
        }
        if (u_is_one<N>(v)) {
#pragma unroll
            for (int j = 0; j < N; j++) out[j] = x2[j];
            return true;
        }
        while (!(u[0] & 1u)) {
            u_shr1<N>(u);
            add_masked<N>(t, x1, 0u - (x1[0] & 1u), modf);  // x1 / 2 mod m
#pragma unroll
            for (int j = 0; j < N; j++) x1[j] = t[j];
            u_shr1<N>(x1);
        }
        while (!(v[0] & 1u)) {
            u_shr1<N>(v);
            add_masked<N>(t, x2, 0u - (x2[0] & 1u), modf);
#pragma unroll
            for (int j = 0; j < N; j++) x2[j] = t[j];
            u_shr1<N>(x2);
        }
        const bool u_ge = sub_n<N>(t, u, v) == 0;  // no borrow: u >= v
        if (u_ge) {  // u -= v, x1 = x1 - x2 mod m
            sub_n<N>(t, u, v);
#pragma unroll
            for (int j = 0; j < N; j++) u[j] = t[j];
            const uint32_t bw = sub_n<N>(t, x1, x2);
            add_masked<N>(x1, t, bw, modf);
        } else {  // v -= u, x2 = x2 - x1 mod m
            sub_n<N>(t, v, u);
#pragma unroll
            for (int j = 0; j < N; j++) v[j] = t[j];
            const uint32_t bw = sub_n<N>(t, x2, x1);
            add_masked<N>(x2, t, bw, modf);
        }
    }
    return false;
}

// a^(p-2) by square-and-multiply over the constant exponent p-2 (Fermat);
// used for single-point normalisation only.
static __device__ __noinline__ Fp fp_inv(const Fp& a) {
    Fp acc = fp_one();
    for (int i = 11; i >= 0; i--) {
        const uint32_t e = FpP::mod(i) - (i == 0 ? 2u : 0u);
        for (int bit = 31; bit >= 0; bit--) {
            acc = fp_sqr(acc);
            if ((e >> bit) & 1u) acc = fp_mul(acc, a);
        }
    }
    return acc;
}

// -------------------------------------------------------------------- Fr ----
struct FrMod { __device__ __forceinline__ uint32_t operator()(int i) const { return FrP::mod(i); } };

__device__ __forceinline__ Fr fr_mul(const Fr& a, const Fr& b) {
    Fr t, r;
    mont_mul_raw<FrP>(t.l, a.l, b.l);
    cond_sub<8>(r.l, t.l, FrMod());
    return r;
}
__device__ __forceinline__ Fr fr_add(const Fr& a, const Fr& b) {
    Fr t, r;
    add_n<8>(t.l, a.l, b.l);
    cond_sub<8>(r.l, t.l, FrMod());
    return r;
}
__device__ __forceinline__ Fr fr_sub(const Fr& a, const Fr& b) {
    Fr t, r;
    uint32_t bw = sub_n<8>(t.l, a.l, b.l);
    add_masked<8>(r.l, t.l, bw, FrMod());
    return r;
}
__device__ __forceinline__ Fr fr_one() {
    Fr r;
#pragma unroll
    for (int j = 0; j < 8; j++) r.l[j] = FrP::one(j);
    return r;
}
__device__ __forceinline__ Fr fr_zero() {
    Fr r;
#pragma unroll
    for (int j = 0; j < 8; j++) r.l[j] = 0;
    return r;
}
// Montgomery -> canonical integer (to_repr): multiply by 1
__device__ __forceinline__ Fr fr_from_mont(const Fr& a) {
    Fr one_raw;
#pragma unroll
    for (int j = 0; j < 8; j++) one_raw.l[j] = j == 0 ? 1u : 0u;
    return fr_mul(a, one_raw);
}
// canonical integer -> Montgomery: multiply by R^2
__device__ __forceinline__ Fr fr_to_mont(const Fr& a) {
    Fr r2;
#pragma unroll
    for (int j = 0; j < 8; j++) r2.l[j] = FrP::r2(j);
    return fr_mul(a, r2);
}

}  // namespace mzk
