/*
 * mzk_oracle.c — CPU restatement of the midnight-zk prover core.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product): loaded by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs.
 *
 * 64-bit limbs with unsigned __int128 products, OpenMP for the parallel parts
 * that the reference runs on rayon.  Every reference algorithm cites the file
 * and lines of midnightntwrk/midnight-zk it restates.  The field and curve
 * primitives (inside the un-vendored `blst` crate in the reference) are
 * restated from published mathematics: Montgomery CIOS (Koc, Acar, Kaliski
 * 1996), Jacobian formulas "add-1998-cmo-2" / "dbl-2009-l" from the Explicit
 * Formulas Database, Fermat inversion, and the ZCash BLS12-381 compressed
 * point format.
 */
#include "mzk_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint64_t u64;
typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------- */
/* Constants                                                                 */
/* ------------------------------------------------------------------------- */

/* r, curves/src/bls12_381/fq.rs:43-48 */
static const u64 FR_MOD[4] = {0xffffffff00000001ULL, 0x53bda402fffe5bfeULL,
                              0x3339d80809a1d805ULL, 0x73eda753299d7d48ULL};
/* p, curves/src/bls12_381/fp.rs:20-27 */
static const u64 FP_MOD[6] = {0xb9feffffffffaaabULL, 0x1eabfffeb153ffffULL,
                              0x6730d2a0f6b0f624ULL, 0x64774b84f38512bfULL,
                              0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL};
/* Montgomery-form constants of Fq, fq.rs:34-41 (GENERATOR), :70-77
 * (ROOT_OF_UNITY), :490-497 (ROOT_OF_UNITY_INV), :501-508 (DELTA), :702-710
 * (ZETA).  They are pinned against the reference source by the golden tests. */
static const u64 FR_GENERATOR[4] = {0x0000000efffffff1ULL, 0x17e363d300189c0fULL,
                                    0xff9c57876f8457b0ULL, 0x351332208fc5a8c4ULL};
static const u64 FR_ROOT_OF_UNITY[4] = {0xb9b58d8c5f0e466aULL, 0x5b1b4c801819d7ecULL,
                                        0x0af53ae352a31e64ULL, 0x5bf3adda19e9b27bULL};
static const u64 FR_ROOT_OF_UNITY_INV[4] = {0x4256481adcf3219aULL, 0x45f37b7f96b6cad3ULL,
                                            0xf9c3f1d75f7a3b27ULL, 0x2d2fc049658afd43ULL};
static const u64 FR_DELTA[4] = {0x70e310d3d146f96aULL, 0x4b64c08919e299e6ULL,
                                0x51e114186a8b970dULL, 0x6185d06627c067cbULL};
static const u64 FR_ZETA[4] = {0x92d9090b093011d2ULL, 0xfc9cbd719d6aa073ULL,
                               0xc1f14ef0cd65a1a6ULL, 0x017f6d35e72fcdebULL};
/* G1 generator, canonical coordinates from curves/README.md:96-101 */
static const u64 G1_GEN_X[6] = {0xfb3af00adb22c6bbULL, 0x6c55e83ff97a1aefULL, 0xa14e3a3f171bac58ULL,
                                0xc3688c4f9774b905ULL, 0x2695638c4fa9ac0fULL, 0x17f1d3a73197d794ULL};
static const u64 G1_GEN_Y[6] = {0x0caa232946c5e7e1ULL, 0xd03cc744a2888ae4ULL, 0x00db18cb2c04b3edULL,
                                0xfcf5e095d5d00af6ULL, 0xa09e30ed741d8ae4ULL, 0x08b3f481e3aaa0f1ULL};

static u64 FR_INV, FP_INV;          /* -m^{-1} mod 2^64 */
static u64 FR_R[4], FR_R2[4];       /* R, R^2 mod r */
static u64 FP_R[6], FP_R2[6];       /* R, R^2 mod p */
static u64 FP_B[6];                 /* 4 in Montgomery form */
static int g_init = 0;

/* ------------------------------------------------------------------------- */
/* Generic multi-precision helpers                                           */
/* ------------------------------------------------------------------------- */

static inline int geq_n(const u64 *a, const u64 *b, int n) {
    for (int i = n - 1; i >= 0; i--) {
        if (a[i] != b[i]) return a[i] > b[i];
    }
    return 1;
}
static inline u64 sub_n(u64 *out, const u64 *a, const u64 *b, int n) {
    u64 borrow = 0;
    for (int i = 0; i < n; i++) {
        u128 d = (u128)a[i] - b[i] - borrow;
        out[i] = (u64)d;
        borrow = (u64)(d >> 127);
    }
    return borrow;
}
static inline u64 add_n(u64 *out, const u64 *a, const u64 *b, int n) {
    u64 c = 0;
    for (int i = 0; i < n; i++) {
        u128 s = (u128)a[i] + b[i] + c;
        out[i] = (u64)s;
        c = (u64)(s >> 64);
    }
    return c;
}
static inline int is_zero_n(const u64 *a, int n) {
    u64 acc = 0;
    for (int i = 0; i < n; i++) acc |= a[i];
    return acc == 0;
}

/* Montgomery CIOS multiplication: out = a*b*2^{-64n} mod m, inputs < m. */
static inline void mont_mul_n(u64 *out, const u64 *a, const u64 *b, const u64 *m, u64 inv, int n) {
    u64 t[8] = {0};
    for (int i = 0; i < n; i++) {
        u64 c = 0;
        for (int j = 0; j < n; j++) {
            u128 s = (u128)a[j] * b[i] + t[j] + c;
            t[j] = (u64)s;
            c = (u64)(s >> 64);
        }
        u128 s = (u128)t[n] + c;
        t[n] = (u64)s;
        t[n + 1] = (u64)(s >> 64);
        u64 q = t[0] * inv;
        s = (u128)q * m[0] + t[0];
        c = (u64)(s >> 64);
        for (int j = 1; j < n; j++) {
            s = (u128)q * m[j] + t[j] + c;
            t[j - 1] = (u64)s;
            c = (u64)(s >> 64);
        }
        s = (u128)t[n] + c;
        t[n - 1] = (u64)s;
        t[n] = t[n + 1] + (u64)(s >> 64);
    }
    if (t[n] || geq_n(t, m, n)) sub_n(t, t, m, n);
    memcpy(out, t, 8 * n);
}
static inline void mod_add_n(u64 *out, const u64 *a, const u64 *b, const u64 *m, int n) {
    u64 t[8];
    u64 c = add_n(t, a, b, n);
    if (c || geq_n(t, m, n)) sub_n(t, t, m, n);
    memcpy(out, t, 8 * n);
}
static inline void mod_sub_n(u64 *out, const u64 *a, const u64 *b, const u64 *m, int n) {
    u64 t[8];
    u64 br = sub_n(t, a, b, n);
    if (br) add_n(t, t, m, n);
    memcpy(out, t, 8 * n);
}
/* -m^{-1} mod 2^64 by Newton iteration */
static u64 neg_inv64(u64 m0) {
    u64 x = 1;
    for (int i = 0; i < 7; i++) x *= 2 - m0 * x;
    return (u64)0 - x;
}
/* R mod m and R^2 mod m by repeated doubling of 1 */
static void compute_r_r2(u64 *r, u64 *r2, const u64 *m, int n) {
    u64 t[8] = {0};
    t[0] = 1;
    for (int i = 0; i < 64 * n * 2; i++) {
        mod_add_n(t, t, t, m, n);
        if (i == 64 * n - 1) memcpy(r, t, 8 * n);
    }
    memcpy(r2, t, 8 * n);
}

static void init_consts(void) {
    if (g_init) return;
    FR_INV = neg_inv64(FR_MOD[0]);
    FP_INV = neg_inv64(FP_MOD[0]);
    compute_r_r2(FR_R, FR_R2, FR_MOD, 4);
    compute_r_r2(FP_R, FP_R2, FP_MOD, 6);
    u64 four[6] = {4, 0, 0, 0, 0, 0};
    mont_mul_n(FP_B, four, FP_R2, FP_MOD, FP_INV, 6);
    g_init = 1;
}
__attribute__((constructor)) static void oracle_ctor(void) { init_consts(); }

/* ------------------------------------------------------------------------- */
/* Fr                                                                        */
/* ------------------------------------------------------------------------- */
/* Fr multiplications counted while counting is on (single-threaded runs
 * only: the work figures of the quotient evaluation come from this count) */
static int g_fr_count_on;
static unsigned long long g_fr_mul_count;
static inline void fr_mul(u64 *o, const u64 *a, const u64 *b) {
    if (g_fr_count_on) g_fr_mul_count++;
    mont_mul_n(o, a, b, FR_MOD, FR_INV, 4);
}
static inline void fr_add(u64 *o, const u64 *a, const u64 *b) { mod_add_n(o, a, b, FR_MOD, 4); }
static inline void fr_sub(u64 *o, const u64 *a, const u64 *b) { mod_sub_n(o, a, b, FR_MOD, 4); }
static void fr_pow(u64 *o, const u64 *a, const u64 *e, int elimbs) {
    u64 acc[4];
    memcpy(acc, FR_R, 32);
    for (int i = elimbs * 64 - 1; i >= 0; i--) {
        fr_mul(acc, acc, acc);
        if ((e[i / 64] >> (i % 64)) & 1) fr_mul(acc, acc, a);
    }
    memcpy(o, acc, 32);
}
static void fr_inv(u64 *o, const u64 *a) {
    u64 e[4];
    u64 two[4] = {2, 0, 0, 0};
    sub_n(e, FR_MOD, two, 4);
    fr_pow(o, a, e, 4);
}

void or_fr_mul(uint64_t out[4], const uint64_t a[4], const uint64_t b[4]) { fr_mul(out, a, b); }
void or_fr_add(uint64_t out[4], const uint64_t a[4], const uint64_t b[4]) { fr_add(out, a, b); }
void or_fr_sub(uint64_t out[4], const uint64_t a[4], const uint64_t b[4]) { fr_sub(out, a, b); }
void or_fr_neg(uint64_t out[4], const uint64_t a[4]) {
    u64 z[4] = {0};
    fr_sub(out, z, a);
}
void or_fr_inv(uint64_t out[4], const uint64_t a[4]) { fr_inv(out, a); }
void or_fr_from_canonical(uint64_t out[4], const uint64_t a[4]) { fr_mul(out, a, FR_R2); }
void or_fr_to_canonical(uint64_t out[4], const uint64_t a[4]) {
    u64 one[4] = {1, 0, 0, 0};
    fr_mul(out, a, one);
}
void or_fr_const(int which, uint64_t out[4]) {
    const u64 *src = FR_R;
    switch (which) {
        case 0: src = FR_R; break;
        case 1: src = FR_R2; break;
        case 2: src = FR_ROOT_OF_UNITY; break;
        case 3: src = FR_ZETA; break;
        case 4: src = FR_ROOT_OF_UNITY_INV; break;
        case 5: src = FR_DELTA; break;
        case 6: src = FR_GENERATOR; break;
    }
    memcpy(out, src, 32);
}

/* ------------------------------------------------------------------------- */
/* Fp                                                                        */
/* ------------------------------------------------------------------------- */
static inline void fp_mul(u64 *o, const u64 *a, const u64 *b) { mont_mul_n(o, a, b, FP_MOD, FP_INV, 6); }
static inline void fp_add(u64 *o, const u64 *a, const u64 *b) { mod_add_n(o, a, b, FP_MOD, 6); }
static inline void fp_sub(u64 *o, const u64 *a, const u64 *b) { mod_sub_n(o, a, b, FP_MOD, 6); }
static inline int fp_is_zero(const u64 *a) { return is_zero_n(a, 6); }
static inline int fp_eq(const u64 *a, const u64 *b) { return memcmp(a, b, 48) == 0; }
static void fp_inv(u64 *o, const u64 *a) {
    u64 e[6];
    u64 two[6] = {2, 0, 0, 0, 0, 0};
    sub_n(e, FP_MOD, two, 6);
    u64 acc[6];
    memcpy(acc, FP_R, 48);
    for (int i = 6 * 64 - 1; i >= 0; i--) {
        fp_mul(acc, acc, acc);
        if ((e[i / 64] >> (i % 64)) & 1) fp_mul(acc, acc, a);
    }
    memcpy(o, acc, 48);
}
void or_fp_mul(uint64_t out[6], const uint64_t a[6], const uint64_t b[6]) { fp_mul(out, a, b); }
void or_fp_add(uint64_t out[6], const uint64_t a[6], const uint64_t b[6]) { fp_add(out, a, b); }
void or_fp_sub(uint64_t out[6], const uint64_t a[6], const uint64_t b[6]) { fp_sub(out, a, b); }
void or_fp_inv(uint64_t out[6], const uint64_t a[6]) { fp_inv(out, a); }
void or_fp_from_canonical(uint64_t out[6], const uint64_t a[6]) { fp_mul(out, a, FP_R2); }
void or_fp_to_canonical(uint64_t out[6], const uint64_t a[6]) {
    u64 one[6] = {1, 0, 0, 0, 0, 0};
    fp_mul(out, a, one);
}
void or_fp_const(int which, uint64_t out[6]) {
    const u64 *src = which == 0 ? FP_R : which == 1 ? FP_R2 : FP_B;
    memcpy(out, src, 48);
}

/* ------------------------------------------------------------------------- */
/* G1 (short Weierstrass y^2 = x^3 + 4 over Fp)                              */
/* ------------------------------------------------------------------------- */
typedef struct { u64 x[6], y[6]; } aff_t;        /* identity: all zero */
typedef struct { u64 x[6], y[6], z[6]; } jac_t;  /* identity: z == 0 */

static inline int aff_is_inf(const aff_t *p) { return fp_is_zero(p->x) && fp_is_zero(p->y); }
static inline int jac_is_inf(const jac_t *p) { return fp_is_zero(p->z); }
static inline void jac_set_inf(jac_t *p) { memset(p, 0, sizeof(*p)); }
static inline void jac_from_aff(jac_t *o, const aff_t *a) {
    if (aff_is_inf(a)) { jac_set_inf(o); return; }
    memcpy(o->x, a->x, 48);
    memcpy(o->y, a->y, 48);
    memcpy(o->z, FP_R, 48);
}

/* dbl-2009-l (a = 0) */
static void jac_double(jac_t *o, const jac_t *p) {
    if (jac_is_inf(p)) { jac_set_inf(o); return; }
    u64 A[6], B[6], C[6], D[6], E[6], F[6], t[6], X3[6], Y3[6], Z3[6];
    fp_mul(A, p->x, p->x);
    fp_mul(B, p->y, p->y);
    fp_mul(C, B, B);
    fp_add(t, p->x, B);
    fp_mul(t, t, t);
    fp_sub(t, t, A);
    fp_sub(t, t, C);
    fp_add(D, t, t);
    fp_add(E, A, A);
    fp_add(E, E, A);
    fp_mul(F, E, E);
    fp_sub(X3, F, D);
    fp_sub(X3, X3, D);
    fp_sub(t, D, X3);
    fp_mul(Y3, E, t);
    fp_add(t, C, C);
    fp_add(t, t, t);
    fp_add(t, t, t);
    fp_sub(Y3, Y3, t);
    fp_mul(Z3, p->y, p->z);
    fp_add(Z3, Z3, Z3);
    memcpy(o->x, X3, 48);
    memcpy(o->y, Y3, 48);
    memcpy(o->z, Z3, 48);
}

/* add-1998-cmo-2 with the doubling / inverse special cases */
static void jac_add(jac_t *o, const jac_t *p, const jac_t *q) {
    if (jac_is_inf(p)) { *o = *q; return; }
    if (jac_is_inf(q)) { *o = *p; return; }
    u64 Z1Z1[6], Z2Z2[6], U1[6], U2[6], S1[6], S2[6], H[6], R[6], t[6];
    fp_mul(Z1Z1, p->z, p->z);
    fp_mul(Z2Z2, q->z, q->z);
    fp_mul(U1, p->x, Z2Z2);
    fp_mul(U2, q->x, Z1Z1);
    fp_mul(t, q->z, Z2Z2);
    fp_mul(S1, p->y, t);
    fp_mul(t, p->z, Z1Z1);
    fp_mul(S2, q->y, t);
    fp_sub(H, U2, U1);
    fp_sub(R, S2, S1);
    if (fp_is_zero(H)) {
        if (fp_is_zero(R)) { jac_double(o, p); return; }
        jac_set_inf(o);
        return;
    }
    u64 HH[6], HHH[6], V[6], X3[6], Y3[6], Z3[6];
    fp_mul(HH, H, H);
    fp_mul(HHH, HH, H);
    fp_mul(V, U1, HH);
    fp_mul(X3, R, R);
    fp_sub(X3, X3, HHH);
    fp_sub(X3, X3, V);
    fp_sub(X3, X3, V);
    fp_sub(t, V, X3);
    fp_mul(Y3, R, t);
    fp_mul(t, S1, HHH);
    fp_sub(Y3, Y3, t);
    fp_mul(Z3, p->z, q->z);
    fp_mul(Z3, Z3, H);
    memcpy(o->x, X3, 48);
    memcpy(o->y, Y3, 48);
    memcpy(o->z, Z3, 48);
}
static void jac_add_aff(jac_t *o, const jac_t *p, const aff_t *q) {
    jac_t qq;
    jac_from_aff(&qq, q);
    jac_add(o, p, &qq);
}
static void aff_neg(aff_t *o, const aff_t *p) {
    *o = *p;
    if (aff_is_inf(p)) return;
    u64 z[6] = {0};
    fp_sub(o->y, z, p->y);
}
static void jac_to_aff(aff_t *o, const jac_t *p) {
    if (jac_is_inf(p)) { memset(o, 0, sizeof(*o)); return; }
    u64 zi[6], zi2[6], zi3[6];
    fp_inv(zi, p->z);
    fp_mul(zi2, zi, zi);
    fp_mul(zi3, zi2, zi);
    fp_mul(o->x, p->x, zi2);
    fp_mul(o->y, p->y, zi3);
}

void or_g1_generator(uint64_t out[12]) {
    fp_mul(out, G1_GEN_X, FP_R2);
    fp_mul(out + 6, G1_GEN_Y, FP_R2);
}
void or_g1_add(uint64_t out[18], const uint64_t a[18], const uint64_t b[18]) {
    jac_add((jac_t *)out, (const jac_t *)a, (const jac_t *)b);
}
void or_g1_double(uint64_t out[18], const uint64_t a[18]) { jac_double((jac_t *)out, (const jac_t *)a); }
void or_g1_to_affine(uint64_t out[12], const uint64_t jac[18]) { jac_to_aff((aff_t *)out, (const jac_t *)jac); }
void or_g1_from_affine(uint64_t out[18], const uint64_t aff[12]) { jac_from_aff((jac_t *)out, (const aff_t *)aff); }
int or_g1_is_on_curve_affine(const uint64_t aff[12]) {
    const aff_t *p = (const aff_t *)aff;
    if (aff_is_inf(p)) return 1;
    u64 l[6], r[6];
    fp_mul(l, p->y, p->y);
    fp_mul(r, p->x, p->x);
    fp_mul(r, r, p->x);
    fp_add(r, r, FP_B);
    return fp_eq(l, r);
}
static void jac_mul_canonical(jac_t *o, const aff_t *p, const u64 k[4]) {
    jac_t acc;
    jac_set_inf(&acc);
    for (int i = 255; i >= 0; i--) {
        jac_double(&acc, &acc);
        if ((k[i / 64] >> (i % 64)) & 1) jac_add_aff(&acc, &acc, p);
    }
    *o = acc;
}
void or_g1_mul(uint64_t out[12], const uint64_t aff[12], const uint64_t scalar_mont[4]) {
    u64 k[4];
    or_fr_to_canonical(k, scalar_mont);
    jac_t r;
    jac_mul_canonical(&r, (const aff_t *)aff, k);
    jac_to_aff((aff_t *)out, &r);
}
/* ZCash format: big-endian x, bit7 compressed, bit6 infinity, bit5 sign of y
 * (y lexicographically largest, i.e. y > (p-1)/2).  Matches the encoding
 * `G1Affine::to_compressed` produces (curves/src/bls12_381/g1.rs:326-333). */
void or_g1_compress(uint8_t out[48], const uint64_t aff[12]) {
    const aff_t *p = (const aff_t *)aff;
    memset(out, 0, 48);
    if (aff_is_inf(p)) { out[0] = 0xc0; return; }
    u64 x[6], y[6], ny[6], z[6] = {0};
    or_fp_to_canonical(x, p->x);
    or_fp_to_canonical(y, p->y);
    fp_sub(ny, z, y); /* p - y */
    for (int i = 0; i < 48; i++) out[47 - i] = (uint8_t)(x[i / 8] >> (8 * (i % 8)));
    out[0] |= 0x80;
    /* y > p - y  <=> y is the larger root */
    if (!geq_n(ny, y, 6)) out[0] |= 0x20;
}

/* The reverse of or_g1_compress, as G1Affine::from_compressed (g1.rs:367-376:
 * blst_p1_uncompress, then the G1 membership check): compression flag set;
 * the infinity flag with every other bit zero is the identity; otherwise
 * x < p, y = (x^3 + 4)^((p+1)/4) must square back (p = 3 mod 4), the sign
 * flag picks y > (p-1)/2, and with check_subgroup [r]P must be the identity.
 * Returns 0 ok, 1 bad encoding, 2 not on the curve, 3 not in G1. */
int or_g1_decompress(uint64_t out[12], const uint8_t in[48], int check_subgroup) {
    aff_t *p = (aff_t *)out;
    memset(out, 0, 96);
    const uint8_t flags = in[0] & 0xe0;
    if (!(flags & 0x80)) return 1;
    if (flags & 0x40) {
        if (in[0] & 0x3f) return 1;
        for (int i = 1; i < 48; i++)
            if (in[i]) return 1;
        return 0;
    }
    u64 x[6] = {0};
    for (int i = 0; i < 48; i++) x[i / 8] |= (u64)(i == 47 ? (in[0] & 0x1f) : in[47 - i]) << (8 * (i % 8));
    if (geq_n(x, FP_MOD, 6)) return 1;
    u64 xm[6], rhs[6], y[6], t[6], e[6], one[6] = {1, 0, 0, 0, 0, 0};
    fp_mul(xm, x, FP_R2);
    fp_mul(t, xm, xm);
    fp_mul(t, t, xm);
    fp_add(rhs, t, FP_B);
    /* e = (p + 1) / 4 */
    add_n(e, FP_MOD, one, 6);
    for (int i = 0; i < 6; i++) e[i] = (e[i] >> 2) | (i < 5 ? e[i + 1] << 62 : 0);
    memcpy(y, FP_R, 48);
    for (int i = 6 * 64 - 1; i >= 0; i--) {
        fp_mul(y, y, y);
        if ((e[i / 64] >> (i % 64)) & 1) fp_mul(y, y, rhs);
    }
    fp_mul(t, y, y);
    if (!fp_eq(t, rhs)) return 2;
    u64 yc[6], nyc[6], z[6] = {0}, ny[6];
    or_fp_to_canonical(yc, y);
    fp_sub(ny, z, y);
    or_fp_to_canonical(nyc, ny);
    const int larger = !geq_n(nyc, yc, 6); /* y > p - y */
    if (larger != !!(flags & 0x20)) memcpy(y, ny, 48);
    memcpy(p->x, xm, 48);
    memcpy(p->y, y, 48);
    if (check_subgroup) {
        jac_t r;
        u64 order[4];
        memcpy(order, FR_MOD, 32);
        jac_mul_canonical(&r, p, order);
        if (!fp_is_zero(r.z)) return 3;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* MSM                                                                       */
/* ------------------------------------------------------------------------- */

void or_msm_naive(uint64_t out[12], const uint64_t *scalars, const uint64_t *bases, size_t n) {
    jac_t acc;
    jac_set_inf(&acc);
    for (size_t i = 0; i < n; i++) {
        u64 k[4];
        or_fr_to_canonical(k, scalars + 4 * i);
        jac_t t;
        jac_mul_canonical(&t, (const aff_t *)(bases + 12 * i), k);
        jac_add(&acc, &acc, &t);
    }
    jac_to_aff((aff_t *)out, &acc);
}

/* get_booth_index, curves/src/msm.rs:13-55 */
int or_booth_index(size_t window_index, size_t window_size, const uint8_t el[32]) {
    size_t skip_bits = window_index * window_size;
    skip_bits = skip_bits > 0 ? skip_bits - 1 : 0;
    size_t skip_bytes = skip_bits / 8;
    uint8_t v[4] = {0, 0, 0, 0};
    for (size_t i = 0; i < 4 && skip_bytes + i < 32; i++) v[i] = el[skip_bytes + i];
    uint32_t tmp = (uint32_t)v[0] | ((uint32_t)v[1] << 8) | ((uint32_t)v[2] << 16) | ((uint32_t)v[3] << 24);
    if (window_index == 0) tmp <<= 1;
    tmp >>= skip_bits - (skip_bytes * 8);
    tmp &= (1u << (window_size + 1)) - 1;
    int sign = (tmp & (1u << window_size)) == 0;
    tmp = (tmp + 1) >> 1;
    if (sign) return (int)tmp;
    return -(int)((~(tmp - 1)) & ((1u << window_size) - 1));
}

static int msm_window_c(size_t n) {
    /* msm.rs:464-470 (and msm_serial :341-347): natural log, ceil */
    if (n < 4) return 1;
    if (n < 32) return 3;
    return (int)ceil(log((double)(uint32_t)n));
}

/* msm_serial, curves/src/msm.rs:338-423 */
typedef struct { int kind; aff_t a; jac_t j; } serial_bucket_t; /* 0 none 1 affine 2 proj */
static void msm_serial(jac_t *acc, const uint8_t (*reprs)[32], const aff_t *bases, size_t n) {
    int c = msm_window_c(n);
    uint8_t acc_or[32] = {0};
    for (size_t i = 0; i < n; i++)
        for (int b = 0; b < 32; b++) acc_or[b] |= reprs[i][b];
    int max_byte_size = 32;
    while (max_byte_size > 0 && acc_or[max_byte_size - 1] == 0) max_byte_size--;
    if (max_byte_size == 0) return;
    int number_of_windows = max_byte_size * 8 / c + 1;
    size_t nb = (size_t)1 << (c - 1);
    serial_bucket_t *buckets = (serial_bucket_t *)malloc(nb * sizeof(serial_bucket_t));
    for (int w = number_of_windows - 1; w >= 0; w--) {
        for (int i = 0; i < c; i++) jac_double(acc, acc);
        for (size_t b = 0; b < nb; b++) buckets[b].kind = 0;
        for (size_t i = 0; i < n; i++) {
            int d = or_booth_index((size_t)w, (size_t)c, reprs[i]);
            if (d == 0) continue;
            aff_t p = bases[i];
            if (d < 0) aff_neg(&p, &bases[i]);
            serial_bucket_t *bk = &buckets[(d < 0 ? -d : d) - 1];
            if (bk->kind == 0) { bk->kind = 1; bk->a = p; }
            else if (bk->kind == 1) { jac_t t; jac_from_aff(&t, &bk->a); jac_add_aff(&bk->j, &t, &p); bk->kind = 2; }
            else jac_add_aff(&bk->j, &bk->j, &p);
        }
        jac_t running;
        jac_set_inf(&running);
        for (size_t b = nb; b-- > 0;) {
            if (buckets[b].kind == 1) jac_add_aff(&running, &running, &buckets[b].a);
            else if (buckets[b].kind == 2) jac_add(&running, &running, &buckets[b].j);
            jac_add(acc, acc, &running);
        }
    }
    free(buckets);
}

/* msm_parallel, curves/src/msm.rs:430-455 (rayon chunks -> OpenMP chunks) */
static void msm_parallel(jac_t *out, const uint8_t (*reprs)[32], const aff_t *bases, size_t n, int threads) {
    jac_set_inf(out);
    if ((size_t)threads >= n || threads <= 1) {
        msm_serial(out, reprs, bases, n);
        return;
    }
    size_t chunk = n / (size_t)threads;
    size_t nchunks = (n + chunk - 1) / chunk;
    jac_t *res = (jac_t *)calloc(nchunks, sizeof(jac_t));
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
    for (size_t ci = 0; ci < nchunks; ci++) {
        size_t lo = ci * chunk, hi = lo + chunk > n ? n : lo + chunk;
        jac_set_inf(&res[ci]);
        msm_serial(&res[ci], reprs + lo, bases + lo, hi - lo);
    }
    for (size_t ci = 0; ci < nchunks; ci++) jac_add(out, out, &res[ci]);
    free(res);
}

/* Schedule / batch_add: 64-wide batch-affine bucket additions,
 * curves/src/msm.rs:58-144 (batch_add) and :273-333 (Schedule). */
#define MSM_BATCH 64
typedef struct { size_t base_idx, buck_idx; int sign; } sched_pt_t;
typedef struct { int some; aff_t p; } abucket_t;
typedef struct {
    abucket_t *buckets;
    sched_pt_t set[MSM_BATCH];
    size_t ptr;
} schedule_t;

static void batch_add(size_t size, abucket_t *buckets, const sched_pt_t *points, const aff_t *bases) {
    u64 t[MSM_BATCH][6], z[MSM_BATCH][6], acc[6];
    memcpy(acc, FP_R, 48);
    for (size_t k = 0; k < size; k++) {
        const sched_pt_t *sp = &points[k];
        abucket_t *bk = &buckets[sp->buck_idx];
        const aff_t *b = &bases[sp->base_idx];
        if (!bk->some) continue;
        if (fp_eq(bk->p.x, b->x)) {
            if (fp_eq(bk->p.y, b->y) ^ !sp->sign) {
                u64 xs[6], three[6];
                fp_mul(xs, b->x, b->x);
                fp_add(three, xs, xs);
                fp_add(three, three, xs);
                fp_add(z[k], bk->p.y, bk->p.y);
                fp_mul(t[k], acc, three);
                fp_mul(acc, acc, z[k]);
                continue;
            }
            bk->some = 0;
            continue;
        }
        fp_sub(z[k], bk->p.x, b->x);
        u64 dy[6];
        if (sp->sign) fp_sub(dy, bk->p.y, b->y);
        else fp_add(dy, bk->p.y, b->y);
        fp_mul(t[k], acc, dy);
        fp_mul(acc, acc, z[k]);
    }
    fp_inv(acc, acc);
    for (size_t k = size; k-- > 0;) {
        const sched_pt_t *sp = &points[k];
        abucket_t *bk = &buckets[sp->buck_idx];
        const aff_t *b = &bases[sp->base_idx];
        if (!bk->some) continue;
        u64 lambda[6], x[6], s[6], y[6];
        fp_mul(lambda, acc, t[k]);
        fp_mul(acc, acc, z[k]);
        fp_mul(x, lambda, lambda);
        fp_add(s, bk->p.x, b->x);
        fp_sub(x, x, s);
        fp_sub(s, b->x, x);
        fp_mul(y, lambda, s);
        if (sp->sign) fp_sub(y, y, b->y);
        else fp_add(y, y, b->y);
        memcpy(bk->p.y, y, 48);
        memcpy(bk->p.x, x, 48);
    }
}
static void sched_execute(schedule_t *s, const aff_t *bases) {
    if (s->ptr != 0) {
        batch_add(s->ptr, s->buckets, s->set, bases);
        s->ptr = 0;
    }
}
static int sched_contains(const schedule_t *s, size_t b) {
    for (size_t i = 0; i < s->ptr; i++)
        if (s->set[i].buck_idx == b) return 1;
    return 0;
}
static void sched_add(schedule_t *s, const aff_t *bases, size_t base_idx, size_t buck_idx, int sign) {
    abucket_t *bk = &s->buckets[buck_idx];
    if (!bk->some) {
        bk->some = 1;
        if (sign) bk->p = bases[base_idx];
        else aff_neg(&bk->p, &bases[base_idx]);
    } else {
        s->set[s->ptr].base_idx = base_idx;
        s->set[s->ptr].buck_idx = buck_idx;
        s->set[s->ptr].sign = sign;
        s->ptr++;
    }
    if (s->ptr == MSM_BATCH) sched_execute(s, bases);
}

static void to_reprs(uint8_t (*reprs)[32], const u64 *scalars, size_t n, int threads) {
#pragma omp parallel for num_threads(threads) schedule(static)
    for (size_t i = 0; i < n; i++) {
        u64 k[4];
        or_fr_to_canonical(k, scalars + 4 * i);
        for (int b = 0; b < 32; b++) reprs[i][b] = (uint8_t)(k[b / 8] >> (8 * (b % 8)));
    }
}

/* msm_best, curves/src/msm.rs:460-532 */
static void msm_best_jac(jac_t *out, const u64 *scalars, const aff_t *bases_in, size_t n, int threads) {
    if (threads < 1) threads = 1;
    int c = msm_window_c(n);
    jac_set_inf(out);
    if (n == 0) return;
    if (c < 10) {
        uint8_t (*reprs)[32] = (uint8_t (*)[32])malloc(n * 32);
        to_reprs(reprs, scalars, n, threads);
        msm_parallel(out, (const uint8_t (*)[32])reprs, bases_in, n, threads);
        free(reprs);
        return;
    }
    /* filter identity bases, to_repr the scalars (msm.rs:477-482) */
    uint8_t (*reprs)[32] = (uint8_t (*)[32])malloc(n * 32);
    aff_t *bases = (aff_t *)malloc(n * sizeof(aff_t));
    size_t m = 0;
    for (size_t i = 0; i < n; i++) {
        if (aff_is_inf(&bases_in[i])) continue;
        u64 k[4];
        or_fr_to_canonical(k, scalars + 4 * i);
        for (int b = 0; b < 32; b++) reprs[m][b] = (uint8_t)(k[b / 8] >> (8 * (b % 8)));
        bases[m] = bases_in[i];
        m++;
    }
    int number_of_windows = 255 / c + 1;
    size_t nb = (size_t)1 << (c - 1);
    jac_t *acc = (jac_t *)calloc((size_t)number_of_windows, sizeof(jac_t));
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
    for (int w = number_of_windows - 1; w >= 0; w--) {
        jac_t *jb = (jac_t *)calloc(nb, sizeof(jac_t)); /* all z == 0: None */
        schedule_t s;
        s.buckets = (abucket_t *)calloc(nb, sizeof(abucket_t));
        s.ptr = 0;
        for (size_t bi = 0; bi < m; bi++) {
            int d = or_booth_index((size_t)w, (size_t)c, reprs[bi]);
            if (d == 0) continue;
            int sign = d > 0;
            size_t buck = (size_t)(d < 0 ? -d : d) - 1;
            if (sched_contains(&s, buck)) {
                aff_t p = bases[bi];
                if (!sign) aff_neg(&p, &bases[bi]);
                jac_add_aff(&jb[buck], &jb[buck], &p);
            } else {
                sched_add(&s, bases, bi, buck, sign);
            }
        }
        sched_execute(&s, bases);
        jac_t running, a;
        jac_set_inf(&running);
        jac_set_inf(&a);
        for (size_t b = nb; b-- > 0;) {
            jac_t t = jb[b];
            if (s.buckets[b].some) jac_add_aff(&t, &t, &s.buckets[b].p);
            jac_add(&running, &running, &t);
            jac_add(&a, &a, &running);
        }
        for (int i = 0; i < c * w; i++) jac_double(&a, &a);
        acc[w] = a;
        free(jb);
        free(s.buckets);
    }
    for (int w = 0; w < number_of_windows; w++) jac_add(out, out, &acc[w]);
    free(acc);
    free(reprs);
    free(bases);
}

void or_msm_best(uint64_t out[12], const uint64_t *scalars, const uint64_t *bases, size_t n, int threads) {
    jac_t r;
    msm_best_jac(&r, scalars, (const aff_t *)bases, n, threads);
    jac_to_aff((aff_t *)out, &r);
}

/* msm_specific: drop zero scalars, then the MSM (kzg/msm.rs:174-201).  The
 * reference dispatches n <= 2^19 to blst's Pippenger and larger n to
 * msm_best; both compute the same unique group element, the oracle uses
 * msm_best for both. */
void or_msm_specific(uint64_t out[12], const uint64_t *scalars, const uint64_t *bases, size_t n, int threads) {
    u64 *s = (u64 *)malloc((n ? n : 1) * 32);
    u64 *b = (u64 *)malloc((n ? n : 1) * 96);
    size_t m = 0;
    for (size_t i = 0; i < n; i++) {
        if (is_zero_n(scalars + 4 * i, 4)) continue;
        memcpy(s + 4 * m, scalars + 4 * i, 32);
        memcpy(b + 12 * m, bases + 12 * i, 96);
        m++;
    }
    if (m == 0) memset(out, 0, 96);
    else or_msm_best(out, s, b, m, threads);
    free(s);
    free(b);
}

void or_fr_inner_product(uint64_t out[4], const uint64_t *s, const uint64_t *r, size_t n, int threads) {
    if (threads < 1) threads = 1;
    u64 *part = (u64 *)calloc((size_t)threads, 32);
#pragma omp parallel num_threads(threads)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        u64 acc[4] = {0}, t[4];
#pragma omp for schedule(static)
        for (size_t i = 0; i < n; i++) {
            fr_mul(t, s + 4 * i, r + 4 * i);
            fr_add(acc, acc, t);
        }
        memcpy(part + 4 * tid, acc, 32);
    }
    u64 acc[4] = {0};
    for (int i = 0; i < threads; i++) fr_add(acc, acc, part + 4 * i);
    memcpy(out, acc, 32);
    free(part);
}

/* ------------------------------------------------------------------------- */
/* Seeded synthetic inputs                                                   */
/* ------------------------------------------------------------------------- */
/* SplitMix64 finaliser over a counter stream: word `ctr` of stream `seed`. */
uint64_t or_rand64(uint64_t seed, uint64_t ctr) {
    u64 z = seed + (ctr + 1) * 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
/* Rejection sampling as Fq::random (fq.rs:382-396): 4 words, top bit masked,
 * accept if < r; element i, attempt a uses counters ((i*64 + a)*4 + w). */
static void rand_fr_one(u64 *out, u64 seed, u64 i) {
    for (u64 a = 0; a < 64; a++) {
        u64 raw[4];
        for (int w = 0; w < 4; w++) raw[w] = or_rand64(seed, (i * 64 + a) * 4 + (u64)w);
        raw[3] &= 0x7fffffffffffffffULL;
        if (!geq_n(raw, FR_MOD, 4)) {
            fr_mul(out, raw, FR_R2);
            return;
        }
    }
    memset(out, 0, 32); /* unreachable in practice: 64 rejections in a row */
}
void or_rand_fr(uint64_t *out, uint64_t seed, uint64_t first, size_t n, int threads) {
    if (threads < 1) threads = 1;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (size_t i = 0; i < n; i++) rand_fr_one(out + 4 * i, seed, first + i);
}

/* [r_i]G by an 8-bit fixed-base table over G, then batch normalisation. */
void or_gen_bases(uint64_t *out, uint64_t seed, uint64_t first, size_t n, int threads) {
    if (threads < 1) threads = 1;
    aff_t g;
    or_g1_generator((u64 *)&g);
    /* table[j][v] = v * 2^(8j) * G, v in 1..255, as affine */
    aff_t *table = (aff_t *)malloc(32 * 256 * sizeof(aff_t));
    jac_t base;
    jac_from_aff(&base, &g);
    for (int j = 0; j < 32; j++) {
        jac_t acc;
        jac_set_inf(&acc);
        memset(&table[j * 256], 0, sizeof(aff_t));
        jac_t row[256];
        for (int v = 1; v < 256; v++) {
            jac_add(&acc, &acc, &base);
            row[v] = acc;
        }
#pragma omp parallel for num_threads(threads)
        for (int v = 1; v < 256; v++) jac_to_aff(&table[j * 256 + v], &row[v]);
        for (int i = 0; i < 8; i++) jac_double(&base, &base);
    }
    jac_t *tmp = (jac_t *)malloc((n ? n : 1) * sizeof(jac_t));
#pragma omp parallel for num_threads(threads) schedule(static)
    for (size_t i = 0; i < n; i++) {
        u64 r[4], k[4];
        rand_fr_one(r, seed, first + i);
        or_fr_to_canonical(k, r);
        jac_t acc;
        jac_set_inf(&acc);
        for (int j = 0; j < 32; j++) {
            int v = (int)((k[j / 8] >> (8 * (j % 8))) & 0xff);
            if (v) jac_add_aff(&acc, &acc, &table[j * 256 + v]);
        }
        tmp[i] = acc;
    }
    /* per-chunk Montgomery batch inversion of z */
#pragma omp parallel num_threads(threads)
    {
        int nt = 1, tid = 0;
#ifdef _OPENMP
        nt = omp_get_num_threads();
        tid = omp_get_thread_num();
#endif
        size_t lo = n * (size_t)tid / (size_t)nt, hi = n * (size_t)(tid + 1) / (size_t)nt;
        if (hi > lo) {
            u64 (*pref)[6] = (u64 (*)[6])malloc((hi - lo) * 48);
            u64 acc[6];
            memcpy(acc, FP_R, 48);
            for (size_t i = lo; i < hi; i++) {
                memcpy(pref[i - lo], acc, 48);
                if (!jac_is_inf(&tmp[i])) fp_mul(acc, acc, tmp[i].z);
            }
            fp_inv(acc, acc);
            for (size_t i = hi; i-- > lo;) {
                aff_t *o = (aff_t *)(out + 12 * i);
                if (jac_is_inf(&tmp[i])) { memset(o, 0, sizeof(*o)); continue; }
                u64 zi[6], zi2[6], zi3[6];
                fp_mul(zi, acc, pref[i - lo]);
                fp_mul(acc, acc, tmp[i].z);
                fp_mul(zi2, zi, zi);
                fp_mul(zi3, zi2, zi);
                fp_mul(o->x, tmp[i].x, zi2);
                fp_mul(o->y, tmp[i].y, zi3);
            }
            free(pref);
        }
    }
    free(tmp);
    free(table);
}

/* ------------------------------------------------------------------------- */
/* FFT, curves/src/fft.rs                                                    */
/* ------------------------------------------------------------------------- */
static inline size_t bitreverse(size_t n, uint32_t log_n) {
    size_t r = 0;
    for (uint32_t i = 0; i < log_n; i++) { r = (r << 1) | (n & 1); n >>= 1; }
    return r;
}
/* compute_twiddles, fft.rs:31-40 */
void or_compute_twiddles(uint64_t *out, const uint64_t omega[4], uint32_t log_n) {
    size_t half = (size_t)1 << (log_n - 1);
    u64 w[4];
    memcpy(w, FR_R, 32);
    for (size_t i = 0; i < half; i++) {
        memcpy(out + 4 * i, w, 32);
        fr_mul(w, w, omega);
    }
}
static void swap_fr(u64 *a, size_t i, size_t j) {
    u64 t[4];
    memcpy(t, a + 4 * i, 32);
    memcpy(a + 4 * i, a + 4 * j, 32);
    memcpy(a + 4 * j, t, 32);
}
/* recursive_butterfly_arithmetic, fft.rs:202-236 (rayon::join -> OpenMP tasks) */
static void rec_butterfly(u64 *a, size_t n, size_t twiddle_chunk, const u64 *tw, int depth) {
    if (n == 2) {
        u64 t[4];
        memcpy(t, a + 4, 32);
        memcpy(a + 4, a, 32);
        fr_add(a, a, t);
        fr_sub(a + 4, a + 4, t);
        return;
    }
    size_t h = n / 2;
    if (depth > 0) {
#pragma omp task
        rec_butterfly(a, h, twiddle_chunk * 2, tw, depth - 1);
#pragma omp task
        rec_butterfly(a + 4 * h, h, twiddle_chunk * 2, tw, depth - 1);
#pragma omp taskwait
    } else {
        rec_butterfly(a, h, twiddle_chunk * 2, tw, 0);
        rec_butterfly(a + 4 * h, h, twiddle_chunk * 2, tw, 0);
    }
    u64 *left = a, *right = a + 4 * h;
    {
        u64 t[4];
        memcpy(t, right, 32);
        memcpy(right, left, 32);
        fr_add(left, left, t);
        fr_sub(right, right, t);
    }
    for (size_t i = 1; i < h; i++) {
        u64 t[4];
        fr_mul(t, right + 4 * i, tw + 4 * (i * twiddle_chunk));
        memcpy(right + 4 * i, left + 4 * i, 32);
        fr_add(left + 4 * i, left + 4 * i, t);
        fr_sub(right + 4 * i, right + 4 * i, t);
    }
}
static int depth_for_threads(int threads) {
    int d = 0;
    while ((1 << d) < 4 * threads) d++;
    return d;
}
/* best_fft_with_twiddles, fft.rs:56-101 */
void or_best_fft(uint64_t *a, const uint64_t *tw, uint32_t log_n, int threads) {
    size_t n = (size_t)1 << log_n;
    if (threads < 1) threads = 1;
    for (size_t k = 0; k < n; k++) {
        size_t rk = bitreverse(k, log_n);
        if (k < rk) swap_fr(a, rk, k);
    }
    if (log_n == 0) return;
    int log_threads = 0;
    while ((2 << log_threads) <= threads) log_threads++;
    if ((int)log_n <= log_threads) {
        size_t chunk = 2, twiddle_chunk = n / 2;
        for (uint32_t s = 0; s < log_n; s++) {
            for (size_t c0 = 0; c0 < n; c0 += chunk) {
                u64 *left = a + 4 * c0, *right = a + 4 * (c0 + chunk / 2);
                u64 t[4];
                memcpy(t, right, 32);
                memcpy(right, left, 32);
                fr_add(left, left, t);
                fr_sub(right, right, t);
                for (size_t i = 0; i + 1 < chunk / 2; i++) {
                    fr_mul(t, right + 4 * (i + 1), tw + 4 * ((i + 1) * twiddle_chunk));
                    memcpy(right + 4 * (i + 1), left + 4 * (i + 1), 32);
                    fr_add(left + 4 * (i + 1), left + 4 * (i + 1), t);
                    fr_sub(right + 4 * (i + 1), right + 4 * (i + 1), t);
                }
            }
            chunk *= 2;
            twiddle_chunk /= 2;
        }
    } else {
        int depth = depth_for_threads(threads);
#pragma omp parallel num_threads(threads)
#pragma omp single
        rec_butterfly(a, n, 1, tw, threads > 1 ? depth : 0);
    }
}

/* Gentleman-Sande butterfly, fq.rs:336-343: d = x0 - x1; x0 += x1; x1 = d*tw */
static inline void gs_bfly(u64 *x0, u64 *x1, const u64 *tw) {
    u64 d[4];
    fr_sub(d, x0, x1);
    fr_add(x0, x0, x1);
    fr_mul(x1, d, tw);
}
/* recursive_dif_pruned, fft.rs:148-186 */
static void rec_dif_pruned(u64 *a, size_t n, size_t tc, const u64 *tw, size_t nz, int depth) {
    if (nz == 0) return;
    if (n == 2) {
        gs_bfly(a, a + 4, tw);
        return;
    }
    size_t h = n / 2;
    if (nz <= h) {
        for (size_t i = 0; i < nz; i++) fr_mul(a + 4 * (i + h), a + 4 * i, tw + 4 * (i * tc));
    } else {
        for (size_t i = 0; i < h; i++) gs_bfly(a + 4 * i, a + 4 * (i + h), tw + 4 * (i * tc));
    }
    size_t child = nz < h ? nz : h;
    if (depth > 0) {
#pragma omp task
        rec_dif_pruned(a, h, tc * 2, tw, child, depth - 1);
#pragma omp task
        rec_dif_pruned(a + 4 * h, h, tc * 2, tw, child, depth - 1);
#pragma omp taskwait
    } else {
        rec_dif_pruned(a, h, tc * 2, tw, child, 0);
        rec_dif_pruned(a + 4 * h, h, tc * 2, tw, child, 0);
    }
}
/* fft_dif_pruned_fq, fft.rs:133-143 */
void or_fft_dif_pruned(uint64_t *a, const uint64_t *tw, uint32_t log_n, size_t n_real, int threads) {
    size_t n = (size_t)1 << log_n;
    if (threads < 1) threads = 1;
    int depth = depth_for_threads(threads);
#pragma omp parallel num_threads(threads)
#pragma omp single
    rec_dif_pruned(a, n, 1, tw, n_real, threads > 1 ? depth : 0);
    for (size_t k = 0; k < n; k++) {
        size_t rk = bitreverse(k, log_n);
        if (k < rk) swap_fr(a, rk, k);
    }
}

/* DFT by definition: out_j = sum_i a_i omega^{ij} (independent check) */
void or_dft_naive(uint64_t *out, const uint64_t *a, const uint64_t omega[4], size_t n) {
    u64 wj[4];
    memcpy(wj, FR_R, 32);
    for (size_t j = 0; j < n; j++) {
        u64 acc[4] = {0}, p[4], t[4];
        memcpy(p, FR_R, 32);
        for (size_t i = 0; i < n; i++) {
            fr_mul(t, a + 4 * i, p);
            fr_add(acc, acc, t);
            fr_mul(p, p, wj);
        }
        memcpy(out + 4 * j, acc, 32);
        fr_mul(wj, wj, omega);
    }
}

/* ------------------------------------------------------------------------- */
/* EvaluationDomain, proofs/src/poly/domain.rs:54-414                        */
/* ------------------------------------------------------------------------- */
struct or_domain {
    uint32_t k, extended_k;
    u64 omega[4], omega_inv[4], extended_omega[4], extended_omega_inv[4];
    u64 g_coset[4], g_coset_inv[4];
    u64 ifft_divisor[4], extended_ifft_divisor[4], barycentric_weight[4];
    u64 *t_evaluations;
    size_t t_len;
    u64 *tw_omega, *tw_omega_inv, *tw_ext, *tw_ext_inv;
};

static void fr_from_u64(u64 *o, u64 v) {
    u64 t[4] = {v, 0, 0, 0};
    fr_mul(o, t, FR_R2);
}
static int fr_eq(const u64 *a, const u64 *b) { return memcmp(a, b, 32) == 0; }

/* EvaluationDomain::new, domain.rs:54-167 */
or_domain *or_domain_new(uint32_t j, uint32_t k) {
    or_domain *d = (or_domain *)calloc(1, sizeof(or_domain));
    u64 quotient_poly_degree = (u64)(j - 1);
    u64 n = (u64)1 << k;
    uint32_t extended_k = k;
    while (((u64)1 << extended_k) < n * quotient_poly_degree) extended_k++;
    d->k = k;
    d->extended_k = extended_k;
    u64 ext[4];
    memcpy(ext, FR_ROOT_OF_UNITY, 32);
    for (uint32_t i = extended_k; i < 32; i++) fr_mul(ext, ext, ext);
    memcpy(d->extended_omega, ext, 32);
    u64 om[4];
    memcpy(om, ext, 32);
    for (uint32_t i = k; i < extended_k; i++) fr_mul(om, om, om);
    memcpy(d->omega, om, 32);
    memcpy(d->g_coset, FR_ZETA, 32);
    fr_mul(d->g_coset_inv, FR_ZETA, FR_ZETA);
    /* t evaluations: t(zeta * ext_omega^i) = zeta^n ext_omega^{in} - 1, inverted */
    u64 nn[4] = {n, 0, 0, 0};
    u64 orig[4], step[4], cur[4];
    fr_pow(orig, d->g_coset, nn, 1);
    fr_pow(step, d->extended_omega, nn, 1);
    d->t_len = (size_t)1 << (extended_k - k);
    d->t_evaluations = (u64 *)malloc(d->t_len * 32);
    memcpy(cur, orig, 32);
    for (size_t i = 0; i < d->t_len; i++) {
        fr_sub(d->t_evaluations + 4 * i, cur, FR_R);
        fr_inv(d->t_evaluations + 4 * i, d->t_evaluations + 4 * i);
        fr_mul(cur, cur, step);
    }
    fr_from_u64(d->ifft_divisor, n);
    fr_inv(d->ifft_divisor, d->ifft_divisor);
    fr_from_u64(d->extended_ifft_divisor, (u64)1 << extended_k);
    fr_inv(d->extended_ifft_divisor, d->extended_ifft_divisor);
    fr_from_u64(d->barycentric_weight, n);
    fr_inv(d->barycentric_weight, d->barycentric_weight);
    fr_inv(d->extended_omega_inv, d->extended_omega);
    fr_inv(d->omega_inv, d->omega);
    size_t half = (size_t)1 << (k - 1), ehalf = (size_t)1 << (extended_k - 1);
    d->tw_omega = (u64 *)malloc(half * 32);
    d->tw_omega_inv = (u64 *)malloc(half * 32);
    d->tw_ext = (u64 *)malloc(ehalf * 32);
    d->tw_ext_inv = (u64 *)malloc(ehalf * 32);
    or_compute_twiddles(d->tw_omega, d->omega, k);
    or_compute_twiddles(d->tw_omega_inv, d->omega_inv, k);
    or_compute_twiddles(d->tw_ext, d->extended_omega, extended_k);
    or_compute_twiddles(d->tw_ext_inv, d->extended_omega_inv, extended_k);
    (void)fr_eq;
    return d;
}
void or_domain_free(or_domain *d) {
    if (!d) return;
    free(d->t_evaluations);
    free(d->tw_omega);
    free(d->tw_omega_inv);
    free(d->tw_ext);
    free(d->tw_ext_inv);
    free(d);
}
uint32_t or_domain_k(const or_domain *d) { return d->k; }
uint32_t or_domain_extended_k(const or_domain *d) { return d->extended_k; }
void or_domain_get(const or_domain *d, int which, int idx, uint64_t out[4]) {
    const u64 *src = d->omega;
    switch (which) {
        case 0: src = d->omega; break;
        case 1: src = d->omega_inv; break;
        case 2: src = d->extended_omega; break;
        case 3: src = d->g_coset; break;
        case 4: src = d->g_coset_inv; break;
        case 5: src = d->ifft_divisor; break;
        case 6: src = d->extended_ifft_divisor; break;
        case 7: src = d->t_evaluations + 4 * (size_t)idx; break;
        case 8: src = d->extended_omega_inv; break;
        case 9: src = d->barycentric_weight; break;
    }
    memcpy(out, src, 32);
}
static void scale_all(u64 *a, size_t n, const u64 *s, int threads) {
#pragma omp parallel for num_threads(threads) schedule(static)
    for (size_t i = 0; i < n; i++) fr_mul(a + 4 * i, a + 4 * i, s);
}
/* distribute_powers_zeta, domain.rs:398-414 */
static void distribute_powers_zeta(const or_domain *d, u64 *a, size_t n, int into, int threads) {
    const u64 *c1 = into ? d->g_coset : d->g_coset_inv;
    const u64 *c2 = into ? d->g_coset_inv : d->g_coset;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (size_t i = 0; i < n; i++) {
        size_t r = i % 3;
        if (r == 1) fr_mul(a + 4 * i, a + 4 * i, c1);
        else if (r == 2) fr_mul(a + 4 * i, a + 4 * i, c2);
    }
}
/* lagrange_to_coeff + ifft, domain.rs:249-264, :389-396 */
void or_domain_lagrange_to_coeff(const or_domain *d, uint64_t *a, int threads) {
    if (threads < 1) threads = 1;
    or_best_fft(a, d->tw_omega_inv, d->k, threads);
    scale_all(a, (size_t)1 << d->k, d->ifft_divisor, threads);
}
/* coeff_to_lagrange, domain.rs:268-277 */
void or_domain_coeff_to_lagrange(const or_domain *d, uint64_t *a, int threads) {
    if (threads < 1) threads = 1;
    or_best_fft(a, d->tw_omega, d->k, threads);
}
/* coeff_to_extended, domain.rs:285-305 */
void or_domain_coeff_to_extended(const or_domain *d, const uint64_t *in, uint64_t *out, int threads) {
    if (threads < 1) threads = 1;
    size_t n = (size_t)1 << d->k, en = (size_t)1 << d->extended_k;
    memcpy(out, in, n * 32);
    distribute_powers_zeta(d, out, n, 1, threads);
    memset(out + 4 * n, 0, (en - n) * 32);
    or_fft_dif_pruned(out, d->tw_ext, d->extended_k, n, threads);
}
/* extended_to_coeff, domain.rs:312-328 */
void or_domain_extended_to_coeff(const or_domain *d, uint64_t *a, int threads) {
    if (threads < 1) threads = 1;
    size_t en = (size_t)1 << d->extended_k;
    or_best_fft(a, d->tw_ext_inv, d->extended_k, threads);
    scale_all(a, en, d->extended_ifft_divisor, threads);
    distribute_powers_zeta(d, a, en, 0, threads);
}
/* extended_to_lagrange, domain.rs:335-357 */
void or_domain_extended_to_lagrange(const or_domain *d, uint64_t *a, uint64_t *out, int threads) {
    if (threads < 1) threads = 1;
    size_t n = (size_t)1 << d->k, en = (size_t)1 << d->extended_k;
    or_best_fft(a, d->tw_ext_inv, d->extended_k, threads);
    scale_all(a, en, d->extended_ifft_divisor, threads);
    memcpy(out, a, n * 32);
    distribute_powers_zeta(d, out, n, 0, threads);
    or_best_fft(out, d->tw_omega, d->k, threads);
}
/* divide_by_vanishing_poly, domain.rs:361-380 */
void or_domain_divide_by_vanishing_poly(const or_domain *d, uint64_t *a, int threads) {
    if (threads < 1) threads = 1;
    size_t en = (size_t)1 << d->extended_k;
    size_t mask = d->t_len - 1;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (size_t i = 0; i < en; i++) fr_mul(a + 4 * i, a + 4 * i, d->t_evaluations + 4 * (i & mask));
}

/* ------------------------------------------------------------------------- */
/* eval_polynomial, proofs/src/utils/arithmetic.rs:59-87: chunked Horner,     */
/* chunk results scaled by point^start and summed.                           */
/* ------------------------------------------------------------------------- */
void or_eval_polynomial(uint64_t out[4], const uint64_t *poly, size_t n, const uint64_t point[4], int threads) {
    if (threads < 1) threads = 1;
    size_t chunk = (n + (size_t)threads - 1) / (size_t)threads;
    if (chunk == 0) chunk = 1;
    size_t nchunks = (n + chunk - 1) / chunk;
    u64 *parts = (u64 *)calloc(nchunks ? nchunks : 1, 32);
#pragma omp parallel for num_threads(threads) schedule(static, 1)
    for (size_t c = 0; c < nchunks; c++) {
        size_t lo = c * chunk, hi = lo + chunk > n ? n : lo + chunk;
        u64 acc[4] = {0}, t[4];
        for (size_t i = hi; i-- > lo;) {
            fr_mul(t, acc, point);
            fr_add(acc, t, poly + 4 * i);
        }
        u64 e[1] = {(u64)lo};
        fr_pow(t, point, e, 1);
        fr_mul(parts + 4 * c, acc, t);
    }
    u64 acc[4] = {0};
    for (size_t c = 0; c < nchunks; c++) fr_add(acc, acc, parts + 4 * c);
    memcpy(out, acc, 32);
    free(parts);
}

/* ------------------------------------------------------------------------- */
/* Grand products and running sums of the permutation and logup arguments    */
/* ------------------------------------------------------------------------- */

static int fr_is_zero(const u64 *a) { return (a[0] | a[1] | a[2] | a[3]) == 0; }

/* ff 0.13 BatchInvert (crate `ff`, a dependency of the reference that is not
 * vendored; used at permutation/prover.rs:139 and logup/prover.rs:221,232):
 * Montgomery's simultaneous inversion, forward products skipping zeros, one
 * inversion, backward pass; zero elements are left unchanged. */
void or_fr_batch_invert(uint64_t *a, size_t n) {
    u64 *pre = (u64 *)malloc((n ? n : 1) * 32);
    u64 acc[4];
    memcpy(acc, FR_R, 32);
    for (size_t i = 0; i < n; i++) {
        memcpy(pre + 4 * i, acc, 32);
        if (!fr_is_zero(a + 4 * i)) fr_mul(acc, acc, a + 4 * i);
    }
    fr_inv(acc, acc);
    for (size_t i = n; i-- > 0;) {
        if (fr_is_zero(a + 4 * i)) continue;
        u64 t[4], inv[4];
        fr_mul(inv, pre + 4 * i, acc); /* 1 / a_i */
        fr_mul(t, acc, a + 4 * i);     /* drop a_i from the running inverse */
        memcpy(acc, t, 32);
        memcpy(a + 4 * i, inv, 32);
    }
    free(pre);
}

/* permutation/prover.rs:81-255 (Stages 1, 2 A-C): per set of chunk_len
 * columns, modified_values[i] = prod_j (p_j(w^i) + delta^(s chunk_len + j) w^i
 * beta + gamma) / prod_j (p_j(w^i) + beta s_j(w^i) + gamma); z[0] = 1,
 * z[r] = z[r-1] modified[r-1]; the last blinding_factors rows are the blinds;
 * set s is then multiplied (every row, blinds included) by the product of the
 * earlier sets' z[n - blinding_factors - 1]. */
void or_permutation_z(const uint64_t *const *values, const uint64_t *const *sigmas, uint32_t n_cols,
                      uint32_t chunk_len, uint32_t k, const uint64_t omega[4], const uint64_t beta[4],
                      const uint64_t gamma[4], uint32_t blinding_factors, const uint64_t *blinds,
                      uint64_t *const *z_out) {
    const size_t n = (size_t)1 << k;
    const uint32_t n_sets = (n_cols + chunk_len - 1) / chunk_len;
    u64 *mv = (u64 *)malloc(n * 32);
    u64 correction[4];
    memcpy(correction, FR_R, 32);
    for (uint32_t s = 0; s < n_sets; s++) {
        const uint32_t c0 = s * chunk_len, c1 = c0 + chunk_len < n_cols ? c0 + chunk_len : n_cols;
        for (size_t i = 0; i < n; i++) memcpy(mv + 4 * i, FR_R, 32);
        for (uint32_t c = c0; c < c1; c++)
            for (size_t i = 0; i < n; i++) {
                u64 t[4];
                fr_mul(t, beta, sigmas[c] + 4 * i);
                fr_add(t, t, gamma);
                fr_add(t, t, values[c] + 4 * i);
                fr_mul(mv + 4 * i, mv + 4 * i, t);
            }
        or_fr_batch_invert(mv, n);
        u64 deltaomega[4], e[1] = {(u64)c0};
        fr_pow(deltaomega, FR_DELTA, e, 1);
        for (uint32_t c = c0; c < c1; c++) {
            u64 dw[4];
            memcpy(dw, deltaomega, 32);
            for (size_t i = 0; i < n; i++) {
                u64 t[4];
                fr_mul(t, dw, beta);
                fr_add(t, t, gamma);
                fr_add(t, t, values[c] + 4 * i);
                fr_mul(mv + 4 * i, mv + 4 * i, t);
                fr_mul(dw, dw, omega);
            }
            fr_mul(deltaomega, deltaomega, FR_DELTA);
        }
        u64 *z = z_out[s];
        memcpy(z, FR_R, 32);
        for (size_t r = 1; r < n; r++) fr_mul(z + 4 * r, z + 4 * (r - 1), mv + 4 * (r - 1));
        for (uint32_t b = 0; b < blinding_factors; b++) memcpy(z + 4 * (n - blinding_factors + b), blinds + 4 * ((size_t)s * blinding_factors + b), 32);
        u64 last[4];
        memcpy(last, z + 4 * (n - blinding_factors - 1), 32);
        for (size_t i = 0; i < n; i++) fr_mul(z + 4 * i, z + 4 * i, correction);
        fr_mul(correction, correction, last); /* the next set's correction */
    }
    free(mv);
}

/* logup/prover.rs:195-300: T = 1/(t + beta) and per chunk of compressed input
 * columns h = sum_j 1/(f_j + beta) (each column batch-inverted on its own);
 * logderivative[i] = selector[i] (sum over chunks of h[i]) - m[i] T[i];
 * aggregator = [0, running sums of logderivative] taken to n - blinding_factors
 * rows, then the blinding values. */
void or_logup(const uint64_t *const *inputs, const uint32_t *chunk_cols, uint32_t n_chunks, const uint64_t *table,
              const uint64_t *selector, const uint64_t *multiplicities, size_t n, const uint64_t beta[4],
              uint32_t blinding_factors, const uint64_t *blinds, uint64_t *const *helpers_out,
              uint64_t *aggregator_out) {
    u64 *tden = (u64 *)malloc(n * 32), *col = (u64 *)malloc(n * 32);
    for (size_t i = 0; i < n; i++) fr_add(tden + 4 * i, beta, table + 4 * i);
    or_fr_batch_invert(tden, n);
    uint32_t ci = 0;
    for (uint32_t c = 0; c < n_chunks; c++) {
        u64 *h = helpers_out[c];
        memset(h, 0, n * 32);
        for (uint32_t j = 0; j < chunk_cols[c]; j++, ci++) {
            for (size_t i = 0; i < n; i++) fr_add(col + 4 * i, beta, inputs[ci] + 4 * i);
            or_fr_batch_invert(col, n);
            for (size_t i = 0; i < n; i++) fr_add(h + 4 * i, h + 4 * i, col + 4 * i);
        }
    }
    u64 state[4] = {0, 0, 0, 0};
    memset(aggregator_out, 0, 32);
    for (size_t i = 0; i + 1 < n - blinding_factors; i++) {
        u64 sum[4] = {0, 0, 0, 0}, t[4], u[4];
        for (uint32_t c = 0; c < n_chunks; c++) fr_add(sum, sum, helpers_out[c] + 4 * i);
        fr_mul(t, selector + 4 * i, sum);
        fr_mul(u, multiplicities + 4 * i, tden + 4 * i);
        fr_sub(t, t, u);
        fr_add(state, state, t);
        memcpy(aggregator_out + 4 * (i + 1), state, 32);
    }
    for (uint32_t b = 0; b < blinding_factors; b++) memcpy(aggregator_out + 4 * (n - blinding_factors + b), blinds + 4 * b, 32);
    free(tden);
    free(col);
}

/* params.rs:47-57 suffix_sum: out[i] = sum_{j >= i} in[j] (affine in and out) */
void or_g1_suffix_sum(const uint64_t *in, size_t n, uint64_t *out) {
    u64 acc[18] = {0}, p[18], t[18];
    for (size_t i = n; i-- > 0;) {
        or_g1_from_affine(p, in + 12 * i);
        or_g1_add(t, acc, p);
        memcpy(acc, t, sizeof(acc));
        or_g1_to_affine(out + 12 * i, acc);
    }
}

/* params.rs:160-209 unsafe_setup, G1 part, for secret s and n = 2^k with the
 * domain's root omega: g[i] = [s^i]G, lag[i] = [(s^n - 1)/n w^i/(s - w^i)]G,
 * then the two suffix sums. */
void or_srs_setup(const uint64_t s[4], uint32_t k, const uint64_t omega[4], uint64_t *g, uint64_t *lag,
                  uint64_t *delta, uint64_t *ddelta) {
    const size_t n = (size_t)1 << k;
    u64 gen[12], sp[4], w[4], sn[4], e[1] = {(u64)n}, ninv[4], nn[4], mult[4], t[4], u[4];
    or_g1_generator(gen);
    memcpy(sp, FR_R, 32);
    for (size_t i = 0; i < n; i++) {
        or_g1_mul(g + 12 * i, gen, sp);
        fr_mul(sp, sp, s);
    }
    fr_pow(sn, s, e, 1);
    fr_sub(sn, sn, FR_R);
    u64 nc[4] = {(u64)n, 0, 0, 0};
    fr_mul(nn, nc, FR_R2);
    fr_inv(ninv, nn);
    fr_mul(mult, sn, ninv);
    memcpy(w, FR_R, 32);
    for (size_t i = 0; i < n; i++) {
        fr_sub(t, s, w);
        fr_inv(t, t);
        fr_mul(u, mult, w);
        fr_mul(u, u, t);
        or_g1_mul(lag + 12 * i, gen, u);
        fr_mul(w, w, omega);
    }
    or_g1_suffix_sum(lag, n, delta);
    or_g1_suffix_sum(delta, n, ddelta);
}

/* kzg/mod.rs:125-147 poly_inner_product: out[i] = sum_p scalars[p] polys[p][i],
 * shorter polynomials zero-extended to the longest (out_len). */
void or_poly_inner_product(const uint64_t *const *polys, const size_t *lens, size_t m, const uint64_t *scalars,
                           uint64_t *out, size_t out_len) {
    memset(out, 0, out_len * 32);
    for (size_t p = 0; p < m; p++)
        for (size_t i = 0; i < lens[p] && i < out_len; i++) {
            u64 t[4];
            fr_mul(t, polys[p] + 4 * i, scalars + 4 * p);
            fr_add(out + 4 * i, out + 4 * i, t);
        }
}

/* Fr multiplication counter: on != 0 resets and starts it, on == 0 stops it;
 * returns the count so far */
unsigned long long or_fr_mul_counter(int on) {
    if (on) g_fr_mul_count = 0;
    g_fr_count_on = on;
    return g_fr_mul_count;
}

/* element-wise product out[i] = a[i] * b[i] (test-input construction) */
void or_fr_mul_vec(const uint64_t *a, const uint64_t *b, uint64_t *out, size_t n) {
    for (size_t i = 0; i < n; i++) fr_mul(out + 4 * i, a + 4 * i, b + 4 * i);
}

/* utils/arithmetic.rs:106-125: quotient of a(X) by (X - b), n - 1 coefficients:
 * from the top, q = a_{i+1} - tmp, tmp = q * (-b). */
void or_kate_division(const uint64_t *a, size_t n, const uint64_t b[4], uint64_t *q) {
    u64 nb[4], tmp[4] = {0, 0, 0, 0}, zero[4] = {0, 0, 0, 0};
    fr_sub(nb, zero, b);
    for (size_t i = n - 1; i-- > 0;) {
        u64 lead[4];
        fr_sub(lead, a + 4 * (i + 1), tmp);
        memcpy(q + 4 * i, lead, 32);
        fr_mul(tmp, lead, nb);
    }
}

/* ------------------------------------------------------------------------- */
/* Quotient numerator, proofs/src/plonk/evaluation.rs:818-1114               */
/* ------------------------------------------------------------------------- */
/* get_rotation_idx, evaluation.rs:13-16 */
static size_t rot_idx(size_t idx, int rot, uint32_t log_scale, uint32_t log_n) {
    size_t mask = ((size_t)1 << log_n) - 1;
    return (idx + (size_t)((intptr_t)rot << log_scale)) & mask;
}

static void quotient_eval(const or_quotient_desc *d, const or_domain *dom, int divide, const uint64_t *gate_values,
                          uint64_t *out, int threads);

void or_quotient_eval(const or_quotient_desc *d, const or_domain *dom, int divide, uint64_t *out, int threads) {
    quotient_eval(d, dom, divide, NULL, out, threads);
}

/* the same with the custom gates' Horner-in-y value of every row given
 * (gate_values: 2^extended_k Fr): circuits whose gates are flattened programs */
void or_quotient_eval_gates(const or_quotient_desc *d, const or_domain *dom, int divide, const uint64_t *gate_values,
                            uint64_t *out, int threads) {
    quotient_eval(d, dom, divide, gate_values, out, threads);
}

static void quotient_eval(const or_quotient_desc *d, const or_domain *dom, int divide, const uint64_t *gate_values,
                          uint64_t *out, int threads) {
    if (threads < 1) threads = 1;
    const uint32_t log_n = d->extended_k, log_scale = d->extended_k - d->k;
    const size_t E = (size_t)1 << log_n;
    const int last_rotation = -(int)(d->blinding_factors + 1);
    u64 delta_start[4];
    fr_mul(delta_start, d->beta, d->g_coset); /* beta * g_coset (evaluation.rs:864) */
#pragma omp parallel for num_threads(threads) schedule(static)
    for (size_t idx = 0; idx < E; idx++) {
        u64 v[4], t[4], u[4], w[4];
        const size_t r_next = rot_idx(idx, 1, log_scale, log_n);
        const size_t r_last = rot_idx(idx, last_rotation, log_scale, log_n);
        /* custom gate: Horner(0, [gate], y) = gate (evaluation.rs:849-852, :680-689) */
        if (gate_values) {
            memcpy(v, gate_values + 4 * idx, 32);
        } else {
            const u64 *ql = d->fixed[d->gate_fixed[0]] + 4 * idx, *qr = d->fixed[d->gate_fixed[1]] + 4 * idx;
            const u64 *qm = d->fixed[d->gate_fixed[2]] + 4 * idx, *qo = d->fixed[d->gate_fixed[3]] + 4 * idx;
            const u64 *qc = d->fixed[d->gate_fixed[4]] + 4 * idx;
            const u64 *a = d->advice[d->gate_advice[0]] + 4 * idx, *b = d->advice[d->gate_advice[1]] + 4 * idx;
            const u64 *c = d->advice[d->gate_advice[2]] + 4 * idx;
            fr_mul(v, ql, a);
            fr_mul(t, qr, b);
            fr_add(v, v, t);
            fr_mul(t, a, b);
            fr_mul(t, t, qm);
            fr_add(v, v, t);
            fr_mul(t, qo, c);
            fr_add(v, v, t);
            fr_add(v, v, qc);
        }
        /* permutation (evaluation.rs:857-943) */
        if (d->n_perm_sets) {
            const u64 *l0 = d->l0 + 4 * idx, *ll = d->l_last + 4 * idx, *la = d->l_active + 4 * idx;
            const u64 *z0 = d->perm_z[0] + 4 * idx, *zl = d->perm_z[d->n_perm_sets - 1] + 4 * idx;
            fr_mul(v, v, d->y);
            fr_sub(t, FR_R, z0);
            fr_mul(t, t, l0);
            fr_add(v, v, t);
            fr_mul(v, v, d->y);
            fr_mul(t, zl, zl);
            fr_sub(t, t, zl);
            fr_mul(t, t, ll);
            fr_add(v, v, t);
            for (uint32_t s = 1; s < d->n_perm_sets; s++) {
                fr_mul(v, v, d->y);
                fr_sub(t, d->perm_z[s] + 4 * idx, d->perm_z[s - 1] + 4 * r_last);
                fr_mul(t, t, l0);
                fr_add(v, v, t);
            }
            /* current_delta = beta * g_coset * omega^idx (omega: extended) */
            u64 cur[4], ew[4];
            u64 e1[1] = {(u64)idx};
            /* the reference steps omega^idx by one multiplication per row
             * (beta_term *= omega, evaluation.rs:941); counted as that */
            const int counting = g_fr_count_on;
            g_fr_count_on = 0;
            fr_pow(ew, d->extended_omega, e1, 1);
            g_fr_count_on = counting;
            if (counting) g_fr_mul_count++;
            fr_mul(cur, delta_start, ew);
            uint32_t col = 0;
            for (uint32_t s = 0; s < d->n_perm_sets; s++) {
                u64 left[4], right[4];
                memcpy(left, d->perm_z[s] + 4 * r_next, 32);
                memcpy(right, d->perm_z[s] + 4 * idx, 32);
                uint32_t end = col + d->chunk_len;
                if (end > d->n_perm_cols) end = d->n_perm_cols;
                for (uint32_t j = col; j < end; j++) {
                    const u64 *val = (d->perm_col_kind[j] == 0 ? d->advice : d->perm_col_kind[j] == 1 ? d->fixed : d->instance)[d->perm_col_index[j]] + 4 * idx;
                    fr_mul(t, d->beta, d->perm_sigma[j] + 4 * idx);
                    fr_add(t, t, val);
                    fr_add(t, t, d->gamma);
                    fr_mul(left, left, t);
                }
                for (uint32_t j = col; j < end; j++) {
                    const u64 *val = (d->perm_col_kind[j] == 0 ? d->advice : d->perm_col_kind[j] == 1 ? d->fixed : d->instance)[d->perm_col_index[j]] + 4 * idx;
                    fr_add(t, val, cur);
                    fr_add(t, t, d->gamma);
                    fr_mul(right, right, t);
                    fr_mul(cur, cur, FR_DELTA);
                }
                col = end;
                fr_mul(v, v, d->y);
                fr_sub(t, left, right);
                fr_mul(t, t, la);
                fr_add(v, v, t);
            }
        }
        /* lookup (evaluation.rs:1034-1090), one input expression and one helper */
        if (d->has_lookup) {
            const u64 *l0 = d->l0 + 4 * idx, *ll = d->l_last + 4 * idx, *la = d->l_active + 4 * idx;
            const u64 *Z = d->lookup_z + 4 * idx, *h = d->lookup_h + 4 * idx, *m = d->lookup_m + 4 * idx;
            fr_mul(v, v, d->y);
            fr_add(t, l0, ll);
            fr_mul(t, t, Z);
            fr_add(v, v, t);
            /* compressed input = Horner(0, [a], theta) = a; product = a + beta;
               sum of partial products = 1 */
            u64 f[4];
            const u64 *a = d->advice[d->lookup_input_advice] + 4 * idx;
            memset(f, 0, 32);
            fr_mul(f, f, d->theta);
            fr_add(f, f, a);
            fr_add(f, f, d->beta);
            fr_mul(v, v, d->y);
            fr_mul(t, h, f);
            fr_add(v, v, t);
            fr_sub(v, v, FR_R);
            /* accumulator: l_active * ((Z(wX) - Z(X) - s*h) * (t + beta) + m) */
            u64 tbl[4], sel[4];
            memset(tbl, 0, 32);
            fr_mul(tbl, tbl, d->theta);
            fr_add(tbl, tbl, d->fixed[d->lookup_table_fixed] + 4 * idx);
            fr_add(tbl, tbl, d->beta);
            if (d->lookup_selector_fixed < 0) memcpy(sel, FR_R, 32);
            else memcpy(sel, d->fixed[d->lookup_selector_fixed] + 4 * idx, 32);
            fr_sub(u, d->lookup_z + 4 * r_next, Z);
            fr_mul(w, sel, h);
            fr_sub(u, u, w);
            fr_mul(u, u, tbl);
            fr_add(u, u, m);
            fr_mul(u, u, la);
            fr_mul(v, v, d->y);
            fr_add(v, v, u);
        }
        if (divide) fr_mul(v, v, dom->t_evaluations + 4 * (idx & (dom->t_len - 1)));
        memcpy(out + 4 * idx, v, 32);
    }
}
