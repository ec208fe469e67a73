// host_ec.hpp — host-side Fp / G1 arithmetic of the runtime.
//
// Used for the last few group operations of an MSM (combining the per-window
// sums with c doublings between windows, one inversion to normalise) where a
// single GPU thread would be latency-bound for a millisecond.  64-bit limbs,
// Montgomery R = 2^384, the same representation as the device code and the
// reference's blst_fp, so device results are reinterpreted without conversion.
#pragma once
#include <cstdint>
#include <cstring>

namespace mzk {
namespace host {

typedef unsigned __int128 u128;

struct Fp6 { uint64_t l[6]; };
struct Xyzz6 { Fp6 x, y, zz, zzz; };

static const uint64_t P6[6] = {0xb9feffffffffaaabULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL,
                               0x64774b84f38512bfULL, 0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL};
static const uint64_t P6_INV = 0x89f3fffcfffcfffdULL;  // -p^{-1} mod 2^64
static const uint64_t ONE6[6] = {0x760900000002fffdULL, 0xebf4000bc40c0002ULL, 0x5f48985753c758baULL,
                                 0x77ce585370525745ULL, 0x5c071a97a256ec6dULL, 0x15f65ec3fa80e493ULL};

inline bool geq6(const uint64_t* a, const uint64_t* b) {
    for (int i = 5; i >= 0; i--)
        if (a[i] != b[i]) return a[i] > b[i];
    return true;
}
inline uint64_t sub6(uint64_t* o, const uint64_t* a, const uint64_t* b) {
    uint64_t br = 0;
    for (int i = 0; i < 6; i++) {
        u128 d = (u128)a[i] - b[i] - br;
        o[i] = (uint64_t)d;
        br = (uint64_t)(d >> 127);
    }
    return br;
}
inline uint64_t add6(uint64_t* o, const uint64_t* a, const uint64_t* b) {
    uint64_t c = 0;
    for (int i = 0; i < 6; i++) {
        u128 s = (u128)a[i] + b[i] + c;
        o[i] = (uint64_t)s;
        c = (uint64_t)(s >> 64);
    }
    return c;
}
// reduce a lazily reduced device value (< 2p) to [0, p)
inline Fp6 canon(const Fp6& a) {
    Fp6 r = a;
    if (geq6(r.l, P6)) sub6(r.l, r.l, P6);
    return r;
}
inline bool is_zero(const Fp6& a) {
    Fp6 c = canon(a);
    uint64_t acc = 0;
    for (int i = 0; i < 6; i++) acc |= c.l[i];
    return acc == 0;
}
inline Fp6 mul(const Fp6& a, const Fp6& b) {
    uint64_t t[8] = {0};
    for (int i = 0; i < 6; i++) {
        uint64_t c = 0;
        for (int j = 0; j < 6; j++) {
            u128 s = (u128)a.l[j] * b.l[i] + t[j] + c;
            t[j] = (uint64_t)s;
            c = (uint64_t)(s >> 64);
        }
        u128 s = (u128)t[6] + c;
        t[6] = (uint64_t)s;
        t[7] = (uint64_t)(s >> 64);
        uint64_t q = t[0] * P6_INV;
        s = (u128)q * P6[0] + t[0];
        c = (uint64_t)(s >> 64);
        for (int j = 1; j < 6; j++) {
            s = (u128)q * P6[j] + t[j] + c;
            t[j - 1] = (uint64_t)s;
            c = (uint64_t)(s >> 64);
        }
        s = (u128)t[6] + c;
        t[5] = (uint64_t)s;
        t[6] = t[7] + (uint64_t)(s >> 64);
    }
    Fp6 r;
    if (t[6] || geq6(t, P6)) sub6(t, t, P6);
    std::memcpy(r.l, t, 48);
    return r;
}
inline Fp6 add(const Fp6& a, const Fp6& b) {
    Fp6 r;
    uint64_t c = add6(r.l, a.l, b.l);
    if (c || geq6(r.l, P6)) sub6(r.l, r.l, P6);
    return r;
}
inline Fp6 sub(const Fp6& a, const Fp6& b) {
    Fp6 r;
    if (sub6(r.l, a.l, b.l)) add6(r.l, r.l, P6);
    return r;
}
inline Fp6 one() {
    Fp6 r;
    std::memcpy(r.l, ONE6, 48);
    return r;
}
inline Fp6 inv(const Fp6& a) {  // a^(p-2)
    uint64_t e[6];
    std::memcpy(e, P6, 48);
    e[0] -= 2;
    Fp6 acc = one();
    for (int i = 6 * 64 - 1; i >= 0; i--) {
        acc = mul(acc, acc);
        if ((e[i / 64] >> (i % 64)) & 1) acc = mul(acc, a);
    }
    return acc;
}

inline bool inf(const Xyzz6& p) { return is_zero(p.zz); }
inline Xyzz6 infinity() {
    Xyzz6 r;
    std::memset(&r, 0, sizeof(r));
    return r;
}
inline Xyzz6 canon(const Xyzz6& p) {
    Xyzz6 r{canon(p.x), canon(p.y), canon(p.zz), canon(p.zzz)};
    return r;
}
// dbl-2008-s-1 and add-2008-s (Explicit-Formulas Database, a = 0)
inline Xyzz6 dbl(const Xyzz6& p) {
    if (inf(p)) return infinity();
    Fp6 u = add(p.y, p.y), v = mul(u, u), w = mul(u, v), s = mul(p.x, v);
    Fp6 xx = mul(p.x, p.x), m = add(add(xx, xx), xx);
    Xyzz6 r;
    r.x = sub(mul(m, m), add(s, s));
    r.y = sub(mul(m, sub(s, r.x)), mul(w, p.y));
    r.zz = mul(v, p.zz);
    r.zzz = mul(w, p.zzz);
    return r;
}
inline Xyzz6 add(const Xyzz6& a, const Xyzz6& b) {
    if (inf(a)) return b;
    if (inf(b)) return a;
    Fp6 u1 = mul(a.x, b.zz), u2 = mul(b.x, a.zz), s1 = mul(a.y, b.zzz), s2 = mul(b.y, a.zzz);
    Fp6 p = sub(u2, u1), r = sub(s2, s1);
    if (is_zero(p)) {
        if (is_zero(r)) return dbl(a);
        return infinity();
    }
    Fp6 pp = mul(p, p), ppp = mul(p, pp), q = mul(u1, pp);
    Xyzz6 o;
    o.x = sub(sub(mul(r, r), ppp), add(q, q));
    o.y = sub(mul(r, sub(q, o.x)), mul(s1, ppp));
    o.zz = mul(mul(a.zz, b.zz), pp);
    o.zzz = mul(mul(a.zzz, b.zzz), ppp);
    return o;
}
// XYZZ -> blst_p1-style Jacobian with Z = 1 (identity: all zero), 18 limbs
inline void to_jacobian_normalised(const Xyzz6& p, uint64_t out[18]) {
    std::memset(out, 0, 18 * 8);
    if (inf(p)) return;
    Fp6 t = inv(p.zzz);
    Fp6 zi = mul(p.zz, t);
    Fp6 x = mul(p.x, mul(zi, zi)), y = mul(p.y, t);
    std::memcpy(out, x.l, 48);
    std::memcpy(out + 6, y.l, 48);
    std::memcpy(out + 12, ONE6, 48);
}

}  // namespace host
}  // namespace mzk

namespace mzk {
namespace host {

// ---- Fr (scalar field r, 4 x u64 Montgomery, R = 2^256) for domain set-up ----
struct Fr4 { uint64_t l[4]; };

static const uint64_t R4[4] = {0xffffffff00000001ULL, 0x53bda402fffe5bfeULL, 0x3339d80809a1d805ULL,
                               0x73eda753299d7d48ULL};
static const uint64_t R4_INV = 0xfffffffeffffffffULL;  // -r^{-1} mod 2^64
static const uint64_t FR_ONE4[4] = {0x00000001fffffffeULL, 0x5884b7fa00034802ULL, 0x998c4fefecbc4ff5ULL,
                                    0x1824b159acc5056fULL};
static const uint64_t FR_R2_4[4] = {0xc999e990f3f29c6dULL, 0x2b6cedcb87925c23ULL, 0x05d314967254398fULL,
                                    0x0748d9d99f59ff11ULL};

// DELTA = GENERATOR^(2^S) in Montgomery form (curves/src/bls12_381/fq.rs:501-508)
static const uint64_t FR_DELTA4[4] = {0x70e310d3d146f96aULL, 0x4b64c08919e299e6ULL, 0x51e114186a8b970dULL,
                                      0x6185d06627c067cbULL};

inline bool fr_geq(const uint64_t* a, const uint64_t* b) {
    for (int i = 3; i >= 0; i--)
        if (a[i] != b[i]) return a[i] > b[i];
    return true;
}
inline Fr4 fr_mul(const Fr4& a, const Fr4& b) {
    uint64_t t[6] = {0};
    for (int i = 0; i < 4; i++) {
        uint64_t c = 0;
        for (int j = 0; j < 4; j++) {
            u128 s = (u128)a.l[j] * b.l[i] + t[j] + c;
            t[j] = (uint64_t)s;
            c = (uint64_t)(s >> 64);
        }
        u128 s = (u128)t[4] + c;
        t[4] = (uint64_t)s;
        t[5] = (uint64_t)(s >> 64);
        uint64_t q = t[0] * R4_INV;
        s = (u128)q * R4[0] + t[0];
        c = (uint64_t)(s >> 64);
        for (int j = 1; j < 4; j++) {
            s = (u128)q * R4[j] + t[j] + c;
            t[j - 1] = (uint64_t)s;
            c = (uint64_t)(s >> 64);
        }
        s = (u128)t[4] + c;
        t[3] = (uint64_t)s;
        t[4] = t[5] + (uint64_t)(s >> 64);
    }
    Fr4 r;
    if (t[4] || fr_geq(t, R4)) {
        uint64_t br = 0;
        for (int i = 0; i < 4; i++) {
            u128 d = (u128)t[i] - R4[i] - br;
            t[i] = (uint64_t)d;
            br = (uint64_t)(d >> 127);
        }
    }
    std::memcpy(r.l, t, 32);
    return r;
}
inline Fr4 fr_sub(const Fr4& a, const Fr4& b) {
    Fr4 r;
    uint64_t br = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a.l[i] - b.l[i] - br;
        r.l[i] = (uint64_t)d;
        br = (uint64_t)(d >> 127);
    }
    if (br) {
        uint64_t c = 0;
        for (int i = 0; i < 4; i++) {
            u128 s = (u128)r.l[i] + R4[i] + c;
            r.l[i] = (uint64_t)s;
            c = (uint64_t)(s >> 64);
        }
    }
    return r;
}
inline Fr4 fr_one() {
    Fr4 r;
    std::memcpy(r.l, FR_ONE4, 32);
    return r;
}
inline Fr4 fr_from_u64(uint64_t v) {
    Fr4 a = {{v, 0, 0, 0}}, r2;
    std::memcpy(r2.l, FR_R2_4, 32);
    return fr_mul(a, r2);
}
inline Fr4 fr_pow(const Fr4& a, const uint64_t* e, int limbs) {
    Fr4 acc = fr_one();
    for (int i = limbs * 64 - 1; i >= 0; i--) {
        acc = fr_mul(acc, acc);
        if ((e[i / 64] >> (i % 64)) & 1) acc = fr_mul(acc, a);
    }
    return acc;
}
inline Fr4 fr_inv(const Fr4& a) {
    uint64_t e[4];
    std::memcpy(e, R4, 32);
    e[0] -= 2;
    return fr_pow(a, e, 4);
}
inline bool fr_eq(const Fr4& a, const Fr4& b) { return std::memcmp(a.l, b.l, 32) == 0; }

}  // namespace host
}  // namespace mzk
