// transcript.hpp — the prover's Fiat-Shamir transcript and the host-side
// scalar and point encodings it hashes.
//
// CircuitTranscript<Blake2bState> (proofs/src/transcript/mod.rs:83-150,
// implementors.rs:13-30): one keyed BLAKE2b-512 state (key "Domain separator
// for transcript"); absorbing an element feeds a 1 byte then its encoding;
// squeezing feeds a 0 byte and reads the digest of everything fed so far
// without resetting the state; a challenge is the 64-byte digest read as a
// little-endian integer mod r (Fq::from_uniform_bytes, fq.rs:712-736).  G1
// points are absorbed and written compressed (ZCash format, 48 bytes,
// implementors.rs:138-156), scalars as 32-byte little-endian canonical values
// (:158-175).  BLAKE2b itself follows RFC 7693 (parameter block with key
// length and personalisation, 12 rounds of the G function over the SIGMA
// message schedule).
#pragma once
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "host_ec.hpp"

namespace mzk {
namespace host {

// ---------------------------------------------------------------- BLAKE2b --
class Blake2b {
   public:
    // digest length 1..64, key up to 64 bytes, personalisation up to 16 bytes
    Blake2b(size_t out_len, const uint8_t* key, size_t key_len, const uint8_t* personal, size_t personal_len) {
        out_len_ = out_len;
        for (int i = 0; i < 8; i++) h_[i] = kIv[i];
        h_[0] ^= 0x01010000ull ^ ((uint64_t)key_len << 8) ^ (uint64_t)out_len;
        uint8_t pers[16] = {0};
        std::memcpy(pers, personal, personal_len);
        h_[6] ^= load64(pers);
        h_[7] ^= load64(pers + 8);
        if (key_len) {
            uint8_t block[128] = {0};
            std::memcpy(block, key, key_len);
            update(block, 128);
        }
    }
    void update(const uint8_t* in, size_t len) {
        while (len > 0) {
            if (buf_len_ == 128) {  // a full block is compressed only once more input follows
                t_ += 128;
                compress(buf_, false);
                buf_len_ = 0;
            }
            const size_t take = std::min(len, 128 - buf_len_);
            std::memcpy(buf_ + buf_len_, in, take);
            buf_len_ += take;
            in += take;
            len -= take;
        }
    }
    // digest of everything absorbed so far; the state is not modified
    void digest(uint8_t* out) const {
        Blake2b c = *this;
        c.t_ += c.buf_len_;
        std::memset(c.buf_ + c.buf_len_, 0, 128 - c.buf_len_);
        c.compress(c.buf_, true);
        uint8_t full[64];
        for (int i = 0; i < 8; i++)
            for (int b = 0; b < 8; b++) full[8 * i + b] = (uint8_t)(c.h_[i] >> (8 * b));
        std::memcpy(out, full, out_len_);
    }

   private:
    static constexpr uint64_t kIv[8] = {0x6a09e667f3bcc908ull, 0xbb67ae8584caa73bull, 0x3c6ef372fe94f82bull,
                                        0xa54ff53a5f1d36f1ull, 0x510e527fade682d1ull, 0x9b05688c2b3e6c1full,
                                        0x1f83d9abfb41bd6bull, 0x5be0cd19137e2179ull};
    static constexpr uint8_t kSigma[12][16] = {
        {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
        {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4}, {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
        {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13}, {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
        {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11}, {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
        {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5}, {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0},
        {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3}};
    static uint64_t load64(const uint8_t* p) {
        uint64_t v = 0;
        for (int i = 7; i >= 0; i--) v = (v << 8) | p[i];
        return v;
    }
    static uint64_t rotr(uint64_t x, int n) { return (x >> n) | (x << (64 - n)); }
    void compress(const uint8_t* block, bool last) {
        uint64_t m[16], v[16];
        for (int i = 0; i < 16; i++) m[i] = load64(block + 8 * i);
        for (int i = 0; i < 8; i++) {
            v[i] = h_[i];
            v[i + 8] = kIv[i];
        }
        v[12] ^= t_;  // byte counter, low word (inputs here stay far below 2^64 bytes)
        if (last) v[14] = ~v[14];
        for (int r = 0; r < 12; r++) {
            const uint8_t* s = kSigma[r];
            auto g = [&](int a, int b, int c, int d, uint64_t x, uint64_t y) {
                v[a] = v[a] + v[b] + x;
                v[d] = rotr(v[d] ^ v[a], 32);
                v[c] = v[c] + v[d];
                v[b] = rotr(v[b] ^ v[c], 24);
                v[a] = v[a] + v[b] + y;
                v[d] = rotr(v[d] ^ v[a], 16);
                v[c] = v[c] + v[d];
                v[b] = rotr(v[b] ^ v[c], 63);
            };
            g(0, 4, 8, 12, m[s[0]], m[s[1]]);
            g(1, 5, 9, 13, m[s[2]], m[s[3]]);
            g(2, 6, 10, 14, m[s[4]], m[s[5]]);
            g(3, 7, 11, 15, m[s[6]], m[s[7]]);
            g(0, 5, 10, 15, m[s[8]], m[s[9]]);
            g(1, 6, 11, 12, m[s[10]], m[s[11]]);
            g(2, 7, 8, 13, m[s[12]], m[s[13]]);
            g(3, 4, 9, 14, m[s[14]], m[s[15]]);
        }
        for (int i = 0; i < 8; i++) h_[i] ^= v[i] ^ v[i + 8];
    }
    uint64_t h_[8];
    uint64_t t_ = 0;
    uint8_t buf_[128] = {0};
    size_t buf_len_ = 0;
    size_t out_len_ = 64;
};

// ------------------------------------------------------------ Fr helpers --
inline Fr4 fr_add(const Fr4& a, const Fr4& b) {
    Fr4 r;
    uint64_t c = 0;
    for (int i = 0; i < 4; i++) {
        u128 s = (u128)a.l[i] + b.l[i] + c;
        r.l[i] = (uint64_t)s;
        c = (uint64_t)(s >> 64);
    }
    if (c || fr_geq(r.l, R4)) {
        uint64_t br = 0;
        for (int i = 0; i < 4; i++) {
            u128 d = (u128)r.l[i] - R4[i] - br;
            r.l[i] = (uint64_t)d;
            br = (uint64_t)(d >> 127);
        }
    }
    return r;
}
inline Fr4 fr_zero() { return Fr4{{0, 0, 0, 0}}; }
inline Fr4 fr_neg(const Fr4& a) { return fr_sub(fr_zero(), a); }
inline bool fr_is_zero(const Fr4& a) { return (a.l[0] | a.l[1] | a.l[2] | a.l[3]) == 0; }
inline Fr4 fr_pow_u64(const Fr4& a, uint64_t e) {
    const uint64_t ee[1] = {e};
    return fr_pow(a, ee, 1);
}
inline Fr4 fr_r2() {
    Fr4 r;
    std::memcpy(r.l, FR_R2_4, 32);
    return r;
}
// canonical value of a Montgomery element (one multiplication by 1)
inline void fr_to_canonical(const Fr4& a, uint64_t out[4]) {
    const Fr4 one_raw = {{1, 0, 0, 0}};
    const Fr4 c = fr_mul(a, one_raw);
    std::memcpy(out, c.l, 32);
}
inline void fr_to_bytes(const Fr4& a, uint8_t out[32]) {
    uint64_t c[4];
    fr_to_canonical(a, c);
    for (int i = 0; i < 4; i++)
        for (int b = 0; b < 8; b++) out[8 * i + b] = (uint8_t)(c[i] >> (8 * b));
}
// Fq::from_uniform_bytes (fq.rs:712-736): a0 R^2 + a1 R^3 with a0, a1 the two
// little-endian 256-bit halves, i.e. the 512-bit integer mod r in Montgomery form
inline Fr4 fr_from_uniform(const uint8_t b[64]) {
    Fr4 a0, a1;
    for (int i = 0; i < 4; i++) {
        uint64_t w0 = 0, w1 = 0;
        for (int k = 7; k >= 0; k--) {
            w0 = (w0 << 8) | b[8 * i + k];
            w1 = (w1 << 8) | b[32 + 8 * i + k];
        }
        a0.l[i] = w0;
        a1.l[i] = w1;
    }
    const Fr4 r2 = fr_r2(), r3 = fr_mul(r2, r2);
    return fr_add(fr_mul(a0, r2), fr_mul(a1, r3));
}

// ------------------------------------------------------------ G1 encoding --
// canonical Fp value of a Montgomery element, big-endian bytes
inline void fp_to_be48(const Fp6& a, uint8_t out[48]) {
    Fp6 raw_one;
    std::memset(raw_one.l, 0, sizeof(raw_one.l));
    raw_one.l[0] = 1;
    const Fp6 c = canon(mul(canon(a), raw_one));
    for (int i = 0; i < 6; i++)
        for (int b = 0; b < 8; b++) out[47 - (8 * i + b)] = (uint8_t)(c.l[i] >> (8 * b));
}
// (p - 1) / 2, the bound of the ZCash "larger y" flag
static const uint64_t P6_HALF[6] = {0xdcff7fffffffd555ULL, 0x0f55ffff58a9ffffULL, 0xb39869507b587b12ULL,
                                    0xb23ba5c279c2895fULL, 0x258dd3db21a5d66bULL, 0x0d0088f51cbff34dULL};
// out18: the MSM result layout (Jacobian x, y, z with z = 1 in Montgomery
// form, or all zero for the identity)
inline bool g1_is_identity(const uint64_t* p18) {
    uint64_t acc = 0;
    for (int i = 12; i < 18; i++) acc |= p18[i];
    return acc == 0;
}
// G1Affine::to_compressed (curves/src/bls12_381/g1.rs:326-334)
inline void g1_compress(const uint64_t* p18, uint8_t out[48]) {
    if (g1_is_identity(p18)) {
        std::memset(out, 0, 48);
        out[0] = 0xc0;
        return;
    }
    Fp6 x, y;
    std::memcpy(x.l, p18, 48);
    std::memcpy(y.l, p18 + 6, 48);
    fp_to_be48(x, out);
    Fp6 raw_one;
    std::memset(raw_one.l, 0, sizeof(raw_one.l));
    raw_one.l[0] = 1;
    const Fp6 yc = canon(mul(canon(y), raw_one));
    bool larger = false;
    for (int i = 5; i >= 0; i--)
        if (yc.l[i] != P6_HALF[i]) {
            larger = yc.l[i] > P6_HALF[i];
            break;
        }
    out[0] |= 0x80;
    if (larger) out[0] |= 0x20;
}
// G1Affine::to_uncompressed (g1.rs:486-488), the RawBytesUnchecked form
inline void g1_uncompressed(const uint64_t* p18, uint8_t out[96]) {
    std::memset(out, 0, 96);
    if (g1_is_identity(p18)) {
        out[0] = 0x40;
        return;
    }
    Fp6 x, y;
    std::memcpy(x.l, p18, 48);
    std::memcpy(y.l, p18 + 6, 48);
    fp_to_be48(x, out);
    fp_to_be48(y, out + 48);
}

// ------------------------------------------------------------- transcript --
class Transcript {
   public:
    Transcript() : h_(64, reinterpret_cast<const uint8_t*>(kKey), sizeof(kKey) - 1, nullptr, 0) {}
    void common_bytes(const uint8_t* b, size_t len) {
        const uint8_t prefix = 1;
        h_.update(&prefix, 1);
        h_.update(b, len);
    }
    void common_fr(const Fr4& v) {
        uint8_t b[32];
        fr_to_bytes(v, b);
        common_bytes(b, 32);
    }
    void write_fr(const Fr4& v) {
        uint8_t b[32];
        fr_to_bytes(v, b);
        common_bytes(b, 32);
        proof_.insert(proof_.end(), b, b + 32);
    }
    void write_point(const uint64_t* p18) {
        uint8_t b[48];
        g1_compress(p18, b);
        common_bytes(b, 48);
        proof_.insert(proof_.end(), b, b + 48);
    }
    Fr4 squeeze() {
        const uint8_t prefix = 0;
        h_.update(&prefix, 1);
        uint8_t d[64];
        h_.digest(d);
        return fr_from_uniform(d);
    }
    const std::vector<uint8_t>& proof() const { return proof_; }

   private:
    static constexpr char kKey[] = "Domain separator for transcript";
    Blake2b h_;
    std::vector<uint8_t> proof_;
};

}  // namespace host
}  // namespace mzk
