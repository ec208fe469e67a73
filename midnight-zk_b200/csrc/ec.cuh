// ec.cuh — BLS12-381 G1 (y^2 = x^3 + 4 over Fp) group law on the device.
//
// Bucket accumulators use extended Jacobian "XYZZ" coordinates
// (x = X/ZZ, y = Y/ZZZ, ZZ^3 = ZZZ^2), whose mixed addition with an affine
// point costs 8M + 2S and needs no inversion.  Formulas are madd-2008-s,
// add-2008-s, mdbl-2008-s-1 and dbl-2008-s-1 of the Explicit-Formulas Database
// (Bernstein, Lange) for short Weierstrass curves with a = 0.  Infinity is
// ZZ == 0 (bit pattern); affine infinity is the all-zero point, the encoding
// of blst_p1_affine used by the reference (curves/src/bls12_381/g1.rs:761-763).
#pragma once
#include "field.cuh"

namespace mzk {

struct Affine { Fp x, y; };
struct Xyzz { Fp x, y, zz, zzz; };

__device__ __forceinline__ bool aff_is_inf(const Affine& p) { return fp_is_zero_raw(p.x) && fp_is_zero_raw(p.y); }
__device__ __forceinline__ bool xyzz_is_inf(const Xyzz& p) { return fp_is_zero_raw(p.zz); }
__device__ __forceinline__ void xyzz_set_inf(Xyzz& p) {
    p.x = fp_zero();
    p.y = fp_zero();
    p.zz = fp_zero();
    p.zzz = fp_zero();
}
__device__ __forceinline__ Xyzz xyzz_from_affine(const Affine& a) {
    Xyzz r;
    if (aff_is_inf(a)) {
        xyzz_set_inf(r);
        return r;
    }
    r.x = a.x;
    r.y = a.y;
    r.zz = fp_one();
    r.zzz = fp_one();
    return r;
}

// mdbl-2008-s-1: 2*(x, y) for an affine point
__device__ __forceinline__ Xyzz xyzz_dbl_affine(const Affine& p) {
    Fp u = fp_dbl(p.y);
    Fp v = fp_sqr(u);
    Fp w = fp_mul(u, v);
    Fp s = fp_mul(p.x, v);
    Fp xx = fp_sqr(p.x);
    Fp m = fp_add(fp_dbl(xx), xx);
    Xyzz r;
    r.x = fp_sub(fp_sqr(m), fp_dbl(s));
    r.y = fp_sub(fp_mul(m, fp_sub(s, r.x)), fp_mul(w, p.y));
    r.zz = v;
    r.zzz = w;
    return r;
}

// dbl-2008-s-1 (a = 0)
__device__ __forceinline__ Xyzz xyzz_dbl(const Xyzz& p) {
    if (xyzz_is_inf(p)) return p;
    Fp u = fp_dbl(p.y);
    Fp v = fp_sqr(u);
    Fp w = fp_mul(u, v);
    Fp s = fp_mul(p.x, v);
    Fp xx = fp_sqr(p.x);
    Fp m = fp_add(fp_dbl(xx), xx);
    Xyzz r;
    r.x = fp_sub(fp_sqr(m), fp_dbl(s));
    r.y = fp_sub(fp_mul(m, fp_sub(s, r.x)), fp_mul(w, p.y));
    r.zz = fp_mul(v, p.zz);
    r.zzz = fp_mul(w, p.zzz);
    return r;
}

// madd-2008-s: acc += (x2, y2) with all special cases (acc = inf, equal
// points, opposite points).  `q` must not be infinity.
__device__ __forceinline__ void xyzz_add_affine(Xyzz& acc, const Affine& q) {
    if (xyzz_is_inf(acc)) {
        acc.x = q.x;
        acc.y = q.y;
        acc.zz = fp_one();
        acc.zzz = fp_one();
        return;
    }
    Fp u2 = fp_mul(q.x, acc.zz);
    Fp s2 = fp_mul(q.y, acc.zzz);
    Fp p = fp_sub(u2, acc.x);
    Fp r = fp_sub(s2, acc.y);
    if (fp_is_zero(p)) {
        if (fp_is_zero(r)) acc = xyzz_dbl_affine(q);
        else xyzz_set_inf(acc);
        return;
    }
    Fp pp = fp_sqr(p);
    Fp ppp = fp_mul(p, pp);
    Fp q1 = fp_mul(acc.x, pp);
    Fp x3 = fp_sub(fp_sub(fp_sqr(r), ppp), fp_dbl(q1));
    Fp y3 = fp_sub(fp_mul(r, fp_sub(q1, x3)), fp_mul(acc.y, ppp));
    acc.zz = fp_mul(acc.zz, pp);
    acc.zzz = fp_mul(acc.zzz, ppp);
    acc.x = x3;
    acc.y = y3;
}

// madd-2008-s for acc != infinity, scheduled as five pairs of independent
// multiplications with the fewest live temporaries.
__device__ __forceinline__ void xyzz_add_affine_fast(Xyzz& acc, const Affine& q) {
    Fp u2, s2;
    fp_mul2(u2, q.x, acc.zz, s2, q.y, acc.zzz);
    const Fp p = fp_sub(u2, acc.x);
    const Fp r = fp_sub(s2, acc.y);
    if (fp_is_zero(p)) {  // rare: equal or opposite x (branch not taken is never fetched)
        if (fp_is_zero(r)) acc = xyzz_dbl_affine(q);
        else xyzz_set_inf(acc);
        return;
    }
    Fp pp, rr;
    // squares as general products: measured faster here than the dedicated
    // squaring (fewer registers in the bucket loop)
    fp_mul2(pp, p, p, rr, r, r);
    Fp ppp, q1;
    fp_mul2(ppp, p, pp, q1, acc.x, pp);
    fp_mul2(acc.zz, acc.zz, pp, acc.zzz, acc.zzz, ppp);
    const Fp x3 = fp_sub(fp_sub(rr, ppp), fp_dbl(q1));
    Fp t1, t2;
    fp_mul2(t1, r, fp_sub(q1, x3), t2, acc.y, ppp);
    acc.y = fp_sub(t1, t2);
    acc.x = x3;
}

// add-2008-s: a + b for XYZZ points, all special cases
__device__ __forceinline__ Xyzz xyzz_add(const Xyzz& a, const Xyzz& b) {
    if (xyzz_is_inf(a)) return b;
    if (xyzz_is_inf(b)) return a;
    Fp u1 = fp_mul(a.x, b.zz);
    Fp u2 = fp_mul(b.x, a.zz);
    Fp s1 = fp_mul(a.y, b.zzz);
    Fp s2 = fp_mul(b.y, a.zzz);
    Fp p = fp_sub(u2, u1);
    Fp r = fp_sub(s2, s1);
    if (fp_is_zero(p)) {
        if (fp_is_zero(r)) return xyzz_dbl(a);
        Xyzz z;
        xyzz_set_inf(z);
        return z;
    }
    Fp pp = fp_mul(p, p);  // general products: the dedicated squaring spills in the bucket reduction
    Fp ppp = fp_mul(p, pp);
    Fp q1 = fp_mul(u1, pp);
    Xyzz o;
    o.x = fp_sub(fp_sub(fp_mul(r, r), ppp), fp_dbl(q1));
    o.y = fp_sub(fp_mul(r, fp_sub(q1, o.x)), fp_mul(s1, ppp));
    o.zz = fp_mul(fp_mul(a.zz, b.zz), pp);
    o.zzz = fp_mul(fp_mul(a.zzz, b.zzz), ppp);
    return o;
}

__device__ __forceinline__ Fp fp_select(bool c, const Fp& a, const Fp& b) {
    Fp r;
#pragma unroll
    for (int j = 0; j < 12; j++) r.l[j] = c ? a.l[j] : b.l[j];
    return r;
}
// c ? a : b, limb by limb in registers
__device__ __forceinline__ Xyzz xyzz_select(bool c, const Xyzz& a, const Xyzz& b) {
    Xyzz r;
    r.x = fp_select(c, a.x, b.x);
    r.y = fp_select(c, a.y, b.y);
    r.zz = fp_select(c, a.zz, b.zz);
    r.zzz = fp_select(c, a.zzz, b.zzz);
    return r;
}

// k * p for a small non-negative k (double-and-add, MSB first)
__device__ __forceinline__ Xyzz xyzz_mul_small(const Xyzz& p, uint32_t k) {
    Xyzz acc;
    xyzz_set_inf(acc);
    for (int bit = 31; bit >= 0; bit--) {
        acc = xyzz_dbl(acc);
        if ((k >> bit) & 1u) acc = xyzz_add(acc, p);
    }
    return acc;
}

// XYZZ -> affine, canonical coordinates; infinity -> all zero
__device__ __forceinline__ Affine xyzz_to_affine(const Xyzz& p) {
    Affine a;
    if (xyzz_is_inf(p)) {
        a.x = fp_zero();
        a.y = fp_zero();
        return a;
    }
    // 1/ZZZ, then 1/ZZ = (ZZ/ZZZ)^2
    Fp t = fp_inv(p.zzz);
    Fp zi = fp_mul(p.zz, t);
    Fp zi2 = fp_sqr(zi);
    a.x = fp_canonical(fp_mul(p.x, zi2));
    a.y = fp_canonical(fp_mul(p.y, t));
    return a;
}

// Vectorised 96-byte affine load (six 16-byte loads through the read-only path)
__device__ __forceinline__ Affine load_affine(const Affine* base, uint32_t idx) {
    const uint4* src = reinterpret_cast<const uint4*>(base + idx);
    Affine a;
    uint4 v[6];
#pragma unroll
    for (int k = 0; k < 6; k++) v[k] = __ldg(src + k);
#pragma unroll
    for (int k = 0; k < 3; k++) {
        a.x.l[4 * k + 0] = v[k].x;
        a.x.l[4 * k + 1] = v[k].y;
        a.x.l[4 * k + 2] = v[k].z;
        a.x.l[4 * k + 3] = v[k].w;
        a.y.l[4 * k + 0] = v[k + 3].x;
        a.y.l[4 * k + 1] = v[k + 3].y;
        a.y.l[4 * k + 2] = v[k + 3].z;
        a.y.l[4 * k + 3] = v[k + 3].w;
    }
    return a;
}

}  // namespace mzk
