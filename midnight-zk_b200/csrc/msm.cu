// msm.cu — Pippenger multi-scalar multiplication over BLS12-381 G1.
//
// Replaces curves::msm::msm_best (curves/src/msm.rs:460-532) and the
// blst Pippenger behind G1Affine::multi_exp_affine (g1.rs:427-446) that
// proofs::poly::kzg::msm::msm_specific (kzg/msm.rs:174-201) dispatches to.
// The result is the same group element; the schedule is built for the GPU:
//
//  1. histogram   one thread per scalar: Montgomery -> canonical (one Fr
//                 multiplication by 1, the reference's `to_repr`), signed
//                 c-bit window digits d_w in [-2^(c-1), 2^(c-1)], count of
//                 entries per key (window, |d|-1) with warp-aggregated atomics;
//                 the digits are also stored, window-major.
//  2. scan        exclusive prefix sum of the counts = start of every bucket
//                 in the sorted entry array (a counting sort).
//  3. scatter     one window at a time from the stored digits: each
//                 (point index | sign) goes to its bucket's slice; a window's
//                 slices (4n bytes) stay in L2 while it is scattered, so the
//                 random 4-byte writes leave L2 as whole sectors.  Zero digits
//                 produce no entry, so zero and sparse scalars cost nothing
//                 (msm_specific drops zero scalars).
//  4. accumulate  the sorted entries split into equal chunks, one per thread:
//                 every thread walks its chunk adding points into an XYZZ
//                 accumulator (mixed addition, affine bases gathered from HBM).
//                 Buckets entirely inside a chunk are written directly; a bucket
//                 cut by a chunk edge leaves partial sums.  Equal chunks keep
//                 every thread busy whatever the scalar distribution.
//  5. fixup       the chunk where a cut bucket starts sums its partials.
//  6. reduce      per window, sum_b (b+1) B_b: running sums over groups of 16
//                 buckets (one thread per group), then the weighted group sums
//                 sum_g g R_g by bit planes (plain tree sums), one block each.
//  7. finish      one thread per window folds the planes into the window sum.
//  8. host        sum_w 2^(c w) S_w (c doublings between windows) and the
//                 affine normalisation on the host: a few hundred group
//                 operations that one GPU thread would take ~1 ms for.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "ec.cuh"
#include "host_ec.hpp"
#include "runtime.hpp"

namespace mzk {

namespace {

constexpr int kGroupLog = 6;       // log2 of the buckets per running-sum group (fewer when nb is smaller)
constexpr int kAccThreads = 128;   // threads per block of the accumulate kernel
constexpr int kReduceThreads = 128;
constexpr uint32_t kNoKey = 0xffffffffu;

struct MsmShape {
    int c;          // window width in bits
    int windows;    // number of windows
    uint32_t nb;    // buckets per window = 2^(c-1)
    uint32_t keys;  // windows * nb
    int glen_log;   // log2 of the buckets per running-sum group
    uint32_t groups;  // running-sum groups per window = nb >> glen_log
    int planes;     // log2(groups)
};

// glen_log: log2 of the buckets per running-sum group, at most c - 1
MsmShape make_shape(int c, int glen_log = kGroupLog) {
    MsmShape s;
    s.c = c;
    s.windows = (256 + c - 1) / c;
    s.nb = 1u << (c - 1);
    s.keys = s.nb * (uint32_t)s.windows;
    s.glen_log = c - 1 < glen_log ? c - 1 : glen_log;
    s.groups = s.nb >> s.glen_log;
    s.planes = 0;
    while ((1u << s.planes) < s.groups) s.planes++;
    return s;
}

// Running-sum group length for a call whose windows hold `keys` buckets in
// all: long groups (fewer plane sums) while there are still >= 32768 groups
// to fill the GPU, shorter ones for small MSMs, whose group chains would
// otherwise be latency-bound (a group is one thread's chain of 2L additions).
int group_log_for(uint64_t keys) {
    int g = 2;
    while (g < kGroupLog && (keys >> (g + 1)) >= 32768) g++;
    return g;
}

__device__ __forceinline__ uint32_t fr_limb(const Fr& s, int i) {
    uint32_t v = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) v = (i == j) ? s.l[j] : v;
    return v;
}

// bits [bit, bit + c) of the canonical scalar, c <= 31
__device__ __forceinline__ uint32_t window_bits(const Fr& s, int bit, int c) {
    const int limb = bit >> 5, sh = bit & 31;
    uint64_t v = (uint64_t)fr_limb(s, limb) | ((uint64_t)fr_limb(s, limb + 1) << 32);
    return (uint32_t)(v >> sh) & ((1u << c) - 1u);
}

__device__ __forceinline__ Fr load_fr(const Fr* p, size_t i) {
    const uint4* src = reinterpret_cast<const uint4*>(p + i);
    uint4 a = __ldg(src), b = __ldg(src + 1);
    Fr r;
    r.l[0] = a.x; r.l[1] = a.y; r.l[2] = a.z; r.l[3] = a.w;
    r.l[4] = b.x; r.l[5] = b.y; r.l[6] = b.z; r.l[7] = b.w;
    return r;
}

// Signed digit recoding: returns key (window * nb + |d| - 1) or kNoKey for a
// zero digit, and the sign; carries between windows through `carry`.
__device__ __forceinline__ uint32_t next_digit(const Fr& s, int w, int c, uint32_t nb, uint32_t& carry, bool& neg) {
    uint32_t v = window_bits(s, w * c, c) + carry;
    uint32_t mag;
    if (v > nb) {  // v - 2^c is negative
        mag = (1u << c) - v;
        carry = 1;
        neg = true;
    } else {
        mag = v;
        carry = 0;
        neg = false;
    }
    return mag == 0 ? kNoKey : (uint32_t)w * nb + (mag - 1);
}

// digits (optional): every point's signed digit per window, window-major
// (digits[w * n + i] = key | sign << 31, kNoKey for a zero digit), for the
// window-by-window scatter
__global__ void k_histogram(const Fr* __restrict__ scalars, size_t n, int c, int windows, uint32_t nb,
                            uint32_t* __restrict__ counts, uint32_t* __restrict__ digits) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    for (size_t base = (size_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const size_t i = base + threadIdx.x;
        const bool valid = i < n;
        Fr s = valid ? fr_from_mont(load_fr(scalars, i)) : fr_zero();
        uint32_t carry = 0;
        for (int w = 0; w < windows; w++) {
            bool neg;
            uint32_t key = next_digit(s, w, c, nb, carry, neg);
            if (!valid) key = kNoKey;
            if (digits && valid) digits[(size_t)w * n + i] = key == kNoKey ? kNoKey : key | (neg ? 0x80000000u : 0u);
            const uint32_t peers = __match_any_sync(0xffffffffu, key);
            if (key != kNoKey && lane == __ffs(peers) - 1) atomicAdd(&counts[key], (uint32_t)__popc(peers));
        }
    }
}

// All-windows scatter of the fixed-scratch path (n <= 2^16, whose sorted
// array fits in L2): windows whose cursor atomics a warp keeps in flight.
constexpr int kScatterWindows = 8;

// The cursor of bucket `key` is cursor[key] (= offsets + 1 of the caller):
// it starts at the bucket's first slot (the exclusive scan written one place
// to the right) and each atomic returns absolute positions.  After the
// scatter cursor[key] = end of bucket key = start of bucket key + 1, so the
// array from offsets[0] = 0 is exactly the bucket offset table.
__device__ __forceinline__ void scatter_group(const uint32_t (&key)[kScatterWindows],
                                              const bool (&neg)[kScatterWindows], uint32_t value, int lane,
                                              uint32_t* __restrict__ cursor, uint32_t* __restrict__ sorted) {
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t peers[kScatterWindows], slot[kScatterWindows];
#pragma unroll
    for (int j = 0; j < kScatterWindows; j++) {
        peers[j] = __match_any_sync(0xffffffffu, key[j]);
        slot[j] = 0;
        if (key[j] != kNoKey && lane == __ffs(peers[j]) - 1) slot[j] = atomicAdd(&cursor[key[j]], (uint32_t)__popc(peers[j]));
    }
#pragma unroll
    for (int j = 0; j < kScatterWindows; j++) {
        const uint32_t first = __shfl_sync(0xffffffffu, slot[j], __ffs(peers[j]) - 1);
        if (key[j] != kNoKey) sorted[first + (uint32_t)__popc(peers[j] & lt_mask)] = value | (neg[j] ? 0x80000000u : 0u);
    }
}

// The scatter of one window from the stored digits.  Its entries go to that
// window's slice of the sorted array (4n bytes: 67 MB at 2^24, inside the
// 126 MB L2), so the scattered 4-byte writes merge into whole sectors in L2
// instead of each costing a DRAM sector read and write.
__global__ void k_scatter_window(const uint32_t* __restrict__ digits_w, size_t n, uint32_t* __restrict__ cursor,
                                 uint32_t* __restrict__ sorted) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (size_t base = (size_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const size_t i = base + threadIdx.x;
        const uint32_t d = i < n ? __ldg(digits_w + i) : kNoKey;
        const uint32_t key = d == kNoKey ? kNoKey : d & 0x7fffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(peers) - 1;
        uint32_t slot = 0;
        if (key != kNoKey && lane == leader) slot = atomicAdd(&cursor[key], (uint32_t)__popc(peers));
        slot = __shfl_sync(0xffffffffu, slot, leader);
        if (key != kNoKey) sorted[slot + (uint32_t)__popc(peers & lt_mask)] = (uint32_t)i | (d & 0x80000000u);
    }
}

__global__ void k_scatter(const Fr* __restrict__ scalars, size_t n, int c, int windows, uint32_t nb,
                          uint32_t* __restrict__ cursor, uint32_t* __restrict__ sorted) {
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    for (size_t base = (size_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const size_t i = base + threadIdx.x;
        const bool valid = i < n;
        Fr s = valid ? fr_from_mont(load_fr(scalars, i)) : fr_zero();
        uint32_t carry = 0;
        for (int w0 = 0; w0 < windows; w0 += kScatterWindows) {
            uint32_t key[kScatterWindows];
            bool neg[kScatterWindows];
#pragma unroll
            for (int j = 0; j < kScatterWindows; j++) {
                key[j] = kNoKey;
                neg[j] = false;
                if (w0 + j < windows) {
                    key[j] = next_digit(s, w0 + j, c, nb, carry, neg[j]);
                    if (!valid) key[j] = kNoKey;
                }
            }
            scatter_group(key, neg, (uint32_t)i, lane, cursor, sorted);
        }
    }
}

// ---- exclusive scan of u32 (3 phases) ----
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* smem_warp, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (int)(blockDim.x >> 5) ? smem_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        smem_warp[lane] = w;
    }
    __syncthreads();
    total = smem_warp[(blockDim.x >> 5) - 1];
    uint32_t prefix = warp > 0 ? smem_warp[warp - 1] : 0;
    __syncthreads();
    return prefix + x - v;
}

__global__ void k_scan_tiles(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t len,
                             uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t sw[32];
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems], sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = base + k < len ? in[base + k] : 0;
        sum += v[k];
    }
    uint32_t total;
    uint32_t pre = block_exclusive_scan(sum, sw, total);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < len) out[base + k] = pre;
        pre += v[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_sums(uint32_t* __restrict__ tile_sums, uint32_t tiles) {
    __shared__ uint32_t sw[32];
    uint32_t carry = 0;
    for (uint32_t b = 0; b < tiles; b += blockDim.x) {
        const uint32_t i = b + threadIdx.x;
        uint32_t v = i < tiles ? tile_sums[i] : 0, total;
        uint32_t pre = block_exclusive_scan(v, sw, total);
        if (i < tiles) tile_sums[i] = pre + carry;
        carry += total;
    }
}

__global__ void k_scan_add(uint32_t* __restrict__ out, uint32_t len, const uint32_t* __restrict__ tile_sums) {
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    const uint32_t add = tile_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (base + k < len) out[base + k] += add;
}

// ---- bucket accumulation ----
__device__ __forceinline__ uint32_t find_key(const uint32_t* offsets, uint32_t keys, uint32_t pos) {
    // largest k in [0, keys) with offsets[k] <= pos (offsets[keys] = total > pos)
    uint32_t lo = 0, hi = keys;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (offsets[mid] <= pos) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void store_xyzz(Xyzz* dst, const Xyzz& v) {
    uint4* d = reinterpret_cast<uint4*>(dst);
    const uint32_t* s = reinterpret_cast<const uint32_t*>(&v);
#pragma unroll
    for (int k = 0; k < 12; k++) d[k] = make_uint4(s[4 * k], s[4 * k + 1], s[4 * k + 2], s[4 * k + 3]);
}
__device__ __forceinline__ Xyzz load_xyzz(const Xyzz* src) {
    Xyzz v;
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(&v);
#pragma unroll
    for (int k = 0; k < 12; k++) {
        uint4 q = s[k];
        d[4 * k] = q.x;
        d[4 * k + 1] = q.y;
        d[4 * k + 2] = q.z;
        d[4 * k + 3] = q.w;
    }
    return v;
}

__device__ __forceinline__ void chunk_range(uint32_t total, uint32_t t, uint32_t nthreads, uint32_t& s, uint32_t& e) {
    const uint32_t len = (total + nthreads - 1) / nthreads;
    s = min(total, t * len);
    e = min(total, s + len);
}

// One flat loop over the chunk, so every thread of a warp runs the same number
// of additions whatever its bucket boundaries; a boundary only costs a short
// divergent flush.
__device__ __forceinline__ void flush_bucket(const Xyzz& acc, uint32_t k, uint32_t seg_lo, uint32_t seg_hi, uint32_t s,
                                             uint32_t e, uint32_t t, Xyzz* buckets, Xyzz* partials, int* owner_key) {
    if (seg_lo >= s && seg_hi <= e) {
        store_xyzz(&buckets[k], acc);
    } else if (seg_lo < s) {
        store_xyzz(&partials[2 * (size_t)t], acc);
    } else {
        store_xyzz(&partials[2 * (size_t)t + 1], acc);
        owner_key[t] = (int)k;
    }
}

__global__ void __launch_bounds__(kAccThreads, 1) k_accumulate(const Affine* __restrict__ bases,
                                                            const uint32_t* __restrict__ sorted,
                                                            const uint32_t* __restrict__ offsets, uint32_t keys,
                                                            Xyzz* __restrict__ buckets, Xyzz* __restrict__ partials,
                                                            int* __restrict__ owner_key) {
    const uint32_t nthreads = gridDim.x * blockDim.x;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t total = offsets[keys];
    uint32_t s, e;
    chunk_range(total, t, nthreads, s, e);
    owner_key[t] = -1;
    if (s >= e) return;
    uint32_t k = find_key(offsets, keys, s);
    uint32_t seg_lo = offsets[k], seg_hi = offsets[k + 1];
    // the end of the following bucket, loaded one bucket ahead (offsets has
    // keys + 2 entries, so k + 2 <= keys + 1 is in range)
    uint32_t nxt_hi = __ldg(offsets + k + 2);
    Xyzz acc;
    xyzz_set_inf(acc);
    // the next entry's base is loaded one iteration ahead, and the entry after
    // it (its index) two ahead, to hide the gather latency
    uint32_t ent = __ldg(sorted + s);
    uint32_t ent2 = s + 1 < e ? __ldg(sorted + s + 1) : 0u;
    Affine nxt = load_affine(bases, ent & 0x7fffffffu);
    for (uint32_t j = s; j < e; j++) {
        if (j == seg_hi) {
            flush_bucket(acc, k, seg_lo, seg_hi, s, e, t, buckets, partials, owner_key);
            xyzz_set_inf(acc);
            k++;
            seg_lo = seg_hi;
            seg_hi = nxt_hi;
            while (seg_hi <= j) {  // empty buckets
                k++;
                seg_lo = seg_hi;
                seg_hi = offsets[k + 1];
            }
            nxt_hi = __ldg(offsets + k + 2);
        }
        Affine p = nxt;
        const uint32_t cur = ent;
        if (j + 1 < e) {
            ent = ent2;
            nxt = load_affine(bases, ent & 0x7fffffffu);
            if (j + 2 < e) ent2 = __ldg(sorted + j + 2);
        }
        if (aff_is_inf(p)) continue;
        p.y = fp_select((cur >> 31) != 0, fp_neg(p.y), p.y);
        if (xyzz_is_inf(acc)) {
            acc.x = p.x;
            acc.y = p.y;
            acc.zz = fp_one();
            acc.zzz = fp_one();
        } else {
            xyzz_add_affine_fast(acc, p);
        }
    }
    flush_bucket(acc, k, seg_lo, seg_hi, s, e, t, buckets, partials, owner_key);
}

// A cut bucket is finished by the chunk where it starts.  Short spans are summed
// by that thread; a bucket spanning many chunks (a heavy bucket: scalars 0/1,
// a nearly empty top window) is queued for k_fixup_long.
constexpr uint32_t kShortSpan = 32;

__global__ void k_fixup(const uint32_t* __restrict__ offsets, uint32_t keys, const Xyzz* __restrict__ partials,
                        const int* __restrict__ owner_key, Xyzz* __restrict__ buckets, uint32_t* __restrict__ long_count,
                        uint2* __restrict__ long_list) {
    const uint32_t nthreads = gridDim.x * blockDim.x;  // same grid as k_accumulate
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = owner_key[t];
    if (k < 0) return;
    const uint32_t total = offsets[keys];
    const uint32_t len = (total + nthreads - 1) / nthreads;
    const uint32_t last = (offsets[k + 1] - 1) / len;
    if (last - t > kShortSpan) {
        const uint32_t slot = atomicAdd(long_count, 1u);
        long_list[slot] = make_uint2(t, last);
        return;
    }
    Xyzz acc = load_xyzz(&partials[2 * (size_t)t + 1]);
    for (uint32_t u = t + 1; u <= last; u++) acc = xyzz_add(acc, load_xyzz(&partials[2 * (size_t)u]));
    store_xyzz(&buckets[k], acc);
}

// one block per queued heavy bucket: strided partial sums, then a tree
__global__ void __launch_bounds__(kReduceThreads) k_fixup_long(const int* __restrict__ owner_key,
                                                               const Xyzz* __restrict__ partials,
                                                               const uint32_t* __restrict__ long_count,
                                                               const uint2* __restrict__ long_list,
                                                               Xyzz* __restrict__ buckets) {
    extern __shared__ uint4 smem_raw[];
    Xyzz* sm = reinterpret_cast<Xyzz*>(smem_raw);
    for (uint32_t item = blockIdx.x; item < *long_count; item += gridDim.x) {
        const uint2 tl = long_list[item];
        const uint32_t t = tl.x, last = tl.y;
        Xyzz acc;
        if (threadIdx.x == 0) acc = load_xyzz(&partials[2 * (size_t)t + 1]);
        else xyzz_set_inf(acc);
        for (uint32_t u = t + 1 + threadIdx.x; u <= last; u += blockDim.x)
            acc = xyzz_add(acc, load_xyzz(&partials[2 * (size_t)u]));
        sm[threadIdx.x] = acc;
        __syncthreads();
        for (int off = blockDim.x >> 1; off > 0; off >>= 1) {
            if ((int)threadIdx.x < off) sm[threadIdx.x] = xyzz_add(sm[threadIdx.x], sm[threadIdx.x + off]);
            __syncthreads();
        }
        if (threadIdx.x == 0) store_xyzz(&buckets[owner_key[t]], sm[0]);
        __syncthreads();
    }
}

// ---- bucket reduction over a table of windows ----
//
// A window's sum S = sum_{b=1}^{nb} b * B_b is reduced in three steps:
//   1. running sums over groups of L = 2^glen_log consecutive buckets, top
//      first: R_g = sum of the group's buckets, T_g = sum_i (i+1) B_{gL+i};
//   2. plane sums: Q_j = sum of R_g over the groups g with bit j set, and
//      T = sum_g T_g (each plane split over `split` blocks, then merged);
//   3. S = T + L * sum_j 2^j Q_j (Horner, one thread per window).
// One table row per window serves a single MSM and a batch of MSMs alike.
struct WinDev {
    uint32_t key_start;    // first bucket key of the window
    uint32_t nb;           // buckets in the window
    uint32_t group_start;  // first running-sum group of the window
    uint32_t plane_start;  // first of its planes + 1 plane slots
    uint32_t glen_log;     // log2 of the buckets per group
    int planes;            // log2 of the groups per window
};

__device__ __forceinline__ uint32_t find_win(const WinDev* wins, uint32_t n_wins, uint32_t v, bool by_plane) {
    uint32_t lo = 0, hi = n_wins;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((by_plane ? wins[mid].plane_start : wins[mid].group_start) <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The bucket sets of an MSM over the same keys (one per part of a pipelined
// MSM), added bucket by bucket; a key is empty in a set when its offsets
// say so (its bucket is then never written)
struct BucketSets {
    const Xyzz* buckets[kMaxMsmParts];
    const uint32_t* offsets[kMaxMsmParts];
    uint32_t n;
};

__global__ void __launch_bounds__(kReduceThreads) k_group_sums(const BucketSets sets,
                                                               const WinDev* __restrict__ wins, uint32_t n_wins,
                                                               uint32_t total_groups, Xyzz* __restrict__ run_out,
                                                               Xyzz* __restrict__ tot_out) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= total_groups) return;
    const WinDev wd = wins[find_win(wins, n_wins, gid, false)];
    const uint32_t key0 = wd.key_start + ((gid - wd.group_start) << wd.glen_log);
    Xyzz run, tot;
    xyzz_set_inf(run);
    xyzz_set_inf(tot);
    for (int b = (1 << wd.glen_log) - 1; b >= 0; b--) {
        const uint32_t key = key0 + (uint32_t)b;
#pragma unroll
        for (uint32_t s = 0; s < kMaxMsmParts; s++)
            if (s < sets.n && sets.offsets[s][key + 1] > sets.offsets[s][key])
                run = xyzz_add(run, load_xyzz(&sets.buckets[s][key]));
        tot = xyzz_add(tot, run);
    }
    store_xyzz(&run_out[gid], run);
    store_xyzz(&tot_out[gid], tot);
}

// block b: plane slot b / split, part b % split of the window's groups.
// Slot plane < planes sums R_g over the g with bit `plane` set; slot plane ==
// planes sums T_g over all g.
__global__ void __launch_bounds__(kReduceThreads) k_plane_sums(const Xyzz* __restrict__ run,
                                                               const Xyzz* __restrict__ tot,
                                                               const WinDev* __restrict__ wins, uint32_t n_wins,
                                                               uint32_t split, Xyzz* __restrict__ partial) {
    extern __shared__ uint4 smem_raw[];
    Xyzz* sm = reinterpret_cast<Xyzz*>(smem_raw);
    const uint32_t slot = blockIdx.x / split, part = blockIdx.x % split;
    const WinDev wd = wins[find_win(wins, n_wins, slot, true)];
    const int plane = (int)(slot - wd.plane_start);
    const uint32_t groups = wd.nb >> wd.glen_log;
    const uint32_t chunk = (groups + split - 1) / split;
    const uint32_t g_end = min(groups, (part + 1) * chunk);
    const Xyzz* src = (plane == wd.planes ? tot : run) + wd.group_start;
    Xyzz acc;
    xyzz_set_inf(acc);
    for (uint32_t g = part * chunk + threadIdx.x; g < g_end; g += blockDim.x)
        if (plane == wd.planes || ((g >> plane) & 1u)) acc = xyzz_add(acc, load_xyzz(&src[g]));
    sm[threadIdx.x] = acc;
    __syncthreads();
    for (int off = blockDim.x >> 1; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) sm[threadIdx.x] = xyzz_add(sm[threadIdx.x], sm[threadIdx.x + off]);
        __syncthreads();
    }
    if (threadIdx.x == 0) store_xyzz(&partial[blockIdx.x], sm[0]);
}

// q[slot] = sum of the slot's `split` partial plane sums
__global__ void k_plane_merge(const Xyzz* __restrict__ partial, uint32_t slots, uint32_t split,
                              Xyzz* __restrict__ q) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= slots) return;
    Xyzz acc = load_xyzz(&partial[(size_t)slot * split]);
    for (uint32_t p = 1; p < split; p++) acc = xyzz_add(acc, load_xyzz(&partial[(size_t)slot * split + p]));
    store_xyzz(&q[slot], acc);
}

// S = T + L * sum_j 2^j Q_j, one thread per window
__global__ void k_window_finish(const Xyzz* __restrict__ q_all, const WinDev* __restrict__ wins, uint32_t n_wins,
                                Xyzz* __restrict__ out) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n_wins) return;
    const WinDev wd = wins[w];
    const Xyzz* q = q_all + wd.plane_start;
    Xyzz acc;
    xyzz_set_inf(acc);
    for (int j = wd.planes - 1; j >= 0; j--) {
        acc = xyzz_dbl(acc);
        acc = xyzz_add(acc, load_xyzz(&q[j]));
    }
    for (uint32_t b = 0; b < wd.glen_log; b++) acc = xyzz_dbl(acc);
    acc = xyzz_add(acc, load_xyzz(&q[wd.planes]));
    store_xyzz(&out[w], acc);
}

// the table rows of one MSM's windows, appended to `wins`
void append_windows(const MsmShape& sh, uint64_t key_base, std::vector<WinDev>& wins, uint64_t& groups,
                    uint64_t& slots) {
    for (int w = 0; w < sh.windows; w++) {
        WinDev wd;
        wd.key_start = (uint32_t)(key_base + (uint64_t)w * sh.nb);
        wd.nb = sh.nb;
        wd.group_start = (uint32_t)groups;
        wd.plane_start = (uint32_t)slots;
        wd.glen_log = (uint32_t)sh.glen_log;
        wd.planes = sh.planes;
        wins.push_back(wd);
        groups += sh.groups;
        slots += (uint64_t)sh.planes + 1;
    }
}

// blocks per plane slot: enough blocks to fill the GPU, at most one per
// kReduceThreads groups of the largest window, at most 16
uint32_t plane_split(uint64_t slots, uint32_t max_groups, int num_sms) {
    const uint64_t want = ((uint64_t)num_sms * 8 + slots - 1) / slots;
    const uint64_t cap = std::max<uint64_t>(1, max_groups / kReduceThreads);
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>({want, cap, 16}));
}

// steps 1-3 on `st`.  partial holds slots * split plane partials and may be
// q itself when split == 1; q holds slots plane sums.  Returns the launch
// error, if any; adds the launches to *launches when given.
cudaError_t launch_reduce(const BucketSets& sets, const WinDev* d_wins, uint32_t n_wins, uint64_t groups,
                          uint64_t slots, uint32_t split, Xyzz* run, Xyzz* tot, Xyzz* partial, Xyzz* q, Xyzz* wsum,
                          uint64_t* launches, cudaStream_t st) {
    k_group_sums<<<(uint32_t)((groups + kReduceThreads - 1) / kReduceThreads), kReduceThreads, 0, st>>>(
        sets, d_wins, n_wins, (uint32_t)groups, run, tot);
    k_plane_sums<<<(uint32_t)(slots * split), kReduceThreads, kReduceThreads * sizeof(Xyzz), st>>>(
        run, tot, d_wins, n_wins, split, split == 1 ? q : partial);
    uint64_t n = 3;
    if (split > 1) {
        k_plane_merge<<<(uint32_t)((slots + 63) / 64), 64, 0, st>>>(partial, (uint32_t)slots, split, q);
        n++;
    }
    k_window_finish<<<(n_wins + 31) / 32, 32, 0, st>>>(q, d_wins, n_wins, wsum);
    if (launches) *launches += n;
    return cudaGetLastError();
}

Status scan_u32(Context* ctx, const uint32_t* in, uint32_t* out, uint32_t len, cudaStream_t st) {
    const uint32_t tiles = (len + kScanTile - 1) / kScanTile;
    void* sums;
    MZK_TRY(ctx->ensure("scan_sums", (size_t)tiles * 4 + 64, &sums));
    k_scan_tiles<<<tiles, kScanThreads, 0, st>>>(in, out, len, (uint32_t*)sums);
    MZK_LAUNCH_CHECK(ctx);
    k_scan_sums<<<1, kScanThreads, 0, st>>>((uint32_t*)sums, tiles);
    MZK_LAUNCH_CHECK(ctx);
    k_scan_add<<<tiles, kScanThreads, 0, st>>>(out, len, (const uint32_t*)sums);
    MZK_LAUNCH_CHECK(ctx);
    return OK;
}

}  // namespace

// Window width by a cost model: W = ceil(256/c) windows of n mixed additions
// (10 Fp mul) plus 2 * 2^(c-1) full additions (14 Fp mul) for the bucket sums.
int msm_pick_window(size_t n) {
    double best = 1e300;
    int bc = 8;
    for (int c = 6; c <= 20; c++) {
        const int w = (256 + c - 1) / c;
        const double cost = (double)w * ((double)n * 10.0 + (double)(1u << c) * 14.0 + 2048.0);
        if (cost < best) {
            best = cost;
            bc = c;
        }
    }
    return bc;
}

Status msm_g1_device(Context* ctx, const void* d_scalars, const void* d_bases, size_t n, uint64_t* out18,
                     cudaStream_t st, cudaEvent_t bases_ready) {
    const MsmPart whole{0, n, nullptr, bases_ready};
    return msm_g1_parts(ctx, d_scalars, d_bases, n, out18, st, &whole, 1);
}

// Each part is sorted and accumulated into its own bucket set, in order on
// `st`; the running-sum groups then add the bucket sets key by key.  The sort
// and accumulation scratch (counts, sorted entries, chunk partials) is shared:
// stream order finishes one part's use before the next part's writes.
Status msm_g1_parts(Context* ctx, const void* d_scalars, const void* d_bases, size_t n, uint64_t* out18,
                    cudaStream_t st, const MsmPart* parts, int n_parts) {
    std::memset(out18, 0, 18 * 8);
    if (n == 0) return OK;
    if (n >= 0x80000000ull) {
        set_error("msm: n must be < 2^31");
        return ERR_ARG;
    }
    if (n_parts < 1 || n_parts > kMaxMsmParts || parts[0].begin != 0 || parts[n_parts - 1].end != n) {
        set_error("msm: parts must cover [0, n) in 1.." + std::to_string(kMaxMsmParts) + " pieces");
        return ERR_ARG;
    }
    size_t max_part = 0;
    for (int p = 0; p < n_parts; p++) {
        if (parts[p].end <= parts[p].begin || (p > 0 && parts[p].begin != parts[p - 1].end)) {
            set_error("msm: parts must be non-empty and contiguous");
            return ERR_ARG;
        }
        max_part = std::max(max_part, parts[p].end - parts[p].begin);
    }
    const int c = msm_window_for(ctx, n);
    if (c < 5 || c > 24) {
        set_error("msm: window width must be in [5, 24]");
        return ERR_ARG;
    }
    const MsmShape sh = make_shape(c, group_log_for(make_shape(c).keys));
    const size_t entries_cap = (size_t)sh.windows * max_part;
    if (entries_cap >= 0xffffffffull) {
        set_error("msm: n * windows exceeds 2^32 entries");
        return ERR_ARG;
    }
    // accumulate grid: persistent, sized to fill the GPU once
    int acc_blocks_per_sm = 0;
    MZK_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&acc_blocks_per_sm, k_accumulate, kAccThreads, 0));
    if (acc_blocks_per_sm < 1) acc_blocks_per_sm = 1;
    const uint32_t acc_blocks = (uint32_t)(ctx->num_sms * acc_blocks_per_sm);
    const uint32_t acc_threads = acc_blocks * kAccThreads;

    void *counts, *sorted, *partials, *owner, *run, *tot, *planes, *wsum;
    void *offsets[kMaxMsmParts] = {}, *buckets[kMaxMsmParts] = {};
    static const char* const kOffsetNames[kMaxMsmParts] = {"msm_offsets", "msm_offsets2", "msm_offsets3",
                                                            "msm_offsets4"};
    static const char* const kBucketNames[kMaxMsmParts] = {"msm_buckets", "msm_buckets2", "msm_buckets3",
                                                            "msm_buckets4"};
    MZK_TRY(ctx->ensure("msm_counts", ((size_t)sh.keys + 1) * 4, &counts));
    for (int p = 0; p < n_parts; p++) {
        MZK_TRY(ctx->ensure(kOffsetNames[p], ((size_t)sh.keys + 2) * 4, &offsets[p]));
        MZK_TRY(ctx->ensure(kBucketNames[p], (size_t)sh.keys * sizeof(Xyzz), &buckets[p]));
    }
    MZK_TRY(ctx->ensure("msm_sorted", entries_cap * 4, &sorted));
    void* digits;
    MZK_TRY(ctx->ensure("msm_digits", entries_cap * 4, &digits));
    MZK_TRY(ctx->ensure("msm_partials", (size_t)acc_threads * 2 * sizeof(Xyzz), &partials));
    MZK_TRY(ctx->ensure("msm_owner", (size_t)acc_threads * 4, &owner));
    void *long_count, *long_list;
    MZK_TRY(ctx->ensure("msm_long_count", 64, &long_count));
    MZK_TRY(ctx->ensure("msm_long_list", (size_t)acc_threads * sizeof(uint2), &long_list));
    std::vector<WinDev> wins;
    uint64_t total_groups = 0, slots = 0;
    append_windows(sh, 0, wins, total_groups, slots);
    const uint32_t split = plane_split(slots, sh.groups, ctx->num_sms);
    void *d_wins, *q;
    MZK_TRY(ctx->ensure("msm_wins", wins.size() * sizeof(WinDev), &d_wins));
    MZK_TRY(ctx->ensure("msm_run", total_groups * sizeof(Xyzz), &run));
    MZK_TRY(ctx->ensure("msm_tot", total_groups * sizeof(Xyzz), &tot));
    MZK_TRY(ctx->ensure("msm_planes", slots * split * sizeof(Xyzz), &planes));
    MZK_TRY(ctx->ensure("msm_q", slots * sizeof(Xyzz), &q));
    MZK_TRY(ctx->ensure("msm_wsum", (size_t)sh.windows * sizeof(Xyzz), &wsum));
    // pinned staging: window sums and the parts' entry counts (read back),
    // then the window table (uploaded without the sync a pageable copy implies)
    void* host_wsum;
    const size_t tab_off = (size_t)sh.windows * sizeof(Xyzz) + 64;
    MZK_TRY(ctx->ensure_pinned(tab_off + wins.size() * sizeof(WinDev), &host_wsum));
    WinDev* host_tab = reinterpret_cast<WinDev*>(static_cast<char*>(host_wsum) + tab_off);
    std::memcpy(host_tab, wins.data(), wins.size() * sizeof(WinDev));
    uint32_t* host_entries =
        reinterpret_cast<uint32_t*>(static_cast<char*>(host_wsum) + (size_t)sh.windows * sizeof(Xyzz));

    const Fr* sc = static_cast<const Fr*>(d_scalars);
    const Affine* ba = static_cast<const Affine*>(d_bases);
    const int pt_threads = 256;

    MZK_CUDA_CHECK(cudaMemcpyAsync(d_wins, host_tab, wins.size() * sizeof(WinDev), cudaMemcpyHostToDevice, st));
    for (int p = 0; p < n_parts; p++) {
        const MsmPart& part = parts[p];
        const size_t np = part.end - part.begin;
        uint32_t* off = static_cast<uint32_t*>(offsets[p]);
        const uint32_t pt_blocks =
            (uint32_t)std::min<size_t>((np + pt_threads - 1) / pt_threads, (size_t)ctx->num_sms * 16);
        if (part.scalars_ready) MZK_CUDA_CHECK(cudaStreamWaitEvent(st, part.scalars_ready, 0));
        MZK_TRY(ctx->phase_begin(PH_HISTOGRAM, st));
        MZK_CUDA_CHECK(cudaMemsetAsync(counts, 0, ((size_t)sh.keys + 1) * 4, st));
        k_histogram<<<pt_blocks, pt_threads, 0, st>>>(sc + part.begin, np, sh.c, sh.windows, sh.nb,
                                                      (uint32_t*)counts, (uint32_t*)digits);
        MZK_LAUNCH_CHECK(ctx);
        MZK_TRY(ctx->phase_end(st));
        MZK_TRY(ctx->phase_begin(PH_SCAN, st));
        // exclusive scan one place to the right: off[key + 1] = start of key
        MZK_CUDA_CHECK(cudaMemsetAsync(off, 0, 4, st));
        MZK_TRY(scan_u32(ctx, (const uint32_t*)counts, off + 1, sh.keys + 1, st));
        MZK_TRY(ctx->phase_end(st));
        MZK_TRY(ctx->phase_begin(PH_SCATTER, st));
        for (int w = 0; w < sh.windows; w++) {
            k_scatter_window<<<pt_blocks, pt_threads, 0, st>>>((const uint32_t*)digits + (size_t)w * np, np,
                                                               off + 1, (uint32_t*)sorted);
            MZK_LAUNCH_CHECK(ctx);
        }
        MZK_TRY(ctx->phase_end(st));
        if (part.bases_ready) MZK_CUDA_CHECK(cudaStreamWaitEvent(st, part.bases_ready, 0));
        MZK_TRY(ctx->phase_begin(PH_ACCUMULATE, st));
        k_accumulate<<<acc_blocks, kAccThreads, 0, st>>>(ba + part.begin, (const uint32_t*)sorted, off, sh.keys,
                                                        (Xyzz*)buckets[p], (Xyzz*)partials, (int*)owner);
        MZK_LAUNCH_CHECK(ctx);
        MZK_TRY(ctx->phase_end(st));
        MZK_TRY(ctx->phase_begin(PH_FIXUP, st));
        MZK_CUDA_CHECK(cudaMemsetAsync(long_count, 0, 4, st));
        k_fixup<<<acc_blocks, kAccThreads, 0, st>>>(off, sh.keys, (const Xyzz*)partials, (const int*)owner,
                                                   (Xyzz*)buckets[p], (uint32_t*)long_count, (uint2*)long_list);
        MZK_LAUNCH_CHECK(ctx);
        k_fixup_long<<<ctx->num_sms * 2, kReduceThreads, kReduceThreads * sizeof(Xyzz), st>>>(
            (const int*)owner, (const Xyzz*)partials, (const uint32_t*)long_count, (const uint2*)long_list,
            (Xyzz*)buckets[p]);
        MZK_LAUNCH_CHECK(ctx);
        MZK_TRY(ctx->phase_end(st));
        MZK_CUDA_CHECK(cudaMemcpyAsync(host_entries + p, off + sh.keys, 4, cudaMemcpyDeviceToHost, st));
    }
    MZK_TRY(ctx->phase_begin(PH_REDUCE, st));
    BucketSets sets{};
    sets.n = (uint32_t)n_parts;
    for (int p = 0; p < n_parts; p++) {
        sets.buckets[p] = (const Xyzz*)buckets[p];
        sets.offsets[p] = (const uint32_t*)offsets[p];
    }
    MZK_CUDA_CHECK(launch_reduce(sets, (const WinDev*)d_wins, (uint32_t)wins.size(),
                                 total_groups, slots, split, (Xyzz*)run, (Xyzz*)tot, (Xyzz*)planes, (Xyzz*)q,
                                 (Xyzz*)wsum, &ctx->launches, st));
    MZK_TRY(ctx->phase_end(st));
    MZK_CUDA_CHECK(cudaMemcpyAsync(host_wsum, wsum, (size_t)sh.windows * sizeof(Xyzz), cudaMemcpyDeviceToHost, st));
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    ctx->phase_collect();
    ctx->last_c = sh.c;
    ctx->last_windows = sh.windows;
    ctx->last_entries = 0;
    for (int p = 0; p < n_parts; p++) ctx->last_entries += host_entries[p];

    // host: sum_w 2^(c w) S_w by Horner, then normalise
    const host::Xyzz6* hs = static_cast<const host::Xyzz6*>(host_wsum);
    host::Xyzz6 acc = host::infinity();
    for (int w = sh.windows - 1; w >= 0; w--) {
        for (int b = 0; b < sh.c; b++) acc = host::dbl(acc);
        acc = host::add(acc, host::canon(hs[w]));
    }
    host::to_jacobian_normalised(acc, out18);
    return OK;
}

}  // namespace mzk

namespace mzk {

// ---------------------------------------------------------------------------
// Batched MSMs over one shared device SRS.
//
// Many MSMs (a proof's commitments, or many proofs' commitments) run as one
// MSM of MSMs: every item keeps its own window width, its keys are laid out
// back to back in one key space, so ONE counting sort orders all entries and
// ONE accumulate launch balances the work of all items across the GPU (an
// item of 2^12 points and one of 2^22 share the same chunks).  Only the final
// combination of each item's window sums is per item.  Bases of item m are
// bases[base_offset_m .. base_offset_m + n_m), like commit_many's
// `bases[..size]` prefix of the SRS (proofs/src/poly/kzg/mod.rs:98-103).
// ---------------------------------------------------------------------------
namespace {

struct BatchItemDev {
    const Fr* scalars;
    uint32_t n, point_start, base_offset;
    uint32_t c, windows, nb, key_start;
    uint32_t fixed;  // 1: the windows share one bucket set, window w reads table row w
};

__device__ __forceinline__ uint32_t find_item(const BatchItemDev* items, uint32_t n_items, uint32_t p) {
    uint32_t lo = 0, hi = n_items;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (items[mid].point_start <= p) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Counts per key of every item's digits, and every point's digit per window,
// window-major (digits[w * total_points + p] = key | sign << 31, kNoKey for a
// zero digit or a window past the item's), for the window-by-window scatter.
__global__ void k_digits_batch(const BatchItemDev* __restrict__ items, uint32_t n_items, uint32_t total_points,
                               int max_windows, uint32_t* __restrict__ counts, uint32_t* __restrict__ digits) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    for (uint32_t base = blockIdx.x * blockDim.x; base < total_points; base += stride) {
        const uint32_t p = base + threadIdx.x;
        const bool valid = p < total_points;
        BatchItemDev it = items[valid ? find_item(items, n_items, p) : 0];
        const uint32_t local = p - it.point_start;
        Fr s = valid ? fr_from_mont(load_fr(it.scalars, local)) : fr_zero();
        uint32_t carry = 0;
        for (int w = 0; w < max_windows; w++) {
            bool neg = false;
            uint32_t key = kNoKey;
            if (valid && w < (int)it.windows) {
                key = next_digit(s, w, (int)it.c, it.nb, carry, neg);
                if (key != kNoKey) key += it.key_start - (it.fixed ? (uint32_t)w * it.nb : 0u);
            }
            const uint32_t peers = __match_any_sync(0xffffffffu, key);
            if (key != kNoKey && lane == __ffs(peers) - 1) atomicAdd(&counts[key], (uint32_t)__popc(peers));
            if (valid) digits[(size_t)w * total_points + p] = key == kNoKey ? kNoKey : key | (neg ? 0x80000000u : 0u);
        }
    }
}


// The batch scatter of window w of every item from the stored digits: the
// entries land in the items' window-w slices (4 bytes per point of the batch),
// which stay in L2 while the window is scattered.
// row_off: w x the table stride (fixed items read window w from table row w)
__global__ void k_scatter_window_batch(const uint32_t* __restrict__ digits_w, const BatchItemDev* __restrict__ items,
                                       uint32_t n_items, uint32_t total_points, uint32_t row_off,
                                       uint32_t* __restrict__ cursor, uint32_t* __restrict__ sorted) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (uint32_t base = blockIdx.x * blockDim.x; base < total_points; base += stride) {
        const uint32_t p = base + threadIdx.x;
        const uint32_t d = p < total_points ? __ldg(digits_w + p) : kNoKey;
        const uint32_t key = d == kNoKey ? kNoKey : d & 0x7fffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(peers) - 1;
        uint32_t slot = 0;
        if (key != kNoKey && lane == leader) slot = atomicAdd(&cursor[key], (uint32_t)__popc(peers));
        slot = __shfl_sync(0xffffffffu, slot, leader);
        if (key != kNoKey) {
            const BatchItemDev& it = items[find_item(items, n_items, p)];
            const uint32_t point = it.base_offset + (p - it.point_start) + (it.fixed ? row_off : 0u);
            sorted[slot + (uint32_t)__popc(peers & lt_mask)] = point | (d & 0x80000000u);
        }
    }
}
}  // namespace

namespace {
// row j+1 of a window table from row j: [2^c] P, normalised
__global__ void __launch_bounds__(256) k_window_row(const Affine* __restrict__ prev, Affine* __restrict__ next,
                                                    uint64_t n, int c) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Xyzz p = xyzz_from_affine(prev[i]);
        for (int b = 0; b < c; b++) p = xyzz_dbl(p);
        next[i] = xyzz_to_affine(p);
    }
}
}  // namespace

uint32_t msm_table_rows(int c) { return (uint32_t)make_shape(c).windows; }

Status msm_window_table(Context* ctx, void* d_table, uint64_t len, int c, uint32_t rows, cudaStream_t st) {
    if (c < 5 || c > 24 || rows < msm_table_rows(c) || len == 0 || (uint64_t)rows * len >= 0x80000000ull) {
        set_error("window table: c in [5, 24], at least msm_table_rows(c) rows, rows x len < 2^31");
        return ERR_ARG;
    }
    Affine* t = static_cast<Affine*>(d_table);
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((len + 255) / 256, (uint64_t)ctx->num_sms * 8);
    for (uint32_t j = 1; j < rows; j++) {
        k_window_row<<<blocks, 256, 0, st>>>(t + (j - 1) * len, t + j * len, len, c);
        MZK_LAUNCH_CHECK(ctx);
    }
    return OK;
}

Status msm_g1_batch_device(Context* ctx, const void* d_bases, size_t bases_len, const BatchItem* items, size_t count,
                           uint64_t* out, cudaStream_t st, const MsmTable* table) {
    if (table) {
        if (table->d_table != d_bases || table->stride != bases_len || table->rows < msm_table_rows(table->c) ||
            table->rows * table->stride >= 0x80000000ull) {
            set_error("msm batch: the window table must start at the bases and cover the windows of its width");
            return ERR_ARG;
        }
    }
    std::memset(out, 0, count * 18 * 8);
    std::vector<BatchItemDev> hi;
    std::vector<WinDev> hw;
    std::vector<size_t> item_of;  // position in `items` of every device item
    uint64_t points = 0, keys = 0, entries = 0, groups = 0, slots = 0;
    uint32_t max_groups = 1;
    int max_windows = 0;
    // the group length follows the buckets of the whole batch
    auto uses_table = [&](uint64_t n) { return table && n >= table->min_n; };
    uint64_t all_keys = 0;
    for (size_t m = 0; m < count; m++)
        if (items[m].n)
            all_keys += uses_table(items[m].n) ? make_shape(table->c).nb
                                                : make_shape(msm_window_for(ctx, items[m].n)).keys;
    const int glen_log = group_log_for(all_keys);
    for (size_t m = 0; m < count; m++) {
        const BatchItem& it = items[m];
        if (it.n == 0) continue;
        if (!it.d_scalars) {
            set_error("msm batch: null scalars in item " + std::to_string(m));
            return ERR_ARG;
        }
        if (it.base_offset + it.n > bases_len || it.base_offset + it.n >= 0x80000000ull) {
            set_error("msm batch: item " + std::to_string(m) + " reads past the bases");
            return ERR_ARG;
        }
        const bool fixed = uses_table(it.n);
        const int c = fixed ? table->c : msm_window_for(ctx, it.n);
        const MsmShape sh = make_shape(c, glen_log);
        BatchItemDev d;
        d.scalars = static_cast<const Fr*>(it.d_scalars);
        d.n = (uint32_t)it.n;
        d.point_start = (uint32_t)points;
        d.base_offset = (uint32_t)it.base_offset;
        d.c = (uint32_t)sh.c;
        d.windows = (uint32_t)sh.windows;
        d.nb = sh.nb;
        d.key_start = (uint32_t)keys;
        d.fixed = fixed ? 1u : 0u;
        if (fixed) {  // one window row: every window's digits land in the same buckets
            MsmShape one = sh;
            one.windows = 1;
            append_windows(one, keys, hw, groups, slots);
            keys += sh.nb;
        } else {
            append_windows(sh, keys, hw, groups, slots);
            keys += sh.keys;
        }
        max_groups = std::max(max_groups, sh.groups);
        points += it.n;
        entries += (uint64_t)sh.windows * it.n;
        max_windows = std::max(max_windows, sh.windows);
        hi.push_back(d);
        item_of.push_back(m);
    }
    if (hi.empty()) return OK;
    if (points >= 0xffffffffull || keys >= 0xffffffffull || entries >= 0xffffffffull) {
        set_error("msm batch: more than 2^32 points, keys or entries");
        return ERR_ARG;
    }
    int acc_blocks_per_sm = 0;
    MZK_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&acc_blocks_per_sm, k_accumulate, kAccThreads, 0));
    if (acc_blocks_per_sm < 1) acc_blocks_per_sm = 1;
    const uint32_t acc_blocks = (uint32_t)(ctx->num_sms * acc_blocks_per_sm);
    const uint32_t acc_threads = acc_blocks * kAccThreads;
    const size_t n_wins = hw.size();
    void *d_items, *d_wins, *counts, *offsets, *sorted, *buckets, *partials, *owner, *long_count, *long_list, *run, *tot,
        *planes, *wsum;
    MZK_TRY(ctx->ensure("batch_items", hi.size() * sizeof(BatchItemDev), &d_items));
    MZK_TRY(ctx->ensure("batch_wins", n_wins * sizeof(WinDev), &d_wins));
    MZK_TRY(ctx->ensure("msm_counts", (keys + 1) * 4, &counts));
    MZK_TRY(ctx->ensure("msm_offsets", (keys + 2) * 4, &offsets));
    MZK_TRY(ctx->ensure("msm_sorted", entries * 4, &sorted));
    void* digits;
    MZK_TRY(ctx->ensure("msm_digits", (size_t)max_windows * points * 4, &digits));
    MZK_TRY(ctx->ensure("msm_buckets", keys * sizeof(Xyzz), &buckets));
    MZK_TRY(ctx->ensure("msm_partials", (size_t)acc_threads * 2 * sizeof(Xyzz), &partials));
    MZK_TRY(ctx->ensure("msm_owner", (size_t)acc_threads * 4, &owner));
    MZK_TRY(ctx->ensure("msm_long_count", 64, &long_count));
    MZK_TRY(ctx->ensure("msm_long_list", (size_t)acc_threads * sizeof(uint2), &long_list));
    MZK_TRY(ctx->ensure("msm_run", groups * sizeof(Xyzz), &run));
    MZK_TRY(ctx->ensure("msm_tot", groups * sizeof(Xyzz), &tot));
    const uint32_t split = plane_split(slots, max_groups, ctx->num_sms);
    void* q;
    MZK_TRY(ctx->ensure("msm_planes", slots * split * sizeof(Xyzz), &planes));
    MZK_TRY(ctx->ensure("msm_q", slots * sizeof(Xyzz), &q));
    MZK_TRY(ctx->ensure("msm_wsum", n_wins * sizeof(Xyzz), &wsum));
    // pinned staging: window sums (read back), then the item and window tables
    void* host_wsum;
    const size_t items_off = n_wins * sizeof(Xyzz) + 64;
    const size_t wins_off = items_off + ((hi.size() * sizeof(BatchItemDev) + 255) & ~(size_t)255);
    MZK_TRY(ctx->ensure_pinned(wins_off + n_wins * sizeof(WinDev), &host_wsum));
    char* staging = static_cast<char*>(host_wsum);
    std::memcpy(staging + items_off, hi.data(), hi.size() * sizeof(BatchItemDev));
    std::memcpy(staging + wins_off, hw.data(), n_wins * sizeof(WinDev));
    MZK_CUDA_CHECK(cudaMemcpyAsync(d_items, staging + items_off, hi.size() * sizeof(BatchItemDev),
                                   cudaMemcpyHostToDevice, st));
    MZK_CUDA_CHECK(cudaMemcpyAsync(d_wins, staging + wins_off, n_wins * sizeof(WinDev), cudaMemcpyHostToDevice, st));

    const uint32_t n_items = (uint32_t)hi.size();
    const int pt_threads = 256;
    const uint32_t pt_blocks =
        (uint32_t)std::min<uint64_t>((points + pt_threads - 1) / pt_threads, (uint64_t)ctx->num_sms * 16);
    MZK_TRY(ctx->phase_begin(PH_HISTOGRAM, st));
    MZK_CUDA_CHECK(cudaMemsetAsync(counts, 0, (keys + 1) * 4, st));
    k_digits_batch<<<pt_blocks, pt_threads, 0, st>>>((const BatchItemDev*)d_items, n_items, (uint32_t)points,
                                                    max_windows, (uint32_t*)counts, (uint32_t*)digits);
    MZK_LAUNCH_CHECK(ctx);
    MZK_TRY(ctx->phase_end(st));
    MZK_TRY(ctx->phase_begin(PH_SCAN, st));
    MZK_CUDA_CHECK(cudaMemsetAsync(offsets, 0, 4, st));
    MZK_TRY(scan_u32(ctx, (const uint32_t*)counts, (uint32_t*)offsets + 1, (uint32_t)keys + 1, st));
    MZK_TRY(ctx->phase_end(st));
    MZK_TRY(ctx->phase_begin(PH_SCATTER, st));
    for (int w = 0; w < max_windows; w++) {
        const uint32_t row_off = table ? (uint32_t)((uint64_t)w * table->stride) : 0u;
        k_scatter_window_batch<<<pt_blocks, pt_threads, 0, st>>>((const uint32_t*)digits + (size_t)w * points,
                                                                 (const BatchItemDev*)d_items, n_items,
                                                                 (uint32_t)points, row_off,
                                                                 (uint32_t*)offsets + 1, (uint32_t*)sorted);
        MZK_LAUNCH_CHECK(ctx);
    }
    MZK_TRY(ctx->phase_end(st));
    MZK_TRY(ctx->phase_begin(PH_ACCUMULATE, st));
    k_accumulate<<<acc_blocks, kAccThreads, 0, st>>>(static_cast<const Affine*>(d_bases), (const uint32_t*)sorted,
                                                    (const uint32_t*)offsets, (uint32_t)keys, (Xyzz*)buckets,
                                                    (Xyzz*)partials, (int*)owner);
    MZK_LAUNCH_CHECK(ctx);
    MZK_TRY(ctx->phase_end(st));
    MZK_TRY(ctx->phase_begin(PH_FIXUP, st));
    MZK_CUDA_CHECK(cudaMemsetAsync(long_count, 0, 4, st));
    k_fixup<<<acc_blocks, kAccThreads, 0, st>>>((const uint32_t*)offsets, (uint32_t)keys, (const Xyzz*)partials,
                                               (const int*)owner, (Xyzz*)buckets, (uint32_t*)long_count,
                                               (uint2*)long_list);
    MZK_LAUNCH_CHECK(ctx);
    k_fixup_long<<<ctx->num_sms * 2, kReduceThreads, kReduceThreads * sizeof(Xyzz), st>>>(
        (const int*)owner, (const Xyzz*)partials, (const uint32_t*)long_count, (const uint2*)long_list,
        (Xyzz*)buckets);
    MZK_LAUNCH_CHECK(ctx);
    MZK_TRY(ctx->phase_end(st));
    MZK_TRY(ctx->phase_begin(PH_REDUCE, st));
    const BucketSets sets{{(const Xyzz*)buckets}, {(const uint32_t*)offsets}, 1};
    MZK_CUDA_CHECK(launch_reduce(sets, (const WinDev*)d_wins, (uint32_t)n_wins, groups, slots, split, (Xyzz*)run,
                                 (Xyzz*)tot, (Xyzz*)planes, (Xyzz*)q, (Xyzz*)wsum, &ctx->launches, st));
    MZK_TRY(ctx->phase_end(st));
    MZK_CUDA_CHECK(cudaMemcpyAsync(host_wsum, wsum, n_wins * sizeof(Xyzz), cudaMemcpyDeviceToHost, st));
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    ctx->phase_collect();
    // host: per item sum_w 2^(c w) S_w by Horner and one inversion (~0.15 ms
    // each, a serial chain of ~250 doublings); items are independent, so a
    // batch spreads them over host threads
    const host::Xyzz6* hs = static_cast<const host::Xyzz6*>(host_wsum);
    std::vector<size_t> first_win(hi.size());
    for (size_t i = 0, w0 = 0; i < hi.size(); w0 += hi[i].fixed ? 1 : hi[i].windows, i++) first_win[i] = w0;
    auto tail = [&](size_t i) {
        host::Xyzz6 acc = host::infinity();
        if (hi[i].fixed) {  // the table rows already carry the 2^(c w) factors
            acc = host::canon(hs[first_win[i]]);
        } else {
            for (int w = (int)hi[i].windows - 1; w >= 0; w--) {
                for (uint32_t b = 0; b < hi[i].c; b++) acc = host::dbl(acc);
                acc = host::add(acc, host::canon(hs[first_win[i] + w]));
            }
        }
        host::to_jacobian_normalised(acc, out + 18 * item_of[i]);
    };
    const size_t cores = std::max(1u, std::thread::hardware_concurrency());
    const size_t nthreads = std::min<size_t>({hi.size() / 2, cores / 2, 32});
    if (nthreads <= 1) {
        for (size_t i = 0; i < hi.size(); i++) tail(i);
    } else {
        std::atomic<size_t> next{0};
        auto worker = [&] {
            for (size_t i; (i = next.fetch_add(1)) < hi.size();) tail(i);
        };
        std::vector<std::thread> pool;
        for (size_t t = 1; t < nthreads; t++) pool.emplace_back(worker);
        worker();
        for (std::thread& th : pool) th.join();
    }
    ctx->last_entries = entries;
    return OK;
}

}  // namespace mzk

namespace mzk {

// ---------------------------------------------------------------------------
// Allocation-free MSM for callers that cannot allocate device memory.
//
// Some hosts own every byte of device memory themselves: a framework that
// hands a custom operation its input and output buffers but no workspace, a
// runtime whose memory pool must not be bypassed, or code running where the
// CUDA allocator may not be called.  For them the MSM below takes its scratch
// from one file-scope device array of fixed size instead of cudaMalloc.  It
// serves n <= kNoAllocMaxN points with the window width clamped to [8, 12].
// Every GPU that loads this library holds the array (about 21 MB) until the
// process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocMaxN = size_t(1) << 16;
constexpr int kNoAllocMinC = 8, kNoAllocMaxC = 12;
constexpr uint32_t kNoAllocAccBlocks = 64;  // fixed accumulate grid (64 x 128 threads)
constexpr int kNoAllocMaxDevices = 64;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
// largest key count over the allowed widths: c = 12 gives 22 windows x 2048
constexpr size_t kNaKeys = 22 * 2048;
constexpr size_t kNaMaxWindows = 32;  // c = 8
constexpr size_t kNaAccThreads = (size_t)kNoAllocAccBlocks * kAccThreads;
constexpr size_t kNaCountsOff = 0;
constexpr size_t kNaOffsetsOff = kNaCountsOff + align256((kNaKeys + 1) * 4);
constexpr size_t kNaSortedOff = kNaOffsetsOff + align256((kNaKeys + 2) * 4);
constexpr size_t kNaBucketsOff = kNaSortedOff + align256(kNaMaxWindows * kNoAllocMaxN * 4);
constexpr size_t kNaPartialsOff = kNaBucketsOff + align256(kNaKeys * sizeof(Xyzz));
constexpr size_t kNaOwnerOff = kNaPartialsOff + align256(kNaAccThreads * 2 * sizeof(Xyzz));
constexpr size_t kNaRunOff = kNaOwnerOff + align256(kNaAccThreads * 4);
// running-sum groups of 2^kNoAllocGroupLog buckets (c >= 8)
constexpr int kNoAllocGroupLog = 4;
constexpr size_t kNaTotOff = kNaRunOff + align256((kNaKeys >> kNoAllocGroupLog) * sizeof(Xyzz));
constexpr size_t kNaPlanesOff = kNaTotOff + align256((kNaKeys >> kNoAllocGroupLog) * sizeof(Xyzz));
constexpr size_t kNaWsumOff = kNaPlanesOff + align256(kNaMaxWindows * 8 * sizeof(Xyzz));
constexpr size_t kNaScanOff = kNaWsumOff + align256(kNaMaxWindows * sizeof(Xyzz));
constexpr size_t kNaWinsOff = kNaScanOff + align256(64 * 4);
constexpr size_t kNaLongOff = kNaWinsOff + align256(kNaMaxWindows * sizeof(WinDev));
constexpr size_t kNaBytes = kNaLongOff + align256(16 + kNaAccThreads * sizeof(uint2));

// The scratch itself.  Host code must not use this name as a device address:
// on the host it is only a stand-in, so kernels get the pointer obtained from
// cudaGetSymbolAddress below.
__device__ __align__(256) unsigned char g_msm_noalloc_scratch[kNaBytes];

// one lock per device: each device has its own copy of the array
std::mutex g_noalloc_mu[kNoAllocMaxDevices];
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};
int g_noalloc_sms[kNoAllocMaxDevices] = {};

// exclusive scan into caller-provided tile sums (no allocation)
Status scan_u32_noalloc(const uint32_t* in, uint32_t* out, uint32_t len, uint32_t* sums, cudaStream_t st) {
    const uint32_t tiles = (len + kScanTile - 1) / kScanTile;
    k_scan_tiles<<<tiles, kScanThreads, 0, st>>>(in, out, len, sums);
    MZK_CUDA_CHECK(cudaGetLastError());
    k_scan_sums<<<1, kScanThreads, 0, st>>>(sums, tiles);
    MZK_CUDA_CHECK(cudaGetLastError());
    k_scan_add<<<tiles, kScanThreads, 0, st>>>(out, len, sums);
    MZK_CUDA_CHECK(cudaGetLastError());
    return OK;
}

Status msm_g1_noalloc_queued(unsigned char* base, int sms, const void* d_scalars, const void* d_bases, size_t n,
                             uint64_t* out18, cudaStream_t st);

Status msm_g1_noalloc(const void* d_scalars, const void* d_bases, size_t n, uint64_t* out18, cudaStream_t st) {
    std::memset(out18, 0, 18 * 8);
    if (n > kNoAllocMaxN) {
        set_error("mzk_msm_g1_noalloc: n = " + std::to_string(n) + " exceeds the fixed scratch limit of " +
                  std::to_string(kNoAllocMaxN) + " points; use mzk_msm_g1_device");
        return ERR_ARG;
    }
    if (n == 0) return OK;
    int dev = 0;
    MZK_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        set_error("mzk_msm_g1_noalloc: device index out of range");
        return ERR_ARG;
    }
    // one lock for this device's array: calls from several host threads take turns
    std::lock_guard<std::mutex> lock(g_noalloc_mu[dev]);
    if (!g_noalloc_ptr[dev]) {
        // set-up, once per device, with that device current
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_msm_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_error(std::string("mzk_msm_g1_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            return ERR_CUDA;
        }
        int sms = 0;
        MZK_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        g_noalloc_sms[dev] = sms;
        g_noalloc_ptr[dev] = p;
    }
    const Status s = msm_g1_noalloc_queued(static_cast<unsigned char*>(g_noalloc_ptr[dev]), g_noalloc_sms[dev],
                                           d_scalars, d_bases, n, out18, st);
    // a failure after work was queued: let that work finish before the lock
    // is released, so the next call cannot race with it on the array
    if (s != OK) cudaStreamSynchronize(st);
    return s;
}

Status msm_g1_noalloc_queued(unsigned char* base, int sms, const void* d_scalars, const void* d_bases, size_t n,
                             uint64_t* out18, cudaStream_t st) {
    int c = msm_pick_window(n);
    c = c < kNoAllocMinC ? kNoAllocMinC : (c > kNoAllocMaxC ? kNoAllocMaxC : c);
    const MsmShape sh = make_shape(c, kNoAllocGroupLog);
    uint32_t* counts = reinterpret_cast<uint32_t*>(base + kNaCountsOff);
    uint32_t* offsets = reinterpret_cast<uint32_t*>(base + kNaOffsetsOff);
    uint32_t* sorted = reinterpret_cast<uint32_t*>(base + kNaSortedOff);
    Xyzz* buckets = reinterpret_cast<Xyzz*>(base + kNaBucketsOff);
    Xyzz* partials = reinterpret_cast<Xyzz*>(base + kNaPartialsOff);
    int* owner = reinterpret_cast<int*>(base + kNaOwnerOff);
    Xyzz* run = reinterpret_cast<Xyzz*>(base + kNaRunOff);
    Xyzz* tot = reinterpret_cast<Xyzz*>(base + kNaTotOff);
    Xyzz* planes = reinterpret_cast<Xyzz*>(base + kNaPlanesOff);
    Xyzz* wsum = reinterpret_cast<Xyzz*>(base + kNaWsumOff);
    uint32_t* scan_sums = reinterpret_cast<uint32_t*>(base + kNaScanOff);

    const Fr* sc = static_cast<const Fr*>(d_scalars);
    const Affine* ba = static_cast<const Affine*>(d_bases);
    const int pt_threads = 256;
    const uint32_t pt_blocks =
        (uint32_t)std::min<size_t>((n + pt_threads - 1) / pt_threads, (size_t)sms * 16);
    // the array keeps the previous call's contents: zero the counters
    MZK_CUDA_CHECK(cudaMemsetAsync(counts, 0, ((size_t)sh.keys + 1) * 4, st));
    k_histogram<<<pt_blocks, pt_threads, 0, st>>>(sc, n, sh.c, sh.windows, sh.nb, counts, nullptr);
    MZK_CUDA_CHECK(cudaGetLastError());
    MZK_CUDA_CHECK(cudaMemsetAsync(offsets, 0, 4, st));
    MZK_TRY(scan_u32_noalloc(counts, offsets + 1, sh.keys + 1, scan_sums, st));
    k_scatter<<<pt_blocks, pt_threads, 0, st>>>(sc, n, sh.c, sh.windows, sh.nb, offsets + 1, sorted);
    MZK_CUDA_CHECK(cudaGetLastError());
    k_accumulate<<<kNoAllocAccBlocks, kAccThreads, 0, st>>>(ba, sorted, offsets, sh.keys, buckets, partials, owner);
    MZK_CUDA_CHECK(cudaGetLastError());
    uint32_t* long_count = reinterpret_cast<uint32_t*>(base + kNaLongOff);
    uint2* long_list = reinterpret_cast<uint2*>(base + kNaLongOff + 16);
    MZK_CUDA_CHECK(cudaMemsetAsync(long_count, 0, 4, st));
    k_fixup<<<kNoAllocAccBlocks, kAccThreads, 0, st>>>(offsets, sh.keys, partials, owner, buckets, long_count,
                                                       long_list);
    MZK_CUDA_CHECK(cudaGetLastError());
    k_fixup_long<<<kNoAllocAccBlocks, kReduceThreads, kReduceThreads * sizeof(Xyzz), st>>>(owner, partials,
                                                                                          long_count, long_list,
                                                                                          buckets);
    MZK_CUDA_CHECK(cudaGetLastError());
    // window table (a copy from pageable memory is staged before the call returns)
    std::vector<WinDev> wins;
    uint64_t total_groups = 0, slots = 0;
    append_windows(sh, 0, wins, total_groups, slots);
    WinDev* d_wins = reinterpret_cast<WinDev*>(base + kNaWinsOff);
    MZK_CUDA_CHECK(cudaMemcpyAsync(d_wins, wins.data(), wins.size() * sizeof(WinDev), cudaMemcpyHostToDevice, st));
    const BucketSets sets{{buckets}, {offsets}, 1};
    MZK_CUDA_CHECK(launch_reduce(sets, d_wins, (uint32_t)wins.size(), total_groups, slots, 1, run, tot, planes, planes,
                                 wsum, nullptr, st));
    // window sums to host memory owned by this function (no pinned allocation)
    host::Xyzz6 hs[kNaMaxWindows];
    MZK_CUDA_CHECK(cudaMemcpyAsync(hs, wsum, (size_t)sh.windows * sizeof(Xyzz), cudaMemcpyDeviceToHost, st));
    MZK_CUDA_CHECK(cudaStreamSynchronize(st));
    host::Xyzz6 acc = host::infinity();
    for (int w = sh.windows - 1; w >= 0; w--) {
        for (int b = 0; b < sh.c; b++) acc = host::dbl(acc);
        acc = host::add(acc, host::canon(hs[w]));
    }
    host::to_jacobian_normalised(acc, out18);
    return OK;
}

}  // namespace

}  // namespace mzk

extern "C" int mzk_msm_g1_noalloc(const uint64_t* d_scalars, const uint64_t* d_bases, size_t n, uint64_t out[18],
                                  void* stream) {
    if (!out || (n && (!d_scalars || !d_bases))) {
        mzk::set_error("mzk_msm_g1_noalloc: null pointer");
        return mzk::ERR_ARG;
    }
    return mzk::msm_g1_noalloc(d_scalars, d_bases, n, out, static_cast<cudaStream_t>(stream));
}
