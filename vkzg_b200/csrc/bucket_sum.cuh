// Bucket sums with batched affine additions.
//
// The reference accumulates each bucket serially in Jacobian coordinates
// (k_phase_a.comp:37-42, k_phase_b_split.comp:43-55: madd-2007-bl, 11 Fp
// multiplies per point).  Here the points of the 128 buckets of one MSM output
// are summed in pairwise rounds: round r adds element pairs
// (2i, 2i+1) of every bucket, so a round is a batch of independent affine
// additions
//   lambda = (y2 - y1) / (x2 - x1),  x3 = lambda^2 - x1 - x2,  y3 = lambda (x1 - x3) - y1
// whose denominators share one inversion (Montgomery's trick across a warp:
// per-lane prefix products, shuffle scans, one divstep inversion).  That is 6
// multiplies per addition plus the amortised inversion.  Doubling (equal
// points), cancellation (P + -P) and the point at infinity ((0,0)) are handled
// per pair, so any input is summed exactly.
//
// Layout: each warp owns two global scratch buffers.  Round 1 reads the source
// points through a loader, later rounds ping-pong between the buffers.  After
// the last round, bucket k's sum is at buf[base[k]] when cnt[k] == 1 (cnt[k] == 0:
// empty bucket, infinity).
#pragma once

#include "device_util.cuh"

namespace vkzg {

#ifndef VKZG_BA_THREADS
#define VKZG_BA_THREADS 256
#endif
constexpr int kBAThreads = VKZG_BA_THREADS; // threads of the batch-affine phase kernels
constexpr int kBABuckets = 128; // buckets per MSM output

// kind: 0 general, 1 doubling, 2 result = a, 3 result = b, 4 result = infinity
__device__ __forceinline__ int pair_kind(const G1A &a, const G1A &b) {
    if (g1a_is_identity(a)) return 3;
    if (g1a_is_identity(b)) return 2;
    if (!fp_eq(a.x, b.x)) return 0;
    return fp_eq(a.y, b.y) ? 1 : 4; // y1 == -y2 (y == 0 has no point on G1)
}

__device__ __forceinline__ Fp pair_denominator(const G1A &a, const G1A &b, int kind) {
    if (kind == 0) return fp_sub(b.x, a.x);
    if (kind == 1) return fp_dbl(a.y);
    return fp_one();
}

// pair_denominator(a, b, pair_kind(a, b)) from the x coordinates when both are
// nonzero and differ (then neither point is (0, 0) and the pair is a general
// addition); otherwise from the full points, which load_a / load_b return.
// The running products of pass 1 need nothing else, so they read 48 bytes per
// point instead of 96.
template <class LoadA, class LoadB>
__device__ __forceinline__ Fp pair_denominator_x(const Fp &ax, const Fp &bx, LoadA load_a, LoadB load_b) {
    if (!fp_is_zero(ax) && !fp_is_zero(bx) && !fp_eq(ax, bx)) return fp_sub(bx, ax);
    const G1A a = load_a(), b = load_b();
    return pair_denominator(a, b, pair_kind(a, b));
}

// INL: the products inlined instead of out-of-line calls
template <bool INL>
__device__ __forceinline__ Fp pmul(const Fp &a, const Fp &b) {
    if constexpr (INL) return fp_mul_inl(a, b);
    else return fp_mul(a, b);
}
template <bool INL>
__device__ __forceinline__ Fp psqr(const Fp &a) {
    if constexpr (INL) return fp_sqr_inl(a);
    else return fp_sqr(a);
}

template <bool INL = false>
__device__ __forceinline__ G1A pair_result(const G1A &a, const G1A &b, int kind, const Fp &inv_den) {
    if (kind == 2) return a;
    if (kind == 3) return b;
    if (kind == 4) {
        G1A z;
        z.x = fp_zero();
        z.y = fp_zero();
        return z;
    }
    Fp num;
    if (kind == 0) {
        num = fp_sub(b.y, a.y);
    } else {
        const Fp xx = psqr<INL>(a.x);
        num = fp_add(fp_dbl(xx), xx);
    }
    const Fp lam = pmul<INL>(num, inv_den);
    G1A r;
    r.x = fp_sub(fp_sub(psqr<INL>(lam), a.x), b.x);
    r.y = fp_sub(pmul<INL>(lam, fp_sub(a.x, r.x)), a.y);
    return r;
}

// bucket containing pair q: largest k with pscan[k] <= q
template <int NB>
__device__ __forceinline__ int ba_bucket_of(const uint32_t *pscan, uint32_t q) {
    int lo = 0, hi = NB - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pscan[mid] <= q) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ------------------------------------------------------------ warp-level form
// One warp sums a bucket space of NB buckets on its own (the 128 buckets of
// NB / 128 MSM outputs side by side): pairwise rounds as above, and each
// round's denominators share one inversion per warp (prefix and suffix products
// by shuffles, one divstep inversion on one lane), so warps never wait on each
// other.  The inversion runs on one lane but costs a whole warp's issue slots,
// which is why several outputs share a bucket space: the more pairs a round
// holds, the smaller that fixed share.  The per-pair prefix products go to the
// warp's global scratch in word-major order (word w of element s of lane l at
// [(s * 12 + w) * 32 + l]), which keeps every access a full 128-byte line.

template <int NB>
struct WarpBuckets {
    uint32_t cnt[NB];
    uint32_t pscan[NB + 1];
    uint32_t base[2][NB + 1];
};

__device__ __forceinline__ Fp fp_shfl_up(const Fp &a, int d) {
    Fp r;
#pragma unroll
    for (int i = 0; i < 12; i++) r.v[i] = __shfl_up_sync(0xffffffffu, a.v[i], d);
    return r;
}
__device__ __forceinline__ Fp fp_shfl_down(const Fp &a, int d) {
    Fp r;
#pragma unroll
    for (int i = 0; i < 12; i++) r.v[i] = __shfl_down_sync(0xffffffffu, a.v[i], d);
    return r;
}
__device__ __forceinline__ Fp fp_shfl_xor(const Fp &a, int mask) {
    Fp r;
#pragma unroll
    for (int i = 0; i < 12; i++) r.v[i] = __shfl_xor_sync(0xffffffffu, a.v[i], mask);
    return r;
}
__device__ __forceinline__ Fp fp_shfl(const Fp &a, int src) {
    Fp r;
#pragma unroll
    for (int i = 0; i < 12; i++) r.v[i] = __shfl_sync(0xffffffffu, a.v[i], src);
    return r;
}

// 1 / a for one value per lane (none zero).
__device__ inline Fp warp_batch_inverse_fp(const Fp &a) {
    const int lane = threadIdx.x & 31;
    Fp pre = a, suf = a;
#pragma unroll 1
    for (int d = 1; d < 32; d <<= 1) {
        const Fp o = fp_shfl_up(pre, d);
        if (lane >= d) pre = fp_mul(pre, o);
        const Fp u = fp_shfl_down(suf, d);
        if (lane + d < 32) suf = fp_mul(suf, u);
    }
    Fp tot = fp_shfl(pre, 31);
    if (lane == 0) tot = fp_inv_fast(tot);
    tot = fp_shfl(tot, 0);
    Fp pre_x = fp_shfl_up(pre, 1), suf_x = fp_shfl_down(suf, 1);
    if (lane == 0) pre_x = fp_one();
    if (lane == 31) suf_x = fp_one();
    return fp_mul(fp_mul(tot, pre_x), suf_x);
}

__device__ __forceinline__ void wb_store_pre(uint32_t *pre, int s, const Fp &v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int w = 0; w < 12; w++) pre[(s * 12 + w) * 32 + lane] = v.v[w];
}
__device__ __forceinline__ Fp wb_load_pre(const uint32_t *pre, int s) {
    const int lane = threadIdx.x & 31;
    Fp v;
#pragma unroll
    for (int w = 0; w < 12; w++) v.v[w] = pre[(s * 12 + w) * 32 + lane];
    return v;
}

// pair and next-element scans over the NB buckets: NB / 32 buckets per lane
template <int NB>
__device__ inline void wb_plan_round(WarpBuckets<NB> &wb, int next) {
    static_assert(NB % 32 == 0, "whole buckets per lane");
    constexpr int per = NB / 32;
    const int lane = threadIdx.x & 31;
    uint32_t p = 0, e = 0;
#pragma unroll
    for (int k = lane * per; k < lane * per + per; k++) {
        p += wb.cnt[k] >> 1;
        e += (wb.cnt[k] + 1) >> 1;
    }
    uint32_t ip = p, ie = e;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t op = __shfl_up_sync(0xffffffffu, ip, d), oe = __shfl_up_sync(0xffffffffu, ie, d);
        if (lane >= d) {
            ip += op;
            ie += oe;
        }
    }
    p = ip - p;
    e = ie - e;
#pragma unroll
    for (int k = lane * per; k < lane * per + per; k++) {
        wb.pscan[k] = p;
        wb.base[next][k] = e;
        p += wb.cnt[k] >> 1;
        e += (wb.cnt[k] + 1) >> 1;
    }
    if (lane == 31) {
        wb.pscan[NB] = ip;
        wb.base[next][NB] = ie;
    }
    __syncwarp();
}

template <int NB, typename Src>
__device__ void wb_round(WarpBuckets<NB> &wb, int next, const Src &src, G1A *dst, uint32_t *pre) {
    const int lane = threadIdx.x & 31;
    const uint32_t P = wb.pscan[NB];
    Fp acc = fp_one();
    int s = 0;
    for (uint32_t q = lane; q < P; q += 32, s++) {
        const int k = ba_bucket_of<NB>(wb.pscan, q);
        const uint32_t i = q - wb.pscan[k];
        const G1A a = src(k, 2 * i), b = src(k, 2 * i + 1);
        wb_store_pre(pre, s, acc);
        acc = fp_mul(acc, pair_denominator(a, b, pair_kind(a, b)));
    }
    Fp inv = warp_batch_inverse_fp(acc);
    for (int t = s - 1; t >= 0; t--) {
        const uint32_t q = lane + (uint32_t)t * 32;
        const int k = ba_bucket_of<NB>(wb.pscan, q);
        const uint32_t i = q - wb.pscan[k];
        const G1A a = src(k, 2 * i), b = src(k, 2 * i + 1);
        const int kind = pair_kind(a, b);
        const Fp den = pair_denominator(a, b, kind);
        const Fp inv_den = fp_mul(inv, wb_load_pre(pre, t));
        inv = fp_mul(inv, den);
        st_vec(&dst[wb.base[next][k] + i], pair_result(a, b, kind, inv_den));
    }
    for (int k = lane; k < NB; k += 32) {
        const uint32_t c = wb.cnt[k];
        if (c & 1u) st_vec(&dst[wb.base[next][k] + (c >> 1)], src(k, c - 1));
    }
    __syncwarp();
    for (int k = lane; k < NB; k += 32) wb.cnt[k] = (wb.cnt[k] + 1) >> 1;
    __syncwarp();
}

// Sums the warp's NB buckets (wb.cnt = initial counts, at most 16 * NB points).
// buf0 >= NB / 128 * 1088 points, buf1 >= NB / 128 * 608, pre >= NB * 3 * 32
// words (NB / 4 pairs per lane).  Round 1 reads src0 only, so wb.base[1] may
// hold src0's own offsets.  Returns the buffer of sums, offsets in
// wb.base[result_slot].
template <int NB, typename Src0>
__device__ G1A *wb_bucket_sums(WarpBuckets<NB> &wb, const Src0 &src0, G1A *buf0, G1A *buf1, uint32_t *pre,
                               int &result_slot) {
    wb_plan_round(wb, 0);
    wb_round(wb, 0, src0, buf0, pre);
    G1A *cur = buf0, *other = buf1;
    int slot = 0;
    for (int round = 0; round < 16; round++) {
        bool more = false;
        for (int k = threadIdx.x & 31; k < NB; k += 32) more |= wb.cnt[k] > 1;
        if (!__any_sync(0xffffffffu, more)) break;
        wb_plan_round(wb, slot ^ 1);
        const G1A *from = cur;
        const uint32_t *fb = wb.base[slot];
        auto src = [from, fb](int k, uint32_t i) { return ld_vec(&from[fb[k] + i]); };
        wb_round(wb, slot ^ 1, src, other, pre);
        slot ^= 1;
        G1A *t = cur;
        cur = other;
        other = t;
    }
    result_slot = slot;
    return cur;
}


} // namespace vkzg
