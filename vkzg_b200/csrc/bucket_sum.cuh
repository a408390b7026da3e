// Bucket sums with batched affine additions.
//
// The reference accumulates each bucket serially in Jacobian coordinates
// (k_phase_a.comp:37-42, k_phase_b_split.comp:43-55: madd-2007-bl, 11 Fp
// multiplies per point).  Here the points of NB buckets (G MSM outputs x 128
// buckets) are summed in pairwise rounds: round r adds element pairs
// (2i, 2i+1) of every bucket, so a round is a batch of independent affine
// additions
//   lambda = (y2 - y1) / (x2 - x1),  x3 = lambda^2 - x1 - x2,  y3 = lambda (x1 - x3) - y1
// whose denominators share one inversion (Montgomery's trick across the block:
// per-thread prefix products, a block product tree, one divstep inversion).
// That is 6 multiplies per addition plus the amortised inversion; the more
// outputs a block carries, the more additions share each round's inversion
// and product-tree latency.  Doubling (equal points), cancellation (P + -P)
// and the point at infinity ((0,0)) are handled per pair, so any input is
// summed exactly.
//
// Layout: the block owns two global scratch buffers.  Round 1 reads the source
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

template <int NB, int NT = kBAThreads>
struct BucketSumShared {
    uint32_t cnt[NB];
    uint32_t pscan[NB + 1];   // exclusive scan of pairs per bucket
    uint32_t base[2][NB + 1]; // element offsets of the current / next list
    uint32_t part[2][NT];
    Fp tree[2 * NT];
};

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
        const Fp xx = fp_sqr(a.x);
        num = fp_add(fp_dbl(xx), xx);
    }
    const Fp lam = fp_mul(num, inv_den);
    G1A r;
    r.x = fp_sub(fp_sub(fp_sqr(lam), a.x), b.x);
    r.y = fp_sub(fp_mul(lam, fp_sub(a.x, r.x)), a.y);
    return r;
}

// Exclusive scans of pair counts and of next-round element counts over the NB
// buckets: each thread sums a contiguous run, one thread scans the partials.
template <int NB, int NT>
__device__ void ba_plan_round(BucketSumShared<NB, NT> &sh, int next) {
    constexpr int per = (NB + NT - 1) / NT;
    const int t = threadIdx.x, lo = t * per;
    uint32_t p = 0, e = 0;
    for (int k = lo; k < lo + per && k < NB; k++) {
        p += sh.cnt[k] >> 1;
        e += (sh.cnt[k] + 1) >> 1;
    }
    sh.part[0][t] = p;
    sh.part[1][t] = e;
    __syncthreads();
    if (t == 0) {
        uint32_t ap = 0, ae = 0;
        for (int q = 0; q < NT; q++) {
            const uint32_t xp = sh.part[0][q], xe = sh.part[1][q];
            sh.part[0][q] = ap;
            sh.part[1][q] = ae;
            ap += xp;
            ae += xe;
        }
        sh.pscan[NB] = ap;
        sh.base[next][NB] = ae;
    }
    __syncthreads();
    p = sh.part[0][t];
    e = sh.part[1][t];
    for (int k = lo; k < lo + per && k < NB; k++) {
        sh.pscan[k] = p;
        sh.base[next][k] = e;
        p += sh.cnt[k] >> 1;
        e += (sh.cnt[k] + 1) >> 1;
    }
    __syncthreads();
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

// One round: pairs of the current list (loaded by `src(k, i)`) into `dst`.
// MAXP bounds the pairs per thread (P <= MAXP * kBAThreads).
template <int NB, int NT, int MAXP, typename Src>
__device__ void ba_round(BucketSumShared<NB, NT> &sh, int next, const Src &src, G1A *dst) {
    const uint32_t P = sh.pscan[NB];
    Fp pre[MAXP];
    Fp acc = fp_one();
    int s = 0;
    for (uint32_t q = threadIdx.x; q < P; q += NT, s++) {
        const int k = ba_bucket_of<NB>(sh.pscan, q);
        const uint32_t i = q - sh.pscan[k];
        const G1A a = src(k, 2 * i), b = src(k, 2 * i + 1);
        pre[s] = acc;
        acc = fp_mul(acc, pair_denominator(a, b, pair_kind(a, b)));
    }
    Fp inv = block_batch_inverse_fp<NT>(acc, sh.tree);
    for (int t = s - 1; t >= 0; t--) {
        const uint32_t q = threadIdx.x + (uint32_t)t * NT;
        const int k = ba_bucket_of<NB>(sh.pscan, q);
        const uint32_t i = q - sh.pscan[k];
        const G1A a = src(k, 2 * i), b = src(k, 2 * i + 1);
        const int kind = pair_kind(a, b);
        const Fp den = pair_denominator(a, b, kind);
        const Fp inv_den = fp_mul(inv, pre[t]);
        inv = fp_mul(inv, den);
        st_vec(&dst[sh.base[next][k] + i], pair_result(a, b, kind, inv_den));
    }
    // odd leftovers move to the end of their bucket's next list
    for (int k = threadIdx.x; k < NB; k += NT) {
        const uint32_t c = sh.cnt[k];
        if (c & 1u) st_vec(&dst[sh.base[next][k] + (c >> 1)], src(k, c - 1));
    }
}

template <int NB, int NT>
__device__ __forceinline__ void ba_halve_counts(BucketSumShared<NB, NT> &sh) {
    __syncthreads();
    for (int k = threadIdx.x; k < NB; k += NT) sh.cnt[k] = (sh.cnt[k] + 1) >> 1;
    __syncthreads();
}

template <int NB, int NT>
__device__ bool ba_any_pair(const BucketSumShared<NB, NT> &sh) {
    return __syncthreads_or(([&] {
        bool m = false;
        for (int k = threadIdx.x; k < NB; k += NT) m |= sh.cnt[k] > 1;
        return m;
    })());
}

// Sums every bucket.  sh.cnt must hold the initial counts; MAXP0 bounds the
// round-1 pairs per thread.  buf0 holds the round-1 output (<= (n + NB) / 2
// points), buf1 the round-2 output.  Returns the buffer holding the sums; their
// offsets are in sh.base[result_slot].
template <int NB, int MAXP0, int NT, typename Src0>
__device__ G1A *ba_bucket_sums(BucketSumShared<NB, NT> &sh, const Src0 &src0, G1A *buf0, G1A *buf1,
                               int &result_slot) {
    // round 1 always runs, so singletons are materialised in buf0 too
    ba_plan_round(sh, 0);
    ba_round<NB, NT, MAXP0>(sh, 0, src0, buf0);
    ba_halve_counts(sh);
    G1A *cur = buf0, *other = buf1;
    int slot = 0;
    for (int round = 0; round < 16; round++) {
        if (!ba_any_pair(sh)) break;
        ba_plan_round(sh, slot ^ 1);
        const G1A *from = cur;
        const uint32_t *fb = sh.base[slot];
        auto src = [from, fb](int k, uint32_t i) { return ld_vec(&from[fb[k] + i]); };
        ba_round<NB, NT, MAXP0>(sh, slot ^ 1, src, other);
        ba_halve_counts(sh);
        slot ^= 1;
        G1A *t = cur;
        cur = other;
        other = t;
    }
    result_slot = slot;
    return cur;
}

} // namespace vkzg
