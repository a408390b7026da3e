// FK20 cell-proof pipeline (reference: src/vkzg.cpp:899-1039 and the k_*.comp
// kernels it dispatches).  Stages:
//   1 k_blob_to_coeffs   blob bytes -> Fr, canonicity flag, inverse NTT-4096 in
//                        shared memory, x 1/4096            (k_blob_to_fr, k_ntt_pass x2)
//   2 k_circulant        64 circulant columns, forward NTT-128, canonical
//                        scalars coeffs[j][i]               (k_build_circulant)
//   3 k_phase_a          per output j: signed-digit recode, bucket sort in
//                        shared memory, fixed-base bucket accumulation over the
//                        position table                     (k_phase_a_sort, k_phase_a)
//   4 k_reduce           sum_k k * B_k, 8 lanes per output  (k_bucket_reduce)
//   5 k_ladder (fold)    u+- = u[j] +- u[j+64], and for plans 3-4 twice more on
//                        the cyclic half: the convolution's parts (k_fold_ladder)
//   6 k_ladder           L[j][d] = 2^(8d) v[j], d < 16      (k_ladder, d < 32: the
//                        taps are split as k1 + k2 z^2 and slots 16..31 read phi(L))
//   7 k_normalize        Jacobian -> affine, block batch inversion, phi images
//                                                           (k_normalize)
//   8 k_phase_b          split-circulant bucket MSM with the fixed taps (k_phase_b_split)
//   4'k_reduce
//   9 k_finish           unfold the parts (C+ +- C-), normalise, compress, write slot brev7(a);
//                        plans 3-4: k_finish_horner, phase B's Horner step first
//                                                           (k_combine_split, k_normalize, k_compress_proofs)
#include "bucket_sum.cuh"
#include "device_util.cuh"
#include "kernels.h"

#include <algorithm>
#include <cstring>
#include <vector>

namespace vkzg {

// ---------------------------------------------------------------- stage 1
constexpr int kNttThreads = 512;

__global__ void __launch_bounds__(kNttThreads) k_blob_to_coeffs(const uint8_t *__restrict__ blobs, Fr *coeffs,
                                                                 const Fr *__restrict__ roots_inv,
                                                                 const Fr *__restrict__ inv_blob_r2, uint32_t *err) {
    extern __shared__ uint4 smem_raw[];
    Fr *s = reinterpret_cast<Fr *>(smem_raw);
    const int b = blockIdx.x;
    const uint8_t *src = blobs + (size_t)b * kBlobBytes;
    bool bad = false;
    // The blob holds f(w_4096^brev12(i)) at slot i: already the bit-reversed
    // order a DIT transform wants.
    for (int i = threadIdx.x; i < kBlobElems; i += kNttThreads) {
        const uint4 *p = reinterpret_cast<const uint4 *>(src + 32 * (size_t)i);
        const uint4 lo = p[0], hi = p[1];
        Fr v;
        v.v[7] = bswap32(lo.x); v.v[6] = bswap32(lo.y); v.v[5] = bswap32(lo.z); v.v[4] = bswap32(lo.w);
        v.v[3] = bswap32(hi.x); v.v[2] = bswap32(hi.y); v.v[1] = bswap32(hi.z); v.v[0] = bswap32(hi.w);
        bad |= !fr_is_canonical(v);
        st_vec(&s[i], fr_from_canonical(v));
    }
    if (bad) atomicOr(&err[b], 1u);
    __syncthreads();
    smem_dit<kNttThreads>(s, 12, 1, 2, 4096, roots_inv);
    const Fr scale = ldg_vec(inv_blob_r2);
    Fr *dst = coeffs + (size_t)b * kBlobElems;
    for (int i = threadIdx.x; i < kBlobElems; i += kNttThreads) st_vec(&dst[i], fr_mul(ld_vec(&s[i]), scale));
}

// ---------------------------------------------------------------- stage 2
// c_i[0] = f[4095-i]; c_i[128-j'] = f[4095-i-64j'] for j' = 1..62; zero
// elsewhere (k_build_circulant.comp:31-41).  8 columns per block.
constexpr int kCircCols = 8;
__global__ void __launch_bounds__(kCircCols * 64) k_circulant(const Fr *__restrict__ coeffs, Fr *scalars,
                                                             const Fr *__restrict__ roots_fwd) {
    __shared__ Fr s[kCircCols * kCells];
    const int b = blockIdx.y, i0 = blockIdx.x * kCircCols;
    const Fr *f = coeffs + (size_t)b * kBlobElems;
    for (int q = threadIdx.x; q < kCircCols * kCells; q += blockDim.x) {
        const int c = q >> 7, t = q & 127, i = i0 + c;
        Fr v = fr_zero();
        if (t == 0) v = ld_vec(&f[kBlobElems - 1 - i]);
        else if (t >= 66) v = ld_vec(&f[kBlobElems - 1 - i - (kCells - t) * kCellElems]);
        st_vec(&s[q], v);
    }
    __syncthreads();
    smem_dif<kCircCols * 64>(s, 7, kCircCols, 128, 2, roots_fwd);
    // s[c][pos] holds coeffs at j = brev7(pos); store canonical coeffs[j][i]
    Fr *out = scalars + (size_t)b * kCells * kCellElems;
    for (int q = threadIdx.x; q < kCircCols * kCells; q += blockDim.x) {
        const int c = q >> 7, pos = q & 127, j = (int)brev_bits((uint32_t)pos, 7);
        st_vec(&out[j * kCellElems + i0 + c], fr_to_canonical(ld_vec(&s[q])));
    }
}

// ---------------------------------------------------------------- stage 3
// Signed base-256 digit dd of a canonical scalar (k_phase_a_sort.comp:31-40).
__device__ __forceinline__ int recode_digit(const Fr &c, int dd, int &carry) {
    int v = (int)((c.v[dd >> 2] >> ((dd & 3) * 8)) & 0xffu) + carry;
    carry = 0;
    if (v > kBuckets) {
        v -= 2 * kBuckets;
        carry = 1;
    }
    return v;
}

// Ranks buckets by descending load so that each warp's threads get similar
// trip counts (the reference's load-class ordering, k_phase_a_sort.comp:74-101).
__device__ __forceinline__ void rank_buckets(const uint32_t *cnt, uint8_t *perm) {
    const int k = threadIdx.x;
    const uint32_t mine = cnt[k];
    int rank = 0;
    for (int q = 0; q < kBuckets; q++) {
        const uint32_t o = cnt[q];
        rank += (o > mine) || (o == mine && q < k);
    }
    perm[rank] = (uint8_t)k;
}

__global__ void __launch_bounds__(kBuckets) k_phase_a(const Fr *__restrict__ scalars, const G1A *__restrict__ pos,
                                                     G1J *buckets) {
    __shared__ uint32_t cnt[kBuckets], start[kBuckets + 1];
    __shared__ uint16_t items[kCellElems * kDigits];
    __shared__ uint8_t perm[kBuckets];
    const int j = blockIdx.x, b = blockIdx.y, tid = threadIdx.x;
    cnt[tid] = 0;
    __syncthreads();
    Fr sc;
    if (tid < kCellElems) {
        sc = ld_vec(&scalars[((size_t)b * kCells + j) * kCellElems + tid]);
        int carry = 0;
        for (int dd = 0; dd < kDigits; dd++) {
            const int v = recode_digit(sc, dd, carry);
            if (v) atomicAdd(&cnt[abs(v) - 1], 1u);
        }
    }
    __syncthreads();
    if (tid == 0) {
        uint32_t acc = 0;
        for (int k = 0; k < kBuckets; k++) {
            start[k] = acc;
            acc += cnt[k];
        }
        start[kBuckets] = acc;
    }
    rank_buckets(cnt, perm);
    __syncthreads();
    cnt[tid] = start[tid];
    __syncthreads();
    if (tid < kCellElems) {
        int carry = 0;
        for (int dd = 0; dd < kDigits; dd++) {
            const int v = recode_digit(sc, dd, carry);
            if (v) {
                const uint32_t slot = atomicAdd(&cnt[abs(v) - 1], 1u);
                items[slot] = (uint16_t)((tid << 6) | (dd << 1) | (v < 0 ? 1 : 0));
            }
        }
    }
    __syncthreads();
    const int bucket = perm[tid];
    const G1A *tj = pos + (size_t)j * kCellElems * kDigits;
    G1J acc = g1_identity();
    for (uint32_t it = start[bucket]; it < start[bucket + 1]; it++) {
        const uint32_t packed = items[it];
        G1A pt = ldg_vec(&tj[(packed >> 6) * kDigits + ((packed >> 1) & 31u)]);
        if (packed & 1u) pt.y = fp_neg(pt.y);
        acc = g1_madd(acc, pt);
    }
    st_vec(&buckets[((size_t)b * kCells + j) * kBuckets + bucket], acc);
}

// ---------------------------------------------------------------- stage 4
// out[o] = sum_{k=1..128} k * B[o][k-1] with 8 lanes per output: lane l runs
// the serial running sum over buckets [16l, 16l+16) giving S_l = sum B and
// W_l = sum (k - 16l + 1) B; then total = sum_l W_l + 16 * sum_l l * S_l
// (the decomposition of field.glsl.inc:478-517), the cross-lane part done by
// lane 0 from shared memory so that only two points per thread stay live.
constexpr int kReduceLanes = 8;
constexpr int kReduceThreads = 128;
__global__ void __launch_bounds__(kReduceThreads) k_reduce(const G1J *__restrict__ buckets, G1J *out, int n_outputs) {
    __shared__ G1J sh_s[kReduceThreads], sh_w[kReduceThreads];
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int o = gid / kReduceLanes, lane = gid % kReduceLanes;
    constexpr int per = kBuckets / kReduceLanes;
    G1J s = g1_identity(), w = g1_identity();
    if (o < n_outputs) {
        const G1J *bk = buckets + (size_t)o * kBuckets + lane * per;
        for (int k = per - 1; k >= 0; k--) {
            s = g1_add(s, ld_vec(&bk[k]));
            w = g1_add(w, s);
        }
    }
    st_vec(&sh_s[threadIdx.x], s);
    st_vec(&sh_w[threadIdx.x], w);
    __syncthreads();
    if (lane != 0 || o >= n_outputs) return;
    // running sums over lanes 7..1: acc = sum_l l * S_l
    G1J run = g1_identity(), acc = g1_identity();
    for (int l = kReduceLanes - 1; l >= 1; l--) {
        run = g1_add(run, ld_vec(&sh_s[threadIdx.x + l]));
        acc = g1_add(acc, run);
        w = g1_add(w, ld_vec(&sh_w[threadIdx.x + l]));
    }
    for (int q = 0; q < 4; q++) acc = g1_dbl(acc); // x 16
    st_vec(&out[o], g1_add(w, acc));
}

// ---------------------------------------------------------------- stages 5-6
// One block per blob, one thread per point.  First the parts of phase B's
// convolution (PartLayout) in shared memory: level l folds the cyclic vector v
// of 2m = 256 >> l points into v[j] + v[j + m] (the next cyclic vector, slots
// [0, m)) and v[j] - v[j + m] (the negacyclic part, slots [m, 2m)); one level is
// the reference's split of the circulant, applied to u before the ladder
// instead of to every ladder row.  Then each thread doubles its folded point
// along the ladder L[j][d] = 2^(8d) v[j], d < kLadderDigits.  The folded points
// stay in shared memory: nothing else reads them.
//
// One level of butterflies over v[0, 2m): thread t < m writes v[t] + v[t + m],
// thread m <= t < 2m writes v[t - m] - v[t], so that a level costs one addition
// of latency rather than two.
__device__ __forceinline__ void butterfly_level(G1J *v, int t, int m) {
    G1J r;
    if (t < 2 * m) {
        const int j = t < m ? t : t - m;
        const G1J y = ld_vec(&v[j + m]);
        r = g1_add(ld_vec(&v[j]), t < m ? y : g1_neg(y));
    }
    __syncthreads();
    if (t < 2 * m) st_vec(&v[t], r);
    __syncthreads();
}

__global__ void __launch_bounds__(kCells) k_ladder(const G1J *__restrict__ u, G1J *ladder, int levels) {
    __shared__ G1J v[kCells];
    const int b = blockIdx.x, t = threadIdx.x;
    st_vec(&v[t], ld_vec(&u[(size_t)b * kCells + t]));
    __syncthreads();
    for (int l = 1; l <= levels; l++) butterfly_level(v, t, kCells >> l);
    G1J acc = ld_vec(&v[t]);
    G1J *dst = ladder + ((size_t)b * kCells + t) * kLadderDigits;
    for (int d = 0; d < kLadderDigits; d++) {
        st_vec(&dst[d], acc);
        if (d + 1 < kLadderDigits)
#pragma unroll 1
            for (int q = 0; q < 8; q++) acc = g1_dbl_inl(acc);
    }
}

// ---------------------------------------------------------------- stage 7
constexpr int kNormThreads = 256;
__global__ void __launch_bounds__(kNormThreads) k_normalize(const G1J *__restrict__ in, G1A *out, int n_points) {
    __shared__ Fp tree[2 * kNormThreads];
    const int gid = blockIdx.x * kNormThreads + threadIdx.x;
    G1J p = gid < n_points ? ld_vec(&in[gid]) : g1_identity();
    const bool inf = fp_is_zero(p.z);
    const Fp zi = block_batch_inverse_fp<kNormThreads>(inf ? fp_one() : p.z, tree);
    if (gid >= n_points) return;
    G1A a;
    if (inf) {
        a.x = fp_zero();
        a.y = fp_zero();
    } else {
        const Fp z2 = fp_sqr(zi);
        a.x = fp_mul(p.x, z2);
        a.y = fp_mul(p.y, fp_mul(z2, zi));
    }
    // in: [row][16] folded ladder; out: [row][32], slot 16 + d = phi(slot d)
    const size_t dst = (size_t)(gid / kLadderDigits) * kDigits + gid % kLadderDigits;
    st_vec(&out[dst], a);
    st_vec(&out[dst + kLadderDigits], g1_phi(a));
}

// ---------------------------------------------------------------- stage 8
// Block a < 64: cyclic half, a >= 64: negacyclic half; a tap that wraps past
// index 0 flips sign in the negacyclic half (k_phase_b_split.comp:43-55).
__global__ void __launch_bounds__(kBuckets) k_phase_b(const G1A *__restrict__ ladder_aff,
                                                     const uint32_t *__restrict__ items_p,
                                                     const uint32_t *__restrict__ off_p,
                                                     const uint32_t *__restrict__ perm_p,
                                                     const uint32_t *__restrict__ items_m,
                                                     const uint32_t *__restrict__ off_m,
                                                     const uint32_t *__restrict__ perm_m, G1J *buckets) {
    const int a = blockIdx.x, b = blockIdx.y;
    const bool minus = a >= kHalf;
    const int aa = a & (kHalf - 1);
    const uint32_t *items = minus ? items_m : items_p;
    const uint32_t *off = minus ? off_m : off_p;
    const int bucket = (int)__ldg(&(minus ? perm_m : perm_p)[threadIdx.x]);
    const G1A *lad = ladder_aff + ((size_t)b * kCells + (minus ? kHalf : 0)) * kDigits;
    G1J acc = g1_identity();
    const uint32_t lo = __ldg(&off[bucket]), hi = __ldg(&off[bucket + 1]);
    for (uint32_t it = lo; it < hi; it++) {
        const uint32_t packed = __ldg(&items[it]);
        const int e = (int)(packed & 0xffu), d = (int)((packed >> 8) & 0xffu);
        const bool neg = ((packed >> 16) & 1u) != (minus && e > aa);
        G1A pt = ld_vec(&lad[((aa - e) & (kHalf - 1)) * kDigits + d]);
        if (neg) pt.y = fp_neg(pt.y);
        acc = g1_madd(acc, pt);
    }
    st_vec(&buckets[((size_t)b * kCells + a) * kBuckets + bucket], acc);
}

// ---------------------------------------------------------------- stage 9
// The parts' results unfold level by level, innermost first (the inverse
// butterflies of k_ladder's fold; the taps carry the factors 1/2): y[a] = C+[a] +
// C-[a], y[a + m] = C+[a] - C-[a].  outp holds the blob's 128 results, one per
// thread of the block.
__device__ __forceinline__ void finish_blob(G1J *outp, Fp *tree, uint8_t *proofs, int b, int t, int levels) {
    __syncthreads();
    for (int l = levels; l >= 1; l--) butterfly_level(outp, t, kCells >> l);
    const G1J p = ld_vec(&outp[t]);
    const bool inf = fp_is_zero(p.z);
    const Fp zi = block_batch_inverse_fp<kCells>(inf ? fp_one() : p.z, tree);
    G1A a;
    if (inf) {
        a.x = fp_zero();
        a.y = fp_zero();
    } else {
        const Fp z2 = fp_sqr(zi);
        a.x = fp_mul(p.x, z2);
        a.y = fp_mul(p.y, fp_mul(z2, zi));
    }
    alignas(16) uint8_t enc[48];
    g1_compress(enc, a);
    uint4 *dst = reinterpret_cast<uint4 *>(proofs + ((size_t)b * kCells + brev_bits((uint32_t)t, 7)) * kProofBytes);
    const uint4 *e4 = reinterpret_cast<const uint4 *>(enc);
    dst[0] = e4[0];
    dst[1] = e4[1];
    dst[2] = e4[2];
}

__global__ void __launch_bounds__(kCells) k_finish(const G1J *__restrict__ c, uint8_t *proofs, int levels) {
    __shared__ Fp tree[2 * kCells];
    __shared__ G1J outp[kCells];
    const int b = blockIdx.x, t = threadIdx.x;
    st_vec(&outp[t], ld_vec(&c[(size_t)b * kCells + t]));
    finish_blob(outp, tree, proofs, b, t, levels);
}

// ------------------------------------------- batch-affine phase A / phase B
// Persistent blocks of kBAWarps independent warps.  A warp's task is
// kWarpOutputs consecutive MSM outputs, whose 128 buckets each it sums as one
// bucket space (wb_bucket_sums), tasks strided over all warps of the grid.
// Output: affine bucket sums bucket_aff[output][k], infinity for empty buckets.
constexpr int kBAWarps = kBAThreads / 32;
constexpr int kWarpNB = kWarpOutputs * kBuckets;
constexpr int kBAMinBlocks = 65536 / (kBAThreads * 128); // at most 128 registers per thread
constexpr size_t kBASmem = kBAWarps * sizeof(WarpBuckets<kWarpNB>);
static_assert(kCells % kWarpOutputs == 0, "a task stays within one blob");
// phase B also stages the tap items (at most one per tap and digit) and their
// bucket offsets of both halves in shared memory
constexpr int kTapItemsMax = kHalf * kDigits;
constexpr size_t kPhaseBSmem = kBASmem + (2 * kTapItemsMax + 2 * (kBuckets + 1)) * sizeof(uint32_t);
static_assert(kBAThreads == VKZG_BA_THREADS, "scratch sized for this block");

struct WarpScratch {
    G1A *buf0, *buf1;
    uint32_t *pre;
    uint16_t *items;
};

__device__ __forceinline__ WarpScratch warp_scratch(G1A *scratch) {
    const size_t wid = (size_t)blockIdx.x * kBAWarps + (threadIdx.x >> 5);
    WarpScratch ws;
    ws.buf0 = scratch + wid * kBAWarpScratchPoints;
    ws.buf1 = ws.buf0 + kWarpOutputs * 1088;
    ws.pre = reinterpret_cast<uint32_t *>(ws.buf1 + kWarpOutputs * 608);
    ws.items = reinterpret_cast<uint16_t *>(ws.buf1 + kWarpOutputs * (608 + 512));
    return ws;
}

// bucket v of the task's space is bucket v % 128 of output o0 + v / 128, which
// sits at out[v] with out = bucket_aff + o0 * 128
__device__ __forceinline__ void store_warp_sums(const WarpBuckets<kWarpNB> &wb, const G1A *res, int slot, G1A *out) {
    for (int k = threadIdx.x & 31; k < kWarpNB; k += 32) {
        G1A v;
        if (wb.cnt[k]) {
            v = ld_vec(&res[wb.base[slot][k]]);
        } else {
            v.x = fp_zero();
            v.y = fp_zero();
        }
        st_vec(&out[k], v);
    }
}

// Tasks are handed out by a global counter rather than by a fixed stride: all
// tasks cost about the same, but warps on an SM that holds fewer of them run
// faster, so taking the next task when done balances the work per SM.
__device__ __forceinline__ int next_task(uint32_t *ctr) {
    uint32_t t = 0;
    if ((threadIdx.x & 31) == 0) t = atomicAdd(ctr, 1u);
    return (int)__shfl_sync(0xffffffffu, t, 0);
}

// Exclusive scan of cnt[0..NB) into a[0..NB] and b[0..NB) (two copies).
template <int NB>
__device__ __forceinline__ void warp_exclusive_scan(const uint32_t *cnt, uint32_t *a, uint32_t *b) {
    constexpr int per = NB / 32;
    const int lane = threadIdx.x & 31;
    uint32_t p = 0;
#pragma unroll
    for (int k = lane * per; k < lane * per + per; k++) p += cnt[k];
    uint32_t ip = p;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, ip, d);
        if (lane >= d) ip += o;
    }
    p = ip - p;
#pragma unroll
    for (int k = lane * per; k < lane * per + per; k++) {
        a[k] = p;
        b[k] = p;
        p += cnt[k];
    }
    if (lane == 31) a[NB] = ip;
    __syncwarp();
}

// Phase A: output o = blob * 128 + j is sum_i sum_d digit_d(s_j[i]) * pos[j][i][d].
// The warp sorts its outputs' (position, digit) items by bucket (counts by
// shared atomics, a scan, a scatter into its scratch) and sums the buckets.
__global__ void __launch_bounds__(kBAThreads, kBAMinBlocks) k_phase_a_affine(const Fr *__restrict__ scalars,
                                                                          const G1A *__restrict__ pos,
                                                                          G1A *bucket_aff, G1A *scratch, int n_out,
                                                                          uint32_t *task_ctr) {
    extern __shared__ uint4 dyn_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpBuckets<kWarpNB> &wb = reinterpret_cast<WarpBuckets<kWarpNB> *>(dyn_smem)[warp];
    const WarpScratch ws = warp_scratch(scratch);
    constexpr int kScalars = kWarpOutputs * kCellElems;
    const int n_tasks = n_out / kWarpOutputs;
    for (int task = next_task(task_ctr); task < n_tasks; task = next_task(task_ctr)) {
        const int o0 = task * kWarpOutputs;
        const Fr *sc_base = scalars + (size_t)o0 * kCellElems;
        for (int k = lane; k < kWarpNB; k += 32) wb.cnt[k] = 0;
        __syncwarp();
        for (int q = lane; q < kScalars; q += 32) {
            const Fr sc = ld_vec(&sc_base[q]);
            const int g = q / kCellElems;
            int carry = 0;
            for (int dd = 0; dd < kDigits; dd++) {
                const int v = recode_digit(sc, dd, carry);
                if (v) atomicAdd(&wb.cnt[g * kBuckets + abs(v) - 1], 1u);
            }
        }
        __syncwarp();
        // item offsets in wb.base[1] (read by round 1 only), cursors in wb.pscan
        warp_exclusive_scan<kWarpNB>(wb.cnt, wb.base[1], wb.pscan);
        for (int q = lane; q < kScalars; q += 32) {
            const Fr sc = ld_vec(&sc_base[q]);
            const int g = q / kCellElems, i = q % kCellElems;
            int carry = 0;
            for (int dd = 0; dd < kDigits; dd++) {
                const int v = recode_digit(sc, dd, carry);
                if (v) {
                    const uint32_t slot = atomicAdd(&wb.pscan[g * kBuckets + abs(v) - 1], 1u);
                    ws.items[slot] = (uint16_t)((i << 6) | (dd << 1) | (v < 0 ? 1 : 0));
                }
            }
        }
        __syncwarp();
        const uint32_t *st = wb.base[1];
        const uint16_t *items = ws.items;
        auto src0 = [=](int k, uint32_t e) {
            const uint32_t packed = items[st[k] + e];
            const G1A *tj = pos + (size_t)((o0 + (k >> 7)) % kCells) * kCellElems * kDigits;
            G1A pt = ldg_vec(&tj[(packed >> 6) * kDigits + ((packed >> 1) & 31u)]);
            if (packed & 1u) pt.y = fp_neg(pt.y);
            return pt;
        };
        int slot = 0;
        const G1A *res = wb_bucket_sums(wb, src0, ws.buf0, ws.buf1, ws.pre, slot);
        store_warp_sums(wb, res, slot, bucket_aff + (size_t)o0 * kBuckets);
        __syncwarp();
    }
}

// Phase B: output (blob b, a) with a < 64 sums the plus-half taps, a >= 64 the
// minus-half taps (negacyclic: tap e > a - 64 flips sign), over the blob's
// normalised ladder points.
__global__ void __launch_bounds__(kBAThreads, kBAMinBlocks) k_phase_b_affine(const G1A *__restrict__ ladder_aff,
                                                                          const uint32_t *__restrict__ g_items_p,
                                                                          const uint32_t *__restrict__ g_off_p,
                                                                          const uint32_t *__restrict__ g_items_m,
                                                                          const uint32_t *__restrict__ g_off_m,
                                                                          G1A *bucket_aff, G1A *scratch,
                                                                          int n_out, uint32_t *task_ctr) {
    extern __shared__ uint4 dyn_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpBuckets<kWarpNB> &wb = reinterpret_cast<WarpBuckets<kWarpNB> *>(dyn_smem)[warp];
    uint32_t *items_p = reinterpret_cast<uint32_t *>(reinterpret_cast<char *>(dyn_smem) + kBASmem);
    uint32_t *items_m = items_p + kTapItemsMax;
    uint32_t *off_p = items_m + kTapItemsMax;
    uint32_t *off_m = off_p + kBuckets + 1;
    for (int k = threadIdx.x; k <= kBuckets; k += kBAThreads) {
        off_p[k] = __ldg(&g_off_p[k]);
        off_m[k] = __ldg(&g_off_m[k]);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < off_p[kBuckets]; k += kBAThreads) items_p[k] = __ldg(&g_items_p[k]);
    for (uint32_t k = threadIdx.x; k < off_m[kBuckets]; k += kBAThreads) items_m[k] = __ldg(&g_items_m[k]);
    __syncthreads();
    const WarpScratch ws = warp_scratch(scratch);
    const int n_tasks = n_out / kWarpOutputs;
    for (int task = next_task(task_ctr); task < n_tasks; task = next_task(task_ctr)) {
        const int o0 = task * kWarpOutputs;
        for (int k = lane; k < kWarpNB; k += 32) {
            const int kk = k & (kBuckets - 1);
            const uint32_t *off = (o0 + (k >> 7)) % kCells >= kHalf ? off_m : off_p;
            wb.cnt[k] = off[kk + 1] - off[kk];
        }
        __syncwarp();
        auto src0 = [=](int k, uint32_t e) {
            const int o = o0 + (k >> 7), kk = k & (kBuckets - 1);
            const int b = o / kCells, a = o % kCells;
            const bool minus = a >= kHalf;
            const int aa = a & (kHalf - 1);
            const uint32_t *items = minus ? items_m : items_p;
            const uint32_t *off = minus ? off_m : off_p;
            const uint32_t packed = items[off[kk] + e];
            const int tap = (int)(packed & 0xffu), d = (int)((packed >> 8) & 0xffu);
            const G1A *lad = ladder_aff + ((size_t)b * kCells + (minus ? kHalf : 0)) * kDigits;
            G1A pt = ld_vec(&lad[((aa - tap) & (kHalf - 1)) * kDigits + d]);
            if (((packed >> 16) & 1u) != (minus && tap > aa)) pt.y = fp_neg(pt.y);
            return pt;
        };
        int slot = 0;
        const G1A *res = wb_bucket_sums(wb, src0, ws.buf0, ws.buf1, ws.pre, slot);
        store_warp_sums(wb, res, slot, bucket_aff + (size_t)o0 * kBuckets);
        __syncwarp();
    }
}

// ------------------------------------------------ phase A over a digit table
// Fixed-base comb: the bases X[j][i] of phase A are setup constants, so with
// the scalar's 256 bits in D signed windows (CombWindows: widths W and W + 1,
// window k at bit b_k) every digit value has its own precomputed point,
//   comb[j][i][entry_off(k) + m - 1] = m 2^(b_k) X[j][i],   m = 1..2^(width_k - 1),
// and output o = (blob, j) is a plain sum of 64 D table points (one per
// nonzero digit, negated for negative digits): no buckets, no bucket
// reduction.  D = 19 (9 windows of 14 bits, 10 of 13) sums 1216 points per
// output against the reference form's 2048 bucket additions plus the
// 128-bucket reduction, for a 90.2 GB table (HBM holds it; the reads are
// 96-byte gathers).  Windows of even widths waste no table: 19 uniform 14-bit
// windows (266 bits) took 122 GB for the same sums.

// Bits [off, off + c) of a canonical 256-bit scalar.
__device__ __forceinline__ uint32_t scalar_window(const Fr &s, int off, int c) {
    const int w = off >> 5, sh = off & 31;
    const uint64_t lo = w < 8 ? s.v[w] : 0u, hi = w + 1 < 8 ? s.v[w + 1] : 0u;
    return (uint32_t)((((hi << 32) | lo) >> sh) & ((1ull << c) - 1));
}

// Plan 3's phase A as grid-wide tree rounds.  The 64 D digit-table points of
// every output form a list; round r adds elements (2i, 2i+1) of every list of
// the chunk at once, with the pairs of all lists dealt to all lanes of the grid
// (pair p to lane p mod lanes).  A round is three launches: pass 1 (each lane's
// running product of its denominators, then the warp's product), one launch
// that inverts every warp's product (32 per warp, one inversion per warp), and
// pass 2 (the lane's inverses and the additions).  No warp waits on a
// one-lane inversion of its own, and every lane has pairs until the lists are
// short.
constexpr int kFlatThreads = 256;
// resident blocks per SM of the grid-wide round kernels (their grid is this
// many blocks per SM, and their register budget follows from it)
#ifndef VKZG_FLAT_BLOCKS_PER_SM
#define VKZG_FLAT_BLOCKS_PER_SM 2
#endif
constexpr int kFlatBlocksPerSM = VKZG_FLAT_BLOCKS_PER_SM;

struct FlatArgs {
    const int16_t *dig;  // [list][64 D] signed digits
    const Fr *scalars;   // [list][64] phase-A scalars (the persistent form recodes them itself)
    const G1A *comb;     // digit table
    size_t per_j;        // points per column j of the table (64 per_i)
    uint32_t per_i;      // points per base column (j, i): win.entries()
    uint32_t dmagic;     // ceil(2^32 / D): t / D = umulhi(t, dmagic) for t < 2^16
    CombWindows win;
    int L;               // 64 D
    const G1A *src;      // round input lists (round 1: the table)
    G1A *dst;            // round output lists
    uint32_t *pre;       // per warp: slots x 12 x 32 words of prefix products
    Fp *others;          // per lane: product of the other lanes' running products
    Fp *tot, *totinv;    // per warp: product of all, and its inverse
    size_t slots;
    int n_lists;
};

// Entry idx of the digit table (kCombEntryBytes apart).
__host__ __device__ __forceinline__ const G1A *comb_at(const G1A *comb, size_t idx) {
    return reinterpret_cast<const G1A *>(reinterpret_cast<const char *>(comb) + idx * kCombEntryBytes);
}
__host__ __device__ __forceinline__ G1A *comb_at(G1A *comb, size_t idx) {
    return reinterpret_cast<G1A *>(reinterpret_cast<char *>(comb) + idx * kCombEntryBytes);
}

// Table entry of element t of list o (scalar i = t / D of the output, window
// k = t mod D) for its digit v != 0.
__device__ __forceinline__ size_t comb_index(const FlatArgs &a, uint32_t o, uint32_t t, int v) {
    const uint32_t i = __umulhi(t, a.dmagic), k = t - i * (uint32_t)a.win.D;
    return (size_t)(o % kCells) * a.per_j + (size_t)i * a.per_i + a.win.entry_off((int)k) + (uint32_t)(abs(v) - 1);
}

// End of every pass-1 kernel: the product of the other lanes' running products
// for each lane, and the warp's product of all of them.  A butterfly over the
// lanes: at level k each lane multiplies in the product of the partner group
// of 2^k lanes (lane ^ 2^k's group), so after five levels every lane holds the
// total, and the five partner groups' products together are the other lanes':
// 9 products per lane, against 11 for a prefix and a suffix scan.
__device__ __forceinline__ void flat_pass1_products(const Fp &acc, Fp *others, Fp *tot, size_t gl, size_t wg) {
    const int lane = threadIdx.x & 31;
    Fp group = acc, rest = fp_shfl_xor(acc, 1);
    group = fp_mul(group, rest);
#pragma unroll 1
    for (int d = 2; d < 32; d <<= 1) {
        const Fp partner = fp_shfl_xor(group, d);
        rest = fp_mul(rest, partner);
        group = fp_mul(group, partner);
    }
    st_vec(&others[gl], rest);
    if (lane == 0) st_vec(&tot[wg], group);
}

// A round's input and output lists, apart from the phase's other arguments:
// a cooperative launch changes them every round while the rest stays in the
// kernel's parameters.
struct RoundIO {
    const G1A *src;
    G1A *dst;
};

template <bool FIRST>
__device__ __forceinline__ G1A flat_load(const FlatArgs &a, RoundIO io, uint32_t o, uint32_t t, uint32_t m) {
    if (FIRST) {
        const int v = a.dig[(size_t)o * a.L + t];
        G1A pt;
        if (v == 0) {
            pt.x = fp_zero();
            pt.y = fp_zero();
            return pt;
        }
        pt = ldg_vec(comb_at(a.comb, comb_index(a, o, t, v)));
        if (v < 0) pt.y = fp_neg(pt.y);
        return pt;
    }
    return ld_vec(&io.src[(size_t)o * m + t]);
}

// the x coordinate of flat_load's point (0 for a zero digit)
template <bool FIRST>
__device__ __forceinline__ Fp flat_load_x(const FlatArgs &a, RoundIO io, uint32_t o, uint32_t t, uint32_t m) {
    if (FIRST) {
        const int v = a.dig[(size_t)o * a.L + t];
        if (v == 0) return fp_zero();
        return ldg_vec(&comb_at(a.comb, comb_index(a, o, t, v))->x);
    }
    return ld_vec(&io.src[(size_t)o * m + t].x);
}

// Signed digits of every scalar in the table's windows (window k: width w_k
// at bit b_k, digits in (-2^(w_k - 1), 2^(w_k - 1)]; the top window takes the
// last carry, the scalars being below 2^255): scalar q = o 64 + i fills
// dig[q D ..].  A block's 128 scalars are recoded into shared memory and
// written out as one contiguous run of 16-byte stores (a thread's own digits
// are D x 2 bytes apart from its neighbour's: direct stores would scatter).
// n_scalars is a multiple of 128 (64 scalars per list, 128 lists per blob).
constexpr int kDigitMaxWindows = kCombMaxWindows;
// the block's group of blockDim.x scalars from q0 (a multiple of 128), staged
// in sd (blockDim.x x D int16, 16-byte aligned); the caller syncs before
// reusing sd
__device__ __forceinline__ void flat_digits_group(const Fr *__restrict__ scalars, int16_t *dig, CombWindows win,
                                                  int q0, int16_t *sd) {
    const Fr sc = ld_vec(&scalars[q0 + threadIdx.x]);
    const int D = win.D;
    int carry = 0;
    for (int k = 0; k < D; k++) {
        const int w = win.width(k);
        const int v = (int)scalar_window(sc, win.bit_off(k), w) + carry;
        carry = v > (1 << (w - 1)) ? 1 : 0;
        sd[threadIdx.x * D + k] = (int16_t)(v - (carry << w));
    }
    __syncthreads();
    const uint4 *src = reinterpret_cast<const uint4 *>(sd);
    uint4 *dst = reinterpret_cast<uint4 *>(dig + (size_t)q0 * D); // 256 D bytes per 128 scalars: 16-byte aligned
    for (int x = threadIdx.x; x < (int)blockDim.x * D / 8; x += blockDim.x) dst[x] = src[x];
}
__global__ void __launch_bounds__(128) k_flat_digits(const Fr *__restrict__ scalars, int16_t *dig, CombWindows win,
                                                    int n_scalars) {
    __shared__ __align__(16) int16_t sd[128 * kDigitMaxWindows];
    const int q0 = blockIdx.x * 128;
    if (q0 >= n_scalars) return;
    flat_digits_group(scalars, dig, win, q0, sd);
}

// Pair p = o h + i of a round (list o, pair i); a lane walks p = gl, gl + NL,
// ... (pass 1) or back (pass 2), stepping (o, i) by (NL / h, NL % h) instead of
// dividing for every pair.  All indices fit in 32 bits (at most 2^32 pairs per
// round: the working set caps a chunk far below that).
__device__ __forceinline__ void pair_step_up(uint32_t &o, uint32_t &i, uint32_t h, uint32_t dq, uint32_t dr) {
    i += dr;
    o += dq;
    if (i >= h) {
        i -= h;
        o++;
    }
}
__device__ __forceinline__ void pair_step_down(uint32_t &o, uint32_t &i, uint32_t h, uint32_t dq, uint32_t dr) {
    if (i < dr) {
        i += h - dr;
        o -= dq + 1;
    } else {
        i -= dr;
        o -= dq;
    }
}

// ---- round 1's digit-table gathers, prefetched one pair ahead
// In the first round every point is a random 96-byte read from a table of tens
// of GB; with a pair's loads issued only when the pair is reached, the lanes
// waited on them (fewer than a quarter of the warps are resident).  Each
// thread instead stages the points of its next pair in shared memory with
// cp.async while it computes the current pair.  The staging is chunk-major,
// [buffer][16-byte chunk][thread], so a warp's reads of one chunk are one
// contiguous 512-byte run (no bank conflicts).
#ifndef VKZG_GATHER_PREFETCH
#define VKZG_GATHER_PREFETCH 1
#endif
constexpr bool kGatherPrefetch = VKZG_GATHER_PREFETCH != 0;
// the same staging in the later rounds, from the round's input lists (a build
// switch, off: their pairs are coalesced runs of lists that stay largely in
// L2, and staged they measured slower, phase A 12.04 against 11.84 ms at 256
// blobs and 18 windows)
#ifndef VKZG_LIST_PREFETCH
#define VKZG_LIST_PREFETCH 0
#endif
constexpr bool kListPrefetch = kGatherPrefetch && VKZG_LIST_PREFETCH != 0;
template <bool FIRST>
constexpr bool kStaged = FIRST ? kGatherPrefetch : kListPrefetch;
constexpr int kStageChunks = 12; // two 96-byte points
constexpr size_t kStage1Bytes = 2 * 6 * kFlatThreads * sizeof(uint4);            // pass 1: x coordinates
constexpr size_t kStage2Bytes = 2 * kStageChunks * kFlatThreads * sizeof(uint4); // pass 2: whole points

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// the digit-table entry of digit v (nonzero) of element t of list o
__device__ __forceinline__ const uint4 *comb_entry(const FlatArgs &a, uint32_t o, uint32_t t, int v) {
    return reinterpret_cast<const uint4 *>(comb_at(a.comb, comb_index(a, o, t, v)));
}

// pass 1 with the x coordinates of each pair staged one pair ahead, from the
// digit table (FIRST) or from the round's input lists
template <bool FIRST>
__device__ __forceinline__ void flat_pass1_staged(const FlatArgs &a, RoundIO io, uint32_t m, uint32_t gl, uint32_t NL) {
    extern __shared__ uint4 stage[];
    uint4 *my = stage + threadIdx.x; // chunk c of buffer b: my[(b * 6 + c) * kFlatThreads]
    const uint32_t wg = gl >> 5;
    const uint32_t h = m >> 1;
    const uint32_t P = (uint32_t)a.n_lists * h;
    const uint32_t dq = NL / h, dr = NL % h;
    uint32_t *pre = a.pre + (size_t)wg * a.slots * 384;
    auto issue = [&](int b, uint32_t o, uint32_t i, int &v0, int &v1) {
        if constexpr (FIRST) {
            const int16_t *d = a.dig + (size_t)o * a.L + 2 * i;
            v0 = d[0];
            v1 = d[1];
            if (v0) {
                const uint4 *src = comb_entry(a, o, 2 * i, v0);
                for (int c = 0; c < 3; c++) cp_async16(&my[(b * 6 + c) * kFlatThreads], src + c);
            }
            if (v1) {
                const uint4 *src = comb_entry(a, o, 2 * i + 1, v1);
                for (int c = 0; c < 3; c++) cp_async16(&my[(b * 6 + 3 + c) * kFlatThreads], src + c);
            }
        } else {
            v0 = v1 = 1; // list points are stored whole, infinity as (0, 0)
            const uint4 *src = reinterpret_cast<const uint4 *>(&io.src[(size_t)o * m + 2 * i]);
            for (int c = 0; c < 3; c++) cp_async16(&my[(b * 6 + c) * kFlatThreads], src + c);
            for (int c = 0; c < 3; c++) cp_async16(&my[(b * 6 + 3 + c) * kFlatThreads], src + 6 + c);
        }
        cp_async_commit();
    };
    auto x_of = [&](int b, int half, int v) {
        Fp x;
        if (v == 0) return fp_zero();
        uint4 *w = reinterpret_cast<uint4 *>(&x);
        for (int c = 0; c < 3; c++) w[c] = my[(b * 6 + 3 * half + c) * kFlatThreads];
        return x;
    };
    Fp acc = fp_one();
    int s = 0, v0 = 0, v1 = 0;
    uint32_t o = gl / h, i = gl % h;
    if (gl < P) issue(0, o, i, v0, v1);
    for (uint32_t p = gl; p < P; p += NL, s++) {
        uint32_t on = o, in = i;
        int w0 = 0, w1 = 0;
        if (p + NL < P) {
            pair_step_up(on, in, h, dq, dr);
            issue((s + 1) & 1, on, in, w0, w1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        const Fp x = x_of(s & 1, 0, v0), y = x_of(s & 1, 1, v1);
        wb_store_pre(pre, s, acc);
        acc = fp_mul(acc, pair_denominator_x(x, y, [&] { return flat_load<FIRST>(a, io, o, 2 * i, m); },
                                             [&] { return flat_load<FIRST>(a, io, o, 2 * i + 1, m); }));
        o = on;
        i = in;
        v0 = w0;
        v1 = w1;
    }
    flat_pass1_products(acc, a.others, a.tot, gl, wg);
}

template <bool FIRST>
__device__ __forceinline__ void flat_pass1_body(const FlatArgs &a, RoundIO io, uint32_t m, uint32_t gl, uint32_t NL) {
    if constexpr (kStaged<FIRST>) {
        flat_pass1_staged<FIRST>(a, io, m, gl, NL);
        return;
    }
    const uint32_t wg = gl >> 5;
    const uint32_t h = m >> 1;
    const uint32_t P = (uint32_t)a.n_lists * h;
    const uint32_t dq = NL / h, dr = NL % h;
    uint32_t *pre = a.pre + (size_t)wg * a.slots * 384;
    Fp acc = fp_one();
    int s = 0;
    uint32_t o = gl / h, i = gl % h;
    for (uint32_t p = gl; p < P; p += NL, s++) {
        const Fp x = flat_load_x<FIRST>(a, io, o, 2 * i, m), y = flat_load_x<FIRST>(a, io, o, 2 * i + 1, m);
        wb_store_pre(pre, s, acc);
        acc = fp_mul(acc, pair_denominator_x(x, y, [&] { return flat_load<FIRST>(a, io, o, 2 * i, m); },
                                             [&] { return flat_load<FIRST>(a, io, o, 2 * i + 1, m); }));
        pair_step_up(o, i, h, dq, dr);
    }
    flat_pass1_products(acc, a.others, a.tot, gl, wg);
}

template <bool FIRST>
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_flat_pass1(FlatArgs a, uint32_t m) {
    flat_pass1_body<FIRST>(a, RoundIO{a.src, a.dst}, m, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// Inverts the n warp products, each by the four lanes of a quad (fp_inv_quad,
// its divstep tables staged in the block's shared memory).  The launch sits on
// the critical path between the passes, so it is latency that counts: all n
// inversions run at once, and one inversion per value has less latency than a
// shared batch inversion (a product scan of 32 values, one inversion, a scan
// back).  Measured per launch of 2368 values, averaged over 50 back-to-back
// launches: 24.7 us at four lanes a value, 31.8 us at one.
constexpr int kInvThreads = 128;
__global__ void __launch_bounds__(kInvThreads) k_flat_invert(const Fp *tot, Fp *totinv, int n) {
    __shared__ uint64_t t4[kDivstepEntries<4>], t2[kDivstepEntries<2>];
    for (int i = threadIdx.x; i < kDivstepEntries<4>; i += kInvThreads) t4[i] = kDivstepTable4.e[i];
    for (int i = threadIdx.x; i < kDivstepEntries<2>; i += kInvThreads) t2[i] = kDivstepTable2.e[i];
    __syncthreads();
    const int k = (int)((blockIdx.x * kInvThreads + threadIdx.x) >> 2);
    // the last block's spare quads invert value n - 1 again (every quad runs whole)
    const Fp r = fp_inv_quad(t4, t2, ld_vec(&tot[min(k, n - 1)]));
    if (k < n && (threadIdx.x & 3) == 2) st_vec(&totinv[k], r);
}
static void launch_flat_invert(const Fp *tot, Fp *totinv, int n, cudaStream_t s) {
    if (n <= 0) return;
    k_flat_invert<<<(4 * n + kInvThreads - 1) / kInvThreads, kInvThreads, 0, s>>>(tot, totinv, n);
}

// Products inlined into this loop instead of called: measured 14.1 against
// 13.1 ms of phase A at 256 blobs (the loop body outgrows the instruction
// cache), so the calls stay.
#ifndef VKZG_PASS2_INLINE
#define VKZG_PASS2_INLINE 0
#endif
constexpr bool kPass2Inline = VKZG_PASS2_INLINE != 0;
// pass 2 with the two points of each pair staged one pair ahead, from the
// digit table (FIRST) or from the round's input lists
template <bool FIRST>
__device__ __forceinline__ void flat_pass2_staged(const FlatArgs &a, RoundIO io, uint32_t m, uint32_t gl, uint32_t NL) {
    extern __shared__ uint4 stage[];
    uint4 *my = stage + threadIdx.x; // chunk c of buffer b: my[(b * kStageChunks + c) * kFlatThreads]
    const uint32_t wg = gl >> 5;
    const uint32_t h = m >> 1, m_next = (m + 1) >> 1;
    const uint32_t P = (uint32_t)a.n_lists * h;
    const uint32_t dq = NL / h, dr = NL % h;
    const uint32_t *pre = a.pre + (size_t)wg * a.slots * 384;
    Fp inv = fp_mul(ld_vec(&a.totinv[wg]), ld_vec(&a.others[gl]));
    const int S = P > gl ? (int)((P - gl + NL - 1) / NL) : 0;
    auto issue = [&](int b, uint32_t o, uint32_t i, int &v0, int &v1) {
        if constexpr (FIRST) {
            const int16_t *d = a.dig + (size_t)o * a.L + 2 * i;
            v0 = d[0];
            v1 = d[1];
            if (v0) {
                const uint4 *src = comb_entry(a, o, 2 * i, v0);
                for (int c = 0; c < 6; c++) cp_async16(&my[(b * kStageChunks + c) * kFlatThreads], src + c);
            }
            if (v1) {
                const uint4 *src = comb_entry(a, o, 2 * i + 1, v1);
                for (int c = 0; c < 6; c++) cp_async16(&my[(b * kStageChunks + 6 + c) * kFlatThreads], src + c);
            }
        } else {
            v0 = v1 = 1; // the pair's two points, 192 contiguous bytes of the list
            const uint4 *src = reinterpret_cast<const uint4 *>(&io.src[(size_t)o * m + 2 * i]);
            for (int c = 0; c < kStageChunks; c++) cp_async16(&my[(b * kStageChunks + c) * kFlatThreads], src + c);
        }
        cp_async_commit();
    };
    auto point = [&](int b, int half, int v) {
        G1A pt;
        if (v == 0) {
            pt.x = fp_zero();
            pt.y = fp_zero();
            return pt;
        }
        uint4 *w = reinterpret_cast<uint4 *>(&pt);
        for (int c = 0; c < 6; c++) w[c] = my[(b * kStageChunks + 6 * half + c) * kFlatThreads];
        if (v < 0) pt.y = fp_neg(pt.y);
        return pt;
    };
    uint32_t o = 0, i = 0;
    int v0 = 0, v1 = 0;
    if (S > 0) {
        const uint32_t p_last = gl + (uint32_t)(S - 1) * NL;
        o = p_last / h;
        i = p_last % h;
        issue((S - 1) & 1, o, i, v0, v1);
    }
    for (int t = S - 1; t >= 0; t--) {
        uint32_t on = o, in = i;
        int w0 = 0, w1 = 0;
        if (t > 0) {
            pair_step_down(on, in, h, dq, dr);
            issue((t - 1) & 1, on, in, w0, w1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        const G1A x = point(t & 1, 0, v0), y = point(t & 1, 1, v1);
        const int kind = pair_kind(x, y);
        const Fp den = pair_denominator(x, y, kind);
        const Fp inv_den = pmul<kPass2Inline>(inv, wb_load_pre(pre, t));
        inv = pmul<kPass2Inline>(inv, den);
        st_vec(&io.dst[(size_t)o * m_next + i], pair_result<kPass2Inline>(x, y, kind, inv_den));
        o = on;
        i = in;
        v0 = w0;
        v1 = w1;
    }
    if (m & 1u)
        for (uint32_t l = gl; l < (uint32_t)a.n_lists; l += NL)
            st_vec(&io.dst[(size_t)l * m_next + h], flat_load<FIRST>(a, io, l, m - 1, m));
}

template <bool FIRST>
__device__ __forceinline__ void flat_pass2_body(const FlatArgs &a, RoundIO io, uint32_t m, uint32_t gl, uint32_t NL) {
    if constexpr (kStaged<FIRST>) {
        flat_pass2_staged<FIRST>(a, io, m, gl, NL);
        return;
    }
    const uint32_t wg = gl >> 5;
    const uint32_t h = m >> 1, m_next = (m + 1) >> 1;
    const uint32_t P = (uint32_t)a.n_lists * h;
    const uint32_t dq = NL / h, dr = NL % h;
    const uint32_t *pre = a.pre + (size_t)wg * a.slots * 384;
    Fp inv = fp_mul(ld_vec(&a.totinv[wg]), ld_vec(&a.others[gl]));
    const int S = P > gl ? (int)((P - gl + NL - 1) / NL) : 0;
    uint32_t o = 0, i = 0;
    if (S > 0) {
        const uint32_t p_last = gl + (uint32_t)(S - 1) * NL;
        o = p_last / h;
        i = p_last % h;
    }
    for (int t = S - 1; t >= 0; t--) {
        if (t < S - 1) pair_step_down(o, i, h, dq, dr);
        const G1A x = flat_load<FIRST>(a, io, o, 2 * i, m), y = flat_load<FIRST>(a, io, o, 2 * i + 1, m);
        const int kind = pair_kind(x, y);
        const Fp den = pair_denominator(x, y, kind);
        const Fp inv_den = pmul<kPass2Inline>(inv, wb_load_pre(pre, t));
        inv = pmul<kPass2Inline>(inv, den);
        st_vec(&io.dst[(size_t)o * m_next + i], pair_result<kPass2Inline>(x, y, kind, inv_den));
    }
    if (m & 1u)
        for (uint32_t l = gl; l < (uint32_t)a.n_lists; l += NL)
            st_vec(&io.dst[(size_t)l * m_next + h], flat_load<FIRST>(a, io, l, m - 1, m));
}

template <bool FIRST>
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_flat_pass2(FlatArgs a, uint32_t m) {
    flat_pass2_body<FIRST>(a, RoundIO{a.src, a.dst}, m, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// The last m <= kTreeTail points of each list (affine, left by the tree
// rounds) summed in Jacobian form: the rounds below that length cost an
// inversion launch each for little work.  Two threads per list, each a chain of
// mixed additions over alternate points, then one addition.
constexpr uint32_t kTreeTail = 10;
// thread t of the tail: half t & 1 of list t >> 1 (all 32 lanes of a warp call
// it together: the halves meet by a shuffle)
__device__ __forceinline__ void flat_finish_body(const G1A *lists, uint32_t m, G1J *points, int n, int t) {
    const int o = t >> 1, h = t & 1;
    G1J acc = g1_identity();
    if (o < n) {
        const G1A *l = lists + (size_t)o * m;
        for (uint32_t k = h; k < m; k += 2) acc = g1_madd(acc, ld_vec(&l[k]));
    }
    G1J other;
#pragma unroll
    for (int w = 0; w < 12; w++) {
        other.x.v[w] = __shfl_xor_sync(0xffffffffu, acc.x.v[w], 1);
        other.y.v[w] = __shfl_xor_sync(0xffffffffu, acc.y.v[w], 1);
        other.z.v[w] = __shfl_xor_sync(0xffffffffu, acc.z.v[w], 1);
    }
    if (o < n && h == 0) st_vec(&points[o], g1_add(acc, other));
}
__global__ void __launch_bounds__(64) k_flat_finish(const G1A *__restrict__ lists, uint32_t m, G1J *points, int n) {
    flat_finish_body(lists, m, points, n, (int)(blockIdx.x * blockDim.x + threadIdx.x));
}

int flat_blocks() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms * kFlatBlocksPerSM;
}

// Working set of the grid-wide rounds for cap blobs and a table of D windows.
FlatSizes flat_sizes(int cap, int windows) {
    FlatSizes z;
    const size_t D = (size_t)windows, L = (size_t)kCellElems * D, lists = (size_t)cap * kCells;
    z.blocks = flat_blocks();
    const size_t lanes = (size_t)z.blocks * kFlatThreads;
    z.dig = lists * L;
    z.buf0 = lists * ((L + 1) / 2);
    z.buf1 = lists * ((L + 3) / 4);
    // phase A: L / 2 pairs per list; phase B: at most 1024 pairs per output (2048 tap items)
    z.slots = (lists * std::max<size_t>(L / 2, 1024) + lanes - 1) / lanes;
    z.pre_words = lanes / 32 * z.slots * 384;
    z.lanes = lanes;
    return z;
}

// Tree rounds from `first_src` (FIRST: the digit table) until every list has
// at most `stop` points (their count left in *m); returns the buffer holding
// the lists and adds the launches to *launched.
template <bool FIRST>
const G1A *run_tree_rounds(FlatArgs a, const G1A *first_src, uint32_t *m_io, uint32_t stop, G1A *buf0, G1A *buf1,
                           int blocks, cudaStream_t s, int *launched) {
    uint32_t m = *m_io;
    const int warps = blocks * kFlatThreads / 32;
    G1A *bufs[2] = {buf0, buf1};
    int out = 0;
    const G1A *cur = first_src;
    bool first = FIRST;
    while (m > stop) {
        a.src = cur;
        a.dst = bufs[out];
        if (first) k_flat_pass1<FIRST><<<blocks, kFlatThreads, kStaged<FIRST> ? kStage1Bytes : 0, s>>>(a, m);
        else k_flat_pass1<false><<<blocks, kFlatThreads, kStaged<false> ? kStage1Bytes : 0, s>>>(a, m);
        launch_flat_invert(a.tot, a.totinv, warps, s);
        if (first) k_flat_pass2<FIRST><<<blocks, kFlatThreads, kStaged<FIRST> ? kStage2Bytes : 0, s>>>(a, m);
        else k_flat_pass2<false><<<blocks, kFlatThreads, kStaged<false> ? kStage2Bytes : 0, s>>>(a, m);
        *launched += 3;
        cur = bufs[out];
        out ^= 1;
        m = (m + 1) >> 1;
        first = false;
    }
    *m_io = m;
    return cur;
}

// The later rounds' pass kernels stage their pairs in dynamic shared memory.
static cudaError_t configure_list_rounds() {
    if (!kListPrefetch) return cudaSuccess;
    cudaError_t e =
        cudaFuncSetAttribute(k_flat_pass1<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStage1Bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_flat_pass2<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStage2Bytes);
}

// Sums of n_lists lists of m points (list o at lists[o m ..]) by the same
// grid-wide rounds, for tests and profiles of the rounds alone (the lists
// buffer is not written unless m == 1).  Returns the launches made.
int launch_tree_sums(const G1A *lists, int n_lists, uint32_t m, G1A *buf0, G1A *buf1, uint32_t *pre, Fp *others,
                     Fp *tot, Fp *totinv, size_t slots, int blocks, G1A *sums, cudaStream_t s) {
    FlatArgs a;
    memset(&a, 0, sizeof a);
    a.pre = pre;
    a.others = others;
    a.tot = tot;
    a.totinv = totinv;
    a.slots = slots;
    a.n_lists = n_lists;
    int launched = 0;
    if (configure_list_rounds() != cudaSuccess) return 0;
    const G1A *res = run_tree_rounds<false>(a, lists, &m, 1, buf0, buf1, blocks, s, &launched);
    cudaMemcpyAsync(sums, res, (size_t)n_lists * sizeof(G1A), cudaMemcpyDeviceToDevice, s);
    count_launches(launched);
    return launched;
}

// The pass bodies as the cooperative kernels call them: inlined (default), or
// out of line with their arguments by value (VKZG_COOP_NOINLINE=1), each then
// with its own register allocation.
#ifndef VKZG_COOP_NOINLINE
#define VKZG_COOP_NOINLINE 0
#endif
#if VKZG_COOP_NOINLINE
#define VKZG_COOP_FN __device__ __noinline__
#else
#define VKZG_COOP_FN __device__ __forceinline__
#endif
template <bool FIRST>
VKZG_COOP_FN void coop_flat_pass1(FlatArgs a, RoundIO io, uint32_t m, uint32_t gl, uint32_t NL) {
    flat_pass1_body<FIRST>(a, io, m, gl, NL);
}
template <bool FIRST>
VKZG_COOP_FN void coop_flat_pass2(FlatArgs a, RoundIO io, uint32_t m, uint32_t gl, uint32_t NL) {
    flat_pass2_body<FIRST>(a, io, m, gl, NL);
}

// The inversions between the passes of a cooperative round: one warp in 32
// inverts the products of warps wg..wg+31, one per lane, so that they spread
// over the SMs as the separate inversion launch does (the first 2368 threads
// of the grid would put them all on a few SMs).
__device__ __noinline__ void coop_invert(const Fp *tot, Fp *totinv, uint32_t n, uint32_t gl, uint32_t NL) {
    (void)NL;
    const uint32_t wg = gl >> 5;
    if (wg & 31u) return;
    const uint32_t t = wg + (gl & 31u);
    if (t < n) st_vec(&totinv[t], fp_inv_fast(ld_vec(&tot[t])));
}

// Cooperative form of run_tree_rounds: every round of the tree in one launch,
// the passes and the inversion between them separated by grid barriers.  The
// phase's arguments stay in the kernel's parameters (only the round's lists
// change from round to round), so the passes compile as in their own kernels.
template <bool FIRST>
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_coop_tree(FlatArgs a, const G1A *first_src, G1A *buf0,
                                                               G1A *buf1, uint32_t m, uint32_t stop, GridSync g) {
    const uint32_t gl = blockIdx.x * blockDim.x + threadIdx.x, NL = gridDim.x * blockDim.x;
    RoundIO io{first_src, buf0};
    if constexpr (FIRST) {
        // the scalars' digits (k_flat_digits), staged in the round's shared
        // memory before pass 1 needs it, then the first round alone (from the
        // digit table, into buf0): its pass bodies differ from the later
        // rounds', and one kernel holding both forms of both passes outgrew
        // its registers and instruction cache
        (void)buf1;
        (void)stop;
        {
            extern __shared__ uint4 stage[];
            int16_t *sd = reinterpret_cast<int16_t *>(stage); // kFlatThreads x D int16 of the staging
            const int n_scalars = a.n_lists * kCellElems;
            for (int q0 = blockIdx.x * kFlatThreads; q0 < n_scalars; q0 += gridDim.x * kFlatThreads) {
                flat_digits_group(a.scalars, const_cast<int16_t *>(a.dig), a.win, q0, sd);
                __syncthreads();
            }
        }
        if (!grid_sync(g)) return;
        coop_flat_pass1<true>(a, io, m, gl, NL);
        if (!grid_sync(g)) return;
        coop_invert(a.tot, a.totinv, NL >> 5, gl, NL);
        if (!grid_sync(g)) return;
        coop_flat_pass2<true>(a, io, m, gl, NL);
    } else {
        while (m > stop) {
            coop_flat_pass1<false>(a, io, m, gl, NL);
            if (!grid_sync(g)) return;
            coop_invert(a.tot, a.totinv, NL >> 5, gl, NL);
            if (!grid_sync(g)) return;
            coop_flat_pass2<false>(a, io, m, gl, NL);
            io.src = io.dst;
            io.dst = io.dst == buf0 ? buf1 : buf0;
            m = (m + 1) >> 1;
            if (m > stop && !grid_sync(g)) return;
        }
    }
}

// the buffer holding the lists after run_tree_rounds' rounds from m down to stop
const G1A *tree_result(const G1A *first_src, uint32_t *m_io, uint32_t stop, G1A *buf0, G1A *buf1) {
    uint32_t m = *m_io;
    const G1A *cur = first_src;
    int out = 0;
    while (m > stop) {
        cur = out ? buf1 : buf0;
        out ^= 1;
        m = (m + 1) >> 1;
    }
    *m_io = m;
    return cur;
}

// a launch with every block resident at once (cudaLaunchAttributeCooperative),
// so that grid barriers inside it complete; capturable into a CUDA graph
template <typename... KArgs, typename... Args>
cudaError_t launch_coop(void (*kernel)(KArgs...), int blocks, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(kFlatThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// polls of a grid barrier before it gives up: far above any round's duration
constexpr uint32_t kSyncSpinLimit = 1u << 24;

GridSync make_sync(const ProofWork &w, int n) {
    GridSync g;
    g.word = w.sync;
    g.err = w.err;
    g.n_err = (uint32_t)n;
    g.spin_limit = kSyncSpinLimit;
    g.expected = (uint32_t)w.flat_blocks;
    return g;
}

// Phase A of plan 3 for n blobs: digits, tree rounds, Jacobian outputs in
// w.points.  Returns the number of kernels launched.
int launch_phase_a_flat(const ProofWork &w, int n, cudaStream_t s) {
    const int D = w.comb_windows, L = kCellElems * D;
    const int lists = n * kCells;
    FlatArgs a;
    a.dig = w.flat_dig;
    a.comb = w.comb;
    a.win = comb_windows(D);
    a.per_i = a.win.entries();
    a.per_j = (size_t)kCellElems * a.per_i;
    a.dmagic = (uint32_t)(((1ull << 32) + (uint64_t)D - 1) / (uint64_t)D);
    a.scalars = w.scalars;
    a.L = L;
    a.pre = w.flat_pre;
    a.others = w.flat_others;
    a.tot = w.flat_tot;
    a.totinv = w.flat_totinv;
    a.slots = w.flat_slots;
    a.n_lists = lists;
    int launched = 0;
    uint32_t m = (uint32_t)L;
    const G1A *res;
    if (w.coop) {
        // round 1 (digit table -> buf0), then the later rounds ping-ponging
        // buf1, buf0, ... as the separate launches do (tree_result)
        const uint32_t m0 = m;
        launch_coop(k_coop_tree<true>, w.flat_blocks, kStage2Bytes, s, a, (const G1A *)nullptr, w.flat_buf[0],
                    w.flat_buf[1], m0, (m0 + 1) >> 1, make_sync(w, n));
        launched++;
        if (((m0 + 1) >> 1) > kTreeTail) {
            launch_coop(k_coop_tree<false>, w.flat_blocks, 0, s, a, (const G1A *)w.flat_buf[0], w.flat_buf[1],
                        w.flat_buf[0], (m0 + 1) >> 1, kTreeTail, make_sync(w, n));
            launched++;
        }
        res = tree_result(nullptr, &m, kTreeTail, w.flat_buf[0], w.flat_buf[1]);
    } else {
        k_flat_digits<<<lists * kCellElems / 128, 128, 0, s>>>(w.scalars, w.flat_dig, a.win, lists * kCellElems);
        launched++;
        res = run_tree_rounds<true>(a, nullptr, &m, kTreeTail, w.flat_buf[0], w.flat_buf[1], w.flat_blocks, s,
                                    &launched);
    }
    k_flat_finish<<<(2 * lists + 63) / 64, 64, 0, s>>>(res, m, w.points, lists);
    return launched + 1;
}

// Plan 3's phase B as grid-wide rounds.  The bucket lists of an output are the
// tap items of its part (PartLayout: the cyclic part and the negacyclic parts
// of the folds), so every output of a part has the same bucket lengths in every
// round: the round structure is a setup constant (FlatBPlan, built on the host)
// and the pairs of all outputs are dealt to all lanes as in phase A.  Round r
// keeps bucket k of output o (part q) at buf[o * stride[r] + base[r][q][k] ..];
// the last round writes each bucket's sum straight to bucket_aff[o][k] (at most
// two elements are left per bucket then) and infinity to the buckets no digit
// reaches, for the reduction.
bool build_flatb_plan(const PartLayout &parts, const uint32_t offsets[][kBuckets + 1], FlatBPlan &pl) {
    memset(&pl, 0, sizeof pl);
    if (parts.n < 1 || parts.n > kFBMaxParts) return false;
    pl.parts = parts;
    uint32_t cnt[kFBMaxParts][kBuckets];
    for (int q = 0; q < parts.n; q++)
        for (int k = 0; k < kBuckets; k++) {
            cnt[q][k] = offsets[q][k + 1] - offsets[q][k];
            if (!cnt[q][k]) pl.empty[q][pl.n_empty[q]++] = (uint8_t)k;
        }
    int r = 0;
    for (;; r++) {
        if (r > kFBMaxRounds) return false;
        bool more = false;
        uint32_t stride = 0;
        for (int q = 0; q < parts.n; q++) {
            uint32_t b = 0, ps = 0, no = 0;
            for (int k = 0; k < kBuckets; k++) {
                pl.cnt[r][q][k] = cnt[q][k];
                pl.base[r][q][k] = b;
                b += cnt[q][k];
                more |= cnt[q][k] > 1;
                if (r < kFBMaxRounds) {
                    pl.pscan[r][q][k] = ps;
                    ps += cnt[q][k] >> 1;
                    if (cnt[q][k] & 1u) pl.odd[r][q][no++] = (uint8_t)k;
                }
            }
            pl.base[r][q][kBuckets] = b;
            stride = std::max(stride, b);
            if (r < kFBMaxRounds) {
                pl.pscan[r][q][kBuckets] = ps;
                pl.pairs[r][q] = ps;
                pl.n_odd[r][q] = no;
            }
        }
        pl.stride[r] = stride;
        if (!more) break;
        for (int q = 0; q < parts.n; q++)
            for (int k = 0; k < kBuckets; k++) cnt[q][k] = (cnt[q][k] + 1) >> 1;
    }
    pl.rounds = r;
    return true;
}

struct FlatBArgs {
    const FlatBPlan *plan;
    const G1A *ladder_aff;
    const uint32_t *items;   // part q's items from kDigits * off[q]
    const uint32_t *offsets; // [kFBMaxParts][kBuckets + 1]
    const G1A *src;
    G1A *dst;
    G1A *bucket_aff; // the last round's destination, [output][kBuckets]
    const G1A *deriv_buf; // [blob][deriv_points] shared pair sums
    uint32_t deriv_points;
    uint32_t deriv_base[kFBMaxParts];
    uint32_t *pre;
    Fp *others, *tot, *totinv;
    size_t slots;
    int n_blobs;
};

// shared copy of one round's plan (and, in round 0, the tap items)
struct FlatBRound {
    uint32_t pscan[kFBMaxParts][kBuckets + 1];
    uint32_t base[kFBMaxParts][kBuckets + 1];
    uint32_t base_next[kFBMaxParts][kBuckets + 1];
    uint32_t cnt[kFBMaxParts][kBuckets];
    uint32_t pairs[kFBMaxParts];
    uint32_t pair_end[kFBMaxParts]; // all blobs' pairs of parts 0..q
    uint32_t size[kFBMaxParts], off[kFBMaxParts], nega[kFBMaxParts];
    uint32_t stride, stride_next;
    int n_parts;
};
constexpr int kPartItemsMax = kCells * kDigits;
constexpr size_t kFlatBSmem =
    sizeof(FlatBRound) + (kPartItemsMax + kFBMaxParts * (kBuckets + 1)) * sizeof(uint32_t);

template <bool FIRST>
__device__ void flatb_stage(const FlatBArgs &a, int r, FlatBRound &sr, uint32_t *items, uint32_t *offs) {
    const FlatBPlan &pl = *a.plan;
    const int np = pl.parts.n;
    for (int x = threadIdx.x; x < np * (kBuckets + 1); x += blockDim.x) {
        const int q = x / (kBuckets + 1), k = x % (kBuckets + 1);
        sr.pscan[q][k] = pl.pscan[r][q][k];
        sr.base[q][k] = pl.base[r][q][k];
        sr.base_next[q][k] = pl.base[r + 1][q][k];
        if (k < kBuckets) sr.cnt[q][k] = pl.cnt[r][q][k];
        if (FIRST) offs[x] = __ldg(&a.offsets[x]);
    }
    if (threadIdx.x == 0) {
        sr.stride = pl.stride[r];
        sr.stride_next = pl.stride[r + 1];
        sr.n_parts = np;
        uint32_t end = 0;
        for (int q = 0; q < np; q++) {
            sr.pairs[q] = pl.pairs[r][q];
            sr.size[q] = pl.parts.size[q];
            sr.off[q] = pl.parts.off[q];
            sr.nega[q] = pl.parts.nega[q];
            end += (uint32_t)a.n_blobs * pl.parts.size[q] * pl.pairs[r][q];
            sr.pair_end[q] = end;
        }
    }
    if (FIRST) {
        __syncthreads();
        for (int q = 0; q < np; q++) {
            const uint32_t b = kDigits * pl.parts.off[q], m = offs[q * (kBuckets + 1) + kBuckets];
            for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) items[b + k] = __ldg(&a.items[b + k]);
        }
    }
    __syncthreads();
}

// point x (< n) of row d of part q of blob b: a ladder row (d < 32) or a shared pair sum
__device__ __forceinline__ const G1A *flatb_src(const FlatBArgs &a, const FlatBRound &sr, uint32_t b, int q,
                                                uint32_t x, int d) {
    if (d < kDigits) return &a.ladder_aff[((size_t)b * kCells + sr.off[q] + x) * kDigits + d];
    return &a.deriv_buf[(size_t)b * a.deriv_points + a.deriv_base[q] + (uint32_t)(d - kDigits) * sr.size[q] + x];
}

// element e of bucket k of output o (part q)
template <bool FIRST>
__device__ __forceinline__ G1A flatb_load(const FlatBArgs &a, RoundIO io, const FlatBRound &sr, const uint32_t *items,
                                          const uint32_t *offs, uint32_t o, int q, int k, uint32_t e) {
    if (FIRST) {
        const uint32_t packed = items[kDigits * sr.off[q] + offs[q * (kBuckets + 1) + k] + e];
        const int tap = (int)(packed & 0xffu), d = (int)((packed >> 8) & 0xffu);
        const uint32_t b = o / kCells, aa = o % kCells - sr.off[q];
        G1A pt = ld_vec(flatb_src(a, sr, b, q, (aa - (uint32_t)tap) & (sr.size[q] - 1), d));
        if (((packed >> 16) & 1u) != (sr.nega[q] && tap > (int)aa)) pt.y = fp_neg(pt.y);
        return pt;
    }
    return ld_vec(&io.src[(size_t)o * sr.stride + sr.base[q][k] + e]);
}

// the x coordinate of flatb_load's point
template <bool FIRST>
__device__ __forceinline__ Fp flatb_load_x(const FlatBArgs &a, RoundIO io, const FlatBRound &sr, const uint32_t *items,
                                           const uint32_t *offs, uint32_t o, int q, int k, uint32_t e) {
    if (FIRST) {
        const uint32_t packed = items[kDigits * sr.off[q] + offs[q * (kBuckets + 1) + k] + e];
        const int tap = (int)(packed & 0xffu), d = (int)((packed >> 8) & 0xffu);
        const uint32_t b = o / kCells, aa = o % kCells - sr.off[q];
        return ld_vec(&flatb_src(a, sr, b, q, (aa - (uint32_t)tap) & (sr.size[q] - 1), d)->x);
    }
    return ld_vec(&io.src[(size_t)o * sr.stride + sr.base[q][k] + e].x);
}

// pair p of the round -> output, part, bucket, index
__device__ __forceinline__ void flatb_pair(const FlatBRound &sr, uint32_t p, uint32_t &o, int &q, int &k,
                                           uint32_t &i) {
    q = 0;
    while (q + 1 < sr.n_parts && p >= sr.pair_end[q]) q++;
    const uint32_t pp = q ? p - sr.pair_end[q - 1] : p;
    const uint32_t per = sr.pairs[q];
    const uint32_t ol = pp / per, r = pp - ol * per;
    const uint32_t m = sr.size[q];
    o = (ol / m) * kCells + sr.off[q] + ol % m;
    k = ba_bucket_of<kBuckets>(sr.pscan[q], r);
    i = r - sr.pscan[q][k];
}

template <bool FIRST>
__device__ __forceinline__ void flatb_pass1_body(const FlatBArgs &a, RoundIO io, int r, uint4 *dyn_smem, uint32_t gl,
                                                 uint32_t NL) {
    FlatBRound &sr = *reinterpret_cast<FlatBRound *>(dyn_smem);
    uint32_t *items = reinterpret_cast<uint32_t *>(&sr + 1), *offs = items + kPartItemsMax;
    flatb_stage<FIRST>(a, r, sr, items, offs);
    const uint32_t wg = gl >> 5;
    const uint32_t P = sr.pair_end[sr.n_parts - 1];
    uint32_t *pre = a.pre + (size_t)wg * a.slots * 384;
    Fp acc = fp_one();
    int s = 0;
    for (uint32_t p = gl; p < P; p += NL, s++) {
        uint32_t o, i;
        int q, k;
        flatb_pair(sr, p, o, q, k, i);
        const Fp x = flatb_load_x<FIRST>(a, io, sr, items, offs, o, q, k, 2 * i);
        const Fp y = flatb_load_x<FIRST>(a, io, sr, items, offs, o, q, k, 2 * i + 1);
        wb_store_pre(pre, s, acc);
        acc = fp_mul(acc, pair_denominator_x(x, y, [&] { return flatb_load<FIRST>(a, io, sr, items, offs, o, q, k, 2 * i); },
                                             [&] { return flatb_load<FIRST>(a, io, sr, items, offs, o, q, k, 2 * i + 1); }));
    }
    flat_pass1_products(acc, a.others, a.tot, gl, wg);
}

template <bool FIRST>
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_flatb_pass1(FlatBArgs a, int r) {
    extern __shared__ uint4 dyn_smem[];
    flatb_pass1_body<FIRST>(a, RoundIO{a.src, a.dst}, r, dyn_smem, blockIdx.x * blockDim.x + threadIdx.x,
                            gridDim.x * blockDim.x);
}

template <bool FIRST>
__device__ __forceinline__ void flatb_pass2_body(const FlatBArgs &a, RoundIO io, int r, uint4 *dyn_smem, uint32_t gl,
                                                 uint32_t NL) {
    FlatBRound &sr = *reinterpret_cast<FlatBRound *>(dyn_smem);
    uint32_t *items = reinterpret_cast<uint32_t *>(&sr + 1), *offs = items + kPartItemsMax;
    flatb_stage<FIRST>(a, r, sr, items, offs);
    const uint32_t wg = gl >> 5;
    const uint32_t P = sr.pair_end[sr.n_parts - 1];
    const uint32_t *pre = a.pre + (size_t)wg * a.slots * 384;
    const bool last = r + 1 == a.plan->rounds;
    Fp inv = fp_mul(ld_vec(&a.totinv[wg]), ld_vec(&a.others[gl]));
    const int S = P > gl ? (int)((P - gl + NL - 1) / NL) : 0;
    for (int t = S - 1; t >= 0; t--) {
        const uint32_t p = gl + (uint32_t)t * NL;
        uint32_t o, i;
        int q, k;
        flatb_pair(sr, p, o, q, k, i);
        const G1A x = flatb_load<FIRST>(a, io, sr, items, offs, o, q, k, 2 * i);
        const G1A y = flatb_load<FIRST>(a, io, sr, items, offs, o, q, k, 2 * i + 1);
        const int kind = pair_kind(x, y);
        const Fp den = pair_denominator(x, y, kind);
        const Fp inv_den = fp_mul(inv, wb_load_pre(pre, t));
        inv = fp_mul(inv, den);
        G1A *d = last ? &a.bucket_aff[(size_t)o * kBuckets + k] : &io.dst[(size_t)o * sr.stride_next + sr.base_next[q][k] + i];
        st_vec(d, pair_result(x, y, kind, inv_den));
    }
    // odd last elements move up unchanged
    const FlatBPlan &pl = *a.plan;
    size_t odd_begin = 0;
    for (int q = 0; q < sr.n_parts; q++) {
        const uint32_t no = pl.n_odd[r][q], m = sr.size[q];
        const size_t odd_q = (size_t)a.n_blobs * m * no;
        // this part's odd elements are x in [odd_begin, odd_begin + odd_q) of the
        // grid-wide sequence; lane gl takes those with x = gl (mod NL)
        const size_t first = odd_begin + (gl + NL - odd_begin % NL) % NL;
        for (size_t x = first; x < odd_begin + odd_q; x += NL) {
            const size_t xx = x - odd_begin;
            const uint32_t ol = (uint32_t)(xx / no), j = (uint32_t)(xx - (size_t)ol * no);
            const int k = pl.odd[r][q][j];
            const uint32_t o = (ol / m) * kCells + sr.off[q] + ol % m;
            const uint32_t c = sr.cnt[q][k];
            G1A *d = last ? &a.bucket_aff[(size_t)o * kBuckets + k]
                          : &io.dst[(size_t)o * sr.stride_next + sr.base_next[q][k] + (c >> 1)];
            st_vec(d, flatb_load<FIRST>(a, io, sr, items, offs, o, q, k, c - 1));
        }
        odd_begin += odd_q;
    }
    if (last) { // infinity in the buckets of a part that no digit reaches
        size_t e_begin = 0;
        for (int q = 0; q < sr.n_parts; q++) {
            const uint32_t ne = pl.n_empty[q], m = sr.size[q];
            const size_t e_q = (size_t)a.n_blobs * m * ne;
            const size_t first = e_begin + (gl + NL - e_begin % NL) % NL;
            for (size_t x = first; x < e_begin + e_q; x += NL) {
                const size_t xx = x - e_begin;
                const uint32_t ol = (uint32_t)(xx / ne), j = (uint32_t)(xx - (size_t)ol * ne);
                const uint32_t o = (ol / m) * kCells + sr.off[q] + ol % m;
                G1A z;
                z.x = fp_zero();
                z.y = fp_zero();
                st_vec(&a.bucket_aff[(size_t)o * kBuckets + pl.empty[q][j]], z);
            }
            e_begin += e_q;
        }
    }
}

template <bool FIRST>
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_flatb_pass2(FlatBArgs a, int r) {
    extern __shared__ uint4 dyn_smem[];
    flatb_pass2_body<FIRST>(a, RoundIO{a.src, a.dst}, r, dyn_smem, blockIdx.x * blockDim.x + threadIdx.x,
                            gridDim.x * blockDim.x);
}

// The shared pair sums of phase B as one grid-wide round: point m of blob b is
// x = m - base of its type; its pair is L_a[x] and s L~_b[x - delta].
struct DerivArgs {
    const DerivType *types;
    const uint16_t *type_of;
    const G1A *ladder_aff;
    G1A *out;
    PartLayout parts;
    uint32_t points; // per blob
    uint32_t *pre;
    Fp *others, *tot, *totinv;
    size_t slots_pre;
    int n_blobs;
};

__device__ __forceinline__ void deriv_pair(const DerivArgs &a, uint32_t p, const G1A *&pa, const G1A *&pb,
                                           bool &neg_b) {
    const uint32_t b = p / a.points, m = p - b * a.points;
    const DerivType ty = a.types[a.type_of[m]];
    const uint32_t n = a.parts.size[ty.part], off = a.parts.off[ty.part];
    const uint32_t x = m - ty.base;
    const bool wrap = x < ty.delta;
    const uint32_t xb = wrap ? x + n - ty.delta : x - ty.delta;
    pa = &a.ladder_aff[((size_t)b * kCells + off + x) * kDigits + ty.row_a];
    pb = &a.ladder_aff[((size_t)b * kCells + off + xb) * kDigits + ty.row_b];
    neg_b = (ty.neg != 0) != (wrap && a.parts.nega[ty.part]);
}

__device__ __forceinline__ void deriv_pass1_body(const DerivArgs &a, uint32_t gl, uint32_t NL) {
    const uint32_t wg = gl >> 5;
    const uint32_t P = (uint32_t)a.n_blobs * a.points;
    uint32_t *pre = a.pre + (size_t)wg * a.slots_pre * 384;
    Fp acc = fp_one();
    int s = 0;
    for (uint32_t p = gl; p < P; p += NL, s++) {
        const G1A *pa, *pb;
        bool nb;
        deriv_pair(a, p, pa, pb, nb);
        wb_store_pre(pre, s, acc);
        acc = fp_mul(acc, pair_denominator_x(ld_vec(&pa->x), ld_vec(&pb->x), [&] { return ld_vec(pa); },
                                             [&] {
                                                 G1A y = ld_vec(pb);
                                                 if (nb) y.y = fp_neg(y.y);
                                                 return y;
                                             }));
    }
    flat_pass1_products(acc, a.others, a.tot, gl, wg);
}
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_deriv_pass1(DerivArgs a) {
    deriv_pass1_body(a, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

__device__ __forceinline__ void deriv_pass2_body(const DerivArgs &a, uint32_t gl, uint32_t NL) {
    const uint32_t wg = gl >> 5;
    const uint32_t P = (uint32_t)a.n_blobs * a.points;
    const uint32_t *pre = a.pre + (size_t)wg * a.slots_pre * 384;
    Fp inv = fp_mul(ld_vec(&a.totinv[wg]), ld_vec(&a.others[gl]));
    const int S = P > gl ? (int)((P - gl + NL - 1) / NL) : 0;
    for (int t = S - 1; t >= 0; t--) {
        const uint32_t p = gl + (uint32_t)t * NL;
        const G1A *pa, *pb;
        bool nb;
        deriv_pair(a, p, pa, pb, nb);
        const G1A x = ld_vec(pa);
        G1A y = ld_vec(pb);
        if (nb) y.y = fp_neg(y.y);
        const int kind = pair_kind(x, y);
        const Fp den = pair_denominator(x, y, kind);
        const Fp inv_den = fp_mul(inv, wb_load_pre(pre, t));
        inv = fp_mul(inv, den);
        st_vec(&a.out[p], pair_result(x, y, kind, inv_den));
    }
}
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_deriv_pass2(DerivArgs a) {
    deriv_pass2_body(a, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// the shared pair sums into w.deriv_buf; returns the launches made (0 without any)
DerivArgs deriv_args(const DeviceTables &t, const ProofWork &w, int n) {
    DerivArgs a;
    a.types = t.deriv;
    a.type_of = t.deriv_of;
    a.ladder_aff = w.ladder_aff;
    a.out = w.deriv_buf;
    a.parts = part_layout(kPartLevels);
    a.points = t.deriv_points;
    a.pre = w.flat_pre;
    a.others = w.flat_others;
    a.tot = w.flat_tot;
    a.totinv = w.flat_totinv;
    a.slots_pre = w.flat_slots;
    a.n_blobs = n;
    return a;
}

int launch_deriv_flat(const DeviceTables &t, const ProofWork &w, int n, cudaStream_t s) {
    if (!t.deriv_points) return 0;
    const DerivArgs a = deriv_args(t, w, n);
    const int blocks = w.flat_blocks, warps = blocks * kFlatThreads / 32;
    k_deriv_pass1<<<blocks, kFlatThreads, 0, s>>>(a);
    launch_flat_invert(a.tot, a.totinv, warps, s);
    k_deriv_pass2<<<blocks, kFlatThreads, 0, s>>>(a);
    return 3;
}

// Phase B of plan 3 into w.bucket_aff; returns the number of kernels launched.
FlatBArgs flatb_args(const DeviceTables &t, const ProofWork &w, int n) {
    FlatBArgs a;
    a.plan = t.fb_plan;
    a.ladder_aff = w.ladder_aff;
    a.items = t.part_items;
    a.offsets = t.part_offsets;
    a.bucket_aff = w.bucket_aff;
    a.deriv_buf = w.deriv_buf;
    a.deriv_points = t.deriv_points;
    for (int q = 0; q < kFBMaxParts; q++) a.deriv_base[q] = t.deriv_base[q];
    a.pre = w.flat_pre;
    a.others = w.flat_others;
    a.tot = w.flat_tot;
    a.totinv = w.flat_totinv;
    a.slots = w.flat_slots;
    a.n_blobs = n;
    return a;
}

VKZG_COOP_FN void coop_deriv_pass1(DerivArgs a, uint32_t gl, uint32_t NL) { deriv_pass1_body(a, gl, NL); }
VKZG_COOP_FN void coop_deriv_pass2(DerivArgs a, uint32_t gl, uint32_t NL) { deriv_pass2_body(a, gl, NL); }
template <bool FIRST>
VKZG_COOP_FN void coop_flatb_pass1(FlatBArgs a, RoundIO io, int r, uint4 *smem, uint32_t gl, uint32_t NL) {
    flatb_pass1_body<FIRST>(a, io, r, smem, gl, NL);
}
template <bool FIRST>
VKZG_COOP_FN void coop_flatb_pass2(FlatBArgs a, RoundIO io, int r, uint4 *smem, uint32_t gl, uint32_t NL) {
    flatb_pass2_body<FIRST>(a, io, r, smem, gl, NL);
}

// Cooperative form of the shared pair sums and phase B's rounds: one launch,
// grid barriers between the passes (the arguments stay in the kernel's
// parameters; only the round's lists change).
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_coop_phase_b(DerivArgs da, int has_deriv, FlatBArgs fa,
                                                                  G1A *buf0, G1A *buf1, int rounds, GridSync g) {
    extern __shared__ uint4 dyn_smem[];
    const uint32_t gl = blockIdx.x * blockDim.x + threadIdx.x, NL = gridDim.x * blockDim.x;
    if (has_deriv) {
        coop_deriv_pass1(da, gl, NL);
        if (!grid_sync(g)) return;
        coop_invert(da.tot, da.totinv, NL >> 5, gl, NL);
        if (!grid_sync(g)) return;
        coop_deriv_pass2(da, gl, NL);
        if (!grid_sync(g)) return;
    }
    RoundIO io{nullptr, buf0};
    for (int r = 0; r < rounds; r++) {
        if (r == 0) coop_flatb_pass1<true>(fa, io, r, dyn_smem, gl, NL);
        else coop_flatb_pass1<false>(fa, io, r, dyn_smem, gl, NL);
        if (!grid_sync(g)) return;
        coop_invert(fa.tot, fa.totinv, NL >> 5, gl, NL);
        if (!grid_sync(g)) return;
        if (r == 0) coop_flatb_pass2<true>(fa, io, r, dyn_smem, gl, NL);
        else coop_flatb_pass2<false>(fa, io, r, dyn_smem, gl, NL);
        io.src = io.dst;
        io.dst = io.dst == buf0 ? buf1 : buf0;
        if (r + 1 < rounds && !grid_sync(g)) return;
    }
}

int launch_phase_b_coop(const DeviceTables &t, const ProofWork &w, int n, cudaStream_t s) {
    launch_coop(k_coop_phase_b, w.flat_blocks, kFlatBSmem, s, deriv_args(t, w, n), t.deriv_points ? 1 : 0,
                flatb_args(t, w, n), w.flatb_buf[0], w.flatb_buf[1], t.fb_rounds, make_sync(w, n));
    return 1;
}

int launch_phase_b_flat(const DeviceTables &t, const ProofWork &w, int n, cudaStream_t s) {
    FlatBArgs a = flatb_args(t, w, n);
    const int blocks = w.flat_blocks, warps = blocks * kFlatThreads / 32;
    G1A *bufs[2] = {w.flatb_buf[0], w.flatb_buf[1]};
    const G1A *cur = nullptr;
    int out = 0, launched = 0;
    for (int r = 0; r < t.fb_rounds; r++) {
        a.src = cur;
        a.dst = bufs[out];
        if (r == 0) k_flatb_pass1<true><<<blocks, kFlatThreads, kFlatBSmem, s>>>(a, r);
        else k_flatb_pass1<false><<<blocks, kFlatThreads, kFlatBSmem, s>>>(a, r);
        launch_flat_invert(a.tot, a.totinv, warps, s);
        if (r == 0) k_flatb_pass2<true><<<blocks, kFlatThreads, kFlatBSmem, s>>>(a, r);
        else k_flatb_pass2<false><<<blocks, kFlatThreads, kFlatBSmem, s>>>(a, r);
        launched += 3;
        cur = bufs[out];
        out ^= 1;
    }
    return launched;
}

// Bases of the digit table: B[j][i][k] = 2^(b_k) X[j][i] (b_k the bit of
// window k), from the position table entry 2^(8 floor(b_k / 8)) X[j][i] and
// (b_k mod 8) doublings.
__global__ void __launch_bounds__(128) k_comb_bases(const G1A *__restrict__ pos, G1A *bases, CombWindows win) {
    const int D = win.D;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= kCells * kCellElems * D) return;
    const int ji = idx / D, k = idx % D, bit = win.bit_off(k);
    G1J p = g1_from_affine(ld_vec(&pos[(size_t)ji * kDigits + (bit >> 3)]));
    for (int r = 0; r < (bit & 7); r++) p = g1_dbl(p);
    G1A a;
    if (fp_is_zero(p.z)) {
        a.x = fp_zero();
        a.y = fp_zero();
    } else {
        const Fp zi = fp_inv_fast(p.z), z2 = fp_sqr(zi);
        a.x = fp_mul(p.x, z2);
        a.y = fp_mul(p.y, fp_mul(z2, zi));
    }
    st_vec(&bases[idx], a);
}

// Rows of the digit table, row[m - 1] = m B for m = 1..H (H = 2^(width - 1) of
// the base's window), built level by level: level L (L = 1, 2, 4, ..., H / 2)
// makes entries L + 1..2L as (L + r) B = r B + L B for r = 1..L (r = L is a
// doubling).  The additions of a level are independent, so one inversion per
// level serves all of them for the warp's kCombRows rows: log2(H) inversions
// per row group instead of one per table entry.  A warp's task is kCombRows
// base columns of one window, so that its rows have one length; the row of
// column ji and window k starts at entry ji per_i + entry_off(k).
constexpr int kCombRows = 8;
constexpr int kCombBuildThreads = 128;

__host__ __device__ inline size_t comb_build_pre_words(int H) { return ((size_t)kCombRows * (H / 2) / 32 + 1) * 384; }

__global__ void __launch_bounds__(kCombBuildThreads) k_comb_table(const G1A *__restrict__ bases, G1A *comb,
                                                                 CombWindows win, int n_cols, uint32_t *pre_all) {
    const int lane = threadIdx.x & 31;
    const int wid = blockIdx.x * (kCombBuildThreads / 32) + (threadIdx.x >> 5);
    const int n_warps = gridDim.x * (kCombBuildThreads / 32);
    uint32_t *pre = pre_all + (size_t)wid * comb_build_pre_words(1 << (win.widest() - 1));
    const int D = win.D;
    const uint32_t per_i = win.entries();
    const int n_tasks = (n_cols + kCombRows - 1) / kCombRows * D;
    for (int task = wid; task < n_tasks; task += n_warps) {
        const int k = task % D, ji0 = task / D * kCombRows;
        const uint32_t nb = (uint32_t)min(kCombRows, n_cols - ji0);
        const uint32_t H = 1u << (win.width(k) - 1), off = win.entry_off(k);
        auto entry = [&](uint32_t rb, uint32_t m) { return comb_at(comb, (size_t)(ji0 + rb) * per_i + off + m); };
        for (uint32_t r = lane; r < nb; r += 32) st_vec(entry(r, 0), ld_vec(&bases[(size_t)(ji0 + r) * D + k]));
        __syncwarp();
        for (uint32_t L = 1; L < H; L <<= 1) {
            const uint32_t P = nb * L;
            Fp acc = fp_one();
            int s = 0;
            for (uint32_t q = lane; q < P; q += 32, s++) {
                const uint32_t rb = q / L, r = q - rb * L + 1;
                const G1A x = ld_vec(entry(rb, r - 1)), y = ld_vec(entry(rb, L - 1));
                wb_store_pre(pre, s, acc);
                acc = fp_mul(acc, pair_denominator(x, y, pair_kind(x, y)));
            }
            Fp inv = warp_batch_inverse_fp(acc);
            for (int t = s - 1; t >= 0; t--) {
                const uint32_t q = lane + (uint32_t)t * 32;
                const uint32_t rb = q / L, r = q - rb * L + 1;
                const G1A x = ld_vec(entry(rb, r - 1)), y = ld_vec(entry(rb, L - 1));
                const int kind = pair_kind(x, y);
                const Fp den = pair_denominator(x, y, kind);
                const Fp inv_den = fp_mul(inv, wb_load_pre(pre, t));
                inv = fp_mul(inv, den);
                st_vec(entry(rb, L + r - 1), pair_result(x, y, kind, inv_den));
            }
            __syncwarp();
        }
    }
}

// Digit table of D windows into comb; scratch holds the bases (128 * 64 * D
// points) followed by the build's prefix products (comb_build_scratch_bytes).
int comb_build_blocks() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms * 4;
}

size_t comb_build_scratch_bytes(int windows) {
    const CombWindows win = comb_windows(windows);
    return (size_t)kCells * kCellElems * win.D * sizeof(G1A) +
           (size_t)comb_build_blocks() * (kCombBuildThreads / 32) * comb_build_pre_words(1 << (win.widest() - 1)) * 4;
}

cudaError_t launch_comb_table(const DeviceTables &t, G1A *comb, void *scratch, int windows, cudaStream_t s) {
    const CombWindows win = comb_windows(windows);
    const int n_cols = kCells * kCellElems, n_bases = n_cols * win.D;
    G1A *bases = reinterpret_cast<G1A *>(scratch);
    uint32_t *pre = reinterpret_cast<uint32_t *>(bases + n_bases);
    k_comb_bases<<<(n_bases + 127) / 128, 128, 0, s>>>(t.pos, bases, win);
    k_comb_table<<<comb_build_blocks(), kCombBuildThreads, 0, s>>>(bases, comb, win, n_cols, pre);
    count_launches(2);
    return cudaGetLastError();
}

// k_reduce over affine bucket sums: s += B_k is a mixed addition.
__global__ void __launch_bounds__(kReduceThreads) k_reduce_affine(const G1A *__restrict__ buckets, G1J *out,
                                                                 int n_outputs) {
    __shared__ G1J sh_s[kReduceThreads], sh_w[kReduceThreads];
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int o = gid / kReduceLanes, lane = gid % kReduceLanes;
    constexpr int per = kBuckets / kReduceLanes;
    G1J s = g1_identity(), w = g1_identity();
    if (o < n_outputs) {
        const G1A *bk = buckets + (size_t)o * kBuckets + lane * per;
        for (int k = per - 1; k >= 0; k--) {
            s = g1_madd(s, ld_vec(&bk[k]));
            w = g1_add(w, s);
        }
    }
    st_vec(&sh_s[threadIdx.x], s);
    st_vec(&sh_w[threadIdx.x], w);
    __syncthreads();
    if (lane != 0 || o >= n_outputs) return;
    G1J run = g1_identity(), acc = g1_identity();
    for (int l = kReduceLanes - 1; l >= 1; l--) {
        run = g1_add(run, ld_vec(&sh_s[threadIdx.x + l]));
        acc = g1_add(acc, run);
        w = g1_add(w, ld_vec(&sh_w[threadIdx.x + l]));
    }
    for (int q = 0; q < 4; q++) acc = g1_dbl(acc);
    st_vec(&out[o], g1_add(w, acc));
}

// ------------------------------------------- batch-affine bucket reduction
// sum_{k=1..128} k B_k = S + sum_{b=0..6} 2^b T_b with A_i = B_{i+1},
// S = sum_i A_i and T_b = sum of A_i over the i with bit b set.  All eight
// sums come out of one halving hierarchy, C^(j+1)_m = C^(j)_2m + C^(j)_2m+1
// (C^(0) = A, C^(7)_0 = S), because T_j = sum of the odd-indexed C^(j)_m:
// 127 additions for the hierarchy plus 120 to add up the odd lists, 247 in all,
// against 256 serial Jacobian additions for the running sum
// (field.glsl.inc:485-489).  Every addition is affine and the schedule is the
// same for every output, so rounds of it run as batch-affine rounds across
// kRedOutputs outputs; a 13-operation Horner step in Jacobian coordinates
// (6 doublings, 7 mixed additions) finishes each output.
constexpr int kRedOps = 247;
constexpr int kRedSlots = kBuckets + kRedOps;   // slots < 128 are the bucket sums themselves
constexpr int kRedMaxRounds = 8;
constexpr int kRedOutputs = 128;                 // outputs per block (one blob)
constexpr int kRedThreads = 256;
constexpr int kRedMaxPairs = 96 * kRedOutputs / kRedThreads; // round 1 has the most operations (96)

// The last kRedTail rounds (8 and 1 operations per output) are not run as
// rounds: the Horner step adds their operands instead, so each Horner term
// T_b (terms 0..6) and S (term 7) is a sum of up to 4 slots of the earlier rounds.
constexpr int kRedTail = 2;
struct ReduceSchedule {
    uint16_t dst[kRedOps], a[kRedOps], b[kRedOps];
    uint16_t round_start[kRedMaxRounds + 1];
    uint16_t term_slot[8][4];
    uint8_t term_n[8];
    int n_rounds; // rounds run as batch-affine rounds
};
__constant__ ReduceSchedule c_red;

static bool build_reduce_schedule(ReduceSchedule &s) {
    struct Op { int dst, a, b, round; };
    std::vector<Op> ops;
    std::vector<int> ready(kRedSlots, 0);
    int next = kBuckets;
    auto add = [&](int a, int b) {
        const int d = next++;
        const int r = std::max(ready[a], ready[b]) + 1;
        ready[d] = r;
        ops.push_back({d, a, b, r});
        return d;
    };
    std::vector<int> cur(kBuckets);
    for (int i = 0; i < kBuckets; i++) cur[i] = i;
    int t_slot[8];
    for (int j = 0; j < 7; j++) {
        std::vector<int> odd;
        for (size_t m = 1; m < cur.size(); m += 2) odd.push_back(cur[m]);
        std::vector<int> nxt;
        for (size_t m = 0; m + 1 < cur.size(); m += 2) nxt.push_back(add(cur[m], cur[m + 1]));
        while (odd.size() > 1) {
            std::vector<int> nl;
            for (size_t q = 0; q + 1 < odd.size(); q += 2) nl.push_back(add(odd[q], odd[q + 1]));
            if (odd.size() & 1) nl.push_back(odd.back());
            odd.swap(nl);
        }
        t_slot[j] = odd[0];
        cur.swap(nxt);
    }
    t_slot[7] = cur[0];
    if ((int)ops.size() != kRedOps) return false;
    std::stable_sort(ops.begin(), ops.end(), [](const Op &x, const Op &y) { return x.round < y.round; });
    int nr = 0;
    for (int q = 0; q < kRedOps; q++) {
        s.dst[q] = (uint16_t)ops[q].dst;
        s.a[q] = (uint16_t)ops[q].a;
        s.b[q] = (uint16_t)ops[q].b;
        nr = std::max(nr, ops[q].round);
    }
    if (nr > kRedMaxRounds || nr <= kRedTail) return false;
    s.n_rounds = nr - kRedTail;
    // Horner terms: a slot made in a tail round expands into its two operands
    std::vector<int> op_of(kRedSlots, -1);
    for (int q = 0; q < kRedOps; q++) op_of[ops[q].dst] = q;
    for (int j = 0; j < 8; j++) {
        std::vector<int> todo{t_slot[j]}, terms;
        while (!todo.empty()) {
            const int x = todo.back();
            todo.pop_back();
            if (x >= kBuckets && ready[x] > s.n_rounds) {
                todo.push_back(ops[op_of[x]].a);
                todo.push_back(ops[op_of[x]].b);
            } else {
                terms.push_back(x);
            }
        }
        if (terms.size() > 4) return false;
        s.term_n[j] = (uint8_t)terms.size();
        for (size_t k = 0; k < terms.size(); k++) s.term_slot[j][k] = (uint16_t)terms[k];
    }
    int q = 0;
    for (int r = 1; r <= nr; r++) {
        s.round_start[r - 1] = (uint16_t)q;
        while (q < kRedOps && ops[q].round == r) q++;
    }
    s.round_start[nr] = (uint16_t)q;
    for (int r = 0; r < nr; r++)
        if ((s.round_start[r + 1] - s.round_start[r]) * kRedOutputs > kRedMaxPairs * kRedThreads) return false;
    return true;
}

// sum_b 2^b T_b + S from the Horner terms (mixed additions of affine slots)
template <class Load>
__device__ __forceinline__ G1J red_horner(Load load) {
    G1J h = g1_identity();
    for (int j = 6; j >= 0; j--) {
        if (j < 6) h = g1_dbl(h);
        for (int k = 0; k < c_red.term_n[j]; k++) h = g1_madd(h, load(c_red.term_slot[j][k]));
    }
    for (int k = 0; k < c_red.term_n[7]; k++) h = g1_madd(h, load(c_red.term_slot[7][k]));
    return h;
}

__global__ void __launch_bounds__(kRedThreads, 2) k_reduce_hier(const G1A *__restrict__ bucket_aff, G1J *out,
                                                              G1A *scratch, int n_outputs) {
    __shared__ Fp tree[2 * kRedThreads];
    const int o0 = blockIdx.x * kRedOutputs;
    const int go = min(kRedOutputs, n_outputs - o0);
    G1A *slots = scratch + (size_t)blockIdx.x * kRedOutputs * kRedOps;
    auto slot = [&](int g, int s) -> G1A * {
        return s < kBuckets ? const_cast<G1A *>(&bucket_aff[((size_t)o0 + g) * kBuckets + s])
                            : &slots[(size_t)g * kRedOps + (s - kBuckets)];
    };
    for (int r = 0; r < c_red.n_rounds; r++) {
        const int q0 = c_red.round_start[r], nops = c_red.round_start[r + 1] - q0;
        const int items = nops * go;
        Fp pre[kRedMaxPairs];
        Fp acc = fp_one();
        int s = 0;
        for (int it = threadIdx.x; it < items; it += kRedThreads, s++) {
            const int g = it / nops, op = q0 + it % nops;
            const G1A a = ld_vec(slot(g, c_red.a[op])), b = ld_vec(slot(g, c_red.b[op]));
            pre[s] = acc;
            acc = fp_mul(acc, pair_denominator(a, b, pair_kind(a, b)));
        }
        Fp inv = block_batch_inverse_fp<kRedThreads>(acc, tree);
        for (int t = s - 1; t >= 0; t--) {
            const int it = threadIdx.x + t * kRedThreads;
            const int g = it / nops, op = q0 + it % nops;
            const G1A a = ld_vec(slot(g, c_red.a[op])), b = ld_vec(slot(g, c_red.b[op]));
            const int kind = pair_kind(a, b);
            const Fp den = pair_denominator(a, b, kind);
            const Fp inv_den = fp_mul(inv, pre[t]);
            inv = fp_mul(inv, den);
            st_vec(slot(g, c_red.dst[op]), pair_result(a, b, kind, inv_den));
        }
        __syncthreads();
    }
    // Horner: H = sum_b 2^b T_b, then + S
    for (int g = threadIdx.x; g < go; g += kRedThreads)
        st_vec(&out[o0 + g], red_horner([&](int x) { return ld_vec(slot(g, x)); }));
}

cudaError_t configure_reduce_schedule() {
    ReduceSchedule s;
    if (!build_reduce_schedule(s)) return cudaErrorInvalidValue;
    return cudaMemcpyToSymbol(c_red, &s, sizeof(s));
}

// The binary-split reduction of plans 3 and 4 as grid-wide rounds: round r of
// the schedule holds the same operations for every output, so its pairs are
// (output, operation) dealt to all lanes as in the phase rounds; the Horner
// tail runs one output per thread.
struct FlatRArgs {
    const G1A *buckets; // [output][128] bucket sums
    G1A *slots;         // [output][kRedOps] intermediate sums
    uint32_t *pre;
    Fp *others, *tot, *totinv;
    size_t slots_pre;
    int n_out;
};

__device__ __forceinline__ G1A *red_slot(const FlatRArgs &a, uint32_t o, int s) {
    return s < kBuckets ? const_cast<G1A *>(&a.buckets[(size_t)o * kBuckets + s])
                        : &a.slots[(size_t)o * kRedOps + (s - kBuckets)];
}

// shared copy of round r's operations (the schedule in constant memory is read
// at a different index by every lane, which constant memory serialises)
struct RedRound {
    uint16_t a[kRedOps], b[kRedOps], d[kRedOps];
    int q0, nops;
};

__device__ void red_stage(RedRound &rr, int r) {
    const int q0 = c_red.round_start[r], nops = c_red.round_start[r + 1] - q0;
    for (int q = threadIdx.x; q < nops; q += blockDim.x) {
        rr.a[q] = c_red.a[q0 + q];
        rr.b[q] = c_red.b[q0 + q];
        rr.d[q] = c_red.dst[q0 + q];
    }
    if (threadIdx.x == 0) {
        rr.q0 = q0;
        rr.nops = nops;
    }
    __syncthreads();
}

__device__ __forceinline__ void flatr_pass1_body(const FlatRArgs &a, int r, RedRound &rr, uint32_t gl, uint32_t NL) {
    red_stage(rr, r);
    const uint32_t wg = gl >> 5;
    const uint32_t nops = (uint32_t)rr.nops;
    const uint32_t P = (uint32_t)a.n_out * nops;
    uint32_t *pre = a.pre + (size_t)wg * a.slots_pre * 384;
    Fp acc = fp_one();
    int s = 0;
    for (uint32_t p = gl; p < P; p += NL, s++) {
        const uint32_t o = p / nops, q = p - o * nops;
        const G1A *pa = red_slot(a, o, rr.a[q]), *pb = red_slot(a, o, rr.b[q]);
        wb_store_pre(pre, s, acc);
        acc = fp_mul(acc, pair_denominator_x(ld_vec(&pa->x), ld_vec(&pb->x), [&] { return ld_vec(pa); },
                                             [&] { return ld_vec(pb); }));
    }
    flat_pass1_products(acc, a.others, a.tot, gl, wg);
}
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_flatr_pass1(FlatRArgs a, int r) {
    __shared__ RedRound rr;
    flatr_pass1_body(a, r, rr, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

__device__ __forceinline__ void flatr_pass2_body(const FlatRArgs &a, int r, RedRound &rr, uint32_t gl, uint32_t NL) {
    red_stage(rr, r);
    const uint32_t wg = gl >> 5;
    const uint32_t nops = (uint32_t)rr.nops;
    const uint32_t P = (uint32_t)a.n_out * nops;
    const uint32_t *pre = a.pre + (size_t)wg * a.slots_pre * 384;
    Fp inv = fp_mul(ld_vec(&a.totinv[wg]), ld_vec(&a.others[gl]));
    const int S = P > gl ? (int)((P - gl + NL - 1) / NL) : 0;
    for (int t = S - 1; t >= 0; t--) {
        const uint32_t p = gl + (uint32_t)t * NL;
        const uint32_t o = p / nops, q = p - o * nops;
        const G1A x = ld_vec(red_slot(a, o, rr.a[q])), y = ld_vec(red_slot(a, o, rr.b[q]));
        const int kind = pair_kind(x, y);
        const Fp den = pair_denominator(x, y, kind);
        const Fp inv_den = fp_mul(inv, wb_load_pre(pre, t));
        inv = fp_mul(inv, den);
        st_vec(red_slot(a, o, rr.d[q]), pair_result(x, y, kind, inv_den));
    }
}
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_flatr_pass2(FlatRArgs a, int r) {
    __shared__ RedRound rr;
    flatr_pass2_body(a, r, rr, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// H = sum_b 2^b T_b (Horner over the 7 bit sums), then + S: the reduction's result.
// One thread per output: at 7.5 M products per 256 blobs the step is near the
// multiply throughput, and splitting an output's terms over lanes or warps
// (measured) only added the combining work.
__global__ void __launch_bounds__(128) k_flatr_horner(FlatRArgs a, G1J *out) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= (uint32_t)a.n_out) return;
    st_vec(&out[o], red_horner([&](int x) { return ld_vec(red_slot(a, o, x)); }));
}

// Phase B's Horner step and stage 9 in one launch (plans 3-4): a block is one
// blob and its 128 threads the blob's outputs, so each thread's Horner result
// goes to shared memory for the unfolding instead of through HBM.
__global__ void __launch_bounds__(kCells) k_finish_horner(FlatRArgs a, uint8_t *proofs, int levels) {
    __shared__ Fp tree[2 * kCells];
    __shared__ G1J outp[kCells];
    const int b = blockIdx.x, t = threadIdx.x;
    const uint32_t o = (uint32_t)b * kCells + (uint32_t)t;
    st_vec(&outp[t], red_horner([&](int x) { return ld_vec(red_slot(a, o, x)); }));
    finish_blob(outp, tree, proofs, b, t, levels);
}

VKZG_COOP_FN void coop_flatr_pass1(FlatRArgs a, int r, RedRound &rr, uint32_t gl, uint32_t NL) {
    flatr_pass1_body(a, r, rr, gl, NL);
}
VKZG_COOP_FN void coop_flatr_pass2(FlatRArgs a, int r, RedRound &rr, uint32_t gl, uint32_t NL) {
    flatr_pass2_body(a, r, rr, gl, NL);
}

// Cooperative form of the reduction's rounds (the Horner step stays its own
// launch: one output per thread, a different register budget).
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_coop_reduce(FlatRArgs a, int rounds, GridSync g) {
    __shared__ RedRound rr;
    const uint32_t gl = blockIdx.x * blockDim.x + threadIdx.x, NL = gridDim.x * blockDim.x;
    for (int r = 0; r < rounds; r++) {
        coop_flatr_pass1(a, r, rr, gl, NL);
        if (!grid_sync(g)) return;
        coop_invert(a.tot, a.totinv, NL >> 5, gl, NL);
        if (!grid_sync(g)) return;
        coop_flatr_pass2(a, r, rr, gl, NL);
        if (r + 1 < rounds && !grid_sync(g)) return;
    }
}

// proofs non-null: the Horner step runs inside stage 9 (k_finish_horner), which
// writes the compressed proofs; else it writes the reduction's results to out.
int launch_reduce_flat(const ProofWork &w, const G1A *buckets, G1J *out, int n_out, cudaStream_t s,
                       uint8_t *proofs = nullptr) {
    // the schedule's round count, computed once (thread-safe static initialisation:
    // serving lanes launch from several threads)
    static const int rounds = [] {
        ReduceSchedule h;
        return build_reduce_schedule(h) ? h.n_rounds : 0;
    }();
    FlatRArgs a;
    a.buckets = buckets;
    a.slots = w.red_scratch;
    a.pre = w.flat_pre;
    a.others = w.flat_others;
    a.tot = w.flat_tot;
    a.totinv = w.flat_totinv;
    a.slots_pre = w.flat_slots;
    a.n_out = n_out;
    const int blocks = w.flat_blocks, warps = blocks * kFlatThreads / 32;
    int launched = 1;
    if (w.coop) {
        launch_coop(k_coop_reduce, blocks, 0, s, a, rounds, make_sync(w, n_out / kCells));
        launched += 1;
    } else {
        for (int r = 0; r < rounds; r++) {
            k_flatr_pass1<<<blocks, kFlatThreads, 0, s>>>(a, r);
            launch_flat_invert(a.tot, a.totinv, warps, s);
            k_flatr_pass2<<<blocks, kFlatThreads, 0, s>>>(a, r);
        }
        launched += 3 * rounds;
    }
    if (proofs) k_finish_horner<<<n_out / kCells, kCells, 0, s>>>(a, proofs, kPartLevels);
    else k_flatr_horner<<<(n_out + 127) / 128, 128, 0, s>>>(a, out);
    return launched;
}

// The ladder to affine form as one grid-wide round (plans 3-4): Z values dealt
// to all lanes, one inversion per warp product, x = X / Z^2, y = Y / Z^3;
// infinity (Z = 0) -> (0, 0); each point is written with its phi image.
struct NormArgs {
    const G1J *in;
    G1A *out;
    uint32_t *pre;
    Fp *others, *tot, *totinv;
    size_t slots_pre;
    uint32_t n;
};

__device__ __forceinline__ void norm_pass1_body(const NormArgs &a, uint32_t gl, uint32_t NL) {
    const uint32_t wg = gl >> 5;
    uint32_t *pre = a.pre + (size_t)wg * a.slots_pre * 384;
    Fp acc = fp_one();
    int s = 0;
    for (uint32_t p = gl; p < a.n; p += NL, s++) {
        const Fp z = ld_vec(&a.in[p].z);
        wb_store_pre(pre, s, acc);
        acc = fp_mul(acc, fp_is_zero(z) ? fp_one() : z);
    }
    flat_pass1_products(acc, a.others, a.tot, gl, wg);
}
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_norm_pass1(NormArgs a) {
    norm_pass1_body(a, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

__device__ __forceinline__ void norm_pass2_body(const NormArgs &a, uint32_t gl, uint32_t NL) {
    const uint32_t wg = gl >> 5;
    const uint32_t *pre = a.pre + (size_t)wg * a.slots_pre * 384;
    Fp inv = fp_mul(ld_vec(&a.totinv[wg]), ld_vec(&a.others[gl]));
    const int S = a.n > gl ? (int)((a.n - gl + NL - 1) / NL) : 0;
    for (int t = S - 1; t >= 0; t--) {
        const uint32_t p = gl + (uint32_t)t * NL;
        const G1J q = ld_vec(&a.in[p]);
        const bool inf = fp_is_zero(q.z);
        const Fp zi = fp_mul(inv, wb_load_pre(pre, t));
        inv = fp_mul(inv, inf ? fp_one() : q.z);
        G1A r;
        if (inf) {
            r.x = fp_zero();
            r.y = fp_zero();
        } else {
            const Fp z2 = fp_sqr(zi);
            r.x = fp_mul(q.x, z2);
            r.y = fp_mul(q.y, fp_mul(z2, zi));
        }
        // in: [row][16] ladder; out: [row][32], slot 16 + d = phi(slot d)
        const size_t dst = (size_t)(p / kLadderDigits) * kDigits + p % kLadderDigits;
        st_vec(&a.out[dst], r);
        st_vec(&a.out[dst + kLadderDigits], g1_phi(r));
    }
}
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_norm_pass2(NormArgs a) {
    norm_pass2_body(a, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// the ladder to affine form with its phi images, into w.ladder_aff; returns the launches made
VKZG_COOP_FN void coop_norm_pass1(NormArgs a, uint32_t gl, uint32_t NL) { norm_pass1_body(a, gl, NL); }
VKZG_COOP_FN void coop_norm_pass2(NormArgs a, uint32_t gl, uint32_t NL) { norm_pass2_body(a, gl, NL); }

// Cooperative form of the ladder's normalisation round.
__global__ void __launch_bounds__(kFlatThreads, kFlatBlocksPerSM) k_coop_norm(NormArgs a, GridSync g) {
    const uint32_t gl = blockIdx.x * blockDim.x + threadIdx.x, NL = gridDim.x * blockDim.x;
    coop_norm_pass1(a, gl, NL);
    if (!grid_sync(g)) return;
    coop_invert(a.tot, a.totinv, NL >> 5, gl, NL);
    if (!grid_sync(g)) return;
    coop_norm_pass2(a, gl, NL);
}

int launch_normalize_flat(const ProofWork &w, int n, cudaStream_t s) {
    const int blocks = w.flat_blocks, warps = blocks * kFlatThreads / 32;
    NormArgs na;
    na.in = w.ladder;
    na.out = w.ladder_aff;
    na.pre = w.flat_pre;
    na.others = w.flat_others;
    na.tot = w.flat_tot;
    na.totinv = w.flat_totinv;
    na.slots_pre = w.flat_slots;
    na.n = (uint32_t)(n * kCells * kLadderDigits);
    if (w.coop) {
        launch_coop(k_coop_norm, blocks, 0, s, na, make_sync(w, n));
        return 1;
    }
    k_norm_pass1<<<blocks, kFlatThreads, 0, s>>>(na);
    launch_flat_invert(na.tot, na.totinv, warps, s);
    k_norm_pass2<<<blocks, kFlatThreads, 0, s>>>(na);
    return 3;
}

// ---------------------------------------------------------------- launcher
// Stages 1-2 (per blob) for blobs [off, off + cnt) of the working set: a host
// upload in pieces runs them on each piece as it lands.
cudaError_t launch_proofs_front(const DeviceTables &t, const ProofWork &w, int off, int cnt, cudaStream_t s) {
    if (cnt <= 0) return cudaSuccess;
    const size_t smem_ntt = (size_t)kBlobElems * sizeof(Fr);
    k_blob_to_coeffs<<<cnt, kNttThreads, smem_ntt, s>>>(w.blobs + (size_t)off * kBlobBytes,
                                                        w.coeffs + (size_t)off * kBlobElems, t.roots_inv,
                                                        t.inv_blob_r2, w.err + off);
    k_circulant<<<dim3(kCellElems / kCircCols, cnt), kCircCols * 64, 0, s>>>(
        w.coeffs + (size_t)off * kBlobElems, w.scalars + (size_t)off * kCells * kCellElems, t.roots_fwd);
    count_launches(2);
    return cudaGetLastError();
}

// ev (nullable): kProofStages + 1 events recorded around the stages.
// skip_front: stages 1-2 already ran (launch_proofs_front).
cudaError_t launch_proofs_timed(const DeviceTables &t, const ProofWork &w, int n, cudaStream_t s, cudaEvent_t *ev,
                                bool skip_front) {
    if (n <= 0) return cudaSuccess;
    int k = 0;
    auto mark = [&]() {
        if (ev) cudaEventRecord(ev[k++], s);
    };
    const size_t smem_ntt = (size_t)kBlobElems * sizeof(Fr);
    const int n_out = n * kCells;
    const int red_blocks = (n_out * kReduceLanes + kReduceThreads - 1) / kReduceThreads;
    const int n_lad = n * kCells * kLadderDigits;
    mark();
    if (!skip_front)
        k_blob_to_coeffs<<<n, kNttThreads, smem_ntt, s>>>(w.blobs, w.coeffs, t.roots_inv, t.inv_blob_r2, w.err);
    mark();
    if (!skip_front)
        k_circulant<<<dim3(kCellElems / kCircCols, n), kCircCols * 64, 0, s>>>(w.coeffs, w.scalars, t.roots_fwd);
    mark();
    // plan: 0 serial Jacobian buckets + serial reduction; 1 batch-affine buckets
    // per warp + binary-split reduction; 2 as 1 with the serial reduction; 3 phase A
    // over the digit table in grid-wide rounds (no reduction), phase B in grid-wide
    // rounds + binary-split reduction; 4 phase A as 1, phase B as 3
    const bool affine = w.plan != 0 && w.ba_blocks > 0;
    const bool comb = w.plan == 3 && w.comb != nullptr && w.flat_dig != nullptr && w.ba_blocks > 0;
    const bool flatb = (w.plan == 3 || w.plan == 4) && w.flat_pre != nullptr && t.fb_rounds > 0 && w.ba_blocks > 0;
    if (!flatb && w.coop) { // the cooperative forms serve plans 3-4 only
        ProofWork w2 = w;
        w2.coop = false;
        return launch_proofs_timed(t, w2, n, s, ev, skip_front);
    }
    const bool hier = w.plan == 1 || w.plan == 3 || w.plan == 4;
    // coefficients, circulant, phase A, its reduction, ladder, normalisation,
    // phase B, its reduction, finish; the launchers add their extra rounds
    int launched = skip_front ? 7 : 9;
    const int ba_grid = std::min(w.ba_blocks, (n_out / kWarpOutputs + kBAWarps - 1) / kBAWarps);
    auto reduce = [&](uint8_t *proofs) {
        if (flatb) launched += launch_reduce_flat(w, w.bucket_aff, w.points, n_out, s, proofs) - 1;
        else if (!affine) k_reduce<<<red_blocks, kReduceThreads, 0, s>>>(w.buckets, w.points, n_out);
        else if (hier)
            k_reduce_hier<<<(n_out + kRedOutputs - 1) / kRedOutputs, kRedThreads, 0, s>>>(w.bucket_aff, w.points,
                                                                                       w.red_scratch, n_out);
        else k_reduce_affine<<<red_blocks, kReduceThreads, 0, s>>>(w.bucket_aff, w.points, n_out);
    };
    // the cooperative launches' barrier words start at zero each step
    if (flatb && w.coop) cudaMemsetAsync(w.sync, 0, 4 * sizeof(uint32_t), s);
    if (comb) {
        cudaMemsetAsync(w.task_ctr, 0, 2 * sizeof(uint32_t), s);
        launched += launch_phase_a_flat(w, n, s) - 2; // no phase-A bucket kernel, no reduction
    } else if (affine) {
        cudaMemsetAsync(w.task_ctr, 0, 2 * sizeof(uint32_t), s);
        k_phase_a_affine<<<ba_grid, kBAThreads, kBASmem, s>>>(w.scalars, t.pos, w.bucket_aff, w.ba_scratch,
                                                               n_out, w.task_ctr);
    } else {
        k_phase_a<<<dim3(kCells, n), kBuckets, 0, s>>>(w.scalars, t.pos, w.buckets);
    }
    mark();
    if (!comb) reduce(nullptr);
    mark();
    // plans 3-4 split phase B into the kPartLevels parts, plans 0-2 into two
    // halves; the fold (stage 5) runs inside the ladder's launch
    const int levels = flatb ? kPartLevels : 1;
    mark();
    k_ladder<<<n, kCells, 0, s>>>(w.points, w.ladder, levels);
    mark();
    if (flatb) launched += launch_normalize_flat(w, n, s) - 1;
    else k_normalize<<<(n_lad + kNormThreads - 1) / kNormThreads, kNormThreads, 0, s>>>(w.ladder, w.ladder_aff, n_lad);
    mark();
    if (flatb && w.coop) {
        launched += launch_phase_b_coop(t, w, n, s) - 1;
    } else if (flatb) {
        launched += launch_deriv_flat(t, w, n, s);
        launched += launch_phase_b_flat(t, w, n, s) - 1;
    } else if (affine) {
        k_phase_b_affine<<<ba_grid, kBAThreads, kPhaseBSmem, s>>>(w.ladder_aff, t.tap_items[0], t.tap_offsets[0],
                                                              t.tap_items[1], t.tap_offsets[1], w.bucket_aff,
                                                              w.ba_scratch, n_out, w.task_ctr + 1);
    } else {
        k_phase_b<<<dim3(kCells, n), kBuckets, 0, s>>>(w.ladder_aff, t.tap_items[0], t.tap_offsets[0],
                                                       t.tap_perm[0], t.tap_items[1], t.tap_offsets[1],
                                                       t.tap_perm[1], w.buckets);
    }
    mark();
    // plans 3-4: phase B's Horner step runs inside stage 9's launch
    reduce(flatb ? w.proofs : nullptr);
    mark();
    if (flatb) launched--;
    else k_finish<<<n, kCells, 0, s>>>(w.points, w.proofs, levels);
    mark();
    count_launches(launched);
    return cudaGetLastError();
}

cudaError_t launch_proofs(const DeviceTables &t, const ProofWork &w, int n, cudaStream_t s) {
    return launch_proofs_timed(t, w, n, s, nullptr, false);
}

// Resident blocks per SM of the batch-affine kernels (sizes their persistent grid).
int batch_affine_blocks_per_sm() {
    int a = 0, b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_phase_a_affine, kBAThreads, kBASmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_phase_b_affine, kBAThreads, kPhaseBSmem);
    return std::max(1, std::min(a, b));
}

size_t reduce_scratch_points(int cap_blobs) { return (size_t)cap_blobs * kCells * kRedOps; }

// True when every cooperative kernel of plans 3-4 fits blocks_per_sm resident
// blocks per SM (the grid of the rounds) and the device takes cooperative launches.
bool coop_supported(int blocks_per_sm) {
    int dev = 0, coop = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop)
        return false;
    int a = 0, b = 0, c = 0, d = 0, e = 0;
    if (cudaFuncSetAttribute(k_coop_phase_b, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFlatBSmem) !=
        cudaSuccess)
        return false;
    if (cudaFuncSetAttribute(k_coop_tree<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStage2Bytes) !=
        cudaSuccess)
        return false;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_coop_tree<true>, kFlatThreads, kStage2Bytes);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_coop_norm, kFlatThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c, k_coop_phase_b, kFlatThreads, kFlatBSmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&d, k_coop_reduce, kFlatThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&e, k_coop_tree<false>, kFlatThreads, 0);
    return std::min(std::min(std::min(a, b), std::min(c, d)), e) >= blocks_per_sm;
}

cudaError_t configure_proof_kernels() {
    cudaError_t e = configure_reduce_schedule();
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_blob_to_coeffs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kBlobElems * sizeof(Fr)));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_phase_a_affine, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBASmem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_flat_pass1<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStage1Bytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_flat_pass2<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStage2Bytes);
    if (e != cudaSuccess) return e;
    e = configure_list_rounds();
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_phase_b_affine, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPhaseBSmem);
}

} // namespace vkzg
