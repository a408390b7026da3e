// Device helpers shared by the proof, recovery and setup kernels: 16-byte
// vector loads/stores of field elements and points, block-wide batch
// inversion, and radix-2 NTT stages over a tile in shared memory.
#pragma once

#include "curve.cuh"
#include "inverse.cuh"

namespace vkzg {

// ------------------------------------------------------------ loads/stores
template <typename T>
__device__ __forceinline__ T ld_vec(const T *p) {
    static_assert(sizeof(T) % 16 == 0, "16-byte multiple");
    T r;
    const uint4 *s = reinterpret_cast<const uint4 *>(p);
    uint4 *d = reinterpret_cast<uint4 *>(&r);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 16); i++) d[i] = s[i];
    return r;
}
// read-only path (table data that no kernel in flight writes)
template <typename T>
__device__ __forceinline__ T ldg_vec(const T *p) {
    T r;
    const uint4 *s = reinterpret_cast<const uint4 *>(p);
    uint4 *d = reinterpret_cast<uint4 *>(&r);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 16); i++) d[i] = __ldg(s + i);
    return r;
}
template <typename T>
__device__ __forceinline__ void st_vec(T *p, const T &v) {
    const uint4 *s = reinterpret_cast<const uint4 *>(&v);
    uint4 *d = reinterpret_cast<uint4 *>(p);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 16); i++) d[i] = s[i];
}

__device__ __forceinline__ G1J g1_shfl_down(const G1J &p, int delta) {
    G1J r;
#pragma unroll
    for (int i = 0; i < 12; i++) {
        r.x.v[i] = __shfl_down_sync(0xffffffffu, p.x.v[i], delta);
        r.y.v[i] = __shfl_down_sync(0xffffffffu, p.y.v[i], delta);
        r.z.v[i] = __shfl_down_sync(0xffffffffu, p.z.v[i], delta);
    }
    return r;
}

// ------------------------------------------------------- batch inversion
// Inverts one Fp per thread across a block of NT threads (power of two) with a
// product tree in shared memory: NT-1 multiplies up, one divstep inversion
// (inverse.cuh) at the root, 2(NT-1) down.  Zero inputs must be replaced by
// one by the caller.
// `tree` holds 2*NT Fp.
template <int NT>
__device__ Fp block_batch_inverse_fp(const Fp &z, Fp *tree) {
    const int t = threadIdx.x;
    // leaves at [NT, 2NT), node k has children 2k, 2k+1, root at 1
    st_vec(&tree[NT + t], z);
    __syncthreads();
    for (int width = NT / 2; width >= 1; width >>= 1) {
        if (t < width) {
            const int k = width + t;
            st_vec(&tree[k], fp_mul(ld_vec(&tree[2 * k]), ld_vec(&tree[2 * k + 1])));
        }
        __syncthreads();
    }
    if (t == 0) st_vec(&tree[1], fp_inv_fast(ld_vec(&tree[1])));
    __syncthreads();
    // push inverses down: inv(child) = inv(parent) * sibling
    for (int width = 1; width < NT; width <<= 1) {
        if (t < width) {
            const int k = width + t;
            const Fp ip = ld_vec(&tree[k]);
            const Fp l = ld_vec(&tree[2 * k]), r = ld_vec(&tree[2 * k + 1]);
            st_vec(&tree[2 * k], fp_mul(ip, r));
            st_vec(&tree[2 * k + 1], fp_mul(ip, l));
        }
        __syncthreads();
    }
    const Fp res = ld_vec(&tree[NT + t]);
    __syncthreads();
    return res;
}

template <int NT>
__device__ Fr block_batch_inverse_fr(const Fr &z, Fr *tree) {
    // the first NT threads of the block hold the values; every thread of the
    // block must call (the barriers), and threads from NT on get their z back
    const int t = threadIdx.x;
    if (t < NT) st_vec(&tree[NT + t], z);
    __syncthreads();
    for (int width = NT / 2; width >= 1; width >>= 1) {
        if (t < width) {
            const int k = width + t;
            st_vec(&tree[k], fr_mul(ld_vec(&tree[2 * k]), ld_vec(&tree[2 * k + 1])));
        }
        __syncthreads();
    }
    if (t == 0) st_vec(&tree[1], fr_inv_fast(ld_vec(&tree[1])));
    __syncthreads();
    for (int width = 1; width < NT; width <<= 1) {
        if (t < width) {
            const int k = width + t;
            const Fr ip = ld_vec(&tree[k]);
            const Fr l = ld_vec(&tree[2 * k]), r = ld_vec(&tree[2 * k + 1]);
            st_vec(&tree[2 * k], fr_mul(ip, r));
            st_vec(&tree[2 * k + 1], fr_mul(ip, l));
        }
        __syncthreads();
    }
    const Fr res = t < NT ? ld_vec(&tree[NT + t]) : z;
    __syncthreads();
    return res;
}

// ------------------------------------------------------------ grid barrier
// A barrier across every block of a cooperative launch (all blocks resident),
// whose every wait is bounded.  word[0] counts arrivals, word[1] is the
// generation the last arrival advances, word[2] is the failure flag: a block
// that waits spin_limit polls without the generation moving (or that finds
// the flag set) sets the flag, marks every error word of err[0..n_err) with
// kSyncFailed and returns false; the kernel then returns, and the other
// blocks, finding the flag set at their next wait, return too.  The words
// start at zero (the launcher clears them); after a barrier the arrival count
// is zero again, so one launch reuses them across its barriers.
constexpr uint32_t kSyncFailed = 0x80000000u; // VKZG_B200_DEVICE_FAILED in include/vkzg_b200.h
struct GridSync {
    uint32_t *word;
    uint32_t *err;
    uint32_t n_err;
    uint32_t spin_limit;
    uint32_t expected; // arrivals that complete a barrier: gridDim.x
};

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

static __device__ __forceinline__ bool grid_sync(const GridSync g) {
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        uint32_t *cnt = g.word, *gen = g.word + 1, *flag = g.word + 2;
        if (ld_acquire_gpu(flag)) {
            ok = 0;
        } else {
            const uint32_t my_gen = ld_acquire_gpu(gen);
            __threadfence();
            if (atomicAdd(cnt, 1u) == g.expected - 1) {
                atomicExch(cnt, 0u);
                __threadfence();
                atomicAdd(gen, 1u);
            } else {
                for (uint32_t spins = 0; ld_acquire_gpu(gen) == my_gen; spins++) {
                    if (spins >= g.spin_limit || ld_acquire_gpu(flag)) {
                        if (atomicExch(flag, 1u) == 0u)
                            for (uint32_t b = 0; b < g.n_err; b++) atomicOr(&g.err[b], kSyncFailed);
                        ok = 0;
                        break;
                    }
                    __nanosleep(100);
                }
            }
            __threadfence();
        }
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// ------------------------------------------------------------ NTT stages
// roots: w_8192^(+-i), i < 8192 (Montgomery).  A transform of length n uses
// w_len^j = roots[j * 8192 / len].
//
// DIT (Cooley-Tukey): bit-reversed input, natural output, lengths 2..n.
// DIF (Gentleman-Sande): natural input, bit-reversed output, lengths n..2.
// Each call runs stages [len_lo, len_hi] over `count` independent n-point
// transforms laid out back to back in `s`, with all NT threads cooperating.
template <int NT>
__device__ void smem_dit(Fr *s, int log_n, int count, int len_lo, int len_hi, const Fr *__restrict__ roots) {
    const int n = 1 << log_n;
    const int total = (n >> 1) * count;
    for (int len = len_lo; len <= len_hi; len <<= 1) {
        const int h = len >> 1, stride = 8192 / len;
        for (int q = threadIdx.x; q < total; q += NT) {
            const int tr = q >> (log_n - 1), k = q & ((n >> 1) - 1);
            const int blk = k / h, j = k - blk * h;
            Fr *base = s + tr * n + blk * len + j;
            const Fr x = ld_vec(base);
            const Fr y = fr_mul(ld_vec(base + h), ldg_vec(&roots[j * stride]));
            st_vec(base, fr_add(x, y));
            st_vec(base + h, fr_sub(x, y));
        }
        __syncthreads();
    }
}

template <int NT>
__device__ void smem_dif(Fr *s, int log_n, int count, int len_hi, int len_lo, const Fr *__restrict__ roots) {
    const int n = 1 << log_n;
    const int total = (n >> 1) * count;
    for (int len = len_hi; len >= len_lo; len >>= 1) {
        const int h = len >> 1, stride = 8192 / len;
        for (int q = threadIdx.x; q < total; q += NT) {
            const int tr = q >> (log_n - 1), k = q & ((n >> 1) - 1);
            const int blk = k / h, j = k - blk * h;
            Fr *base = s + tr * n + blk * len + j;
            const Fr x = ld_vec(base);
            const Fr y = ld_vec(base + h);
            st_vec(base, fr_add(x, y));
            st_vec(base + h, fr_mul(fr_sub(x, y), ldg_vec(&roots[j * stride])));
        }
        __syncthreads();
    }
}

// The same stages two at a time: a radix-4 butterfly on the elements
// j, j + h, j + 2h, j + 3h of each group of 4h does stage len = 2h and stage
// 4h in registers (the same four products per four elements as two radix-2
// stages), so each pair of stages is one read and one write of shared memory
// and one barrier instead of two.  An odd stage count starts (DIT) or ends
// (DIF) with one radix-2 stage at the shortest length.
template <int NT>
__device__ void smem_dit4(Fr *s, int log_n, int count, int len_lo, int len_hi, const Fr *__restrict__ roots) {
    int stages = 0;
    for (int len = len_lo; len <= len_hi; len <<= 1) stages++;
    int len = len_lo;
    if (stages & 1) {
        smem_dit<NT>(s, log_n, count, len, len, roots);
        len <<= 1;
    }
    const int n = 1 << log_n;
    const int total = (n >> 2) * count;
    for (; len < len_hi; len <<= 2) {
        const int h = len >> 1, stride = 8192 / (2 * len); // twiddles of the longer stage: w_{2 len}^j
        for (int q = threadIdx.x; q < total; q += NT) {
            const int tr = q >> (log_n - 2), k = q & ((n >> 2) - 1);
            const int blk = k / h, j = k - blk * h;
            Fr *base = s + tr * n + blk * 4 * h + j;
            const Fr a0 = ld_vec(base), a1 = ld_vec(base + h), a2 = ld_vec(base + 2 * h), a3 = ld_vec(base + 3 * h);
            const Fr w1 = ldg_vec(&roots[2 * j * stride]);        // w_len^j
            const Fr w2 = ldg_vec(&roots[j * stride]);            // w_{2 len}^j
            const Fr w3 = ldg_vec(&roots[(j + h) * stride]);      // w_{2 len}^(j + h)
            Fr t = fr_mul(a1, w1);
            const Fr b0 = fr_add(a0, t), b1 = fr_sub(a0, t);
            t = fr_mul(a3, w1);
            const Fr b2 = fr_add(a2, t), b3 = fr_sub(a2, t);
            t = fr_mul(b2, w2);
            st_vec(base, fr_add(b0, t));
            st_vec(base + 2 * h, fr_sub(b0, t));
            t = fr_mul(b3, w3);
            st_vec(base + h, fr_add(b1, t));
            st_vec(base + 3 * h, fr_sub(b1, t));
        }
        __syncthreads();
    }
}

template <int NT>
__device__ void smem_dif4(Fr *s, int log_n, int count, int len_hi, int len_lo, const Fr *__restrict__ roots) {
    int stages = 0;
    for (int len = len_hi; len >= len_lo; len >>= 1) stages++;
    const int n = 1 << log_n;
    const int total = (n >> 2) * count;
    int len = len_hi; // the longer of each pair of stages
    for (int pairs = stages >> 1; pairs > 0; pairs--, len >>= 2) {
        const int h = len >> 2, stride = 8192 / len; // w_len^j and w_{len/2}^j = w_len^(2j)
        for (int q = threadIdx.x; q < total; q += NT) {
            const int tr = q >> (log_n - 2), k = q & ((n >> 2) - 1);
            const int blk = k / h, j = k - blk * h;
            Fr *base = s + tr * n + blk * 4 * h + j;
            const Fr a0 = ld_vec(base), a1 = ld_vec(base + h), a2 = ld_vec(base + 2 * h), a3 = ld_vec(base + 3 * h);
            const Fr w2 = ldg_vec(&roots[j * stride]);            // w_len^j
            const Fr w3 = ldg_vec(&roots[(j + h) * stride]);      // w_len^(j + h)
            const Fr w1 = ldg_vec(&roots[2 * j * stride]);        // w_{len/2}^j
            const Fr t0 = fr_add(a0, a2), t2 = fr_mul(fr_sub(a0, a2), w2);
            const Fr t1 = fr_add(a1, a3), t3 = fr_mul(fr_sub(a1, a3), w3);
            st_vec(base, fr_add(t0, t1));
            st_vec(base + h, fr_mul(fr_sub(t0, t1), w1));
            st_vec(base + 2 * h, fr_add(t2, t3));
            st_vec(base + 3 * h, fr_mul(fr_sub(t2, t3), w1));
        }
        __syncthreads();
    }
    if (stages & 1) smem_dif<NT>(s, log_n, count, len, len, roots);
}

} // namespace vkzg
