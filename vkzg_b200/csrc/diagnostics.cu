// Throughput probes for the integer roofline: the device's 32-bit IMAD issue
// rate and the library's own Fp / Fr Montgomery multiply rates.  The reference
// has no counterpart; its README quotes only end-to-end timings.
#include "../../include/vkzg_b200.h"
#include "bucket_sum.cuh"
#include "device_util.cuh"
#include "kernels.h"

#include <vector>

namespace vkzg {

constexpr int kProbeIters = 4096;

// 8 independent mad.lo chains per thread: 8 * kProbeIters IMAD per thread.
__global__ void __launch_bounds__(256) k_probe_imad(uint32_t seed, uint32_t *sink) {
    uint32_t a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + threadIdx.x * 8 + k;
    const uint32_t m = seed | 1u;
    for (int i = 0; i < kProbeIters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(m), "r"(a[(k + 1) & 7]));
    }
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) acc ^= a[k];
    if (acc == 0x12345678u) sink[0] = acc;
}

// 8 independent mad.wide.u32 chains per thread (64-bit addend and result):
// 8 * kProbeIters wide multiply-adds per thread.
__global__ void __launch_bounds__(256) k_probe_imad_wide(uint32_t seed, uint32_t *sink) {
    uint64_t a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = seed + threadIdx.x * 8 + k;
    const uint32_t m = seed | 1u;
    for (int i = 0; i < kProbeIters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++)
            asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(a[k]) : "r"(m), "r"((uint32_t)a[(k + 1) & 7]));
    }
    uint64_t acc = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) acc ^= a[k];
    if ((uint32_t)acc == 0x12345678u) sink[0] = (uint32_t)(acc >> 32);
}

// 8 independent fma.rn.f64 chains per thread
__global__ void __launch_bounds__(256) k_probe_dfma(uint32_t seed, uint32_t *sink) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = 1.0 + 1e-9 * (seed + threadIdx.x * 8 + k);
    const double m = 1.0 - 1e-12 * seed;
    for (int i = 0; i < kProbeIters; i++) {
#pragma unroll
        for (int k = 0; k < 8; k++) asm volatile("fma.rn.f64 %0, %0, %1, %2;" : "+d"(a[k]) : "d"(m), "d"(a[(k + 1) & 7]));
    }
    double acc = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) acc += a[k];
    if (acc == 0.125) sink[0] = 1u;
}

// one inversion per thread on pseudo-random values below p (the scalar form)
template <bool VAR>
__global__ void __launch_bounds__(64) k_probe_inv(uint32_t seed, int n, uint32_t *sink) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    Fp x;
    uint32_t h = seed * 0x9e3779b9u + (uint32_t)t * 0x85ebca6bu;
#pragma unroll
    for (int k = 0; k < 12; k++) {
        h ^= h >> 15;
        h *= 0x2c1b3c6du;
        h ^= h >> 12;
        x.v[k] = h;
    }
    x.v[11] &= 0x0fffffffu;
    const Fp y = fp_inv_fast<VAR>(x);
    if (y.v[0] == 0x12345678u) sink[0] = y.v[1];
}

// the same values inverted four lanes a value, as k_flat_invert does
__global__ void __launch_bounds__(128) k_probe_inv_quad(uint32_t seed, int n, uint32_t *sink) {
    __shared__ uint64_t t4[kDivstepEntries<4>], t2[kDivstepEntries<2>];
    for (int i = threadIdx.x; i < kDivstepEntries<4>; i += blockDim.x) t4[i] = kDivstepTable4.e[i];
    for (int i = threadIdx.x; i < kDivstepEntries<2>; i += blockDim.x) t2[i] = kDivstepTable2.e[i];
    __syncthreads();
    const int t = min((int)((blockIdx.x * blockDim.x + threadIdx.x) >> 2), n - 1);
    Fp x;
    uint32_t h = seed * 0x9e3779b9u + (uint32_t)t * 0x85ebca6bu;
#pragma unroll
    for (int k = 0; k < 12; k++) {
        h ^= h >> 15;
        h *= 0x2c1b3c6du;
        h ^= h >> 12;
        x.v[k] = h;
    }
    x.v[11] &= 0x0fffffffu;
    const Fp y = fp_inv_quad(t4, t2, x);
    if (y.v[0] == 0x12345678u) sink[0] = y.v[1];
}

__device__ __noinline__ Fp fp_mul_ks_call(Fp a, Fp b) {
    Fp r;
    mont_mul_ks<12>(r.v, a.v, b.v);
    return r;
}

__device__ __noinline__ Fp fp_mul_ks2_call(Fp a, Fp b) {
    Fp r;
    mont_mul_ks<12, 2>(r.v, a.v, b.v);
    return r;
}

__device__ __noinline__ Fp fp_sqr_ks_call(Fp a) {
    Fp r;
    mont_sqr_ks<12>(r.v, a.v);
    return r;
}

__device__ __noinline__ Fp fp_mul_f64_call(Fp a, Fp b) { return f64::mont_mul(a, b); }
__device__ __noinline__ Fp fp_sqr_f64_call(Fp a) { return f64::mont_sqr(a); }

// independent Fp products per thread (2 chains); OP 0: fp_mul, 1: fp_sqr, 2: the
// one-level Karatsuba product, 3: the Karatsuba square, 4: the two-level product,
// 5: the FP64-pipe product, 6: the FP64-pipe square, 7: even warps the
// Karatsuba product and odd warps the FP64-pipe product (both pipes at once)
template <int OP>
__global__ void __launch_bounds__(128) k_probe_fp(uint32_t seed, int iters, uint32_t *sink) {
    Fp a = fp_one(), b = fp_one();
    a.v[0] ^= seed + threadIdx.x;
    b.v[1] ^= seed * 3u + blockIdx.x;
    const Fp c = a;
    const bool odd_warp = (threadIdx.x >> 5) & 1;
    if constexpr (OP == 8 || OP == 9) { // four independent chains per thread, half the iterations
        Fp d = b, e = a;
        d.v[2] ^= 5u;
        e.v[3] ^= 7u;
        for (int i = 0; i < iters / 2; i++) {
            if (OP == 8) {
                a = fp_mul_f64_call(a, c);
                b = fp_mul_f64_call(b, c);
                d = fp_mul_f64_call(d, c);
                e = fp_mul_f64_call(e, c);
            } else {
                a = fp_mul_ks_call(a, c);
                b = fp_mul_ks_call(b, c);
                d = fp_mul_ks_call(d, c);
                e = fp_mul_ks_call(e, c);
            }
        }
        if ((a.v[0] ^ b.v[0] ^ d.v[0] ^ e.v[0]) == 0x12345678u) sink[0] = a.v[1];
        return;
    } else {
    for (int i = 0; i < iters; i++) {
        if (OP == 5 || (OP == 7 && odd_warp)) {
            a = fp_mul_f64_call(a, c);
            b = fp_mul_f64_call(b, c);
        } else if (OP == 6) {
            a = fp_sqr_f64_call(a);
            b = fp_sqr_f64_call(b);
        } else if (OP == 7) {
            a = fp_mul_ks_call(a, c);
            b = fp_mul_ks_call(b, c);
        } else if (OP == 0) {
            a = fp_mul(a, c);
            b = fp_mul(b, c);
        } else if (OP == 1) {
            a = fp_sqr(a);
            b = fp_sqr(b);
        } else if (OP == 2) {
            a = fp_mul_ks_call(a, c);
            b = fp_mul_ks_call(b, c);
        } else if (OP == 3) {
            a = fp_sqr_ks_call(a);
            b = fp_sqr_ks_call(b);
        } else {
            a = fp_mul_ks2_call(a, c);
            b = fp_mul_ks2_call(b, c);
        }
    }
    if ((a.v[0] ^ b.v[0]) == 0x12345678u) sink[0] = a.v[1];
    }
}

// OP 0: fr_mul (CIOS), 1: the Karatsuba product
template <int OP>
__global__ void __launch_bounds__(256) k_probe_fr(uint32_t seed, int iters, uint32_t *sink) {
    Fr a = fr_one(), b = fr_one();
    a.v[0] ^= seed + threadIdx.x;
    b.v[1] ^= seed * 3u + blockIdx.x;
    const Fr c = a;
    for (int i = 0; i < iters; i++) {
        if (OP == 0) {
            a = fr_mul(a, c);
            b = fr_mul(b, c);
        } else {
            mont_mul_ks<8>(a.v, a.v, c.v);
            mont_mul_ks<8>(b.v, b.v, c.v);
        }
    }
    if ((a.v[0] ^ b.v[0]) == 0x12345678u) sink[0] = a.v[1];
}

// Sums caller-chosen points into 128 buckets with the batch-affine routine of
// the proof kernels (one block), so tests can drive its special cases: repeated
// points (doubling), P + -P, the point at infinity.
__global__ void __launch_bounds__(32) k_bucket_sums_selftest(const G1A *points, const uint32_t *start, G1A *sums,
                                                            G1A *scratch) {
    __shared__ WarpBuckets<kBABuckets> wb;
    for (int k = threadIdx.x; k < kBABuckets; k += 32) wb.cnt[k] = start[k + 1] - start[k];
    __syncwarp();
    auto src0 = [points, start](int k, uint32_t i) { return ld_vec(&points[start[k] + i]); };
    int slot = 0;
    const G1A *res = wb_bucket_sums(wb, src0, scratch, scratch + 1088, reinterpret_cast<uint32_t *>(scratch + 1696),
                                    slot);
    for (int k = threadIdx.x; k < kBABuckets; k += 32) {
        G1A v;
        if (wb.cnt[k]) {
            v = ld_vec(&res[wb.base[slot][k]]);
        } else {
            v.x = fp_zero();
            v.y = fp_zero();
        }
        st_vec(&sums[k], v);
    }
}

// Seeded pseudo-random coordinates below 2^380 < p (a timing workload for the
// tree rounds: field elements, not curve points).
__global__ void k_seed_lists(G1A *pts, size_t n, uint64_t seed) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
    G1A a;
    uint32_t *w = reinterpret_cast<uint32_t *>(&a);
    for (int k = 0; k < 24; k++) {
        z += 0x9E3779B97F4A7C15ull;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        w[k] = (uint32_t)(x ^ (x >> 31));
    }
    a.x.v[11] &= 0x0fffffffu;
    a.y.v[11] &= 0x0fffffffu;
    st_vec(&pts[i], a);
}

} // namespace vkzg

using namespace vkzg;

// 96-byte (x || y canonical big-endian, all zero = infinity) <-> Montgomery affine
static G1A point_from_be(const uint8_t *xy) {
    G1A a;
    bool inf = true;
    for (int c = 0; c < 2; c++) {
        Fp v;
        for (int limb = 0; limb < 12; limb++) {
            const uint8_t *b = xy + 48 * c + (11 - limb) * 4;
            v.v[limb] = ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | b[3];
        }
        inf &= fp_is_zero(v);
        (c == 0 ? a.x : a.y) = fp_from_canonical(v);
    }
    if (inf) a.x = a.y = fp_zero();
    return a;
}

static void point_to_be(const G1A &p, uint8_t *xy) {
    const bool inf = g1a_is_identity(p);
    for (int c = 0; c < 2; c++) {
        const Fp v = inf ? fp_zero() : fp_to_canonical(c == 0 ? p.x : p.y);
        for (int limb = 0; limb < 12; limb++) {
            uint8_t *b = xy + 48 * c + (11 - limb) * 4;
            b[0] = (uint8_t)(v.v[limb] >> 24);
            b[1] = (uint8_t)(v.v[limb] >> 16);
            b[2] = (uint8_t)(v.v[limb] >> 8);
            b[3] = (uint8_t)v.v[limb];
        }
    }
}

// points_xy: n affine points, 96 bytes each (x || y, canonical big-endian; all
// zero = infinity); bucket_of: n bucket indices < 128.  sums_xy: 128 x 96 bytes.
// At most 2048 points.
extern "C" vkzg_result vkzg_b200_bucket_sums_selftest(const uint8_t *points_xy, const uint32_t *bucket_of, size_t n,
                                                      uint8_t *sums_xy) {
    if (!points_xy || !bucket_of || !sums_xy || n > 2048) return VKZG_ERR_BADARGS;
    std::vector<uint32_t> start(kBABuckets + 1, 0);
    for (size_t i = 0; i < n; i++) {
        if (bucket_of[i] >= (uint32_t)kBABuckets) return VKZG_ERR_BADARGS;
        start[bucket_of[i] + 1]++;
    }
    for (int k = 0; k < kBABuckets; k++) start[k + 1] += start[k];
    std::vector<uint32_t> cur(start.begin(), start.end() - 1);
    std::vector<G1A> pts(n > 0 ? n : 1);
    for (size_t i = 0; i < n; i++) pts[cur[bucket_of[i]]++] = point_from_be(points_xy + 96 * i);
    G1A *d_pts = nullptr, *d_sums = nullptr, *d_scratch = nullptr;
    uint32_t *d_start = nullptr;
    vkzg_result rc = VKZG_OK;
    if (cudaMalloc(&d_pts, pts.size() * sizeof(G1A)) != cudaSuccess ||
        cudaMalloc(&d_sums, kBABuckets * sizeof(G1A)) != cudaSuccess ||
        cudaMalloc(&d_scratch, (1088 + 608 + 512) * sizeof(G1A)) != cudaSuccess ||
        cudaMalloc(&d_start, start.size() * 4) != cudaSuccess) {
        rc = VKZG_ERR_MALLOC;
    } else {
        std::vector<G1A> sums(kBABuckets);
        if (cudaMemcpy(d_pts, pts.data(), pts.size() * sizeof(G1A), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(d_start, start.data(), start.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
            rc = VKZG_ERR_GPU;
        } else {
            k_bucket_sums_selftest<<<1, 32>>>(d_pts, d_start, d_sums, d_scratch);
            if (cudaDeviceSynchronize() != cudaSuccess ||
                cudaMemcpy(sums.data(), d_sums, kBABuckets * sizeof(G1A), cudaMemcpyDeviceToHost) != cudaSuccess)
                rc = VKZG_ERR_GPU;
        }
        if (rc == VKZG_OK)
            for (int k = 0; k < kBABuckets; k++) point_to_be(sums[k], sums_xy + 96 * k);
    }
    cudaFree(d_pts);
    cudaFree(d_sums);
    cudaFree(d_scratch);
    cudaFree(d_start);
    return rc;
}

// which: 0 = 32-bit IMAD issue rate (T/s), 1 = Fp multiplies (G/s), 2 = Fr multiplies (G/s)
extern "C" vkzg_result vkzg_b200_microbench(int which, double *result) {
    if (!result || which < 0 || which > 17) return VKZG_ERR_BADARGS;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return VKZG_ERR_GPU;
    uint32_t *sink = nullptr;
    cudaEvent_t e0, e1;
    if (cudaMalloc(&sink, 16) != cudaSuccess) return VKZG_ERR_MALLOC;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int fp_iters = 256, fr_iters = 1024;
    double best = 0.0;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        double ops = 0.0;
        if (which == 10 || which == 11 || which == 17) {
            const int n = sms * 16; // the warps of the round kernels' grid, one inversion each
            if (which == 10) k_probe_inv<true><<<(n + 63) / 64, 64>>>(rep + 1, n, sink);
            else if (which == 11) k_probe_inv<false><<<(n + 63) / 64, 64>>>(rep + 1, n, sink);
            else k_probe_inv_quad<<<(4 * n + 127) / 128, 128>>>(rep + 1, n, sink);
            ops = 1.0;
        } else if (which == 0 || which == 8 || which == 9) {
            const int blocks = sms * 8;
            if (which == 0) k_probe_imad<<<blocks, 256>>>(rep + 1, sink);
            else if (which == 8) k_probe_imad_wide<<<blocks, 256>>>(rep + 1, sink);
            else k_probe_dfma<<<blocks, 256>>>(rep + 1, sink);
            ops = (double)blocks * 256 * 8 * kProbeIters;
        } else if (which != 2 && which != 5) {
            const int blocks = sms * 4;
            if (which == 1) k_probe_fp<0><<<blocks, 128>>>(rep + 1, fp_iters, sink);
            else if (which == 3) k_probe_fp<1><<<blocks, 128>>>(rep + 1, fp_iters, sink);
            else if (which == 4) k_probe_fp<2><<<blocks, 128>>>(rep + 1, fp_iters, sink);
            else if (which == 6) k_probe_fp<3><<<blocks, 128>>>(rep + 1, fp_iters, sink);
            else if (which == 7) k_probe_fp<4><<<blocks, 128>>>(rep + 1, fp_iters, sink);
            else if (which == 12) k_probe_fp<5><<<blocks, 128>>>(rep + 1, fp_iters, sink);
            else if (which == 13) k_probe_fp<6><<<blocks, 128>>>(rep + 1, fp_iters, sink);
            else if (which == 14) k_probe_fp<7><<<blocks, 128>>>(rep + 1, fp_iters, sink);
            else if (which == 15) k_probe_fp<8><<<blocks, 128>>>(rep + 1, fp_iters, sink);
            else k_probe_fp<9><<<blocks, 128>>>(rep + 1, fp_iters, sink);
            ops = (double)blocks * 128 * 2 * fp_iters;
        } else {
            const int blocks = sms * 8;
            if (which == 2) k_probe_fr<0><<<blocks, 256>>>(rep + 1, fr_iters, sink);
            else k_probe_fr<1><<<blocks, 256>>>(rep + 1, fr_iters, sink);
            ops = (double)blocks * 256 * 2 * fr_iters;
        }
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            cudaFree(sink);
            return VKZG_ERR_GPU;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (which == 10 || which == 11 || which == 17) { // launch time in microseconds, the smallest
            const double us = ms * 1e3;
            if (rep > 0 && (best == 0.0 || us < best)) best = us;
            continue;
        }
        const double rate = ops / (ms * 1e-3) / ((which == 0 || which == 8 || which == 9) ? 1e12 : 1e9);
        if (rep > 0 && rate > best) best = rate;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    *result = best;
    return VKZG_OK;
}

// Grid barriers alone, in a cooperative launch of two 256-thread blocks per
// SM: `rounds` barriers, each block counting the ones it passed.  With
// extra_arrivals > 0 a barrier waits for more blocks than the grid has, so no
// barrier can complete: every wait runs out after spin_limit polls, sets the
// failure flag and marks the error words, and every block returns.
__global__ void __launch_bounds__(256) k_sync_probe(GridSync g, int rounds, uint32_t *passed) {
    for (int r = 0; r < rounds; r++) {
        if (!grid_sync(g)) return;
        if (threadIdx.x == 0) atomicAdd(passed, 1u);
    }
}

extern "C" vkzg_result vkzg_b200_grid_sync_selftest(uint32_t extra_arrivals, uint32_t spin_limit, int rounds,
                                                    uint32_t *barriers_passed, uint32_t *failed_flag,
                                                    uint32_t *error_words_marked) {
    if (!barriers_passed || !failed_flag || !error_words_marked || rounds < 0 || rounds > 1000 ||
        extra_arrivals > 1024)
        return VKZG_ERR_BADARGS;
    int dev = 0, sms = 0, coop = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop)
        return VKZG_ERR_GPU;
    const int blocks = 2 * sms;
    constexpr uint32_t kErrWords = 8;
    uint32_t *d = nullptr; // [0..4) barrier words, [4] passed, [8..16) error words
    if (cudaMalloc(&d, 16 * sizeof(uint32_t)) != cudaSuccess) return VKZG_ERR_MALLOC;
    vkzg_result rc = VKZG_OK;
    if (cudaMemset(d, 0, 16 * sizeof(uint32_t)) != cudaSuccess) rc = VKZG_ERR_GPU;
    GridSync g;
    g.word = d;
    g.err = d + 8;
    g.n_err = kErrWords;
    g.spin_limit = spin_limit;
    g.expected = (uint32_t)blocks + extra_arrivals;
    uint32_t *passed = d + 4;
    if (rc == VKZG_OK) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)blocks);
        cfg.blockDim = dim3(256);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (cudaLaunchKernelEx(&cfg, k_sync_probe, g, rounds, passed) != cudaSuccess ||
            cudaDeviceSynchronize() != cudaSuccess)
            rc = VKZG_ERR_GPU;
    }
    uint32_t h[16] = {};
    if (rc == VKZG_OK && cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) rc = VKZG_ERR_GPU;
    cudaFree(d);
    if (rc != VKZG_OK) return rc;
    *barriers_passed = h[4];
    *failed_flag = h[2];
    uint32_t marked = 0;
    for (uint32_t i = 0; i < kErrWords; i++) marked += (h[8 + i] & kSyncFailed) ? 1u : 0u;
    *error_words_marked = marked;
    return VKZG_OK;
}

// fp_inv_quad (four lanes a value, as the proof rounds' inversion launches)
// against fp_inv_fast (one lane) on n seeded pseudo-random values below p, the
// first four 0, 1, 2 and p - 1: the number of 32-bit words that differ.
__device__ Fp selftest_value(uint32_t seed, int t) {
    Fp x;
    uint32_t h = seed * 0x9e3779b9u + (uint32_t)t * 0x85ebca6bu;
#pragma unroll
    for (int k = 0; k < 12; k++) {
        h ^= h >> 15;
        h *= 0x2c1b3c6du;
        h ^= h >> 12;
        x.v[k] = h;
    }
    x.v[11] &= 0x0fffffffu;
    if (t < 3) {
#pragma unroll
        for (int k = 0; k < 12; k++) x.v[k] = k == 0 ? (uint32_t)t : 0u;
    } else if (t == 3) {
#pragma unroll
        for (int k = 0; k < 12; k++) x.v[k] = fp_p(k) - (k == 0 ? 1u : 0u);
    }
    return x;
}
__global__ void __launch_bounds__(128) k_inverse_selftest(uint32_t seed, int n, uint32_t *mismatch) {
    __shared__ uint64_t t4[kDivstepEntries<4>], t2[kDivstepEntries<2>];
    for (int i = threadIdx.x; i < kDivstepEntries<4>; i += blockDim.x) t4[i] = kDivstepTable4.e[i];
    for (int i = threadIdx.x; i < kDivstepEntries<2>; i += blockDim.x) t2[i] = kDivstepTable2.e[i];
    __syncthreads();
    const int k = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 2);
    const Fp x = selftest_value(seed, min(k, n - 1));
    const Fp q = fp_inv_quad(t4, t2, x);
    if (k < n && (threadIdx.x & 3) == 2) {
        const Fp s = fp_inv_fast(x);
        uint32_t bad = 0;
#pragma unroll
        for (int i = 0; i < 12; i++) bad += q.v[i] != s.v[i] ? 1u : 0u;
        if (bad) atomicAdd(mismatch, bad);
    }
}

extern "C" vkzg_result vkzg_b200_inverse_selftest(int n, uint32_t seed, uint32_t *mismatched_words) {
    if (!mismatched_words || n <= 0 || n > (1 << 20)) return VKZG_ERR_BADARGS;
    uint32_t *d = nullptr;
    if (cudaMalloc(&d, sizeof(uint32_t)) != cudaSuccess) return VKZG_ERR_MALLOC;
    vkzg_result rc = VKZG_OK;
    if (cudaMemset(d, 0, sizeof(uint32_t)) != cudaSuccess) rc = VKZG_ERR_GPU;
    if (rc == VKZG_OK) {
        k_inverse_selftest<<<(4 * n + 127) / 128, 128>>>(seed, n, d);
        count_launches(1);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = VKZG_ERR_GPU;
    }
    uint32_t h = 0;
    if (rc == VKZG_OK && cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) rc = VKZG_ERR_GPU;
    cudaFree(d);
    if (rc == VKZG_OK) *mismatched_words = h;
    return rc;
}

// Sums n_lists lists of m points each with the proof path's grid-wide
// batch-affine tree rounds (plan 3's phase-A rounds, without the digit table).
// points_xy: n_lists * m points of 96 bytes (list o first), or NULL for seeded
// pseudo-random coordinates generated on the device (a timing workload).
// sums_xy (may be NULL): n_lists x 96 bytes.  *ms (may be NULL): device time of
// the rounds.
extern "C" vkzg_result vkzg_b200_tree_sums_selftest(const uint8_t *points_xy, size_t n_lists, uint32_t m,
                                                    uint64_t seed, uint8_t *sums_xy, double *ms) {
    if (n_lists == 0 || m == 0 || n_lists > (1u << 24) || (size_t)n_lists * m > (1ull << 27))
        return VKZG_ERR_BADARGS;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return VKZG_ERR_GPU;
    const int blocks = sms * 2;
    const size_t lanes = (size_t)blocks * 256, total = n_lists * (size_t)m;
    const size_t slots = (n_lists * (size_t)(m / 2) + lanes - 1) / lanes + 1;
    G1A *lists = nullptr, *buf0 = nullptr, *buf1 = nullptr, *sums = nullptr;
    uint32_t *pre = nullptr;
    Fp *others = nullptr, *tot = nullptr, *totinv = nullptr;
    vkzg_result rc = VKZG_OK;
    if (cudaMalloc(&lists, total * sizeof(G1A)) != cudaSuccess ||
        cudaMalloc(&buf0, n_lists * (size_t)((m + 1) / 2) * sizeof(G1A)) != cudaSuccess ||
        cudaMalloc(&buf1, n_lists * (size_t)((m + 3) / 4 + 1) * sizeof(G1A)) != cudaSuccess ||
        cudaMalloc(&sums, n_lists * sizeof(G1A)) != cudaSuccess ||
        cudaMalloc(&pre, lanes / 32 * slots * 384 * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&others, lanes * sizeof(Fp)) != cudaSuccess ||
        cudaMalloc(&tot, lanes / 32 * sizeof(Fp)) != cudaSuccess ||
        cudaMalloc(&totinv, lanes / 32 * sizeof(Fp)) != cudaSuccess) {
        rc = VKZG_ERR_MALLOC;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (rc == VKZG_OK) {
        if (points_xy) {
            std::vector<G1A> pts(total);
            for (size_t i = 0; i < total; i++) pts[i] = point_from_be(points_xy + 96 * i);
            if (cudaMemcpy(lists, pts.data(), total * sizeof(G1A), cudaMemcpyHostToDevice) != cudaSuccess)
                rc = VKZG_ERR_GPU;
        } else {
            k_seed_lists<<<(unsigned)((total + 255) / 256), 256>>>(lists, total, seed);
        }
    }
    if (rc == VKZG_OK) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        launch_tree_sums(lists, (int)n_lists, m, buf0, buf1, pre, others, tot, totinv, slots, blocks, sums, 0);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) rc = VKZG_ERR_GPU;
    }
    if (rc == VKZG_OK && ms) {
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        *ms = t;
    }
    if (rc == VKZG_OK && sums_xy) {
        std::vector<G1A> out(n_lists);
        if (cudaMemcpy(out.data(), sums, n_lists * sizeof(G1A), cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = VKZG_ERR_GPU;
        } else {
            for (size_t o = 0; o < n_lists; o++) point_to_be(out[o], sums_xy + 96 * o);
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(lists);
    cudaFree(buf0);
    cudaFree(buf1);
    cudaFree(sums);
    cudaFree(pre);
    cudaFree(others);
    cudaFree(tot);
    cudaFree(totinv);
    return rc;
}
