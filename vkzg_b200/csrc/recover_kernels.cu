// Cell recovery (reference: src/vkzg.cpp:1086-1164, k_cells_to_fr,
// k_vanishing_poly, k_ntt_pass, k_ew_mul, k_ew_div, k_fr_to_cells).
//
// The reference computes, per blob,
//   out = FFT( 7^-i/N * IFFT( FFT(7^i/N * IFFT(E . FFT(Z))) / FFT(7^i . Z) ) )
// with Z(x) = Zs(x^64), Zs = prod over missing cells m of (x - w_128^brev7(m)).
// Because Z(x) = Zs(x^64), its values on the 8192-point domain and on the
// coset 7.domain take only 128 distinct values each:
//   Z(w^k)   = Zs(w_128^(k mod 128)),   Z(7 w^k) = Zs(7^64 w_128^(k mod 128)).
// k_recover_prep evaluates those 2 x 128 values directly (and batch-inverts the
// coset ones), which replaces two of the reference's six 8192-point NTTs and
// its per-element Fermat division with exactly the same field values.
//
// k_recover_cluster then runs the remaining four transforms for one blob per
// cluster of four blocks.  The wire order of cells is the bit-reversed order of
// the evaluation domain, so a DIT inverse (bit-reversed in, natural out) and a
// DIF forward (natural in, bit-reversed out) chain with no permutation pass.
#include "device_util.cuh"
#include "kernels.h"

#include <cooperative_groups.h>
#include <mutex>

namespace vkzg {

namespace cg = cooperative_groups;

// zv[c] = Zs(w_128^brev7(c)) * R   (R folded in so raw cell words need no
//                                    separate Montgomery conversion)
// inv_zc[c] = 1 / Zs(7^64 w_128^brev7(c))
__global__ void __launch_bounds__(kCells) k_recover_prep(const uint8_t *__restrict__ present,
                                                        const Fr *__restrict__ roots_fwd, Fr seven64, Fr *zv,
                                                        Fr *inv_zc, uint32_t *err) {
    __shared__ uint8_t miss_root[kCells];
    __shared__ int n_miss;
    __shared__ Fr tree[2 * kCells];
    const int b = blockIdx.x, c = threadIdx.x;
    if (c == 0) {
        int n = 0;
        for (int i = 0; i < kCells; i++)
            if (!present[(size_t)b * kCells + i]) miss_root[n++] = (uint8_t)brev_bits((uint32_t)i, 7);
        n_miss = n;
        if (err) err[b] = n > kCellElems ? 1u : 0u;
    }
    __syncthreads();
    const Fr x = ldg_vec(&roots_fwd[brev_bits((uint32_t)c, 7) * 64]);
    const Fr xc = fr_mul(x, seven64);
    Fr pv = fr_one(), pc = fr_one();
    for (int m = 0; m < n_miss; m++) {
        const Fr r = ldg_vec(&roots_fwd[(int)miss_root[m] * 64]);
        pv = fr_mul(pv, fr_sub(x, r));
        pc = fr_mul(pc, fr_sub(xc, r));
    }
    st_vec(&zv[(size_t)b * kCells + c], fr_mul(pv, Fr{VK_FR_R2}));
    const Fr inv = block_batch_inverse_fr<kCells>(pc, tree);
    st_vec(&inv_zc[(size_t)b * kCells + c], inv);
}

// ------------------------------------------------ transforms
// One blob is spread over a cluster of four blocks, each holding a quarter
// (2048 elements, 64 KB) of the blob in its own shared memory.  The inner 11
// stages of every transform run per quarter; the two outermost stages (the
// pairs k, k+2048 and k, k+4096), fused with the pointwise coset shift and the
// first two stages of the next transform, run as a radix-4 step on the groups
// {k, k+2048, k+4096, k+6144}, one element from each block's shared memory over
// the cluster's distributed shared memory.  No global scratch is used, and a
// block is a quarter of the per-blob work (three fit on an SM), so a batch's
// last blobs finish sooner than with one 128 KB block per blob, which ran two
// 4096-point halves in turn with the outer stage streamed through global
// memory (130 k against 143 k blobs/s at 256 blobs).
constexpr int kRecQuarter = kExtElems / 4;
constexpr int kRecQThreads = 256;

__device__ void cluster_dit_scale_dif(cg::cluster_group &cl, Fr *s, const Fr *__restrict__ roots_fwd,
                                      const Fr *__restrict__ roots_inv, const Fr *__restrict__ shift) {
    Fr *q0 = cl.map_shared_rank(s, 0), *q1 = cl.map_shared_rank(s, 1);
    Fr *q2 = cl.map_shared_rank(s, 2), *q3 = cl.map_shared_rank(s, 3);
    const int first = (int)cl.block_rank() * (kRecQuarter / 4);
    for (int i = threadIdx.x; i < kRecQuarter / 4; i += kRecQThreads) {
        const int k = first + i;
        Fr a0 = ld_vec(&q0[k]), a1 = ld_vec(&q1[k]), a2 = ld_vec(&q2[k]), a3 = ld_vec(&q3[k]);
        // inverse DIT, length 4096: (k, k+2048) and (k+4096, k+6144), twiddle w^(2k)
        const Fr w4 = ldg_vec(&roots_inv[2 * k]);
        Fr t = fr_mul(a1, w4);
        a1 = fr_sub(a0, t);
        a0 = fr_add(a0, t);
        t = fr_mul(a3, w4);
        a3 = fr_sub(a2, t);
        a2 = fr_add(a2, t);
        // inverse DIT, length 8192: (k, k+4096) twiddle w^k, (k+2048, k+6144) twiddle w^(k+2048)
        t = fr_mul(a2, ldg_vec(&roots_inv[k]));
        a2 = fr_sub(a0, t);
        a0 = fr_add(a0, t);
        t = fr_mul(a3, ldg_vec(&roots_inv[k + kRecQuarter]));
        a3 = fr_sub(a1, t);
        a1 = fr_add(a1, t);
        // pointwise shift
        a0 = fr_mul(a0, ldg_vec(&shift[k]));
        a1 = fr_mul(a1, ldg_vec(&shift[k + kRecQuarter]));
        a2 = fr_mul(a2, ldg_vec(&shift[k + 2 * kRecQuarter]));
        a3 = fr_mul(a3, ldg_vec(&shift[k + 3 * kRecQuarter]));
        // forward DIF, length 8192: (k, k+4096) twiddle w^k, (k+2048, k+6144) twiddle w^(k+2048)
        t = fr_sub(a0, a2);
        a0 = fr_add(a0, a2);
        a2 = fr_mul(t, ldg_vec(&roots_fwd[k]));
        t = fr_sub(a1, a3);
        a1 = fr_add(a1, a3);
        a3 = fr_mul(t, ldg_vec(&roots_fwd[k + kRecQuarter]));
        // forward DIF, length 4096: (k, k+2048) and (k+4096, k+6144), twiddle w^(2k)
        const Fr v4 = ldg_vec(&roots_fwd[2 * k]);
        t = fr_sub(a0, a1);
        a0 = fr_add(a0, a1);
        a1 = fr_mul(t, v4);
        t = fr_sub(a2, a3);
        a2 = fr_add(a2, a3);
        a3 = fr_mul(t, v4);
        st_vec(&q0[k], a0);
        st_vec(&q1[k], a1);
        st_vec(&q2[k], a2);
        st_vec(&q3[k], a3);
    }
}

#ifndef VKZG_REC_BLOCKS_PER_SM
#define VKZG_REC_BLOCKS_PER_SM 3
#endif
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(kRecQThreads, VKZG_REC_BLOCKS_PER_SM)
    k_recover_cluster(const uint8_t *__restrict__ cells, uint8_t *out, const Fr *__restrict__ zv,
                      const Fr *__restrict__ inv_zc, const Fr *__restrict__ roots_fwd,
                      const Fr *__restrict__ roots_inv, const Fr *__restrict__ shift_fwd,
                      const Fr *__restrict__ shift_inv) {
    extern __shared__ uint4 smem_raw[];
    Fr *s = reinterpret_cast<Fr *>(smem_raw);
    cg::cluster_group cl = cg::this_cluster();
    const int b = blockIdx.x >> 2;
    const int first = (int)cl.block_rank() * kRecQuarter; // this block's positions
    const uint8_t *src = cells + ((size_t)b * kExtElems + first) * 32;
    const Fr *zvb = zv + (size_t)b * kCells;
    const Fr *izb = inv_zc + (size_t)b * kCells;

    // A: X = E . Z on the domain (bit-reversed), inverse DIT inner stages
    for (int q = threadIdx.x; q < kRecQuarter; q += kRecQThreads) {
        const uint4 *w = reinterpret_cast<const uint4 *>(src + 32 * (size_t)q);
        const uint4 lo = w[0], hi = w[1];
        Fr v;
        v.v[7] = bswap32(lo.x); v.v[6] = bswap32(lo.y); v.v[5] = bswap32(lo.z); v.v[4] = bswap32(lo.w);
        v.v[3] = bswap32(hi.x); v.v[2] = bswap32(hi.y); v.v[1] = bswap32(hi.z); v.v[0] = bswap32(hi.w);
        st_vec(&s[q], fr_mul(ld_vec(&zvb[(first + q) >> 6]), v)); // raw word second
    }
    __syncthreads();
    smem_dit<kRecQThreads>(s, 11, 1, 2, kRecQuarter, roots_inv);
    cl.sync();
    // B: finish the IFFT, x 7^k / N, first two stages of the coset FFT
    cluster_dit_scale_dif(cl, s, roots_fwd, roots_inv, shift_fwd);
    cl.sync();
    // C: coset FFT inner stages, divide by Z on the coset, inverse DIT inner stages
    smem_dif<kRecQThreads>(s, 11, 1, kRecQuarter, 2, roots_fwd);
    for (int q = threadIdx.x; q < kRecQuarter; q += kRecQThreads)
        st_vec(&s[q], fr_mul(ld_vec(&s[q]), ld_vec(&izb[(first + q) >> 6])));
    __syncthreads();
    smem_dit<kRecQThreads>(s, 11, 1, 2, kRecQuarter, roots_inv);
    cl.sync();
    // D: finish the coset IFFT, x 7^-k / N / R, first two stages of the final FFT
    cluster_dit_scale_dif(cl, s, roots_fwd, roots_inv, shift_inv);
    cl.sync();
    // E: final FFT inner stages; bit-reversed output = wire order (no shared
    // memory of another block is touched after the last cluster barrier)
    smem_dif<kRecQThreads>(s, 11, 1, kRecQuarter, 2, roots_fwd);
    uint8_t *dst = out + ((size_t)b * kExtElems + first) * 32;
    for (int q = threadIdx.x; q < kRecQuarter; q += kRecQThreads) {
        const Fr v = ld_vec(&s[q]);
        uint4 *w = reinterpret_cast<uint4 *>(dst + 32 * (size_t)q);
        w[0] = make_uint4(bswap32(v.v[7]), bswap32(v.v[6]), bswap32(v.v[5]), bswap32(v.v[4]));
        w[1] = make_uint4(bswap32(v.v[3]), bswap32(v.v[2]), bswap32(v.v[1]), bswap32(v.v[0]));
    }
}

static void launch_recover_transforms(const DeviceTables &t, const uint8_t *cells, uint8_t *out, const Fr *zv,
                                      const Fr *inv_zc, int n, cudaStream_t s) {
    k_recover_cluster<<<4 * n, kRecQThreads, kRecQuarter * sizeof(Fr), s>>>(cells, out, zv, inv_zc, t.roots_fwd,
                                                                            t.roots_inv, t.shift_fwd, t.shift_inv);
}

static Fr host_seven64() {
    Fr seven = fr_from_u32(7), acc = seven;
    for (int i = 0; i < 6; i++) acc = fr_mul(acc, acc); // 7^64
    return acc;
}

cudaError_t launch_recover_timed(const DeviceTables &t, const RecoverWork &w, int n, cudaStream_t s,
                                 cudaEvent_t *ev) {
    if (n <= 0) return cudaSuccess;
    static const Fr seven64 = host_seven64();
    if (ev) cudaEventRecord(ev[0], s);
    k_recover_prep<<<n, kCells, 0, s>>>(w.present, t.roots_fwd, seven64, w.zv, w.inv_zc, w.err);
    if (ev) cudaEventRecord(ev[1], s);
    launch_recover_transforms(t, w.cells, w.out, w.zv, w.inv_zc, n, s);
    if (ev) cudaEventRecord(ev[2], s);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_recover(const DeviceTables &t, const RecoverWork &w, int n, cudaStream_t s) {
    return launch_recover_timed(t, w, n, s, nullptr);
}

cudaError_t configure_recover_kernels() {
    return cudaFuncSetAttribute(k_recover_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kRecQuarter * sizeof(Fr)));
}

// ------------------------------------------ allocation-free recovery variant
// Scratch for vkzg_b200_recover_cells_device_noalloc: a fixed array in the
// module's device memory instead of the prover's cudaMalloc'd working set.
// Per blob: Z on the domain and 1/Z on the coset (128 elements each; the
// transforms work in shared memory).  Every GPU that loads this library holds
// it (128 KiB) until the process exits; all calls share it.
constexpr int kNoAllocMaxBlobs = 16;
constexpr size_t kNoAllocPerBlob = 2 * kCells;
static __device__ __align__(256) Fr g_noalloc_scratch[kNoAllocMaxBlobs * kNoAllocPerBlob];

namespace {
std::mutex g_noalloc_mutex;
Fr *g_noalloc_addr[64] = {};
} // namespace

// Device address of g_noalloc_scratch on the current device.  The host-side
// symbol is only a stand-in; the address is fetched once per device.
static cudaError_t noalloc_scratch_address(Fr **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[dev] = reinterpret_cast<Fr *>(ptr);
    }
    *out = g_noalloc_addr[dev];
    return cudaSuccess;
}

int noalloc_max_blobs() { return kNoAllocMaxBlobs; }

// Same two kernels as launch_recover, with the Z tables carved out of
// g_noalloc_scratch.  Nothing in the scratch needs to start at zero: the prep
// kernel writes zv / inv_zc before the transforms read them.
cudaError_t launch_recover_noalloc(const DeviceTables &t, const uint8_t *cells, const uint8_t *present, uint8_t *out,
                                   uint32_t *err, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (n > kNoAllocMaxBlobs) return cudaErrorInvalidValue;
    Fr *base = nullptr;
    cudaError_t e = noalloc_scratch_address(&base);
    if (e != cudaSuccess) return e;
    Fr *zv = base;
    Fr *inv_zc = zv + (size_t)kNoAllocMaxBlobs * kCells;
    static const Fr seven64 = host_seven64();
    k_recover_prep<<<n, kCells, 0, s>>>(present, t.roots_fwd, seven64, zv, inv_zc, err);
    launch_recover_transforms(t, cells, out, zv, inv_zc, n, s);
    count_launches(2);
    return cudaGetLastError();
}

} // namespace vkzg
