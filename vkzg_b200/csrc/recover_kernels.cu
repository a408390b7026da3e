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
// k_recover_main then runs the remaining four transforms for one blob per
// block.  The wire order of cells is the bit-reversed order of the evaluation
// domain, so a DIT inverse (bit-reversed in, natural out) and a DIF forward
// (natural in, bit-reversed out) chain with no permutation pass.  An 8192-point
// transform is split at its outermost radix-2 stage: the inner 12 stages run on
// one 4096-element half at a time in shared memory (128 KB), and the stage
// that pairs k with k+4096 runs as a streaming pass over global scratch,
// fused with the pointwise coset shift and the next transform's first stage.
#include "device_util.cuh"
#include "kernels.h"

#include <mutex>

namespace vkzg {

constexpr int kRecThreads = 512;

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

// Outermost DIT stage of an inverse 8192 transform, pointwise scale by
// shift[k], then outermost DIF stage of a forward transform, in place on g.
__device__ void stream_dit_scale_dif(Fr *g, const Fr *__restrict__ roots_fwd, const Fr *__restrict__ roots_inv,
                                     const Fr *__restrict__ shift) {
    for (int j = threadIdx.x; j < kBlobElems; j += kRecThreads) {
        const Fr u = ld_vec(&g[j]);
        const Fr v = fr_mul(ld_vec(&g[j + kBlobElems]), ldg_vec(&roots_inv[j]));
        const Fr c0 = fr_mul(fr_add(u, v), ldg_vec(&shift[j]));
        const Fr c1 = fr_mul(fr_sub(u, v), ldg_vec(&shift[j + kBlobElems]));
        st_vec(&g[j], fr_add(c0, c1));
        st_vec(&g[j + kBlobElems], fr_mul(fr_sub(c0, c1), ldg_vec(&roots_fwd[j])));
    }
}

__global__ void __launch_bounds__(kRecThreads, 1) k_recover_main(const uint8_t *__restrict__ cells, uint8_t *out,
                                                                 Fr *scratch, const Fr *__restrict__ zv,
                                                                 const Fr *__restrict__ inv_zc,
                                                                 const Fr *__restrict__ roots_fwd,
                                                                 const Fr *__restrict__ roots_inv,
                                                                 const Fr *__restrict__ shift_fwd,
                                                                 const Fr *__restrict__ shift_inv) {
    extern __shared__ uint4 smem_raw[];
    Fr *s = reinterpret_cast<Fr *>(smem_raw);
    const int b = blockIdx.x;
    Fr *g = scratch + (size_t)b * kExtElems;
    const uint8_t *src = cells + (size_t)b * kExtElems * 32;
    const Fr *zvb = zv + (size_t)b * kCells;
    const Fr *izb = inv_zc + (size_t)b * kCells;

    // A: X = E . Z on the domain (bit-reversed), inverse DIT inner stages
    for (int h = 0; h < 2; h++) {
        for (int q = threadIdx.x; q < kBlobElems; q += kRecThreads) {
            const int p = h * kBlobElems + q;
            const uint4 *w = reinterpret_cast<const uint4 *>(src + 32 * (size_t)p);
            const uint4 lo = w[0], hi = w[1];
            Fr v;
            v.v[7] = bswap32(lo.x); v.v[6] = bswap32(lo.y); v.v[5] = bswap32(lo.z); v.v[4] = bswap32(lo.w);
            v.v[3] = bswap32(hi.x); v.v[2] = bswap32(hi.y); v.v[1] = bswap32(hi.z); v.v[0] = bswap32(hi.w);
            st_vec(&s[q], fr_mul(ld_vec(&zvb[p >> 6]), v)); // raw word second
        }
        __syncthreads();
        smem_dit<kRecThreads>(s, 12, 1, 2, 4096, roots_inv);
        for (int q = threadIdx.x; q < kBlobElems; q += kRecThreads) st_vec(&g[h * kBlobElems + q], ld_vec(&s[q]));
        __syncthreads();
    }
    // B: finish IFFT, x 7^k / N, first stage of the coset FFT
    stream_dit_scale_dif(g, roots_fwd, roots_inv, shift_fwd);
    __syncthreads();
    // C: coset FFT inner stages, divide by Z on the coset, inverse DIT inner stages
    for (int h = 0; h < 2; h++) {
        for (int q = threadIdx.x; q < kBlobElems; q += kRecThreads) st_vec(&s[q], ld_vec(&g[h * kBlobElems + q]));
        __syncthreads();
        smem_dif<kRecThreads>(s, 12, 1, 4096, 2, roots_fwd);
        for (int q = threadIdx.x; q < kBlobElems; q += kRecThreads) {
            const int p = h * kBlobElems + q;
            st_vec(&s[q], fr_mul(ld_vec(&s[q]), ld_vec(&izb[p >> 6])));
        }
        __syncthreads();
        smem_dit<kRecThreads>(s, 12, 1, 2, 4096, roots_inv);
        for (int q = threadIdx.x; q < kBlobElems; q += kRecThreads) st_vec(&g[h * kBlobElems + q], ld_vec(&s[q]));
        __syncthreads();
    }
    // D: finish the coset IFFT, x 7^-k / N / R, first stage of the final FFT
    stream_dit_scale_dif(g, roots_fwd, roots_inv, shift_inv);
    __syncthreads();
    // E: final FFT inner stages; bit-reversed output = wire order.  The 1/R in
    // shift_inv leaves each value's canonical form in its limbs.
    uint8_t *dst = out + (size_t)b * kExtElems * 32;
    for (int h = 0; h < 2; h++) {
        for (int q = threadIdx.x; q < kBlobElems; q += kRecThreads) st_vec(&s[q], ld_vec(&g[h * kBlobElems + q]));
        __syncthreads();
        smem_dif<kRecThreads>(s, 12, 1, 4096, 2, roots_fwd);
        for (int q = threadIdx.x; q < kBlobElems; q += kRecThreads) {
            const Fr v = ld_vec(&s[q]);
            uint4 *w = reinterpret_cast<uint4 *>(dst + 32 * (size_t)(h * kBlobElems + q));
            w[0] = make_uint4(bswap32(v.v[7]), bswap32(v.v[6]), bswap32(v.v[5]), bswap32(v.v[4]));
            w[1] = make_uint4(bswap32(v.v[3]), bswap32(v.v[2]), bswap32(v.v[1]), bswap32(v.v[0]));
        }
        __syncthreads();
    }
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
    k_recover_main<<<n, kRecThreads, kBlobElems * sizeof(Fr), s>>>(w.cells, w.out, w.scratch, w.zv, w.inv_zc,
                                                                   t.roots_fwd, t.roots_inv, t.shift_fwd,
                                                                   t.shift_inv);
    if (ev) cudaEventRecord(ev[2], s);
    count_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_recover(const DeviceTables &t, const RecoverWork &w, int n, cudaStream_t s) {
    return launch_recover_timed(t, w, n, s, nullptr);
}

cudaError_t configure_recover_kernels() {
    return cudaFuncSetAttribute(k_recover_main, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kBlobElems * sizeof(Fr)));
}

// ------------------------------------------ allocation-free recovery variant
// Scratch for vkzg_b200_recover_cells_device_noalloc: a fixed array in the
// module's device memory instead of the prover's cudaMalloc'd working set.
// Per blob: the 8192-element transform buffer, then Z on the domain and
// 1/Z on the coset (128 elements each).  Every GPU that loads this library
// holds it (4.125 MiB) until the process exits; all calls share it.
constexpr int kNoAllocMaxBlobs = 16;
constexpr size_t kNoAllocPerBlob = kExtElems + 2 * kCells;
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

// Same two kernels as launch_recover, with the per-blob scratch carved out of
// g_noalloc_scratch.  Nothing in the scratch needs to start at zero: the prep
// kernel writes zv / inv_zc and the main kernel writes each transform buffer
// before reading it.
cudaError_t launch_recover_noalloc(const DeviceTables &t, const uint8_t *cells, const uint8_t *present, uint8_t *out,
                                   uint32_t *err, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (n > kNoAllocMaxBlobs) return cudaErrorInvalidValue;
    Fr *base = nullptr;
    cudaError_t e = noalloc_scratch_address(&base);
    if (e != cudaSuccess) return e;
    Fr *work = base;
    Fr *zv = base + (size_t)kNoAllocMaxBlobs * kExtElems;
    Fr *inv_zc = zv + (size_t)kNoAllocMaxBlobs * kCells;
    static const Fr seven64 = host_seven64();
    k_recover_prep<<<n, kCells, 0, s>>>(present, t.roots_fwd, seven64, zv, inv_zc, err);
    k_recover_main<<<n, kRecThreads, kBlobElems * sizeof(Fr), s>>>(cells, out, work, zv, inv_zc, t.roots_fwd,
                                                                   t.roots_inv, t.shift_fwd, t.shift_inv);
    count_launches(2);
    return cudaGetLastError();
}

} // namespace vkzg
