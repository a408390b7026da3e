// Cell recovery (reference: src/vkzg.cpp:1086-1164, k_cells_to_fr,
// k_vanishing_poly, k_ntt_pass, k_ew_mul, k_ew_div, k_fr_to_cells).
//
// The reference computes, per blob,
//   out = FFT( 7^-i/N * IFFT( FFT(7^i/N * IFFT(E . FFT(Z))) / FFT(7^i . Z) ) )
// with Z(x) = Zs(x^64), Zs = prod over missing cells m of (x - w_128^brev7(m)).
// Because Z(x) = Zs(x^64), its values on the 8192-point domain and on the
// coset 7.domain take only 128 distinct values each:
//   Z(w^k)   = Zs(w_128^(k mod 128)),   Z(7 w^k) = Zs(7^64 w_128^(k mod 128)).
// Each cluster evaluates those values directly (the coset inverses as products
// over the present cells' roots), which replaces two of the reference's six
// 8192-point NTTs and its per-element Fermat division with exactly the same
// field values, and then
// runs the remaining four transforms.  The wire order of cells is the
// bit-reversed order of the evaluation domain, so a DIT inverse (bit-reversed
// in, natural out) and a DIF forward (natural in, bit-reversed out) chain with
// no permutation pass.
#include "device_util.cuh"
#include "kernels.h"

#include <cooperative_groups.h>

namespace vkzg {

namespace cg = cooperative_groups;

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
// memory (130 k blobs/s at 256 blobs, against 143 k for this form).
constexpr int kRecQuarter = kExtElems / 4;
constexpr int kQCells = kCells / 4; // cells per quarter
constexpr int kRecQThreads = 256;
constexpr int kZSlice = kCells / (kRecQThreads / kQCells); // list entries per thread
static_assert(kZSlice * kRecQThreads == kCells * kQCells, "Z partial products: whole slices");

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

// three blocks per SM (80 registers; 64 KB of shared memory each) measured
// faster than two with more registers: 143 k against 138 k blobs/s
#ifndef VKZG_REC_MIN_BLOCKS
#define VKZG_REC_MIN_BLOCKS 3
#endif
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(kRecQThreads, VKZG_REC_MIN_BLOCKS)
    k_recover_cluster(const uint8_t *__restrict__ cells, const uint8_t *__restrict__ present, uint8_t *out,
                      const Fr *__restrict__ roots_fwd, const Fr *__restrict__ roots_inv,
                      const Fr *__restrict__ shift_fwd, const Fr *__restrict__ shift_inv, Fr seven64,
                      Fr coset_scale, uint32_t *err) {
    extern __shared__ uint4 smem_raw[];
    Fr *s = reinterpret_cast<Fr *>(smem_raw);
    __shared__ uint8_t root_of[kCells];
    __shared__ int warp_miss[kCells / 32];
    __shared__ Fr zq[kQCells], izq[kQCells];
    cg::cluster_group cl = cg::this_cluster();
    const int b = blockIdx.x >> 2;
    const int rank = (int)cl.block_rank();
    const int first = rank * kRecQuarter; // this block's positions: cells 32 rank .. 32 rank + 31
    const uint8_t *src = cells + ((size_t)b * kExtElems + first) * 32;

    // Z on the domain needs the roots w_128^brev7(m) of the missing cells m; its
    // inverse on the coset needs no inversion: the 128 roots are all the 128th
    // roots of unity, so for y = 7^64 x (x one of them)
    //   prod over all m of (y - root_m) = y^128 - 1 = 7^8192 - 1,
    //   1 / Zs(y) = prod over present m of (y - root_m) / (7^8192 - 1).
    // root_of lists the missing cells' roots first, then the present ones.
    int before_m = 0, before_p = 0;
    bool missing = false;
    if (threadIdx.x < kCells) { // warps 0-3, whole warps
        missing = present[(size_t)b * kCells + threadIdx.x] == 0;
        const unsigned ball = __ballot_sync(0xffffffffu, missing);
        const unsigned lower = (1u << (threadIdx.x & 31)) - 1u;
        before_m = __popc(ball & lower);
        before_p = __popc(~ball & lower);
        if ((threadIdx.x & 31) == 0) warp_miss[threadIdx.x >> 5] = __popc(ball);
    }
    __syncthreads();
    int n_miss = 0;
    for (int w = 0; w < kCells / 32; w++) {
        if (w < (int)(threadIdx.x >> 5)) {
            before_m += warp_miss[w];
            before_p += 32 - warp_miss[w];
        }
        n_miss += warp_miss[w];
    }
    if (threadIdx.x < kCells)
        root_of[missing ? before_m : n_miss + before_p] = (uint8_t)brev_bits(threadIdx.x, 7);
    if (err && rank == 0 && threadIdx.x == 0) err[b] = n_miss > kCellElems ? 1u : 0u;
    __syncthreads();
    // this block's 32 cells: thread (sub, j) multiplies list entries 16 sub ..
    // 16 sub + 15 into a domain and a coset partial product, kept in the (not yet
    // used) shared buffer as [sub][domain / coset][j]
    {
        const int j = threadIdx.x & 31, sub = threadIdx.x >> 5;
        const Fr x = ldg_vec(&roots_fwd[brev_bits((uint32_t)(rank * kQCells + j), 7) * 64]);
        const Fr xc = fr_mul(x, seven64);
        Fr dom = fr_one(), cos = fr_one();
        for (int i = sub * kZSlice; i < (sub + 1) * kZSlice; i++) {
            const Fr r = ldg_vec(&roots_fwd[(int)root_of[i] * 64]);
            if (i < n_miss) dom = fr_mul(dom, fr_sub(x, r));
            else cos = fr_mul(cos, fr_sub(xc, r));
        }
        st_vec(&s[(2 * sub) * kQCells + j], dom);
        st_vec(&s[(2 * sub + 1) * kQCells + j], cos);
    }
    __syncthreads();
    if (threadIdx.x < 2 * kQCells) {
        const int j = threadIdx.x & 31, kind = threadIdx.x >> 5;
        Fr v = ld_vec(&s[kind * kQCells + j]);
        for (int sub = 1; sub < kRecQThreads / kQCells; sub++) v = fr_mul(v, ld_vec(&s[(2 * sub + kind) * kQCells + j]));
        if (kind == 0) st_vec(&zq[j], fr_mul(v, Fr{VK_FR_R2})); // R folded in: cell words are raw
        else st_vec(&izq[j], fr_mul(v, coset_scale));
    }
    __syncthreads();

    // A: X = E . Z on the domain (bit-reversed), inverse DIT inner stages
    for (int q = threadIdx.x; q < kRecQuarter; q += kRecQThreads) {
        const uint4 *w = reinterpret_cast<const uint4 *>(src + 32 * (size_t)q);
        const uint4 lo = w[0], hi = w[1];
        Fr v;
        v.v[7] = bswap32(lo.x); v.v[6] = bswap32(lo.y); v.v[5] = bswap32(lo.z); v.v[4] = bswap32(lo.w);
        v.v[3] = bswap32(hi.x); v.v[2] = bswap32(hi.y); v.v[1] = bswap32(hi.z); v.v[0] = bswap32(hi.w);
        st_vec(&s[q], fr_mul(ld_vec(&zq[q >> 6]), v)); // raw word second
    }
    __syncthreads();
    smem_dit4<kRecQThreads>(s, 11, 1, 2, kRecQuarter, roots_inv);
    cl.sync();
    // B: finish the IFFT, x 7^k / N, first two stages of the coset FFT
    cluster_dit_scale_dif(cl, s, roots_fwd, roots_inv, shift_fwd);
    cl.sync();
    // C: coset FFT inner stages, divide by Z on the coset, inverse DIT inner stages
    smem_dif4<kRecQThreads>(s, 11, 1, kRecQuarter, 2, roots_fwd);
    for (int q = threadIdx.x; q < kRecQuarter; q += kRecQThreads)
        st_vec(&s[q], fr_mul(ld_vec(&s[q]), ld_vec(&izq[q >> 6])));
    __syncthreads();
    smem_dit4<kRecQThreads>(s, 11, 1, 2, kRecQuarter, roots_inv);
    cl.sync();
    // D: finish the coset IFFT, x 7^-k / N / R, first two stages of the final FFT
    cluster_dit_scale_dif(cl, s, roots_fwd, roots_inv, shift_inv);
    cl.sync();
    // E: final FFT inner stages; bit-reversed output = wire order (no shared
    // memory of another block is touched after the last cluster barrier)
    smem_dif4<kRecQThreads>(s, 11, 1, kRecQuarter, 2, roots_fwd);
    uint8_t *dst = out + ((size_t)b * kExtElems + first) * 32;
    for (int q = threadIdx.x; q < kRecQuarter; q += kRecQThreads) {
        const Fr v = ld_vec(&s[q]);
        uint4 *w = reinterpret_cast<uint4 *>(dst + 32 * (size_t)q);
        w[0] = make_uint4(bswap32(v.v[7]), bswap32(v.v[6]), bswap32(v.v[5]), bswap32(v.v[4]));
        w[1] = make_uint4(bswap32(v.v[3]), bswap32(v.v[2]), bswap32(v.v[1]), bswap32(v.v[0]));
    }
}

static Fr host_seven64() {
    Fr seven = fr_from_u32(7), acc = seven;
    for (int i = 0; i < 6; i++) acc = fr_mul(acc, acc); // 7^64
    return acc;
}

// 1 / (7^8192 - 1): the product of y - w over all 128th roots of unity w is
// y^128 - 1, and y^128 = 7^8192 for every y on the coset 7^64 w_128^j
static Fr host_coset_scale() {
    Fr acc = fr_from_u32(7);
    for (int i = 0; i < 13; i++) acc = fr_mul(acc, acc); // 7^8192
    return fr_inv(fr_sub(acc, fr_one()));
}

static cudaError_t launch_recover_cluster(const DeviceTables &t, const uint8_t *cells, const uint8_t *present,
                                          uint8_t *out, uint32_t *err, int n, cudaStream_t s) {
    static const Fr seven64 = host_seven64();
    static const Fr coset_scale = host_coset_scale();
    k_recover_cluster<<<4 * n, kRecQThreads, kRecQuarter * sizeof(Fr), s>>>(
        cells, present, out, t.roots_fwd, t.roots_inv, t.shift_fwd, t.shift_inv, seven64, coset_scale, err);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_recover_timed(const DeviceTables &t, const RecoverWork &w, int n, cudaStream_t s,
                                 cudaEvent_t *ev) {
    if (n <= 0) return cudaSuccess;
    if (ev) cudaEventRecord(ev[0], s);
    const cudaError_t e = launch_recover_cluster(t, w.cells, w.present, w.out, w.err, n, s);
    if (ev) cudaEventRecord(ev[1], s);
    return e;
}

cudaError_t launch_recover(const DeviceTables &t, const RecoverWork &w, int n, cudaStream_t s) {
    return launch_recover_timed(t, w, n, s, nullptr);
}

cudaError_t configure_recover_kernels() {
    return cudaFuncSetAttribute(k_recover_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kRecQuarter * sizeof(Fr)));
}

// ------------------------------------------ allocation-free recovery variant
// vkzg_b200_recover_cells_device_noalloc: the same kernel, which keeps all of
// its working state in shared memory and needs no scratch, on the caller's
// buffers; the 16-blob limit is part of that entry point's contract.
constexpr int kNoAllocMaxBlobs = 16;

int noalloc_max_blobs() { return kNoAllocMaxBlobs; }

cudaError_t launch_recover_noalloc(const DeviceTables &t, const uint8_t *cells, const uint8_t *present, uint8_t *out,
                                   uint32_t *err, int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    if (n > kNoAllocMaxBlobs) return cudaErrorInvalidValue;
    return launch_recover_cluster(t, cells, present, out, err, n, s);
}

} // namespace vkzg
