// Cells of a blob: the 2x Reed-Solomon extension (EIP-7594 compute_cells), the
// half of compute_cells_and_kzg_proofs the reference leaves out
// (include/vkzg.h:16-18).  Its expected output is pinned by the cells in the
// reference's test vectors (tests/vectors/compute_cells_and_kzg_proofs_*,
// spans 1..128, which tests/vectors.h:88-95 skips).
//
// Per blob, one block: inverse NTT-4096 of the blob (bit-reversed evaluations
// -> natural coefficients f, as in the proof path), then the forward NTT-8192
// of f zero-padded, whose bit-reversed output order is the cells' wire order.
// The outermost DIF stage of that transform pairs k with k+4096, where the
// upper input half is zero: it reduces to (f[k], f[k] w_8192^k).  So the block
// keeps f in shared memory for the lower half and parks f . w^k in global
// scratch for the upper half.  The 1/4096 scale carries an extra 1/R, so the
// Montgomery limbs of every output are its canonical value.
#include "device_util.cuh"
#include "kernels.h"

namespace vkzg {

constexpr int kCellsThreads = 512;

__global__ void __launch_bounds__(kCellsThreads, 1) k_blob_to_cells(const uint8_t *__restrict__ blobs, uint8_t *cells,
                                                                   Fr *scratch, const Fr *__restrict__ roots_fwd,
                                                                   const Fr *__restrict__ roots_inv, Fr scale,
                                                                   uint32_t *err) {
    extern __shared__ uint4 smem_raw[];
    Fr *s = reinterpret_cast<Fr *>(smem_raw);
    const int b = blockIdx.x;
    const uint8_t *src = blobs + (size_t)b * kBlobBytes;
    Fr *g = scratch + (size_t)b * kExtElems;
    bool bad = false;
    for (int i = threadIdx.x; i < kBlobElems; i += kCellsThreads) {
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
    smem_dit<kCellsThreads>(s, 12, 1, 2, 4096, roots_inv);
    // f (scaled by 1/(4096 R)); upper half of the first DIF stage to scratch
    for (int k = threadIdx.x; k < kBlobElems; k += kCellsThreads) {
        const Fr f = fr_mul(ld_vec(&s[k]), scale);
        st_vec(&s[k], f);
        st_vec(&g[k], fr_mul(f, ldg_vec(&roots_fwd[k])));
    }
    __syncthreads();
    uint8_t *dst = cells + (size_t)b * kExtElems * 32;
    for (int h = 0; h < 2; h++) {
        if (h == 1) {
            for (int q = threadIdx.x; q < kBlobElems; q += kCellsThreads) st_vec(&s[q], ld_vec(&g[q]));
            __syncthreads();
        }
        smem_dif<kCellsThreads>(s, 12, 1, 4096, 2, roots_fwd);
        for (int q = threadIdx.x; q < kBlobElems; q += kCellsThreads) {
            const Fr v = ld_vec(&s[q]);
            uint4 *w = reinterpret_cast<uint4 *>(dst + 32 * (size_t)(h * kBlobElems + q));
            w[0] = make_uint4(bswap32(v.v[7]), bswap32(v.v[6]), bswap32(v.v[5]), bswap32(v.v[4]));
            w[1] = make_uint4(bswap32(v.v[3]), bswap32(v.v[2]), bswap32(v.v[1]), bswap32(v.v[0]));
        }
        __syncthreads();
    }
}

cudaError_t launch_cells(const DeviceTables &t, const uint8_t *blobs, uint8_t *cells, Fr *scratch, uint32_t *err,
                         int n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    // (1/4096) / R: the canonical integer of the Montgomery constant 1/4096
    static const Fr scale = fr_to_canonical(fr_inv(fr_from_u32(kBlobElems)));
    k_blob_to_cells<<<n, kCellsThreads, kBlobElems * sizeof(Fr), s>>>(blobs, cells, scratch, t.roots_fwd,
                                                                      t.roots_inv, scale, err);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t configure_cells_kernels() {
    return cudaFuncSetAttribute(k_blob_to_cells, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kBlobElems * sizeof(Fr)));
}

} // namespace vkzg
