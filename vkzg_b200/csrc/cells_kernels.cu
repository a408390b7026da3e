// Cells of a blob: the 2x Reed-Solomon extension (EIP-7594 compute_cells), the
// half of compute_cells_and_kzg_proofs the reference leaves out
// (include/vkzg.h:16-18).  Its expected output is pinned by the cells in the
// reference's test vectors (tests/vectors/compute_cells_and_kzg_proofs_*,
// spans 1..128, which tests/vectors.h:88-95 skips).
//
// Per blob, one block.  The wire order of the 8192 extended evaluations is
// bit-reversed: position p holds the value at w_8192^brev13(p), and for p < 4096
// brev13(p) = 2 brev12(p), so the first 64 cells are the blob itself (its
// element p is the value at w_4096^brev12(p)); those bytes are copied.  The
// other 64 cells are the values on the coset w_8192 D_4096: the forward NTT-4096
// of f_k w_8192^k, f the blob's coefficients from an inverse NTT-4096
// (bit-reversed evaluations -> natural coefficients, as in the proof path), and
// that DIF transform's bit-reversed output is the cells' wire order.  The
// 1/4096 scale carries an extra 1/R, so the Montgomery limbs of every output
// are its canonical value.
#include "device_util.cuh"
#include "kernels.h"

namespace vkzg {

constexpr int kCellsThreads = 512;

__global__ void __launch_bounds__(kCellsThreads, 1) k_blob_to_cells(const uint8_t *__restrict__ blobs, uint8_t *cells,
                                                                   const Fr *__restrict__ roots_fwd,
                                                                   const Fr *__restrict__ roots_inv, Fr scale,
                                                                   uint32_t *err) {
    extern __shared__ uint4 smem_raw[];
    Fr *s = reinterpret_cast<Fr *>(smem_raw);
    const int b = blockIdx.x;
    const uint8_t *src = blobs + (size_t)b * kBlobBytes;
    uint8_t *dst = cells + (size_t)b * kExtElems * 32;
    bool bad = false;
    for (int i = threadIdx.x; i < kBlobElems; i += kCellsThreads) {
        const uint4 *p = reinterpret_cast<const uint4 *>(src + 32 * (size_t)i);
        const uint4 lo = p[0], hi = p[1];
        uint4 *w = reinterpret_cast<uint4 *>(dst + 32 * (size_t)i); // first half of the cells: the blob
        w[0] = lo;
        w[1] = hi;
        Fr v;
        v.v[7] = bswap32(lo.x); v.v[6] = bswap32(lo.y); v.v[5] = bswap32(lo.z); v.v[4] = bswap32(lo.w);
        v.v[3] = bswap32(hi.x); v.v[2] = bswap32(hi.y); v.v[1] = bswap32(hi.z); v.v[0] = bswap32(hi.w);
        bad |= !fr_is_canonical(v);
        st_vec(&s[i], fr_from_canonical(v));
    }
    if (bad) atomicOr(&err[b], 1u);
    __syncthreads();
    smem_dit<kCellsThreads>(s, 12, 1, 2, 4096, roots_inv);
    // f_k w_8192^k, f scaled by 1/(4096 R)
    for (int k = threadIdx.x; k < kBlobElems; k += kCellsThreads)
        st_vec(&s[k], fr_mul(fr_mul(ld_vec(&s[k]), scale), ldg_vec(&roots_fwd[k])));
    __syncthreads();
    smem_dif<kCellsThreads>(s, 12, 1, 4096, 2, roots_fwd);
    for (int q = threadIdx.x; q < kBlobElems; q += kCellsThreads) {
        const Fr v = ld_vec(&s[q]);
        uint4 *w = reinterpret_cast<uint4 *>(dst + 32 * (size_t)(kBlobElems + q));
        w[0] = make_uint4(bswap32(v.v[7]), bswap32(v.v[6]), bswap32(v.v[5]), bswap32(v.v[4]));
        w[1] = make_uint4(bswap32(v.v[3]), bswap32(v.v[2]), bswap32(v.v[1]), bswap32(v.v[0]));
    }
}

cudaError_t launch_cells(const DeviceTables &t, const uint8_t *blobs, uint8_t *cells, uint32_t *err, int n,
                         cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    // (1/4096) / R: the canonical integer of the Montgomery constant 1/4096
    static const Fr scale = fr_to_canonical(fr_inv(fr_from_u32(kBlobElems)));
    k_blob_to_cells<<<n, kCellsThreads, kBlobElems * sizeof(Fr), s>>>(blobs, cells, t.roots_fwd, t.roots_inv, scale,
                                                                      err);
    count_launches(1);
    return cudaGetLastError();
}

cudaError_t configure_cells_kernels() {
    return cudaFuncSetAttribute(k_blob_to_cells, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kBlobElems * sizeof(Fr)));
}

} // namespace vkzg
