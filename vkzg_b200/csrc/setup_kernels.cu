// FK20 position table from the G1 monomial setup, on the device.  The
// reference ships this table precomputed (src/precomputed_tables.cpp:16-58,
// file missing from its tree); this is the standard FK20 precomputation:
//   s_i[t] = [tau^(4031 - i - 64t)]G1 for t < 63, infinity for t >= 63
//   X[.][i] = FFT_128 over G1 of s_i
//   T[j][i][d] = 2^(8d) X[j][i]   (affine, Montgomery)
// which is what k_phase_a.comp:35,39 indexes.
#include "device_util.cuh"
#include "kernels.h"

namespace vkzg {

__global__ void __launch_bounds__(128) k_setup_decompress(const uint8_t *__restrict__ comp, G1A *out, uint32_t *err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kBlobElems) return;
    uint8_t b[48];
    for (int q = 0; q < 48; q++) b[q] = comp[48 * (size_t)k + q];
    G1A a;
    if (!g1_decompress(a, b)) {
        atomicOr(err, 1u);
        a.x = fp_zero();
        a.y = fp_zero();
    }
    st_vec(&out[k], a);
}

// One block per column i; DIT with bit-reversed input.  Twiddle products are
// scalar multiplications by the canonical root w_len^j.
__global__ void __launch_bounds__(64) k_setup_columns(const G1A *__restrict__ mono, G1J *x_out,
                                                     const Fr *__restrict__ roots_fwd) {
    __shared__ G1J s[kCells];
    const int i = blockIdx.x, t = threadIdx.x;
    for (int q = t; q < kCells; q += 64) {
        G1J v = g1_identity();
        if (q < kCellElems - 1) v = g1_from_affine(ld_vec(&mono[kBlobElems - kCellElems - 1 - i - kCellElems * q]));
        st_vec(&s[brev_bits((uint32_t)q, 7)], v);
    }
    __syncthreads();
    for (int len = 2; len <= kCells; len <<= 1) {
        const int h = len >> 1, blk = t / h, j = t - blk * h;
        G1J *base = s + blk * len + j;
        const G1J a = ld_vec(base);
        G1J c = ld_vec(base + h);
        if (j != 0) c = g1_mul_scalar(c, fr_to_canonical(ldg_vec(&roots_fwd[j * (8192 / len)])));
        __syncthreads();
        st_vec(base, g1_add(a, c));
        st_vec(base + h, g1_sub(a, c));
        __syncthreads();
    }
    for (int q = t; q < kCells; q += 64) st_vec(&x_out[q * kCellElems + i], ld_vec(&s[q]));
}

__global__ void __launch_bounds__(128) k_setup_ladder(const G1J *__restrict__ x, G1J *lad) {
    const int ji = blockIdx.x * blockDim.x + threadIdx.x; // j * 64 + i
    if (ji >= kCells * kCellElems) return;
    G1J acc = ld_vec(&x[ji]);
    for (int d = 0; d < kDigits; d++) {
        st_vec(&lad[(size_t)ji * kDigits + d], acc);
        if (d + 1 < kDigits)
            for (int q = 0; q < 8; q++) acc = g1_dbl(acc);
    }
}

// Jacobian -> affine with a block-wide batch inversion (same as the proof
// path's normaliser, kept local to this translation unit).
__global__ void __launch_bounds__(256) k_setup_normalize(const G1J *__restrict__ in, G1A *out, int n) {
    __shared__ Fp tree[512];
    const int gid = blockIdx.x * 256 + threadIdx.x;
    const G1J p = gid < n ? ld_vec(&in[gid]) : g1_identity();
    const bool inf = fp_is_zero(p.z);
    const Fp zi = block_batch_inverse_fp<256>(inf ? fp_one() : p.z, tree);
    if (gid >= n) return;
    G1A a;
    if (inf) {
        a.x = fp_zero();
        a.y = fp_zero();
    } else {
        const Fp z2 = fp_sqr(zi);
        a.x = fp_mul(p.x, z2);
        a.y = fp_mul(p.y, fp_mul(z2, zi));
    }
    st_vec(&out[gid], a);
}

size_t setup_scratch_bytes() {
    return sizeof(G1A) * kBlobElems + sizeof(G1J) * kCells * kCellElems + sizeof(G1J) * kPositionPoints;
}

cudaError_t launch_setup_tables(const uint8_t *d_g1_monomial, G1A *pos, const Fr *roots_fwd, void *scratch,
                                uint32_t *d_err, cudaStream_t s) {
    G1A *mono = reinterpret_cast<G1A *>(scratch);
    G1J *x = reinterpret_cast<G1J *>(mono + kBlobElems);
    G1J *lad = x + kCells * kCellElems;
    k_setup_decompress<<<kBlobElems / 128, 128, 0, s>>>(d_g1_monomial, mono, d_err);
    k_setup_columns<<<kCellElems, 64, 0, s>>>(mono, x, roots_fwd);
    k_setup_ladder<<<kCells * kCellElems / 128, 128, 0, s>>>(x, lad);
    k_setup_normalize<<<(int)(kPositionPoints / 256), 256, 0, s>>>(lad, pos, (int)kPositionPoints);
    count_launches(4);
    return cudaGetLastError();
}

} // namespace vkzg
