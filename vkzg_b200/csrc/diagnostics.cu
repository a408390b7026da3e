// Throughput probes for the integer roofline: the device's 32-bit IMAD issue
// rate and the library's own Fp / Fr Montgomery multiply rates.  The reference
// has no counterpart; its README quotes only end-to-end timings.
#include "../../include/vkzg_b200.h"
#include "device_util.cuh"
#include "kernels.h"

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

// independent Fp products per thread (2 chains)
__global__ void __launch_bounds__(128) k_probe_fp(uint32_t seed, int iters, uint32_t *sink) {
    Fp a = fp_one(), b = fp_one();
    a.v[0] ^= seed + threadIdx.x;
    b.v[1] ^= seed * 3u + blockIdx.x;
    const Fp c = a;
    for (int i = 0; i < iters; i++) {
        a = fp_mul(a, c);
        b = fp_mul(b, c);
    }
    if ((a.v[0] ^ b.v[0]) == 0x12345678u) sink[0] = a.v[1];
}

__global__ void __launch_bounds__(256) k_probe_fr(uint32_t seed, int iters, uint32_t *sink) {
    Fr a = fr_one(), b = fr_one();
    a.v[0] ^= seed + threadIdx.x;
    b.v[1] ^= seed * 3u + blockIdx.x;
    const Fr c = a;
    for (int i = 0; i < iters; i++) {
        a = fr_mul(a, c);
        b = fr_mul(b, c);
    }
    if ((a.v[0] ^ b.v[0]) == 0x12345678u) sink[0] = a.v[1];
}

} // namespace vkzg

using namespace vkzg;

// which: 0 = 32-bit IMAD issue rate (T/s), 1 = Fp multiplies (G/s), 2 = Fr multiplies (G/s)
extern "C" vkzg_result vkzg_b200_microbench(int which, double *result) {
    if (!result || which < 0 || which > 2) return VKZG_ERR_BADARGS;
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
        if (which == 0) {
            const int blocks = sms * 8;
            k_probe_imad<<<blocks, 256>>>(rep + 1, sink);
            ops = (double)blocks * 256 * 8 * kProbeIters;
        } else if (which == 1) {
            const int blocks = sms * 4;
            k_probe_fp<<<blocks, 128>>>(rep + 1, fp_iters, sink);
            ops = (double)blocks * 128 * 2 * fp_iters;
        } else {
            const int blocks = sms * 8;
            k_probe_fr<<<blocks, 256>>>(rep + 1, fr_iters, sink);
            ops = (double)blocks * 256 * 2 * fr_iters;
        }
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
            cudaFree(sink);
            return VKZG_ERR_GPU;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double rate = ops / (ms * 1e-3) / (which == 0 ? 1e12 : 1e9);
        if (rep > 0 && rate > best) best = rate;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    *result = best;
    return VKZG_OK;
}
