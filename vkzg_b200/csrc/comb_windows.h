// The digit table's window layout (plan 3's phase A), shared by the kernels,
// the host code and the host-side tests; no CUDA headers needed.
#pragma once

#include <stdint.h>

namespace vkzg {

// The digit table's windows: a scalar's 256 bits in D windows as even as they
// go, the first R = 256 mod D of W + 1 bits and the rest of W = 256 / D bits
// (D x W + R = 256 exactly, which signed digits of scalars below 2^255 need).
// Window k holds the multiples m = 1..2^(width - 1) of its base, so a base
// column (j, i) has entries() points; phase A sums 64 D of them per output.
// D = 32: 8-bit windows, 3.2 GB; 24: 16 of 11 bits and 8 of 10, 16.1 GB; 23:
// 20.9 GB; 20: 58.0 GB; 19: 9 of 14 bits and 10 of 13, 90.2 GB; 18: 4 of 15
// bits and 14 of 14, 141.7 GB (17 windows would take 232 GB).
#if defined(__CUDACC__)
#define VKZG_HD __host__ __device__ __forceinline__
#else
#define VKZG_HD inline
#endif
struct CombWindows {
    int D, W, R;
    VKZG_HD int width(int k) const { return W + (k < R ? 1 : 0); }
    VKZG_HD int bit_off(int k) const { return k * W + (k < R ? k : R); }
    // first entry of window k within a base column's entries
    VKZG_HD uint32_t entry_off(int k) const {
        return k < R ? (uint32_t)k << W : ((uint32_t)R << W) + ((uint32_t)(k - R) << (W - 1));
    }
    VKZG_HD uint32_t entries() const { return ((uint32_t)R << W) + ((uint32_t)(D - R) << (W - 1)); }
    VKZG_HD int widest() const { return W + (R ? 1 : 0); }
};
VKZG_HD CombWindows comb_windows(int D) { return CombWindows{D, 256 / D, 256 % D}; }
#undef VKZG_HD

} // namespace vkzg
