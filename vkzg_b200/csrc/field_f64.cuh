// Fp Montgomery products on the FP64 pipe.
//
// The integer multiply-add pipe is what bounds every Fp-product kernel here
// (each 32 x 32-bit partial product is one mad.lo or mad.hi; a 381-bit product
// is 516 of them).  B200 issues fma.rn.f64 at the same rate as IMAD, on its own
// pipe, and one double FMA covers a 50 x 50-bit partial product.  This file
// computes the same function as fp_mul / fp_sqr -- a b 2^-384 mod p, canonical
// in [0, p) -- with the partial products on the FP64 pipe and the column sums
// on the integer ALU.
//
// Limbs.  A value below 2^381 is eight limbs of 50 bits, each an exact double.
// For limbs |a|, |b| < 2^50 the product a b (below 2^100 in magnitude) splits
// exactly into h 2^50 + lo with two FMAs:
//   x = fma(a, b, 3 2^101)      x lies in [2^102, 2^103), whose ulp is 2^50, so
//                               x = 3 2^101 + h 2^50 with h = round(a b / 2^50)
//   y = fma(a, b, K - x)        K = 3 2^101 + 3 2^51, K - x = 3 2^51 - h 2^50 is
//                               exact, and y = lo + 3 2^51 lies in [2^52, 2^53)
//                               whose ulp is 1, so y is exact
// The bit patterns of x and y are then h and lo plus a constant: the column
// sums are formed as 64-bit integer sums of the patterns, with the constants
// taken out once by starting each column at minus their total (wrapping
// modulo 2^64 is harmless: the true sums are far below 2^63).  This is the
// published technique of computing exact integer partial products with
// double-precision FMA (Emmart, Zheng and Weems, "Faster modular
// exponentiation using double precision floating point arithmetic on the
// GPU", ARITH 2018), restated here for 50-bit limbs and this field.
//
// Reduction.  Word-serial Montgomery reduction (separated operand scanning)
// with digits of 50 bits for rounds 0..6 and 34 bits for round 7: 7 x 50 + 34 =
// 384, so the quotient m is the unique m < 2^384 with T + m p = 0 mod 2^384 --
// the same m, hence the same (T + m p) / 2^384 < 2p, as the 32-bit-word
// reduction computes.  Each round's digit m_k = (column k mod 2^50) (-p^-1)
// mod 2^50 takes four 32-bit multiplies on the (otherwise idle) integer pipe.
// A final conditional subtraction of p gives the canonical result, so these
// functions are interchangeable with fp_mul / fp_sqr bit for bit.
//
// Host builds compile the same sequence with std::fma (correctly rounded, as
// fma.rn.f64 is), which is how the CPU tests check it against the integer
// products.
//
// field.cuh includes this file once Fp, the modulus words and the carry
// primitives are defined; include field.cuh, not this file.
#pragma once

#include <string.h>

#include <type_traits>
#include <utility>
#if !defined(__CUDA_ARCH__)
#include <cmath>
#endif

namespace vkzg {
namespace f64 {

constexpr uint64_t kLimbMask = (1ull << 50) - 1;
constexpr double kSplitHi = 0x3p101;              // 3 2^101
constexpr double kSplitLo = 0x1.8000000000006p102; // 3 2^101 + 3 2^51
constexpr double kTwo52 = 0x1p52;
constexpr uint64_t kBitsX = 0x4658000000000000ull; // pattern of 3 2^101
constexpr uint64_t kBitsY = 0x4338000000000000ull; // pattern of 3 2^51
constexpr uint64_t kBits52 = 0x4330000000000000ull; // pattern of 2^52
// -p^-1 mod 2^50 (its low 34 bits are -p^-1 mod 2^34)
constexpr uint32_t kPinvLo = 0xfffcfffdu, kPinvHi = 0x3fffcu;

// p in 50-bit limbs, as exact doubles
VK_HD constexpr double p_limb(int j) {
    return j == 0 ? (double)0x2ffffffffaaabull : j == 1 ? (double)0x3ac54ffffee7full
         : j == 2 ? (double)0x30f6241eabfffull : j == 3 ? (double)0x2fd9cc34a83daull
         : j == 4 ? (double)0x0774b84f38512ull : j == 5 ? (double)0x1ed90d2eb35d9ull
         : j == 6 ? (double)0x397fe69a4b1baull : (double)0x680447a8ull;
}

VK_HD uint64_t dbits(double x) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    memcpy(&u, &x, 8);
    return u;
#endif
}
VK_HD double from_bits(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double x;
    memcpy(&x, &u, 8);
    return x;
#endif
}
VK_HD double dfma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
VK_HD double dsub(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
VK_HD double dadd(double a, double b) {
#if defined(__CUDA_ARCH__)
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
VK_HD uint32_t umulhi(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

// a b = h 2^50 + lo: the patterns of h (for column k + 1) and lo (column k).
VK_HD void limb_product(double a, double b, uint64_t &hi, uint64_t &lo) {
    const double x = dfma(a, b, kSplitHi);
    const double y = dfma(a, b, dsub(kSplitLo, x));
    hi += dbits(x);
    lo += dbits(y);
}

// Terms that land in column k: products (i, j) with i + j = k (low halves)
// and i + j = k - 1 (high halves), over the product and the reduction.
VK_HD constexpr int pairs_summing_to(int k, bool sq) {
    int n = 0;
    for (int i = 0; i < 8; i++)
        for (int j = sq ? i : 0; j < 8; j++)
            if (i + j == k) n++;
    return n;
}
VK_HD constexpr int reduction_lo_terms(int k) { // round r adds m_r p_j: low half to column r + j
    int n = 0;
    for (int r = 0; r < 8; r++)
        if (k >= r && k <= r + 7) n++;
    return n;
}
VK_HD constexpr uint64_t column_start(int k, bool sq) {
    const uint64_t lo = (uint64_t)(pairs_summing_to(k, sq) + reduction_lo_terms(k));
    const uint64_t hi = (uint64_t)(pairs_summing_to(k - 1, sq) + reduction_lo_terms(k - 1));
    return 0ull - lo * kBitsY - hi * kBitsX;
}
// The sixteen starting values, each forced to a compile-time constant.
template <bool SQ, int... K>
VK_HD void init_columns(uint64_t *c, std::integer_sequence<int, K...>) {
    ((c[K] = std::integral_constant<uint64_t, column_start(K, SQ)>::value), ...);
}

// Eight 50-bit limbs of a 12-word value below 2^381.
VK_HD void to_limbs(double *x, const uint32_t *w) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int s = 50 * i, wi = s >> 5, off = s & 31;
        uint64_t v = ((uint64_t)w[wi] | ((uint64_t)w[wi + 1] << 32)) >> off;
        if (off > 14 && wi + 2 < 12) v |= (uint64_t)w[wi + 2] << (64 - off);
        x[i] = dsub(from_bits((v & kLimbMask) | kBits52), kTwo52);
    }
}

// Montgomery reduction of the product columns c[0..16) and the canonical
// result's 12 words.
VK_HD Fp reduce_columns(uint64_t *c) {
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const uint32_t lo32 = (uint32_t)c[r], hi32 = (uint32_t)(c[r] >> 32);
        const uint32_t m_lo = lo32 * kPinvLo;
        const uint32_t m_hi = (umulhi(lo32, kPinvLo) + lo32 * kPinvHi + hi32 * kPinvLo) & (r < 7 ? 0x3ffffu : 0x3u);
        const double m = dsub(from_bits(((uint64_t)(m_hi | 0x43300000u) << 32) | m_lo), kTwo52);
#pragma unroll
        for (int j = 0; j < 8; j++) limb_product(m, p_limb(j), c[r + j + 1], c[r + j]);
        if (r < 7) c[r + 1] += (uint64_t)((int64_t)c[r] >> 50);
    }
    // t = (c[7] >> 34) + sum_{k >= 8} c[k] 2^(50 k - 384): digits of 16 bits at
    // bit 0 and 50 bits at 16 + 50 (i - 1), carries propagated upwards.
    uint64_t d[9];
    int64_t acc = (int64_t)c[7] >> 34;
    d[0] = (uint64_t)acc & 0xffffu;
    acc >>= 16;
#pragma unroll
    for (int k = 8; k < 16; k++) {
        acc += (int64_t)c[k];
        d[k - 7] = (uint64_t)acc & kLimbMask;
        acc >>= 50;
    }
    uint32_t w[12];
#pragma unroll
    for (int q = 0; q < 12; q++) {
        const int L = 32 * q;
        const int i = L < 16 ? 0 : 1 + (L - 16) / 50;
        const int si = i == 0 ? 0 : 16 + 50 * (i - 1);
        const int sn = 16 + 50 * i;
        uint64_t v = d[i] >> (L - si);
        if (i + 1 < 9 && sn < L + 32) v |= d[i + 1] << (sn - L);
        w[q] = (uint32_t)v;
    }
    // t < 2p: one conditional subtraction
    CARRY_DECL
    uint32_t s[12], borrow;
    SUB_CC(s[0], w[0], fp_p(0));
#pragma unroll
    for (int i = 1; i < 12; i++) SUBC_CC(s[i], w[i], fp_p(i));
    SUBC(borrow, 0u, 0u);
    Fp r;
#pragma unroll
    for (int i = 0; i < 12; i++) r.v[i] = borrow ? w[i] : s[i];
    return r;
}

VK_HD Fp mont_mul(const Fp &a, const Fp &b) {
    double x[8], y[8];
    to_limbs(x, a.v);
    to_limbs(y, b.v);
    uint64_t c[16];
    init_columns<false>(c, std::make_integer_sequence<int, 16>{});
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) limb_product(x[i], y[j], c[i + j + 1], c[i + j]);
    return reduce_columns(c);
}

// a^2: the cross products once with one factor doubled (|2 a_i a_j| < 2^101
// still rounds inside [2^102, 2^103)), the squares on the diagonal.
VK_HD Fp mont_sqr(const Fp &a) {
    double x[8];
    to_limbs(x, a.v);
    uint64_t c[16];
    init_columns<true>(c, std::make_integer_sequence<int, 16>{});
    double x2[8];
#pragma unroll
    for (int i = 0; i < 8; i++) x2[i] = dadd(x[i], x[i]);
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (j == i) limb_product(x[i], x[i], c[2 * i + 1], c[2 * i]);
            else if (j > i) limb_product(x2[i], x[j], c[i + j + 1], c[i + j]);
        }
    return reduce_columns(c);
}

} // namespace f64
} // namespace vkzg
