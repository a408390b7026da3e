// BLS12-381 base field Fp (381-bit, 12 x 32-bit limbs) and scalar field Fr
// (255-bit, 8 x 32-bit limbs), little-endian limbs in Montgomery form with
// R = 2^384 / 2^256.  The memory image of a value is identical to the
// reference's (src/shaders/field.glsl.inc:1-4), so its setup tables load as-is.
//
// Multiplication is Montgomery: word-serial (CIOS) for Fr, and for Fp one
// Karatsuba level over 6-word halves followed by a separated word-by-word
// reduction.  On the device every product row is a PTX carry chain: each 32x32
// partial product is one mad.lo.cc / madc.hi.cc, with the even-index and
// odd-index products of a row on two separate chains (their 64-bit results
// never overlap, so a row is two passes of n instructions instead of n wide
// multiplies plus carry fix-ups).  The same
// code compiles for the host with the carry flag emulated in a local
// variable, which is how the CPU tests check the exact instruction sequence
// against the oracle.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define VK_HD __host__ __device__ __forceinline__
#define VK_D __device__ __forceinline__
#else
#define VK_HD inline
#define VK_D inline
#endif

namespace vkzg {

// ------------------------------------------------------------- constants
// p = 0x1a0111ea397fe69a4b1ba7b6434bacd764774b84f38512bf6730d2a0f6b0f6241eabfffeb153ffffb9feffffffffaaab
// r = 0x73eda753299d7d483339d80809a1d80553bda402fffe5bfeffffffff00000001
#define VK_FP_P                                                                                       \
    {0xffffaaabu, 0xb9feffffu, 0xb153ffffu, 0x1eabfffeu, 0xf6b0f624u, 0x6730d2a0u, 0xf38512bfu,         \
     0x64774b84u, 0x434bacd7u, 0x4b1ba7b6u, 0x397fe69au, 0x1a0111eau}
#define VK_FP_ONE                                                                                     \
    {0x0002fffdu, 0x76090000u, 0xc40c0002u, 0xebf4000bu, 0x53c758bau, 0x5f489857u, 0x70525745u,         \
     0x77ce5853u, 0xa256ec6du, 0x5c071a97u, 0xfa80e493u, 0x15f65ec3u}
#define VK_FP_R2                                                                                      \
    {0x1c341746u, 0xf4df1f34u, 0x09d104f1u, 0x0a76e6a6u, 0x4c95b6d5u, 0x8de5476cu, 0x939d83c0u,         \
     0x67eb88a9u, 0xb519952du, 0x9a793e85u, 0x92cae3aau, 0x11988fe5u}
#define VK_FP_N0 0xfffcfffdu
#define VK_FR_P {0x00000001u, 0xffffffffu, 0xfffe5bfeu, 0x53bda402u, 0x09a1d805u, 0x3339d808u, 0x299d7d48u, 0x73eda753u}
#define VK_FR_ONE {0xfffffffeu, 0x00000001u, 0x00034802u, 0x5884b7fau, 0xecbc4ff5u, 0x998c4fefu, 0xacc5056fu, 0x1824b159u}
#define VK_FR_R2 {0xf3f29c6du, 0xc999e990u, 0x87925c23u, 0x2b6cedcbu, 0x7254398fu, 0x05d31496u, 0x9f59ff11u, 0x0748d9d9u}
#define VK_FR_N0 0xffffffffu

struct alignas(16) Fp {
    uint32_t v[12];
};
struct alignas(16) Fr {
    uint32_t v[8];
};

// Modulus words as immediates: a switch on a compile-time index lets the
// compiler fold them into the instruction stream (no constant-bank loads).
VK_HD constexpr uint32_t fp_p(int i) {
    return i == 0 ? 0xffffaaabu : i == 1 ? 0xb9feffffu : i == 2 ? 0xb153ffffu : i == 3 ? 0x1eabfffeu
         : i == 4 ? 0xf6b0f624u : i == 5 ? 0x6730d2a0u : i == 6 ? 0xf38512bfu : i == 7 ? 0x64774b84u
         : i == 8 ? 0x434bacd7u : i == 9 ? 0x4b1ba7b6u : i == 10 ? 0x397fe69au : 0x1a0111eau;
}
VK_HD constexpr uint32_t fr_p(int i) {
    return i == 0 ? 0x00000001u : i == 1 ? 0xffffffffu : i == 2 ? 0xfffe5bfeu : i == 3 ? 0x53bda402u
         : i == 4 ? 0x09a1d805u : i == 5 ? 0x3339d808u : i == 6 ? 0x299d7d48u : 0x73eda753u;
}
template <int N>
VK_HD constexpr uint32_t mod_word(int i) {
    return N == 12 ? fp_p(i) : fr_p(i);
}
template <int N>
VK_HD constexpr uint32_t mod_n0() {
    return N == 12 ? VK_FP_N0 : VK_FR_N0;
}

// ------------------------------------------------------------- carry ops
// PTX extended-precision primitives.  On the host, `cf` is the carry flag.
#if defined(__CUDA_ARCH__)
#define CARRY_DECL
#define MAD_LO_CC(d, a, b, c) asm volatile("mad.lo.cc.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c))
#define MADC_LO_CC(d, a, b, c) asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c))
#define MADC_HI_CC(d, a, b, c) asm volatile("madc.hi.cc.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c))
#define MADC_HI(d, a, b, c) asm volatile("madc.hi.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c))
#define ADD_CC(d, a, b) asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define ADDC_CC(d, a, b) asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define ADDC(d, a, b) asm volatile("addc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define SUB_CC(d, a, b) asm volatile("sub.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define SUBC_CC(d, a, b) asm volatile("subc.cc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#define SUBC(d, a, b) asm volatile("subc.u32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b))
#else
#define CARRY_DECL uint32_t cf = 0;
#define MAD_LO_CC(d, a, b, c)                                                                         \
    do {                                                                                              \
        uint64_t _t = (uint64_t)(uint32_t)((uint64_t)(a) * (b)) + (uint32_t)(c);                      \
        d = (uint32_t)_t;                                                                             \
        cf = (uint32_t)(_t >> 32);                                                                    \
    } while (0)
#define MADC_LO_CC(d, a, b, c)                                                                        \
    do {                                                                                              \
        uint64_t _t = (uint64_t)(uint32_t)((uint64_t)(a) * (b)) + (uint32_t)(c) + cf;                 \
        d = (uint32_t)_t;                                                                             \
        cf = (uint32_t)(_t >> 32);                                                                    \
    } while (0)
#define MADC_HI_CC(d, a, b, c)                                                                        \
    do {                                                                                              \
        uint64_t _t = (((uint64_t)(a) * (b)) >> 32) + (uint32_t)(c) + cf;                             \
        d = (uint32_t)_t;                                                                             \
        cf = (uint32_t)(_t >> 32);                                                                    \
    } while (0)
#define MADC_HI(d, a, b, c)                                                                           \
    do {                                                                                              \
        d = (uint32_t)((((uint64_t)(a) * (b)) >> 32) + (uint32_t)(c) + cf);                           \
    } while (0)
#define ADD_CC(d, a, b)                                                                               \
    do {                                                                                              \
        uint64_t _t = (uint64_t)(uint32_t)(a) + (uint32_t)(b);                                        \
        d = (uint32_t)_t;                                                                             \
        cf = (uint32_t)(_t >> 32);                                                                    \
    } while (0)
#define ADDC_CC(d, a, b)                                                                              \
    do {                                                                                              \
        uint64_t _t = (uint64_t)(uint32_t)(a) + (uint32_t)(b) + cf;                                   \
        d = (uint32_t)_t;                                                                             \
        cf = (uint32_t)(_t >> 32);                                                                    \
    } while (0)
#define ADDC(d, a, b)                                                                                 \
    do {                                                                                              \
        d = (uint32_t)((uint64_t)(uint32_t)(a) + (uint32_t)(b) + cf);                                 \
    } while (0)
#define SUB_CC(d, a, b)                                                                               \
    do {                                                                                              \
        uint64_t _t = (uint64_t)(uint32_t)(a) - (uint32_t)(b);                                        \
        d = (uint32_t)_t;                                                                             \
        cf = (uint32_t)(_t >> 63);                                                                    \
    } while (0)
#define SUBC_CC(d, a, b)                                                                              \
    do {                                                                                              \
        uint64_t _t = (uint64_t)(uint32_t)(a) - (uint32_t)(b) - cf;                                   \
        d = (uint32_t)_t;                                                                             \
        cf = (uint32_t)(_t >> 63);                                                                    \
    } while (0)
#define SUBC(d, a, b)                                                                                 \
    do {                                                                                              \
        d = (uint32_t)((uint64_t)(uint32_t)(a) - (uint32_t)(b) - cf);                                 \
    } while (0)
#endif

} // namespace vkzg

#include "field_f64.cuh"

namespace vkzg {

// ------------------------------------------------------- generic n-limb ops
// r = a + b mod m (a, b < m; m < 2^(32n-1) so the raw sum fits in n words).
template <int N>
VK_HD void mod_add(uint32_t *r, const uint32_t *a, const uint32_t *b) {
    CARRY_DECL
    uint32_t t[N], s[N];
    ADD_CC(t[0], a[0], b[0]);
#pragma unroll
    for (int i = 1; i < N; i++) ADDC_CC(t[i], a[i], b[i]);
    SUB_CC(s[0], t[0], mod_word<N>(0));
#pragma unroll
    for (int i = 1; i < N; i++) SUBC_CC(s[i], t[i], mod_word<N>(i));
    uint32_t borrow;
    SUBC(borrow, 0u, 0u); // 0xffffffff when t < m
#pragma unroll
    for (int i = 0; i < N; i++) r[i] = borrow ? t[i] : s[i];
}

// r = a - b mod m
template <int N>
VK_HD void mod_sub(uint32_t *r, const uint32_t *a, const uint32_t *b) {
    CARRY_DECL
    uint32_t t[N];
    SUB_CC(t[0], a[0], b[0]);
#pragma unroll
    for (int i = 1; i < N; i++) SUBC_CC(t[i], a[i], b[i]);
    uint32_t mask;
    SUBC(mask, 0u, 0u); // all ones on borrow
    ADD_CC(r[0], t[0], mod_word<N>(0) & mask);
#pragma unroll
    for (int i = 1; i < N; i++) ADDC_CC(r[i], t[i], mod_word<N>(i) & mask);
}

// Montgomery product, CIOS.  Invariant: the running value t < 2m after each
// row, and t + a*b_i + q*m < 2^(32(n+1)), so n+1 words hold it and the odd
// chain's top word needs no carry-out.
template <int N>
VK_HD void mont_mul(uint32_t *r, const uint32_t *a, const uint32_t *b) {
    CARRY_DECL
    uint32_t t[N + 1];
#pragma unroll
    for (int i = 0; i < N + 1; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        const uint32_t bi = b[i];
        // even products: lo -> t[j], hi -> t[j+1]
        MAD_LO_CC(t[0], a[0], bi, t[0]);
        MADC_HI_CC(t[1], a[0], bi, t[1]);
#pragma unroll
        for (int j = 2; j < N; j += 2) {
            MADC_LO_CC(t[j], a[j], bi, t[j]);
            MADC_HI_CC(t[j + 1], a[j], bi, t[j + 1]);
        }
        ADDC(t[N], t[N], 0u);
        // odd products: lo -> t[j], hi -> t[j+1]
        MAD_LO_CC(t[1], a[1], bi, t[1]);
        MADC_HI_CC(t[2], a[1], bi, t[2]);
#pragma unroll
        for (int j = 3; j < N - 1; j += 2) {
            MADC_LO_CC(t[j], a[j], bi, t[j]);
            MADC_HI_CC(t[j + 1], a[j], bi, t[j + 1]);
        }
        MADC_LO_CC(t[N - 1], a[N - 1], bi, t[N - 1]);
        MADC_HI(t[N], a[N - 1], bi, t[N]);
        // reduction row
        const uint32_t q = t[0] * mod_n0<N>();
        MAD_LO_CC(t[0], q, mod_word<N>(0), t[0]);
        MADC_HI_CC(t[1], q, mod_word<N>(0), t[1]);
#pragma unroll
        for (int j = 2; j < N; j += 2) {
            MADC_LO_CC(t[j], q, mod_word<N>(j), t[j]);
            MADC_HI_CC(t[j + 1], q, mod_word<N>(j), t[j + 1]);
        }
        ADDC(t[N], t[N], 0u);
        MAD_LO_CC(t[1], q, mod_word<N>(1), t[1]);
        MADC_HI_CC(t[2], q, mod_word<N>(1), t[2]);
#pragma unroll
        for (int j = 3; j < N - 1; j += 2) {
            MADC_LO_CC(t[j], q, mod_word<N>(j), t[j]);
            MADC_HI_CC(t[j + 1], q, mod_word<N>(j), t[j + 1]);
        }
        MADC_LO_CC(t[N - 1], q, mod_word<N>(N - 1), t[N - 1]);
        MADC_HI(t[N], q, mod_word<N>(N - 1), t[N]);
        // t[0] == 0: shift one word
#pragma unroll
        for (int j = 0; j < N; j++) t[j] = t[j + 1];
        t[N] = 0;
    }
    // t < 2m < 2^(32n): one conditional subtraction
    uint32_t s[N];
    SUB_CC(s[0], t[0], mod_word<N>(0));
#pragma unroll
    for (int i = 1; i < N; i++) SUBC_CC(s[i], t[i], mod_word<N>(i));
    uint32_t borrow;
    SUBC(borrow, 0u, 0u);
#pragma unroll
    for (int i = 0; i < N; i++) r[i] = borrow ? t[i] : s[i];
}

template <int N>
VK_HD void sos_reduce(uint32_t *r, uint32_t *T);

// T (2n words) = a^2: the cross products a_i a_j (i < j) once, doubled by a
// shift, plus the diagonal; n(n-1) + 2n multiply instructions.
template <int N>
VK_HD void sqr_words(uint32_t *T, const uint32_t *a) {
    CARRY_DECL
#pragma unroll
    for (int i = 0; i < 2 * N; i++) T[i] = 0;
    // Row i adds a_i a_j (j > i) at T[i + j] in two chains of disjoint word
    // pairs (j = i+1, i+3, ... and j = i+2, i+4, ...).  T[i + n + 1] is still zero
    // when row i starts, so each chain's carry stops there.
#pragma unroll
    for (int i = 0; i < N - 1; i++) {
#pragma unroll
        for (int c = 1; c <= 2; c++) {
            const int j0 = i + c;
            if (j0 >= N) continue;
            MAD_LO_CC(T[i + j0], a[i], a[j0], T[i + j0]);
            MADC_HI_CC(T[i + j0 + 1], a[i], a[j0], T[i + j0 + 1]);
            int top = i + j0 + 1;
#pragma unroll
            for (int j = j0 + 2; j < N; j += 2) {
                MADC_LO_CC(T[i + j], a[i], a[j], T[i + j]);
                MADC_HI_CC(T[i + j + 1], a[i], a[j], T[i + j + 1]);
                top = i + j + 1;
            }
#pragma unroll
            for (int k = top + 1; k < i + N + 1; k++) ADDC_CC(T[k], T[k], 0u);
            ADDC(T[i + N + 1], T[i + N + 1], 0u);
        }
    }
    // x2 (the cross sum is below 2^(64n - 1))
#pragma unroll
    for (int k = 2 * N - 1; k > 0; k--) T[k] = (T[k] << 1) | (T[k - 1] >> 31);
    T[0] <<= 1;
    // + a_i^2 at T[2i]
    MAD_LO_CC(T[0], a[0], a[0], T[0]);
    MADC_HI_CC(T[1], a[0], a[0], T[1]);
#pragma unroll
    for (int i = 1; i < N - 1; i++) {
        MADC_LO_CC(T[2 * i], a[i], a[i], T[2 * i]);
        MADC_HI_CC(T[2 * i + 1], a[i], a[i], T[2 * i + 1]);
    }
    MADC_LO_CC(T[2 * N - 2], a[N - 1], a[N - 1], T[2 * N - 2]);
    MADC_HI(T[2 * N - 1], a[N - 1], a[N - 1], T[2 * N - 1]);
}

// Montgomery square a^2 / R mod m: sqr_words, then word-by-word reduction of
// the 2n-word square (separated operand scanning).  n(n-1) + 2n + 2n^2 + n
// multiply instructions against 4n^2 + n for mont_mul(a, a); same result.
template <int N>
VK_HD void mont_sqr(uint32_t *r, const uint32_t *a) {
    uint32_t T[2 * N];
    sqr_words<N>(T, a);
    sos_reduce<N>(r, T);
}

// r = T / R mod m for a 2n-word T < m R (separated operand scanning): row i
// clears T[i] with q m 2^(32 i); its carry out of T[i + n] is owed to
// T[i + n + 1] and added by row i + 1 (the last row owes none: T + q m <
// m R + R m < R^2).  T is clobbered.
template <int N>
VK_HD void sos_reduce(uint32_t *r, uint32_t *T) {
    CARRY_DECL
    uint32_t owed = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        const uint32_t q = T[i] * mod_n0<N>();
        uint32_t ce, co;
        MAD_LO_CC(T[i], q, mod_word<N>(0), T[i]);
        MADC_HI_CC(T[i + 1], q, mod_word<N>(0), T[i + 1]);
#pragma unroll
        for (int j = 2; j < N; j += 2) {
            MADC_LO_CC(T[i + j], q, mod_word<N>(j), T[i + j]);
            MADC_HI_CC(T[i + j + 1], q, mod_word<N>(j), T[i + j + 1]);
        }
        ADDC_CC(T[i + N], T[i + N], owed);
        ADDC(ce, 0u, 0u);
        MAD_LO_CC(T[i + 1], q, mod_word<N>(1), T[i + 1]);
        MADC_HI_CC(T[i + 2], q, mod_word<N>(1), T[i + 2]);
#pragma unroll
        for (int j = 3; j < N; j += 2) {
            MADC_LO_CC(T[i + j], q, mod_word<N>(j), T[i + j]);
            MADC_HI_CC(T[i + j + 1], q, mod_word<N>(j), T[i + j + 1]);
        }
        ADDC(co, 0u, 0u);
        owed = ce + co;
    }
    // T[n..2n) < 2m: one conditional subtraction
    uint32_t s[N];
    SUB_CC(s[0], T[N], mod_word<N>(0));
#pragma unroll
    for (int i = 1; i < N; i++) SUBC_CC(s[i], T[N + i], mod_word<N>(i));
    uint32_t borrow;
    SUBC(borrow, 0u, 0u);
#pragma unroll
    for (int i = 0; i < N; i++) r[i] = borrow ? T[N + i] : s[i];
}

// z (2h words) = x y (h words each), one row per y_i in an even and an odd
// chain of disjoint word pairs.  After row i the partial product is below
// 2^(32(h + i + 1)), so neither chain carries out of word i + h.
template <int H>
VK_HD void mul_words(uint32_t *z, const uint32_t *x, const uint32_t *y) {
    static_assert(H >= 3, "at least three words");
    CARRY_DECL
#pragma unroll
    for (int i = 0; i < 2 * H; i++) z[i] = 0;
#pragma unroll
    for (int i = 0; i < H; i++) {
        const uint32_t yi = y[i];
        if constexpr (H % 2 == 0) {
            // even j: words i .. i+h-1, then the carry into i+h; odd j: i+1 .. i+h
            MAD_LO_CC(z[i], x[0], yi, z[i]);
            MADC_HI_CC(z[i + 1], x[0], yi, z[i + 1]);
#pragma unroll
            for (int j = 2; j < H; j += 2) {
                MADC_LO_CC(z[i + j], x[j], yi, z[i + j]);
                MADC_HI_CC(z[i + j + 1], x[j], yi, z[i + j + 1]);
            }
            ADDC(z[i + H], z[i + H], 0u);
            MAD_LO_CC(z[i + 1], x[1], yi, z[i + 1]);
            MADC_HI_CC(z[i + 2], x[1], yi, z[i + 2]);
#pragma unroll
            for (int j = 3; j < H - 1; j += 2) {
                MADC_LO_CC(z[i + j], x[j], yi, z[i + j]);
                MADC_HI_CC(z[i + j + 1], x[j], yi, z[i + j + 1]);
            }
            MADC_LO_CC(z[i + H - 1], x[H - 1], yi, z[i + H - 1]);
            MADC_HI(z[i + H], x[H - 1], yi, z[i + H]);
        } else {
            // even j: words i .. i+h; odd j: i+1 .. i+h-1, then the carry into i+h
            MAD_LO_CC(z[i], x[0], yi, z[i]);
            MADC_HI_CC(z[i + 1], x[0], yi, z[i + 1]);
#pragma unroll
            for (int j = 2; j < H - 1; j += 2) {
                MADC_LO_CC(z[i + j], x[j], yi, z[i + j]);
                MADC_HI_CC(z[i + j + 1], x[j], yi, z[i + j + 1]);
            }
            MADC_LO_CC(z[i + H - 1], x[H - 1], yi, z[i + H - 1]);
            MADC_HI(z[i + H], x[H - 1], yi, z[i + H]);
            MAD_LO_CC(z[i + 1], x[1], yi, z[i + 1]);
            MADC_HI_CC(z[i + 2], x[1], yi, z[i + 2]);
#pragma unroll
            for (int j = 3; j < H; j += 2) {
                MADC_LO_CC(z[i + j], x[j], yi, z[i + j]);
                MADC_HI_CC(z[i + j + 1], x[j], yi, z[i + j + 1]);
            }
            ADDC(z[i + H], z[i + H], 0u);
        }
    }
}

// z (2h words) = x y through LV Karatsuba levels (each level needs an even word
// count; schoolbook below): x y = x0 y0 + (x0 y1 + x1 y0) 2^(32g) + x1 y1 2^(32h),
// g = h/2, with the middle term x0 y0 + x1 y1 + (x0 - x1)(y1 - y0) taken from
// |x0 - x1| |y1 - y0| and the sign of the factors: 3 products of g words.
template <int H, int LV>
VK_HD void kara_words(uint32_t *z, const uint32_t *x, const uint32_t *y) {
    if constexpr (LV == 0 || H % 2 != 0 || H < 6) {
        mul_words<H>(z, x, y);
    } else {
        constexpr int G = H / 2;
        CARRY_DECL
        kara_words<G, LV - 1>(z, x, y);
        kara_words<G, LV - 1>(z + H, x + G, y + G);
        // dx = |x0 - x1|, dy = |y1 - y0|: the difference, then (t ^ mask) - mask,
        // which negates it when the subtraction borrowed (mask all ones)
        uint32_t dx[G], dy[G], mx, my;
        SUB_CC(dx[0], x[0], x[G]);
#pragma unroll
        for (int i = 1; i < G; i++) SUBC_CC(dx[i], x[i], x[G + i]);
        SUBC(mx, 0u, 0u);
        SUB_CC(dx[0], dx[0] ^ mx, mx);
#pragma unroll
        for (int i = 1; i < G; i++) SUBC_CC(dx[i], dx[i] ^ mx, mx);
        SUB_CC(dy[0], y[G], y[0]);
#pragma unroll
        for (int i = 1; i < G; i++) SUBC_CC(dy[i], y[G + i], y[i]);
        SUBC(my, 0u, 0u);
        SUB_CC(dy[0], dy[0] ^ my, my);
#pragma unroll
        for (int i = 1; i < G; i++) SUBC_CC(dy[i], dy[i] ^ my, my);
        uint32_t M[H];
        kara_words<G, LV - 1>(M, dx, dy);
        // mid = x0 y0 + x1 y1 +- M in h + 1 words (it equals x0 y1 + x1 y0 < 2^(32h + 1));
        // -M is (M ^ s) + 1 with s all ones, the + 1 entering as the carry of s + 1
        const uint32_t s = mx ^ my;
        uint32_t mid[H + 1], dummy;
        ADD_CC(mid[0], z[0], z[H]);
#pragma unroll
        for (int i = 1; i < H; i++) ADDC_CC(mid[i], z[i], z[H + i]);
        ADDC(mid[H], 0u, 0u);
        ADD_CC(dummy, s, 1u);
#pragma unroll
        for (int i = 0; i < H; i++) ADDC_CC(mid[i], mid[i], M[i] ^ s);
        ADDC(mid[H], mid[H], s);
        (void)dummy;
        // z += mid 2^(32g); the full product is below 2^(64h), so the last word takes no carry out
        ADD_CC(z[G], z[G], mid[0]);
#pragma unroll
        for (int i = 1; i <= H; i++) ADDC_CC(z[G + i], z[G + i], mid[i]);
#pragma unroll
        for (int k = G + H + 1; k < 2 * H - 1; k++) ADDC_CC(z[k], z[k], 0u);
        ADDC(z[2 * H - 1], z[2 * H - 1], 0u);
    }
}

// Montgomery product with the 2n-word product through LV Karatsuba levels, then
// the same reduction as mont_sqr; the same bounds as mont_mul (a b < m R).
// One level for 12 words: 3 x 36 word products instead of 144.
template <int N, int LV = 1>
VK_HD void mont_mul_ks(uint32_t *r, const uint32_t *a, const uint32_t *b) {
    uint32_t T[2 * N];
    kara_words<N, LV>(T, a, b);
    sos_reduce<N>(r, T);
}

// Montgomery square through one Karatsuba level: a^2 = a0^2 + 2 a0 a1 2^(32h)
// + a1^2 2^(32n) with 2 a0 a1 = a0^2 + a1^2 - (a0 - a1)^2, three h-word squares.
template <int N>
VK_HD void mont_sqr_ks(uint32_t *r, const uint32_t *a) {
    static_assert(N % 2 == 0 && N >= 8, "even word count");
    constexpr int H = N / 2;
    CARRY_DECL
    uint32_t T[2 * N];
    sqr_words<H>(T, a);
    sqr_words<H>(T + N, a + H);
    uint32_t d[H], md;
    SUB_CC(d[0], a[0], a[H]);
#pragma unroll
    for (int i = 1; i < H; i++) SUBC_CC(d[i], a[i], a[H + i]);
    SUBC(md, 0u, 0u);
    SUB_CC(d[0], d[0] ^ md, md);
#pragma unroll
    for (int i = 1; i < H; i++) SUBC_CC(d[i], d[i] ^ md, md);
    uint32_t M[N];
    sqr_words<H>(M, d);
    // mid = a0^2 + a1^2 - M in n + 1 words (it equals 2 a0 a1 < 2^(32n + 1))
    uint32_t mid[N + 1];
    ADD_CC(mid[0], T[0], T[N]);
#pragma unroll
    for (int i = 1; i < N; i++) ADDC_CC(mid[i], T[i], T[N + i]);
    ADDC(mid[N], 0u, 0u);
    SUB_CC(mid[0], mid[0], M[0]);
#pragma unroll
    for (int i = 1; i < N; i++) SUBC_CC(mid[i], mid[i], M[i]);
    SUBC(mid[N], mid[N], 0u);
    ADD_CC(T[H], T[H], mid[0]);
#pragma unroll
    for (int i = 1; i <= N; i++) ADDC_CC(T[H + i], T[H + i], mid[i]);
#pragma unroll
    for (int k = H + N + 1; k < 2 * N - 1; k++) ADDC_CC(T[k], T[k], 0u);
    ADDC(T[2 * N - 1], T[2 * N - 1], 0u);
    sos_reduce<N>(r, T);
}

template <int N>
VK_HD bool limbs_is_zero(const uint32_t *a) {
    uint32_t acc = 0;
#pragma unroll
    for (int i = 0; i < N; i++) acc |= a[i];
    return acc == 0;
}

template <int N>
VK_HD bool limbs_eq(const uint32_t *a, const uint32_t *b) {
    uint32_t acc = 0;
#pragma unroll
    for (int i = 0; i < N; i++) acc |= a[i] ^ b[i];
    return acc == 0;
}

// ------------------------------------------------------------------- Fp
VK_HD Fp fp_zero() {
    Fp r;
#pragma unroll
    for (int i = 0; i < 12; i++) r.v[i] = 0;
    return r;
}
VK_HD Fp fp_one() { return Fp{VK_FP_ONE}; }
// On the device the 12-limb product is an out-of-line call by default: inlined,
// every point formula becomes thousands of straight-line instructions (an
// instruction-cache and compile-time cost); VKZG_FP_INLINE=1 inlines it.
#ifndef VKZG_FP_INLINE
#define VKZG_FP_INLINE 0
#endif
// The 12-limb product goes through VKZG_FP_KARATSUBA Karatsuba levels
// (mont_mul_ks): one level is 516 multiply instructions against 588 for CIOS,
// about 9% more products per second on the integer pipe; 0 selects CIOS.
#ifndef VKZG_FP_KARATSUBA
#define VKZG_FP_KARATSUBA 1
#endif
// VKZG_FP_F64=1 computes Fp products and squares with the partial products on
// the FP64 pipe (field_f64.cuh); the results are the same bits.
#ifndef VKZG_FP_F64
#define VKZG_FP_F64 0
#endif
// VKZG_FP_SQR_F64=1: squares alone on the FP64 pipe
#ifndef VKZG_FP_SQR_F64
#define VKZG_FP_SQR_F64 VKZG_FP_F64
#endif
#if defined(__CUDA_ARCH__) && !VKZG_FP_INLINE
__device__ __noinline__ Fp fp_mul_call(Fp a, Fp b) {
#if VKZG_FP_F64
    return f64::mont_mul(a, b);
#endif
    Fp r;
#if VKZG_FP_KARATSUBA
    mont_mul_ks<12, VKZG_FP_KARATSUBA>(r.v, a.v, b.v);
#else
    mont_mul<12>(r.v, a.v, b.v);
#endif
    return r;
}
#endif
VK_HD Fp fp_mul(const Fp &a, const Fp &b) {
#if defined(__CUDA_ARCH__) && !VKZG_FP_INLINE
    return fp_mul_call(a, b);
#else
    Fp r;
#if VKZG_FP_KARATSUBA
    mont_mul_ks<12, VKZG_FP_KARATSUBA>(r.v, a.v, b.v);
#else
    mont_mul<12>(r.v, a.v, b.v);
#endif
    return r;
#endif
}
#if defined(__CUDA_ARCH__) && !VKZG_FP_INLINE
__device__ __noinline__ Fp fp_sqr_call(Fp a) {
#if VKZG_FP_SQR_F64
    return f64::mont_sqr(a);
#endif
    Fp r;
#if VKZG_FP_KARATSUBA
    mont_sqr_ks<12>(r.v, a.v);
#else
    mont_sqr<12>(r.v, a.v);
#endif
    return r;
}
#endif
VK_HD Fp fp_sqr(const Fp &a) {
#if defined(__CUDA_ARCH__) && !VKZG_FP_INLINE
    return fp_sqr_call(a);
#else
    Fp r;
#if VKZG_FP_KARATSUBA
    mont_sqr_ks<12>(r.v, a.v);
#else
    mont_sqr<12>(r.v, a.v);
#endif
    return r;
#endif
}
VK_HD Fp fp_add(const Fp &a, const Fp &b) {
    Fp r;
    mod_add<12>(r.v, a.v, b.v);
    return r;
}
VK_HD Fp fp_sub(const Fp &a, const Fp &b) {
    Fp r;
    mod_sub<12>(r.v, a.v, b.v);
    return r;
}
VK_HD Fp fp_dbl(const Fp &a) { return fp_add(a, a); }
VK_HD bool fp_is_zero(const Fp &a) { return limbs_is_zero<12>(a.v); }
VK_HD bool fp_eq(const Fp &a, const Fp &b) { return limbs_eq<12>(a.v, b.v); }
// -0 = 0 (field.glsl.inc:99-102)
VK_HD Fp fp_neg(const Fp &a) { return fp_is_zero(a) ? a : fp_sub(fp_zero(), a); }
VK_HD Fp fp_cneg(const Fp &a, bool neg) { return neg ? fp_neg(a) : a; }

// a^e for a little-endian exponent of `words` 32-bit words (square-and-multiply)
VK_HD Fp fp_pow_words(const Fp &a, const uint32_t *e, int words) {
    Fp acc = fp_one();
    for (int i = words - 1; i >= 0; i--) {
        for (int b = 31; b >= 0; b--) {
            acc = fp_sqr(acc);
            if ((e[i] >> b) & 1u) acc = fp_mul(acc, a);
        }
    }
    return acc;
}
// a^(p-2); zero maps to zero (field.glsl.inc:528-547)
VK_HD Fp fp_inv(const Fp &a) {
    const uint32_t e[12] = {0xffffaaa9u, 0xb9feffffu, 0xb153ffffu, 0x1eabfffeu, 0xf6b0f624u, 0x6730d2a0u,
                            0xf38512bfu, 0x64774b84u, 0x434bacd7u, 0x4b1ba7b6u, 0x397fe69au, 0x1a0111eau};
    return fp_pow_words(a, e, 12);
}
VK_HD Fp fp_to_canonical(const Fp &a) {
    Fp one = fp_zero();
    one.v[0] = 1;
    return fp_mul(a, one);
}
VK_HD Fp fp_from_canonical(const Fp &a) { return fp_mul(Fp{VK_FP_R2}, a); }
// canonical > (p-1)/2 (field.glsl.inc:549-562)
VK_HD bool fp_is_lex_largest(const Fp &c) {
    const uint32_t h[12] = {0xffffd555u, 0xdcff7fffu, 0x58a9ffffu, 0x0f55ffffu, 0x7b587b12u, 0xb3986950u,
                            0x79c2895fu, 0xb23ba5c2u, 0x21a5d66bu, 0x258dd3dbu, 0x1cbff34du, 0x0d0088f5u};
    for (int i = 11; i >= 0; i--) {
        if (c.v[i] != h[i]) return c.v[i] > h[i];
    }
    return false;
}
VK_HD bool fp_is_canonical(const Fp &a) {
    for (int i = 11; i >= 0; i--) {
        if (a.v[i] != fp_p(i)) return a.v[i] < fp_p(i);
    }
    return false;
}
// p = 3 mod 4: sqrt(a) = a^((p+1)/4); returns false when a is not a square
VK_HD bool fp_sqrt(Fp &out, const Fp &a) {
    const uint32_t e[12] = {0xffffeaabu, 0xee7fbfffu, 0xac54ffffu, 0x07aaffffu, 0x3dac3d89u, 0xd9cc34a8u,
                            0x3ce144afu, 0xd91dd2e1u, 0x90d2eb35u, 0x92c6e9edu, 0x8e5ff9a6u, 0x0680447au};
    Fp s = fp_pow_words(a, e, 12);
    if (!fp_eq(fp_sqr(s), a)) return false;
    out = s;
    return true;
}

// ------------------------------------------------------------------- Fr
VK_HD Fr fr_zero() {
    Fr r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.v[i] = 0;
    return r;
}
VK_HD Fr fr_one() { return Fr{VK_FR_ONE}; }
VK_HD Fr fr_mul(const Fr &a, const Fr &b) {
    Fr r;
    mont_mul<8>(r.v, a.v, b.v);
    return r;
}
VK_HD Fr fr_sqr(const Fr &a) { return fr_mul(a, a); }
VK_HD Fr fr_add(const Fr &a, const Fr &b) {
    Fr r;
    mod_add<8>(r.v, a.v, b.v);
    return r;
}
VK_HD Fr fr_sub(const Fr &a, const Fr &b) {
    Fr r;
    mod_sub<8>(r.v, a.v, b.v);
    return r;
}
VK_HD Fr fr_neg(const Fr &a) { return fr_sub(fr_zero(), a); }
VK_HD bool fr_is_zero(const Fr &a) { return limbs_is_zero<8>(a.v); }
VK_HD bool fr_eq(const Fr &a, const Fr &b) { return limbs_eq<8>(a.v, b.v); }
VK_HD Fr fr_pow_words(const Fr &a, const uint32_t *e, int words) {
    Fr acc = fr_one();
    for (int i = words - 1; i >= 0; i--) {
        for (int b = 31; b >= 0; b--) {
            acc = fr_sqr(acc);
            if ((e[i] >> b) & 1u) acc = fr_mul(acc, a);
        }
    }
    return acc;
}
// a^(r-2) (field.glsl.inc:257-275)
VK_HD Fr fr_inv(const Fr &a) {
    const uint32_t e[8] = {0xffffffffu, 0xfffffffeu, 0xfffe5bfeu, 0x53bda402u,
                           0x09a1d805u, 0x3339d808u, 0x299d7d48u, 0x73eda753u};
    return fr_pow_words(a, e, 8);
}
VK_HD Fr fr_to_canonical(const Fr &a) {
    Fr one = fr_zero();
    one.v[0] = 1;
    return fr_mul(a, one);
}
// mont_mul needs its first operand below the modulus; the second may be any
// n-word value (the result is still < 2m before the final subtraction).  So a
// raw 256-bit input, canonical or not, goes second: fr_from_canonical(v) is
// v mod r in Montgomery form for every v < 2^256 (k_cells_to_fr.comp relies on
// the same property).
VK_HD Fr fr_from_canonical(const Fr &a) { return fr_mul(Fr{VK_FR_R2}, a); }
VK_HD bool fr_is_canonical(const Fr &a) {
    for (int i = 7; i >= 0; i--) {
        if (a.v[i] != fr_p(i)) return a.v[i] < fr_p(i);
    }
    return false;
}
VK_HD Fr fr_from_u32(uint32_t x) {
    Fr c = fr_zero();
    c.v[0] = x;
    return fr_from_canonical(c);
}

// 32 big-endian bytes <-> 8 little-endian words
VK_HD Fr fr_load_be(const uint8_t *b) {
    Fr v;
#pragma unroll
    for (int limb = 0; limb < 8; limb++) {
        const int off = (7 - limb) * 4;
        v.v[limb] = ((uint32_t)b[off] << 24) | ((uint32_t)b[off + 1] << 16) | ((uint32_t)b[off + 2] << 8) |
                    (uint32_t)b[off + 3];
    }
    return v;
}
VK_HD uint32_t bswap32(uint32_t x) {
    return (x >> 24) | ((x >> 8) & 0xff00u) | ((x << 8) & 0xff0000u) | (x << 24);
}

VK_HD uint32_t brev_bits(uint32_t x, int bits) {
#if defined(__CUDA_ARCH__)
    return __brev(x) >> (32 - bits);
#else
    uint32_t r = 0;
    for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
#endif
}

} // namespace vkzg
