// Host-only: splitting the fixed phase-B tap scalars for the G1 endomorphism
// phi(P) = -z^2 P (curve.cuh g1_phi).  With Z = z^2 (127.4 bits) and
// r = Z^2 - Z + 1, every k < r is k = q Z + rem; centring rem and q (the
// latter through Z^2 = Z - 1 mod r) gives
//     k = k1 + k2 Z (mod r),   |k1|, |k2| <= Z/2 + 1 < 2^126.5,
// so k P = k1 P + (-k2) phi(P): two 16-digit scalars in place of one 32-digit
// scalar, which halves the doublings of the proof ladder.  The reference
// applies the full 255-bit taps (k_phase_b_split.comp); the sums are the same
// group elements.
#pragma once

#include <stdint.h>

namespace vkzg {

typedef unsigned __int128 glv_u128;

constexpr int kGlvDigits = 16; // signed base-256 digits per half

// coefficient of P is (neg[0] ? -1 : 1) mag[0], of phi(P) (neg[1] ? -1 : 1) mag[1]
struct GlvSplit {
    glv_u128 mag[2];
    bool neg[2];
};

inline glv_u128 glv_z2() { return ((glv_u128)0xac45a4010001a402ull << 64) | 0x0000000100000000ull; }

// k: 8 little-endian 32-bit words, k < r (canonical).
inline GlvSplit glv_split(const uint32_t k[8]) {
    glv_u128 lo = 0, hi = 0;
    for (int i = 3; i >= 0; i--) {
        lo = (lo << 32) | k[i];
        hi = (hi << 32) | k[i + 4];
    }
    const glv_u128 Z = glv_z2();
    // quotient by shift-and-subtract: k < r < Z 2^128, so q < 2^128 and the
    // remainder ends below Z with hi = 0
    glv_u128 q = 0;
    for (int bit = 127; bit >= 0; bit--) {
        const glv_u128 shi = bit ? Z >> (128 - bit) : 0, slo = Z << bit;
        if (hi > shi || (hi == shi && lo >= slo)) {
            hi = hi - shi - (lo < slo ? 1 : 0);
            lo -= slo;
            q |= (glv_u128)1 << bit;
        }
    }
    GlvSplit s;
    // k1 = rem in (-Z/2, Z/2]
    if (lo > Z / 2) {
        s.mag[0] = Z - lo;
        s.neg[0] = true;
        q += 1;
    } else {
        s.mag[0] = lo;
        s.neg[0] = false;
    }
    // k2 = q in [0, Z]; above Z/2, (Z - 1) Z = Z^2 - Z = -1 (mod r) gives
    // q Z = (q - (Z - 1)) Z - 1: k2 = q - (Z - 1), k1 - 1
    bool k2_neg = false;
    glv_u128 k2 = q;
    if (q > Z / 2) {
        // k1 -= 1
        if (s.neg[0]) {
            s.mag[0] += 1;
        } else if (s.mag[0] == 0) {
            s.mag[0] = 1;
            s.neg[0] = true;
        } else {
            s.mag[0] -= 1;
        }
        if (q >= Z - 1) {
            k2 = q - (Z - 1);
        } else {
            k2 = (Z - 1) - q;
            k2_neg = true;
        }
    }
    s.mag[1] = k2;
    s.neg[1] = !k2_neg; // phi(P) carries -k2
    return s;
}

// Signed base-256 digits in [-127, 128] (the reference's recoding: a byte
// above 128 becomes byte - 256 with a carry into the next), negated when neg.
// Returns false if kGlvDigits digits do not hold the value.
inline bool glv_digits(glv_u128 mag, bool neg, int dig[kGlvDigits]) {
    int carry = 0;
    for (int d = 0; d < kGlvDigits; d++) {
        int v = (int)((mag >> (8 * d)) & 0xffu) + carry;
        carry = 0;
        if (v > 128) {
            v -= 256;
            carry = 1;
        }
        dig[d] = neg ? -v : v;
    }
    return carry == 0; // the 16 digits span all 128 bits of mag
}

} // namespace vkzg
