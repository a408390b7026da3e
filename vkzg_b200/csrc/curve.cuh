// BLS12-381 G1 (y^2 = x^3 + 4 over Fp).  Jacobian (X:Y:Z) = (X/Z^2, Y/Z^3)
// with Z == 0 as the point at infinity; affine (0, 0) is the point at
// infinity (the reference's conventions, src/shaders/field.glsl.inc:302-310).
// Formulas are the standard EFD ones for a = 0: dbl-2009-l, add-2007-bl,
// madd-2007-bl, each handling P == Q and P == -Q like the reference's.
#pragma once

#include "field.cuh"

namespace vkzg {

struct G1J {
    Fp x, y, z;
};
struct G1A {
    Fp x, y;
};

VK_HD G1J g1_identity() {
    G1J r;
    r.x = fp_zero();
    r.y = fp_one();
    r.z = fp_zero();
    return r;
}
VK_HD bool g1a_is_identity(const G1A &p) { return fp_is_zero(p.x) && fp_is_zero(p.y); }
VK_HD bool g1j_is_identity(const G1J &p) { return fp_is_zero(p.z); }

// The order-3 endomorphism phi(x, y) = (beta x, y), beta the cube root of unity
// 0x5f19672fdf76ce51ba69c6076a0f77eaddb3a93be6f89688de17d813620a00022e01fffffffefffe
// (here in Montgomery form).  On G1, phi(P) = -z^2 P with z = -0xd201000000010000
// the curve parameter; (0, 0) stays (0, 0).
VK_HD G1A g1_phi(const G1A &p) {
    const Fp beta = {{0x798a64e8u, 0x30f1361bu, 0x7ece5a2au, 0xf3b8ddabu, 0xc61577f7u, 0x16a8ca3au,
                      0x74fd029bu, 0xc26a2ff8u, 0x60701c6eu, 0x3636b766u, 0x241b6160u, 0x051ba4abu}};
    G1A r;
    r.x = fp_mul(beta, p.x);
    r.y = p.y;
    return r;
}

VK_HD G1J g1_from_affine(const G1A &a) {
    if (g1a_is_identity(a)) return g1_identity();
    G1J r;
    r.x = a.x;
    r.y = a.y;
    r.z = fp_one();
    return r;
}

// dbl-2009-l: 2M + 5S
VK_HD G1J g1_dbl(const G1J &p) {
    if (fp_is_zero(p.z)) return p;
    const Fp A = fp_sqr(p.x);
    const Fp B = fp_sqr(p.y);
    const Fp C = fp_sqr(B);
    Fp t0 = fp_sqr(fp_add(p.x, B));
    t0 = fp_sub(fp_sub(t0, A), C);
    const Fp D = fp_dbl(t0);
    const Fp E = fp_add(fp_dbl(A), A);
    const Fp F = fp_sqr(E);
    G1J r;
    r.x = fp_sub(F, fp_dbl(D));
    r.y = fp_sub(fp_mul(E, fp_sub(D, r.x)), fp_dbl(fp_dbl(fp_dbl(C))));
    r.z = fp_dbl(fp_mul(p.y, p.z));
    return r;
}

// g1_dbl with the products inlined: the independent products of one doubling
// (X^2, Y^2, Y Z; then B^2, (X + B)^2, E^2) overlap instead of running as
// sequential calls.  For latency-bound chains of doublings (the ladder).
VK_HD Fp fp_mul_inl(const Fp &a, const Fp &b) {
    Fp r;
#if VKZG_FP_KARATSUBA
    mont_mul_ks<12, VKZG_FP_KARATSUBA>(r.v, a.v, b.v);
#else
    mont_mul<12>(r.v, a.v, b.v);
#endif
    return r;
}
VK_HD Fp fp_sqr_inl(const Fp &a) {
    Fp r;
#if VKZG_FP_KARATSUBA
    mont_sqr_ks<12>(r.v, a.v);
#else
    mont_sqr<12>(r.v, a.v);
#endif
    return r;
}
VK_HD G1J g1_dbl_inl(const G1J &p) {
    if (fp_is_zero(p.z)) return p;
    const Fp A = fp_sqr_inl(p.x);
    const Fp B = fp_sqr_inl(p.y);
    const Fp YZ = fp_mul_inl(p.y, p.z);
    const Fp C = fp_sqr_inl(B);
    const Fp XB = fp_add(p.x, B);
    Fp t0 = fp_sqr_inl(XB);
    const Fp E = fp_add(fp_dbl(A), A);
    const Fp F = fp_sqr_inl(E);
    t0 = fp_sub(fp_sub(t0, A), C);
    const Fp D = fp_dbl(t0);
    G1J r;
    r.x = fp_sub(F, fp_dbl(D));
    r.y = fp_sub(fp_mul_inl(E, fp_sub(D, r.x)), fp_dbl(fp_dbl(fp_dbl(C))));
    r.z = fp_dbl(YZ);
    return r;
}

// add-2007-bl: 11M + 5S
VK_HD G1J g1_add(const G1J &a, const G1J &b) {
    if (fp_is_zero(a.z)) return b;
    if (fp_is_zero(b.z)) return a;
    const Fp Z1Z1 = fp_sqr(a.z);
    const Fp Z2Z2 = fp_sqr(b.z);
    const Fp U1 = fp_mul(a.x, Z2Z2);
    const Fp U2 = fp_mul(b.x, Z1Z1);
    const Fp S1 = fp_mul(a.y, fp_mul(b.z, Z2Z2));
    const Fp S2 = fp_mul(b.y, fp_mul(a.z, Z1Z1));
    if (fp_eq(U1, U2)) {
        if (fp_eq(S1, S2)) return g1_dbl(a);
        return g1_identity();
    }
    const Fp H = fp_sub(U2, U1);
    const Fp I = fp_sqr(fp_dbl(H));
    const Fp J = fp_mul(H, I);
    const Fp K = fp_dbl(fp_sub(S2, S1));
    const Fp V = fp_mul(U1, I);
    G1J r;
    r.x = fp_sub(fp_sub(fp_sqr(K), J), fp_dbl(V));
    r.y = fp_sub(fp_mul(K, fp_sub(V, r.x)), fp_dbl(fp_mul(S1, J)));
    r.z = fp_mul(fp_sub(fp_sub(fp_sqr(fp_add(a.z, b.z)), Z1Z1), Z2Z2), H);
    return r;
}

// madd-2007-bl (Jacobian + affine): 7M + 4S
VK_HD G1J g1_madd(const G1J &a, const G1A &b) {
    if (g1a_is_identity(b)) return a;
    if (fp_is_zero(a.z)) {
        G1J r;
        r.x = b.x;
        r.y = b.y;
        r.z = fp_one();
        return r;
    }
    const Fp Z1Z1 = fp_sqr(a.z);
    const Fp U2 = fp_mul(b.x, Z1Z1);
    const Fp S2 = fp_mul(b.y, fp_mul(a.z, Z1Z1));
    if (fp_eq(a.x, U2)) {
        if (fp_eq(a.y, S2)) return g1_dbl(a);
        return g1_identity();
    }
    const Fp H = fp_sub(U2, a.x);
    const Fp HH = fp_sqr(H);
    const Fp I = fp_dbl(fp_dbl(HH));
    const Fp J = fp_mul(H, I);
    const Fp K = fp_dbl(fp_sub(S2, a.y));
    const Fp V = fp_mul(a.x, I);
    G1J r;
    r.x = fp_sub(fp_sub(fp_sqr(K), J), fp_dbl(V));
    r.y = fp_sub(fp_mul(K, fp_sub(V, r.x)), fp_dbl(fp_mul(a.y, J)));
    r.z = fp_sub(fp_sub(fp_sqr(fp_add(a.z, H)), Z1Z1), HH);
    return r;
}

VK_HD G1J g1_neg(const G1J &p) {
    G1J r = p;
    r.y = fp_neg(p.y);
    return r;
}
VK_HD G1J g1_sub(const G1J &a, const G1J &b) { return g1_add(a, g1_neg(b)); }

// double-and-add over a canonical scalar (8 LE words), MSB first
VK_HD G1J g1_mul_scalar(const G1J &p, const Fr &k) {
    G1J acc = g1_identity();
    for (int i = 7; i >= 0; i--) {
        for (int b = 31; b >= 0; b--) {
            acc = g1_dbl(acc);
            if ((k.v[i] >> b) & 1u) acc = g1_add(acc, p);
        }
    }
    return acc;
}

// ZCash compressed encoding from affine Montgomery (k_compress_proofs.comp:25-47):
// 48 bytes BE of canonical x; 0x80 compressed, 0x20 when y > (p-1)/2, 0xc0 for infinity.
VK_HD void g1_compress(uint8_t *out, const G1A &p) {
    if (g1a_is_identity(p)) {
        for (int k = 0; k < 48; k++) out[k] = 0;
        out[0] = 0xc0;
        return;
    }
    const Fp x = fp_to_canonical(p.x);
    const Fp y = fp_to_canonical(p.y);
    for (int limb = 0; limb < 12; limb++) {
        const uint32_t w = x.v[limb];
        const int off = (11 - limb) * 4;
        out[off + 0] = (uint8_t)(w >> 24);
        out[off + 1] = (uint8_t)(w >> 16);
        out[off + 2] = (uint8_t)(w >> 8);
        out[off + 3] = (uint8_t)w;
    }
    out[0] |= 0x80u | (fp_is_lex_largest(y) ? 0x20u : 0u);
}

// Inverse of g1_compress (on-curve check, no subgroup check).  Returns false on
// malformed input.
VK_HD bool g1_decompress(G1A &out, const uint8_t *in) {
    const uint8_t flags = in[0];
    if (!(flags & 0x80u)) return false;
    const bool inf = (flags & 0x40u) != 0, sign = (flags & 0x20u) != 0;
    Fp x;
    for (int limb = 0; limb < 12; limb++) {
        const int off = (11 - limb) * 4;
        x.v[limb] = ((uint32_t)in[off] << 24) | ((uint32_t)in[off + 1] << 16) | ((uint32_t)in[off + 2] << 8) |
                    (uint32_t)in[off + 3];
    }
    x.v[11] &= 0x1fffffffu;
    if (inf) {
        if (sign || !fp_is_zero(x)) return false;
        out.x = fp_zero();
        out.y = fp_zero();
        return true;
    }
    if (!fp_is_canonical(x)) return false;
    const Fp xm = fp_from_canonical(x);
    Fp four = fp_zero();
    four.v[0] = 4;
    const Fp y2 = fp_add(fp_mul(fp_sqr(xm), xm), fp_from_canonical(four));
    Fp y;
    if (!fp_sqrt(y, y2)) return false;
    if (fp_is_lex_largest(fp_to_canonical(y)) != sign) y = fp_neg(y);
    out.x = xm;
    out.y = y;
    return true;
}

} // namespace vkzg
