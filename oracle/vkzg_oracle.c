/*
 * vkzg CPU oracle -- TEST INFRASTRUCTURE ONLY (see vkzg_oracle.h).
 *
 * Scalar restatement of the reference's arithmetic and pipelines.  Limbs are
 * 64-bit here (the reference's are 32-bit), but the Montgomery radices are the
 * same (R = 2^384 for Fp, 2^256 for Fr), so a Montgomery value has the same
 * byte image as the reference's 12 / 8 little-endian 32-bit words.
 *
 * Reference citations are paths within jtraglia/vkzg.
 */
#include "vkzg_oracle.h"

#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ======================================================================
 * Field constants (tools/gen_constants.py:8-9 gives p and r).
 * ====================================================================== */
typedef struct { uint64_t l[6]; } fp_t;
typedef struct { uint64_t l[4]; } fr_t;

static const fp_t FP_P = {{0xb9feffffffffaaabULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL,
                           0x64774b84f38512bfULL, 0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL}};
static const uint64_t FP_INV = 0x89f3fffcfffcfffdULL; /* -p^-1 mod 2^64 */
static const fp_t FP_ONE = {{0x760900000002fffdULL, 0xebf4000bc40c0002ULL, 0x5f48985753c758baULL,
                             0x77ce585370525745ULL, 0x5c071a97a256ec6dULL, 0x15f65ec3fa80e493ULL}};
static const fp_t FP_R2 = {{0xf4df1f341c341746ULL, 0x0a76e6a609d104f1ULL, 0x8de5476c4c95b6d5ULL,
                            0x67eb88a9939d83c0ULL, 0x9a793e85b519952dULL, 0x11988fe592cae3aaULL}};

static const fr_t FR_P = {{0xffffffff00000001ULL, 0x53bda402fffe5bfeULL, 0x3339d80809a1d805ULL,
                           0x73eda753299d7d48ULL}};
static const uint64_t FR_INV = 0xfffffffeffffffffULL; /* -r^-1 mod 2^64 */
static const fr_t FR_ONE = {{0x00000001fffffffeULL, 0x5884b7fa00034802ULL, 0x998c4fefecbc4ff5ULL,
                             0x1824b159acc5056fULL}};
static const fr_t FR_R2 = {{0xc999e990f3f29c6dULL, 0x2b6cedcb87925c23ULL, 0x05d314967254398fULL,
                            0x0748d9d99f59ff11ULL}};

/* ---------------------------------------------------------------- generic
 * Montgomery CIOS over n 64-bit limbs.  field.glsl.inc:116-157 (fp_mul) and
 * :208-248 (fr_mul) are the same algorithm over 32-bit limbs. */
static inline void mont_mul(uint64_t *r, const uint64_t *a, const uint64_t *b, const uint64_t *m,
                            uint64_t inv, int n) {
    uint64_t t[8] = {0};
    for (int i = 0; i < n; i++) {
        u128 c = 0;
        for (int j = 0; j < n; j++) {
            c += (u128)a[j] * b[i] + t[j];
            t[j] = (uint64_t)c;
            c >>= 64;
        }
        c += t[n];
        t[n] = (uint64_t)c;
        t[n + 1] = (uint64_t)(c >> 64);
        uint64_t q = t[0] * inv;
        c = (u128)q * m[0] + t[0];
        c >>= 64;
        for (int j = 1; j < n; j++) {
            c += (u128)q * m[j] + t[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[n];
        t[n - 1] = (uint64_t)c;
        t[n] = t[n + 1] + (uint64_t)(c >> 64);
    }
    /* result < 2m: one conditional subtraction (field.glsl.inc:146-156) */
    uint64_t s[8];
    uint64_t borrow = 0;
    for (int i = 0; i < n; i++) {
        u128 d = (u128)t[i] - m[i] - borrow;
        s[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) & 1;
    }
    int keep = t[n] < borrow; /* negative => keep t */
    for (int i = 0; i < n; i++) r[i] = keep ? t[i] : s[i];
}

static inline void mod_add(uint64_t *r, const uint64_t *a, const uint64_t *b, const uint64_t *m, int n) {
    uint64_t t[8], s[8];
    u128 c = 0;
    for (int i = 0; i < n; i++) {
        c += (u128)a[i] + b[i];
        t[i] = (uint64_t)c;
        c >>= 64;
    }
    uint64_t borrow = 0;
    for (int i = 0; i < n; i++) {
        u128 d = (u128)t[i] - m[i] - borrow;
        s[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) & 1;
    }
    /* moduli leave headroom in the top limb, so the sum never carries out */
    for (int i = 0; i < n; i++) r[i] = borrow ? t[i] : s[i];
}

static inline void mod_sub(uint64_t *r, const uint64_t *a, const uint64_t *b, const uint64_t *m, int n) {
    uint64_t t[8];
    uint64_t borrow = 0;
    for (int i = 0; i < n; i++) {
        u128 d = (u128)a[i] - b[i] - borrow;
        t[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) & 1;
    }
    u128 c = 0;
    for (int i = 0; i < n; i++) {
        c += (u128)t[i] + (borrow ? m[i] : 0);
        r[i] = (uint64_t)c;
        c >>= 64;
    }
}

static inline int limbs_is_zero(const uint64_t *a, int n) {
    uint64_t acc = 0;
    for (int i = 0; i < n; i++) acc |= a[i];
    return acc == 0;
}

static inline int limbs_eq(const uint64_t *a, const uint64_t *b, int n) {
    uint64_t acc = 0;
    for (int i = 0; i < n; i++) acc |= a[i] ^ b[i];
    return acc == 0;
}

/* a < b, little-endian limbs */
static inline int limbs_lt(const uint64_t *a, const uint64_t *b, int n) {
    for (int i = n - 1; i >= 0; i--) {
        if (a[i] != b[i]) return a[i] < b[i];
    }
    return 0;
}

/* ---------------------------------------------------------------- Fp */
static inline void fp_mul(fp_t *r, const fp_t *a, const fp_t *b) { mont_mul(r->l, a->l, b->l, FP_P.l, FP_INV, 6); }
static inline void fp_sqr(fp_t *r, const fp_t *a) { mont_mul(r->l, a->l, a->l, FP_P.l, FP_INV, 6); }
static inline void fp_add(fp_t *r, const fp_t *a, const fp_t *b) { mod_add(r->l, a->l, b->l, FP_P.l, 6); }
static inline void fp_sub(fp_t *r, const fp_t *a, const fp_t *b) { mod_sub(r->l, a->l, b->l, FP_P.l, 6); }
static inline void fp_dbl(fp_t *r, const fp_t *a) { mod_add(r->l, a->l, a->l, FP_P.l, 6); }
static inline int fp_is_zero(const fp_t *a) { return limbs_is_zero(a->l, 6); }
static inline int fp_eq(const fp_t *a, const fp_t *b) { return limbs_eq(a->l, b->l, 6); }
static inline void fp_neg(fp_t *r, const fp_t *a) {
    /* field.glsl.inc:99-102: -0 stays 0 */
    if (fp_is_zero(a)) { *r = *a; return; }
    fp_t z = {{0}};
    fp_sub(r, &z, a);
}

static void fp_pow(fp_t *r, const fp_t *a, const uint64_t *e, int nlimbs) {
    fp_t acc = FP_ONE;
    for (int i = nlimbs - 1; i >= 0; i--) {
        for (int b = 63; b >= 0; b--) {
            fp_sqr(&acc, &acc);
            if ((e[i] >> b) & 1) fp_mul(&acc, &acc, a);
        }
    }
    *r = acc;
}

/* a^(p-2), field.glsl.inc:528-547 */
static void fp_inv(fp_t *r, const fp_t *a) {
    uint64_t e[6];
    memcpy(e, FP_P.l, sizeof e);
    e[0] -= 2;
    fp_pow(r, a, e, 6);
}

/* p = 3 mod 4: sqrt(a) = a^((p+1)/4).  Returns 1 when a is a square. */
static int fp_sqrt(fp_t *r, const fp_t *a) {
    /* (p+1)/4 */
    uint64_t e[6];
    u128 c = 1;
    for (int i = 0; i < 6; i++) {
        c += FP_P.l[i];
        e[i] = (uint64_t)c;
        c >>= 64;
    }
    for (int i = 0; i < 6; i++) e[i] = (e[i] >> 2) | (i < 5 ? e[i + 1] << 62 : 0);
    fp_t s, chk;
    fp_pow(&s, a, e, 6);
    fp_sqr(&chk, &s);
    if (!fp_eq(&chk, a)) return 0;
    *r = s;
    return 1;
}

static void fp_from_canonical(fp_t *r, const fp_t *a) { fp_mul(r, a, &FP_R2); }
static void fp_to_canonical(fp_t *r, const fp_t *a) {
    fp_t one = {{1, 0, 0, 0, 0, 0}};
    fp_mul(r, a, &one);
}

/* ---------------------------------------------------------------- Fr */
static inline void fr_mul(fr_t *r, const fr_t *a, const fr_t *b) { mont_mul(r->l, a->l, b->l, FR_P.l, FR_INV, 4); }
static inline void fr_add(fr_t *r, const fr_t *a, const fr_t *b) { mod_add(r->l, a->l, b->l, FR_P.l, 4); }
static inline void fr_sub(fr_t *r, const fr_t *a, const fr_t *b) { mod_sub(r->l, a->l, b->l, FR_P.l, 4); }
static inline int fr_is_zero(const fr_t *a) { return limbs_is_zero(a->l, 4); }
static inline void fr_neg(fr_t *r, const fr_t *a) {
    fr_t z = {{0}};
    fr_sub(r, &z, a); /* field.glsl.inc:250-252: 0 - 0 = 0 */
}
static void fr_from_canonical(fr_t *r, const fr_t *a) { fr_mul(r, a, &FR_R2); }
static void fr_to_canonical(fr_t *r, const fr_t *a) {
    fr_t one = {{1, 0, 0, 0}};
    fr_mul(r, a, &one);
}
static int fr_is_canonical(const fr_t *a) { return limbs_lt(a->l, FR_P.l, 4); }

static void fr_pow(fr_t *r, const fr_t *a, const uint64_t *e, int nlimbs) {
    fr_t acc = FR_ONE;
    for (int i = nlimbs - 1; i >= 0; i--) {
        for (int b = 63; b >= 0; b--) {
            fr_mul(&acc, &acc, &acc);
            if ((e[i] >> b) & 1) fr_mul(&acc, &acc, a);
        }
    }
    *r = acc;
}

/* a^(r-2), field.glsl.inc:257-275 (zero maps to zero) */
static void fr_inv(fr_t *r, const fr_t *a) {
    uint64_t e[4];
    memcpy(e, FR_P.l, sizeof e);
    e[0] -= 2;
    fr_pow(r, a, e, 4);
}

static void fr_from_u64(fr_t *r, uint64_t v) {
    fr_t c = {{v, 0, 0, 0}};
    fr_from_canonical(r, &c);
}

/* ---------------------------------------------------------------- bytes */
/* 32 big-endian bytes -> 4 little-endian 64-bit limbs (k_blob_to_fr.comp:24-29) */
static void be32_to_limbs(uint64_t *l, const uint8_t *b) {
    for (int i = 0; i < 4; i++) {
        uint64_t v = 0;
        for (int k = 0; k < 8; k++) v = (v << 8) | b[(3 - i) * 8 + k];
        l[i] = v;
    }
}
static void limbs_to_be32(uint8_t *b, const uint64_t *l) {
    for (int i = 0; i < 4; i++)
        for (int k = 0; k < 8; k++) b[(3 - i) * 8 + k] = (uint8_t)(l[i] >> (56 - 8 * k));
}
static void be48_to_limbs(uint64_t *l, const uint8_t *b) {
    for (int i = 0; i < 6; i++) {
        uint64_t v = 0;
        for (int k = 0; k < 8; k++) v = (v << 8) | b[(5 - i) * 8 + k];
        l[i] = v;
    }
}
static void limbs_to_be48(uint8_t *b, const uint64_t *l) {
    for (int i = 0; i < 6; i++)
        for (int k = 0; k < 8; k++) b[(5 - i) * 8 + k] = (uint8_t)(l[i] >> (56 - 8 * k));
}

static uint32_t brev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

/* ======================================================================
 * G1 (field.glsl.inc:281-425).  Jacobian, Z == 0 is infinity; affine (0,0)
 * is infinity.
 * ====================================================================== */
typedef struct { fp_t x, y, z; } g1j_t;
typedef struct { fp_t x, y; } g1a_t;

static g1j_t g1_identity(void) {
    g1j_t r;
    memset(&r, 0, sizeof r);
    r.y = FP_ONE;
    return r;
}
static int g1a_is_identity(const g1a_t *p) { return fp_is_zero(&p->x) && fp_is_zero(&p->y); }

/* dbl-2009-l, field.glsl.inc:312-333 */
static void g1_dbl(g1j_t *r, const g1j_t *p) {
    if (fp_is_zero(&p->z)) { *r = *p; return; }
    fp_t A, B, C, D, E, F, t0, t1, t2;
    fp_sqr(&A, &p->x);
    fp_sqr(&B, &p->y);
    fp_sqr(&C, &B);
    fp_add(&t0, &p->x, &B);
    fp_sqr(&t0, &t0);
    fp_sub(&t0, &t0, &A);
    fp_sub(&t0, &t0, &C);
    fp_dbl(&D, &t0);
    fp_dbl(&E, &A);
    fp_add(&E, &E, &A);
    fp_sqr(&F, &E);
    g1j_t o;
    fp_dbl(&t1, &D);
    fp_sub(&o.x, &F, &t1);
    fp_sub(&t1, &D, &o.x);
    fp_mul(&t1, &E, &t1);
    fp_dbl(&t2, &C);
    fp_dbl(&t2, &t2);
    fp_dbl(&t2, &t2);
    fp_sub(&o.y, &t1, &t2);
    fp_mul(&t0, &p->y, &p->z);
    fp_dbl(&o.z, &t0);
    *r = o;
}

/* add-2007-bl, field.glsl.inc:336-363 */
static void g1_add(g1j_t *r, const g1j_t *a, const g1j_t *b) {
    if (fp_is_zero(&a->z)) { *r = *b; return; }
    if (fp_is_zero(&b->z)) { *r = *a; return; }
    fp_t Z1Z1, Z2Z2, U1, U2, S1, S2, t;
    fp_sqr(&Z1Z1, &a->z);
    fp_sqr(&Z2Z2, &b->z);
    fp_mul(&U1, &a->x, &Z2Z2);
    fp_mul(&U2, &b->x, &Z1Z1);
    fp_mul(&t, &b->z, &Z2Z2);
    fp_mul(&S1, &a->y, &t);
    fp_mul(&t, &a->z, &Z1Z1);
    fp_mul(&S2, &b->y, &t);
    if (fp_eq(&U1, &U2)) {
        if (fp_eq(&S1, &S2)) { g1_dbl(r, a); return; }
        *r = g1_identity();
        return;
    }
    fp_t H, I, J, K, V;
    fp_sub(&H, &U2, &U1);
    fp_dbl(&I, &H);
    fp_sqr(&I, &I);
    fp_mul(&J, &H, &I);
    fp_sub(&K, &S2, &S1);
    fp_dbl(&K, &K);
    fp_mul(&V, &U1, &I);
    g1j_t o;
    fp_sqr(&o.x, &K);
    fp_sub(&o.x, &o.x, &J);
    fp_dbl(&t, &V);
    fp_sub(&o.x, &o.x, &t);
    fp_sub(&t, &V, &o.x);
    fp_mul(&t, &K, &t);
    fp_t s1j;
    fp_mul(&s1j, &S1, &J);
    fp_dbl(&s1j, &s1j);
    fp_sub(&o.y, &t, &s1j);
    fp_add(&o.z, &a->z, &b->z);
    fp_sqr(&o.z, &o.z);
    fp_sub(&o.z, &o.z, &Z1Z1);
    fp_sub(&o.z, &o.z, &Z2Z2);
    fp_mul(&o.z, &o.z, &H);
    *r = o;
}

/* madd-2007-bl, field.glsl.inc:366-396 */
static void g1_madd(g1j_t *r, const g1j_t *a, const g1a_t *b) {
    if (g1a_is_identity(b)) { *r = *a; return; }
    if (fp_is_zero(&a->z)) {
        r->x = b->x;
        r->y = b->y;
        r->z = FP_ONE;
        return;
    }
    fp_t Z1Z1, U2, S2, t;
    fp_sqr(&Z1Z1, &a->z);
    fp_mul(&U2, &b->x, &Z1Z1);
    fp_mul(&t, &a->z, &Z1Z1);
    fp_mul(&S2, &b->y, &t);
    if (fp_eq(&a->x, &U2)) {
        if (fp_eq(&a->y, &S2)) { g1_dbl(r, a); return; }
        *r = g1_identity();
        return;
    }
    fp_t H, HH, I, J, K, V;
    fp_sub(&H, &U2, &a->x);
    fp_sqr(&HH, &H);
    fp_dbl(&I, &HH);
    fp_dbl(&I, &I);
    fp_mul(&J, &H, &I);
    fp_sub(&K, &S2, &a->y);
    fp_dbl(&K, &K);
    fp_mul(&V, &a->x, &I);
    g1j_t o;
    fp_sqr(&o.x, &K);
    fp_sub(&o.x, &o.x, &J);
    fp_dbl(&t, &V);
    fp_sub(&o.x, &o.x, &t);
    fp_sub(&t, &V, &o.x);
    fp_mul(&t, &K, &t);
    fp_t yj;
    fp_mul(&yj, &a->y, &J);
    fp_dbl(&yj, &yj);
    fp_sub(&o.y, &t, &yj);
    fp_add(&o.z, &a->z, &H);
    fp_sqr(&o.z, &o.z);
    fp_sub(&o.z, &o.z, &Z1Z1);
    fp_sub(&o.z, &o.z, &HH);
    *r = o;
}

static void g1_neg(g1j_t *r, const g1j_t *p) {
    *r = *p;
    fp_neg(&r->y, &p->y);
}

static void g1_sub(g1j_t *r, const g1j_t *a, const g1j_t *b) {
    g1j_t nb;
    g1_neg(&nb, b);
    g1_add(r, a, &nb);
}

static g1j_t g1_from_affine(const g1a_t *a) {
    if (g1a_is_identity(a)) return g1_identity();
    g1j_t r;
    r.x = a->x;
    r.y = a->y;
    r.z = FP_ONE;
    return r;
}

static g1a_t g1_to_affine(const g1j_t *p) {
    g1a_t r;
    if (fp_is_zero(&p->z)) {
        memset(&r, 0, sizeof r);
        return r;
    }
    fp_t zi, z2, z3;
    fp_inv(&zi, &p->z);
    fp_sqr(&z2, &zi);
    fp_mul(&z3, &z2, &zi);
    fp_mul(&r.x, &p->x, &z2);
    fp_mul(&r.y, &p->y, &z3);
    return r;
}

/* Montgomery batch normalisation (k_normalize.comp:19-57): one inversion for
 * all points; infinity -> (0,0). */
static void g1_batch_to_affine(g1a_t *out, const g1j_t *in, size_t n) {
    fp_t *pre = (fp_t *)malloc(sizeof(fp_t) * (n ? n : 1));
    fp_t acc = FP_ONE;
    for (size_t i = 0; i < n; i++) {
        pre[i] = acc;
        if (!fp_is_zero(&in[i].z)) fp_mul(&acc, &acc, &in[i].z);
    }
    fp_t inv;
    fp_inv(&inv, &acc);
    for (size_t k = n; k-- > 0;) {
        if (fp_is_zero(&in[k].z)) {
            memset(&out[k], 0, sizeof out[k]);
            continue;
        }
        fp_t zi, z2, z3;
        fp_mul(&zi, &pre[k], &inv);
        fp_mul(&inv, &inv, &in[k].z);
        fp_sqr(&z2, &zi);
        fp_mul(&z3, &z2, &zi);
        g1a_t o;
        fp_mul(&o.x, &in[k].x, &z2);
        fp_mul(&o.y, &in[k].y, &z3);
        out[k] = o;
    }
    free(pre);
}

/* double-and-add, MSB first, on a canonical scalar */
static void g1_mul(g1j_t *r, const g1j_t *p, const fr_t *k_canonical) {
    g1j_t acc = g1_identity();
    for (int i = 3; i >= 0; i--) {
        for (int b = 63; b >= 0; b--) {
            g1_dbl(&acc, &acc);
            if ((k_canonical->l[i] >> b) & 1) g1_add(&acc, &acc, p);
        }
    }
    *r = acc;
}

/* ---------------------------------------------------------------- encoding */
/* (p-1)/2 comparison, field.glsl.inc:549-562 */
static int fp_is_lex_largest(const fp_t *canonical) {
    fp_t half;
    /* (p-1)/2 */
    for (int i = 0; i < 6; i++) half.l[i] = (FP_P.l[i] >> 1) | (i < 5 ? FP_P.l[i + 1] << 63 : 0);
    return limbs_lt(half.l, canonical->l, 6);
}

/* ZCash compressed G1, k_compress_proofs.comp:25-47 */
static void g1_compress(uint8_t *out, const g1a_t *p) {
    if (g1a_is_identity(p)) {
        memset(out, 0, 48);
        out[0] = 0xc0;
        return;
    }
    fp_t x, y;
    fp_to_canonical(&x, &p->x);
    fp_to_canonical(&y, &p->y);
    limbs_to_be48(out, x.l);
    out[0] |= 0x80;
    if (fp_is_lex_largest(&y)) out[0] |= 0x20;
}

/* Inverse of g1_compress; returns 0 on success.  Checks on-curve, not subgroup. */
static int g1_decompress(g1a_t *out, const uint8_t *in) {
    uint8_t b[48];
    memcpy(b, in, 48);
    const int cflag = (b[0] >> 7) & 1, iflag = (b[0] >> 6) & 1, sflag = (b[0] >> 5) & 1;
    if (!cflag) return -1;
    b[0] &= 0x1f;
    if (iflag) {
        for (int i = 0; i < 48; i++)
            if (b[i]) return -1;
        if (sflag) return -1;
        memset(out, 0, sizeof *out);
        return 0;
    }
    fp_t x;
    be48_to_limbs(x.l, b);
    if (!limbs_lt(x.l, FP_P.l, 6)) return -1;
    fp_t xm, y2, four = {{4, 0, 0, 0, 0, 0}}, fourm, y;
    fp_from_canonical(&xm, &x);
    fp_from_canonical(&fourm, &four);
    fp_sqr(&y2, &xm);
    fp_mul(&y2, &y2, &xm);
    fp_add(&y2, &y2, &fourm);
    if (!fp_sqrt(&y, &y2)) return -1;
    fp_t yc;
    fp_to_canonical(&yc, &y);
    if (fp_is_lex_largest(&yc) != sflag) fp_neg(&y, &y);
    out->x = xm;
    out->y = y;
    return 0;
}

/* ======================================================================
 * Roots of unity and Fr NTT.  The reference's roots tables hold
 * w_8192^i and w_8192^-i with w_8192 = 7^((r-1)/8192)
 * (src/precomputed_tables.cpp:43-44; generator 7 from tools/gen_constants.py:56-61).
 * ====================================================================== */
static fr_t g_roots_fwd[8192], g_roots_inv[8192];
static pthread_once_t g_roots_once = PTHREAD_ONCE_INIT;

static void roots_init(void) {
    fr_t seven, w, wi;
    fr_from_u64(&seven, 7);
    /* (r-1)/8192 */
    uint64_t e[4];
    memcpy(e, FR_P.l, sizeof e);
    e[0] -= 1;
    for (int i = 0; i < 4; i++) e[i] = (e[i] >> 13) | (i < 3 ? e[i + 1] << 51 : 0);
    fr_pow(&w, &seven, e, 4);
    fr_inv(&wi, &w);
    g_roots_fwd[0] = FR_ONE;
    g_roots_inv[0] = FR_ONE;
    for (int i = 1; i < 8192; i++) {
        fr_mul(&g_roots_fwd[i], &g_roots_fwd[i - 1], &w);
        fr_mul(&g_roots_inv[i], &g_roots_inv[i - 1], &wi);
    }
}
static void roots_ready(void) { pthread_once(&g_roots_once, roots_init); }

/* In-place radix-2 NTT of size n (power of two <= 8192):
 * out[k] = sum_t in[t] * w_n^(+-kt), unscaled (k_ntt_pass.comp:38-90 computes
 * the same transform in four-step form). */
static void fr_ntt(fr_t *a, int n, int inverse) {
    roots_ready();
    const fr_t *roots = inverse ? g_roots_inv : g_roots_fwd;
    int logn = 0;
    while ((1 << logn) < n) logn++;
    for (int i = 0; i < n; i++) {
        int j = (int)brev((uint32_t)i, logn);
        if (j > i) {
            fr_t t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int h = len >> 1, stride = 8192 / len;
        for (int b = 0; b < n; b += len) {
            for (int j = 0; j < h; j++) {
                fr_t c;
                fr_mul(&c, &a[b + j + h], &roots[j * stride]);
                fr_t s, d;
                fr_add(&s, &a[b + j], &c);
                fr_sub(&d, &a[b + j], &c);
                a[b + j] = s;
                a[b + j + h] = d;
            }
        }
    }
}

/* G1 NTT of size n (points in Jacobian), same shape as fr_ntt. */
static void g1_ntt(g1j_t *a, int n, int inverse) {
    roots_ready();
    const fr_t *roots = inverse ? g_roots_inv : g_roots_fwd;
    int logn = 0;
    while ((1 << logn) < n) logn++;
    for (int i = 0; i < n; i++) {
        int j = (int)brev((uint32_t)i, logn);
        if (j > i) {
            g1j_t t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int h = len >> 1, stride = 8192 / len;
        for (int b = 0; b < n; b += len) {
            for (int j = 0; j < h; j++) {
                g1j_t c;
                if (j == 0) {
                    c = a[b + j + h];
                } else {
                    fr_t k;
                    fr_to_canonical(&k, &roots[j * stride]);
                    g1_mul(&c, &a[b + j + h], &k);
                }
                g1j_t s, d;
                g1_add(&s, &a[b + j], &c);
                g1_sub(&d, &a[b + j], &c);
                a[b + j] = s;
                a[b + j + h] = d;
            }
        }
    }
}

/* ======================================================================
 * Tables (src/precomputed_tables.cpp:16-58, format v1) and their derivation
 * from the monomial setup.
 * ====================================================================== */
#define N_BLOB 4096
#define N_EXT 8192
#define N_CIRC 128
#define N_HALF 64
#define N_TERMS 64
#define N_DIGITS 32
#define N_BUCKETS 128
#define POS_POINTS (N_CIRC * N_TERMS * N_DIGITS) /* 262144 */

struct orc_tables {
    g1a_t *pos;            /* [j][i][d], POS_POINTS affine Montgomery */
    uint32_t *items[2];    /* tap items, plus / minus */
    uint32_t n_items[2];
    uint32_t offsets[2][N_BUCKETS + 1];
    uint32_t perm[2][N_BUCKETS];
    fr_t inv_blob;
};

/* Signed base-256 digits of a canonical scalar, k_phase_a_sort.comp:31-40:
 * digit = byte + carry; above 128 it borrows from the next digit. */
static void recode(int *digits, const fr_t *canonical) {
    int carry = 0;
    for (int dd = 0; dd < N_DIGITS; dd++) {
        int byte = (int)((canonical->l[dd >> 3] >> ((dd & 7) * 8)) & 0xff);
        int v = byte + carry;
        carry = 0;
        if (v > N_BUCKETS) {
            v -= 2 * N_BUCKETS;
            carry = 1;
        }
        digits[dd] = v;
    }
}

/* Phase-B half taps c+-[e] = (c[e] +- c[e+64]) / 2 with
 * c[e] = (1/128) sum_{t<64} w_128^(e t): the IFFT_128 / truncate-to-64 /
 * FFT_128 composition as a circulant (src/layout_defs.h:23-37,
 * k_phase_b_split.comp:43-55, k_combine_split.comp:29-31). */
static void phase_b_taps(fr_t taps[2][N_HALF]) {
    roots_ready();
    fr_t c[N_CIRC];
    fr_t inv128, two, inv2;
    fr_from_u64(&inv128, 128);
    fr_inv(&inv128, &inv128);
    fr_from_u64(&two, 2);
    fr_inv(&inv2, &two);
    for (int e = 0; e < N_CIRC; e++) {
        fr_t acc = {{0}};
        for (int t = 0; t < N_HALF; t++) {
            fr_add(&acc, &acc, &g_roots_fwd[((e * t) % N_CIRC) * (N_EXT / N_CIRC)]);
        }
        fr_mul(&c[e], &acc, &inv128);
    }
    for (int e = 0; e < N_HALF; e++) {
        fr_t s, d;
        fr_add(&s, &c[e], &c[e + N_HALF]);
        fr_sub(&d, &c[e], &c[e + N_HALF]);
        fr_mul(&taps[0][e], &s, &inv2);
        fr_mul(&taps[1][e], &d, &inv2);
    }
}

/* Items e | d<<8 | neg<<16 grouped by bucket |digit|-1, offsets[129], and a
 * bucket order by descending load (k_phase_a_sort.comp:74-101's load classes). */
static int build_tap_items(orc_tables *t) {
    fr_t taps[2][N_HALF];
    phase_b_taps(taps);
    for (int h = 0; h < 2; h++) {
        uint32_t count[N_BUCKETS] = {0};
        int dig[N_HALF][N_DIGITS];
        for (int e = 0; e < N_HALF; e++) {
            fr_t c;
            fr_to_canonical(&c, &taps[h][e]);
            recode(dig[e], &c);
            for (int d = 0; d < N_DIGITS; d++)
                if (dig[e][d]) count[abs(dig[e][d]) - 1]++;
        }
        uint32_t acc = 0;
        for (int k = 0; k < N_BUCKETS; k++) {
            t->offsets[h][k] = acc;
            acc += count[k];
        }
        t->offsets[h][N_BUCKETS] = acc;
        t->n_items[h] = acc;
        t->items[h] = (uint32_t *)malloc(sizeof(uint32_t) * (acc ? acc : 1));
        if (!t->items[h]) return ORC_MALLOC;
        uint32_t cursor[N_BUCKETS];
        memcpy(cursor, t->offsets[h], sizeof cursor);
        for (int e = 0; e < N_HALF; e++) {
            for (int d = 0; d < N_DIGITS; d++) {
                int v = dig[e][d];
                if (!v) continue;
                uint32_t k = (uint32_t)abs(v) - 1;
                t->items[h][cursor[k]++] = (uint32_t)e | ((uint32_t)d << 8) | ((v < 0 ? 1u : 0u) << 16);
            }
        }
        /* descending load, stable (scheduling only; results do not depend on it) */
        uint32_t hist[64] = {0}, pos = 0;
        for (int k = 0; k < N_BUCKETS; k++) {
            uint32_t cls = count[k] < 63 ? count[k] : 63;
            hist[cls]++;
        }
        uint32_t startc[64];
        for (int c = 63; c >= 0; c--) {
            startc[c] = pos;
            pos += hist[c];
        }
        for (int k = 0; k < N_BUCKETS; k++) {
            uint32_t cls = count[k] < 63 ? count[k] : 63;
            t->perm[h][startc[cls]++] = (uint32_t)k;
        }
    }
    return ORC_OK;
}

typedef struct {
    const g1a_t *monomial;
    g1a_t *pos;
    int col_lo, col_hi;
} gen_job;

/* X[.][i] = FFT_128 over G1 of s_i, s_i[t] = [tau^(4031 - i - 64 t)] for t < 63,
 * infinity otherwise; T[j][i][d] = 2^(8d) X[j][i].  This is the standard FK20
 * precomputation; index math follows k_phase_a.comp:35,39. */
static void *gen_columns(void *arg) {
    gen_job *job = (gen_job *)arg;
    g1j_t col[N_CIRC];
    g1j_t *lad = (g1j_t *)malloc(sizeof(g1j_t) * N_CIRC * N_DIGITS);
    for (int i = job->col_lo; i < job->col_hi; i++) {
        for (int tt = 0; tt < N_CIRC; tt++) {
            if (tt < N_TERMS - 1) {
                col[tt] = g1_from_affine(&job->monomial[N_BLOB - N_TERMS - 1 - i - N_TERMS * tt]);
            } else {
                col[tt] = g1_identity();
            }
        }
        g1_ntt(col, N_CIRC, 0);
        for (int j = 0; j < N_CIRC; j++) {
            g1j_t acc = col[j];
            for (int d = 0; d < N_DIGITS; d++) {
                lad[j * N_DIGITS + d] = acc;
                for (int s = 0; s < 8; s++) g1_dbl(&acc, &acc);
            }
        }
        g1a_t *aff = (g1a_t *)malloc(sizeof(g1a_t) * N_CIRC * N_DIGITS);
        g1_batch_to_affine(aff, lad, N_CIRC * N_DIGITS);
        for (int j = 0; j < N_CIRC; j++)
            for (int d = 0; d < N_DIGITS; d++)
                job->pos[((size_t)j * N_TERMS + i) * N_DIGITS + d] = aff[j * N_DIGITS + d];
        free(aff);
    }
    free(lad);
    return NULL;
}

static orc_tables *tables_alloc(void) {
    orc_tables *t = (orc_tables *)calloc(1, sizeof(orc_tables));
    if (!t) return NULL;
    t->pos = (g1a_t *)malloc(sizeof(g1a_t) * POS_POINTS);
    if (!t->pos) {
        free(t);
        return NULL;
    }
    fr_from_u64(&t->inv_blob, N_BLOB);
    fr_inv(&t->inv_blob, &t->inv_blob);
    return t;
}

int orc_tables_from_setup(orc_tables **out, const uint8_t *g1_monomial_compressed, int nthreads) {
    if (!out || !g1_monomial_compressed) return ORC_BADARGS;
    roots_ready();
    g1a_t *mono = (g1a_t *)malloc(sizeof(g1a_t) * N_BLOB);
    if (!mono) return ORC_MALLOC;
    for (int k = 0; k < N_BLOB; k++) {
        if (g1_decompress(&mono[k], g1_monomial_compressed + 48 * k) != 0) {
            free(mono);
            return ORC_SETUP;
        }
    }
    orc_tables *t = tables_alloc();
    if (!t) {
        free(mono);
        return ORC_MALLOC;
    }
    if (nthreads < 1) nthreads = 1;
    if (nthreads > N_TERMS) nthreads = N_TERMS;
    pthread_t th[N_TERMS];
    gen_job jobs[N_TERMS];
    for (int w = 0; w < nthreads; w++) {
        jobs[w].monomial = mono;
        jobs[w].pos = t->pos;
        jobs[w].col_lo = N_TERMS * w / nthreads;
        jobs[w].col_hi = N_TERMS * (w + 1) / nthreads;
        pthread_create(&th[w], NULL, gen_columns, &jobs[w]);
    }
    for (int w = 0; w < nthreads; w++) pthread_join(th[w], NULL);
    free(mono);
    int rc = build_tap_items(t);
    if (rc != ORC_OK) {
        orc_tables_free(t);
        return rc;
    }
    *out = t;
    return ORC_OK;
}

void orc_tables_free(orc_tables *t) {
    if (!t) return;
    free(t->pos);
    free(t->items[0]);
    free(t->items[1]);
    free(t);
}

const uint32_t *orc_tables_position(const orc_tables *t) { return t ? (const uint32_t *)t->pos : NULL; }

/* header, position table, roots fwd/inv, items+/-, offsets+/-, perm+/-, inv_blob
 * (src/precomputed_tables.cpp:34-58) */
size_t orc_tables_file_size(const orc_tables *t) {
    return 16 + (size_t)POS_POINTS * 96 + 2 * (size_t)N_EXT * 32 + 4 * ((size_t)t->n_items[0] + t->n_items[1]) +
           2 * 4 * (N_BUCKETS + 1) + 2 * 4 * N_BUCKETS + 32;
}

int orc_tables_serialize(const orc_tables *t, uint8_t *dst, size_t cap) {
    if (!t || !dst || cap < orc_tables_file_size(t)) return ORC_BADARGS;
    roots_ready();
    uint8_t *p = dst;
    uint32_t hdr[4] = {0x475A4B56u, 1u, t->n_items[0], t->n_items[1]};
    memcpy(p, hdr, 16); p += 16;
    memcpy(p, t->pos, (size_t)POS_POINTS * 96); p += (size_t)POS_POINTS * 96;
    memcpy(p, g_roots_fwd, sizeof g_roots_fwd); p += sizeof g_roots_fwd;
    memcpy(p, g_roots_inv, sizeof g_roots_inv); p += sizeof g_roots_inv;
    memcpy(p, t->items[0], 4 * (size_t)t->n_items[0]); p += 4 * (size_t)t->n_items[0];
    memcpy(p, t->items[1], 4 * (size_t)t->n_items[1]); p += 4 * (size_t)t->n_items[1];
    memcpy(p, t->offsets[0], sizeof t->offsets[0]); p += sizeof t->offsets[0];
    memcpy(p, t->offsets[1], sizeof t->offsets[1]); p += sizeof t->offsets[1];
    memcpy(p, t->perm[0], sizeof t->perm[0]); p += sizeof t->perm[0];
    memcpy(p, t->perm[1], sizeof t->perm[1]); p += sizeof t->perm[1];
    memcpy(p, &t->inv_blob, 32); p += 32;
    return ORC_OK;
}

int orc_tables_write(const orc_tables *t, const char *path) {
    if (!t || !path) return ORC_BADARGS;
    size_t n = orc_tables_file_size(t);
    uint8_t *buf = (uint8_t *)malloc(n);
    if (!buf) return ORC_MALLOC;
    orc_tables_serialize(t, buf, n);
    FILE *f = fopen(path, "wb");
    if (!f) {
        free(buf);
        return ORC_IO;
    }
    int ok = fwrite(buf, 1, n, f) == n;
    fclose(f);
    free(buf);
    return ok ? ORC_OK : ORC_IO;
}

static int read_exact(FILE *f, void *p, size_t n) { return fread(p, 1, n, f) == n; }

int orc_tables_load(orc_tables **out, const char *path) {
    if (!out || !path) return ORC_BADARGS;
    FILE *f = fopen(path, "rb");
    if (!f) return ORC_IO;
    uint32_t hdr[4];
    orc_tables *t = NULL;
    int rc = ORC_SETUP;
    if (!read_exact(f, hdr, 16) || hdr[0] != 0x475A4B56u || hdr[1] != 1u) goto done;
    if (hdr[2] > 65536 || hdr[3] > 65536) goto done;
    t = tables_alloc();
    if (!t) { rc = ORC_MALLOC; goto done; }
    t->n_items[0] = hdr[2];
    t->n_items[1] = hdr[3];
    t->items[0] = (uint32_t *)malloc(4 * (size_t)(hdr[2] ? hdr[2] : 1));
    t->items[1] = (uint32_t *)malloc(4 * (size_t)(hdr[3] ? hdr[3] : 1));
    {
        static fr_t skip[N_EXT]; /* roots: recomputed, not trusted from the file */
        if (!read_exact(f, t->pos, (size_t)POS_POINTS * 96) || !read_exact(f, skip, sizeof skip) ||
            !read_exact(f, skip, sizeof skip) || !read_exact(f, t->items[0], 4 * (size_t)hdr[2]) ||
            !read_exact(f, t->items[1], 4 * (size_t)hdr[3]) || !read_exact(f, t->offsets[0], sizeof t->offsets[0]) ||
            !read_exact(f, t->offsets[1], sizeof t->offsets[1]) || !read_exact(f, t->perm[0], sizeof t->perm[0]) ||
            !read_exact(f, t->perm[1], sizeof t->perm[1]) || !read_exact(f, &t->inv_blob, 32)) {
            goto done;
        }
    }
    rc = ORC_OK;
done:
    fclose(f);
    if (rc != ORC_OK) {
        orc_tables_free(t);
        return rc;
    }
    *out = t;
    return ORC_OK;
}

/* ======================================================================
 * FK20 proofs, reference algorithm (src/vkzg.cpp:899-1039).
 * ====================================================================== */

/* blob bytes -> natural-order coefficients f (k_blob_to_fr.comp, k_ntt_pass
 * inverse 4096 with scale 1/4096: src/vkzg.cpp:921-935).  Returns 0 or
 * ORC_INVALID_BLOB. */
static int blob_to_coeffs(fr_t *f, const uint8_t *blob, const fr_t *inv_blob) {
    int bad = 0;
    for (int i = 0; i < N_BLOB; i++) {
        fr_t v;
        be32_to_limbs(v.l, blob + 32 * i);
        if (!fr_is_canonical(&v)) bad = 1;
        fr_from_canonical(&f[brev((uint32_t)i, 12)], &v);
    }
    fr_ntt(f, N_BLOB, 1);
    for (int i = 0; i < N_BLOB; i++) fr_mul(&f[i], &f[i], inv_blob);
    return bad ? ORC_INVALID_BLOB : ORC_OK;
}

/* coeffs[j][i] = FFT_128(c_i)[j] with c_i[0] = f[4095-i],
 * c_i[128-j'] = f[4095-i-64j'] for j' = 1..62 (k_build_circulant.comp:31-41). */
static void circulant_coeffs(fr_t *coeffs /*[128][64]*/, const fr_t *f) {
    fr_t col[N_CIRC];
    for (int i = 0; i < N_TERMS; i++) {
        memset(col, 0, sizeof col);
        col[0] = f[N_BLOB - 1 - i];
        for (int jj = 1; jj <= 62; jj++) col[N_CIRC - jj] = f[N_BLOB - 1 - i - jj * N_TERMS];
        fr_ntt(col, N_CIRC, 0);
        for (int j = 0; j < N_CIRC; j++) coeffs[j * N_TERMS + i] = col[j];
    }
}

/* sum_{k=1}^{128} k * B[k-1] via the running sum (field.glsl.inc:478-517 with one lane). */
static g1j_t reduce_buckets(const g1j_t *b) {
    g1j_t s = g1_identity(), rs = g1_identity();
    for (int k = N_BUCKETS; k-- > 0;) {
        g1_add(&s, &s, &b[k]);
        g1_add(&rs, &rs, &s);
    }
    return rs;
}

/* Phase A for output j: u[j] = sum_i coeffs[j][i] * X[j][i] with the signed-digit
 * bucket method over the position table (k_phase_a_sort.comp, k_phase_a.comp:30-43,
 * k_bucket_reduce.comp). */
static g1j_t phase_a_one(const orc_tables *t, const fr_t *coeffs_j /*[64]*/, int j) {
    g1j_t buckets[N_BUCKETS];
    for (int k = 0; k < N_BUCKETS; k++) buckets[k] = g1_identity();
    for (int i = 0; i < N_TERMS; i++) {
        fr_t c;
        fr_to_canonical(&c, &coeffs_j[i]);
        int dig[N_DIGITS];
        recode(dig, &c);
        for (int d = 0; d < N_DIGITS; d++) {
            int v = dig[d];
            if (!v) continue;
            g1a_t pt = t->pos[((size_t)j * N_TERMS + i) * N_DIGITS + d];
            if (v < 0) fp_neg(&pt.y, &pt.y);
            g1_madd(&buckets[abs(v) - 1], &buckets[abs(v) - 1], &pt);
        }
    }
    return reduce_buckets(buckets);
}

/* Phase B split form for half h (0 = cyclic, 1 = negacyclic), output aa
 * (k_phase_b_split.comp:21-62). lad: affine L-half [64][32]. */
static g1j_t phase_b_one(const orc_tables *t, const g1a_t *lad, int h, int aa) {
    g1j_t buckets[N_BUCKETS];
    for (int k = 0; k < N_BUCKETS; k++) {
        buckets[k] = g1_identity();
        for (uint32_t it = t->offsets[h][k]; it < t->offsets[h][k + 1]; it++) {
            uint32_t packed = t->items[h][it];
            int e = (int)(packed & 0xff), d = (int)((packed >> 8) & 0xff), sign = (int)((packed >> 16) & 1);
            int src = (aa - e) & (N_HALF - 1);
            g1a_t pt = lad[src * N_DIGITS + d];
            if (sign) fp_neg(&pt.y, &pt.y);
            if (h == 1 && e > aa) fp_neg(&pt.y, &pt.y);
            g1_madd(&buckets[k], &buckets[k], &pt);
        }
    }
    return reduce_buckets(buckets);
}

/* u (128 Jacobian) -> proofs in natural order via ladder, fold, normalise,
 * phase B, combine (src/vkzg.cpp:965-1008). */
static void phase_b_all(const orc_tables *t, const g1j_t *u, g1j_t *out) {
    g1j_t *lad = (g1j_t *)malloc(sizeof(g1j_t) * N_CIRC * N_DIGITS);
    g1j_t *fold = (g1j_t *)malloc(sizeof(g1j_t) * N_CIRC * N_DIGITS);
    g1a_t *aff = (g1a_t *)malloc(sizeof(g1a_t) * N_CIRC * N_DIGITS);
    /* k_ladder.comp:21-25 */
    for (int j = 0; j < N_CIRC; j++) {
        g1j_t acc = u[j];
        for (int d = 0; d < N_DIGITS; d++) {
            lad[j * N_DIGITS + d] = acc;
            for (int s = 0; s < 8; s++) g1_dbl(&acc, &acc);
        }
    }
    /* k_fold_ladder.comp:25-36 */
    for (int j = 0; j < N_HALF; j++) {
        for (int d = 0; d < N_DIGITS; d++) {
            g1_add(&fold[j * N_DIGITS + d], &lad[j * N_DIGITS + d], &lad[(j + N_HALF) * N_DIGITS + d]);
            g1_sub(&fold[(j + N_HALF) * N_DIGITS + d], &lad[j * N_DIGITS + d], &lad[(j + N_HALF) * N_DIGITS + d]);
        }
    }
    g1_batch_to_affine(aff, fold, N_CIRC * N_DIGITS);
    for (int aa = 0; aa < N_HALF; aa++) {
        g1j_t cp = phase_b_one(t, aff, 0, aa);
        g1j_t cm = phase_b_one(t, aff + N_HALF * N_DIGITS, 1, aa);
        /* k_combine_split.comp:29-31 */
        g1_add(&out[aa], &cp, &cm);
        g1_sub(&out[aa + N_HALF], &cp, &cm);
    }
    free(lad);
    free(fold);
    free(aff);
}

static void proofs_to_bytes(uint8_t *proofs, const g1j_t *nat) {
    g1a_t aff[N_CIRC];
    g1_batch_to_affine(aff, nat, N_CIRC);
    for (int a = 0; a < N_CIRC; a++) g1_compress(proofs + 48 * brev((uint32_t)a, 7), &aff[a]);
}

static int proofs_one(const orc_tables *t, uint8_t *proofs, const uint8_t *blob, g1j_t *u_out,
                      fr_t *f_out, fr_t *circ_out, g1j_t *nat_out) {
    fr_t *f = (fr_t *)malloc(sizeof(fr_t) * N_BLOB);
    fr_t *coeffs = (fr_t *)malloc(sizeof(fr_t) * N_CIRC * N_TERMS);
    g1j_t u[N_CIRC], nat[N_CIRC];
    int rc = blob_to_coeffs(f, blob, &t->inv_blob);
    if (rc == ORC_OK) {
        circulant_coeffs(coeffs, f);
        for (int j = 0; j < N_CIRC; j++) u[j] = phase_a_one(t, coeffs + j * N_TERMS, j);
        phase_b_all(t, u, nat);
        if (proofs) proofs_to_bytes(proofs, nat);
        if (u_out) memcpy(u_out, u, sizeof u);
        if (nat_out) memcpy(nat_out, nat, sizeof nat);
        if (f_out) memcpy(f_out, f, sizeof(fr_t) * N_BLOB);
        if (circ_out) memcpy(circ_out, coeffs, sizeof(fr_t) * N_CIRC * N_TERMS);
    }
    free(f);
    free(coeffs);
    return rc;
}

typedef struct {
    const orc_tables *t;
    uint8_t *proofs;
    const uint8_t *blobs;
    uint8_t *cells;
    const uint8_t *present;
    size_t lo, hi;
    int rc;
    int kind; /* 0 proofs, 1 recover, 2 cells */
} batch_job;

static int recover_one(uint8_t *out, const uint8_t *cells, const uint8_t *present);
static int cells_one(uint8_t *cells, const uint8_t *blob);

static void *batch_worker(void *arg) {
    batch_job *j = (batch_job *)arg;
    j->rc = ORC_OK;
    for (size_t b = j->lo; b < j->hi; b++) {
        int rc;
        if (j->kind == 0) {
            rc = proofs_one(j->t, j->proofs + b * N_CIRC * 48, j->blobs + b * (size_t)N_BLOB * 32, NULL, NULL,
                            NULL, NULL);
        } else if (j->kind == 1) {
            rc = recover_one(j->cells + b * (size_t)N_EXT * 32, j->blobs + b * (size_t)N_EXT * 32,
                             j->present + b * N_CIRC);
        } else {
            rc = cells_one(j->cells + b * (size_t)N_EXT * 32, j->blobs + b * (size_t)N_BLOB * 32);
        }
        if (rc != ORC_OK && j->rc == ORC_OK) j->rc = rc;
    }
    return NULL;
}

static int run_batch(batch_job proto, size_t n, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if ((size_t)nthreads > n) nthreads = (int)n;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    batch_job jobs[256];
    for (int w = 0; w < nthreads; w++) {
        jobs[w] = proto;
        jobs[w].lo = n * (size_t)w / (size_t)nthreads;
        jobs[w].hi = n * (size_t)(w + 1) / (size_t)nthreads;
        pthread_create(&th[w], NULL, batch_worker, &jobs[w]);
    }
    int rc = ORC_OK;
    for (int w = 0; w < nthreads; w++) {
        pthread_join(th[w], NULL);
        if (jobs[w].rc != ORC_OK && rc == ORC_OK) rc = jobs[w].rc;
    }
    return rc;
}

int orc_compute_proofs(const orc_tables *t, uint8_t *proofs, const uint8_t *blobs, size_t n, int nthreads) {
    if (!t || !proofs || !blobs) return ORC_BADARGS;
    if (n == 0) return ORC_OK;
    roots_ready();
    batch_job proto;
    memset(&proto, 0, sizeof proto);
    proto.t = t;
    proto.proofs = proofs;
    proto.blobs = blobs;
    proto.kind = 0;
    return run_batch(proto, n, nthreads);
}

static void fr_to_be(uint8_t *out, const fr_t *m) {
    fr_t c;
    fr_to_canonical(&c, m);
    limbs_to_be32(out, c.l);
}

static void g1_to_xy(uint8_t *out96, const g1a_t *a) {
    if (g1a_is_identity(a)) {
        memset(out96, 0, 96);
        return;
    }
    fp_t x, y;
    fp_to_canonical(&x, &a->x);
    fp_to_canonical(&y, &a->y);
    limbs_to_be48(out96, x.l);
    limbs_to_be48(out96 + 48, y.l);
}

int orc_proof_stages(const orc_tables *t, const uint8_t *blob, uint8_t *coeffs_f, uint8_t *circ, uint8_t *u,
                     uint8_t *proofs_nat) {
    if (!t || !blob) return ORC_BADARGS;
    roots_ready();
    fr_t *f = (fr_t *)malloc(sizeof(fr_t) * N_BLOB);
    fr_t *cc = (fr_t *)malloc(sizeof(fr_t) * N_CIRC * N_TERMS);
    g1j_t uu[N_CIRC], nat[N_CIRC];
    int rc = proofs_one(t, NULL, blob, uu, f, cc, nat);
    if (rc == ORC_OK) {
        if (coeffs_f)
            for (int i = 0; i < N_BLOB; i++) fr_to_be(coeffs_f + 32 * i, &f[i]);
        if (circ)
            for (int i = 0; i < N_CIRC * N_TERMS; i++) fr_to_be(circ + 32 * i, &cc[i]);
        g1a_t aff[N_CIRC];
        if (u) {
            g1_batch_to_affine(aff, uu, N_CIRC);
            for (int j = 0; j < N_CIRC; j++) g1_to_xy(u + 96 * j, &aff[j]);
        }
        if (proofs_nat) {
            g1_batch_to_affine(aff, nat, N_CIRC);
            for (int j = 0; j < N_CIRC; j++) g1_to_xy(proofs_nat + 96 * j, &aff[j]);
        }
    }
    free(f);
    free(cc);
    return rc;
}

/* Same u[j] as the reference, then h = IFFT_128(u) in G1, h[64..127] = 0,
 * proofs = FFT_128(h): the textbook FK20 tail, independent of the phase-B
 * tap tables. */
int orc_compute_proofs_g1fft(const orc_tables *t, uint8_t *proofs, const uint8_t *blob) {
    if (!t || !proofs || !blob) return ORC_BADARGS;
    roots_ready();
    fr_t *f = (fr_t *)malloc(sizeof(fr_t) * N_BLOB);
    fr_t *coeffs = (fr_t *)malloc(sizeof(fr_t) * N_CIRC * N_TERMS);
    int rc = blob_to_coeffs(f, blob, &t->inv_blob);
    if (rc == ORC_OK) {
        circulant_coeffs(coeffs, f);
        g1j_t h[N_CIRC];
        for (int j = 0; j < N_CIRC; j++) h[j] = phase_a_one(t, coeffs + j * N_TERMS, j);
        g1_ntt(h, N_CIRC, 1);
        fr_t inv128;
        fr_from_u64(&inv128, N_CIRC);
        fr_inv(&inv128, &inv128);
        fr_to_canonical(&inv128, &inv128);
        for (int k = 0; k < N_HALF; k++) g1_mul(&h[k], &h[k], &inv128);
        for (int k = N_HALF; k < N_CIRC; k++) h[k] = g1_identity();
        g1_ntt(h, N_CIRC, 0);
        proofs_to_bytes(proofs, h);
    }
    free(f);
    free(coeffs);
    return rc;
}

static const fp_t G1_GEN_X = {{0xfb3af00adb22c6bbULL, 0x6c55e83ff97a1aefULL, 0xa14e3a3f171bac58ULL,
                               0xc3688c4f9774b905ULL, 0x2695638c4fa9ac0fULL, 0x17f1d3a73197d794ULL}};
static const fp_t G1_GEN_Y = {{0x0caa232946c5e7e1ULL, 0xd03cc744a2888ae4ULL, 0x00db18cb2c04b3edULL,
                               0xfcf5e095d5d00af6ULL, 0xa09e30ed741d8ae4ULL, 0x08b3f481e3aaa0f1ULL}};

static g1j_t g1_generator(void) {
    g1j_t g;
    fp_from_canonical(&g.x, &G1_GEN_X);
    fp_from_canonical(&g.y, &G1_GEN_Y);
    g.z = FP_ONE;
    return g;
}

/* proof for cell brev7(a) = [q(tau)]G1, q = f div (X^64 - w_128^a). */
int orc_compute_proofs_tau(const uint8_t *tau_be, uint8_t *proofs, const uint8_t *blob) {
    if (!tau_be || !proofs || !blob) return ORC_BADARGS;
    roots_ready();
    fr_t *f = (fr_t *)malloc(sizeof(fr_t) * N_BLOB);
    fr_t inv_blob;
    fr_from_u64(&inv_blob, N_BLOB);
    fr_inv(&inv_blob, &inv_blob);
    int rc = blob_to_coeffs(f, blob, &inv_blob);
    if (rc == ORC_OK) {
        fr_t tau;
        be32_to_limbs(tau.l, tau_be);
        fr_from_canonical(&tau, &tau);
        fr_t *q = (fr_t *)malloc(sizeof(fr_t) * N_BLOB);
        g1j_t g = g1_generator(), nat[N_CIRC];
        for (int a = 0; a < N_CIRC; a++) {
            const fr_t *x = &g_roots_fwd[a * (N_EXT / N_CIRC)];
            memset(q, 0, sizeof(fr_t) * N_BLOB);
            for (int k = N_BLOB - 1; k >= N_TERMS; k--) {
                fr_t tq;
                fr_mul(&tq, x, &q[k]);
                fr_add(&q[k - N_TERMS], &f[k], &tq);
            }
            /* Horner at tau over q[0..4031] */
            fr_t acc = {{0}};
            for (int k = N_BLOB - N_TERMS - 1; k >= 0; k--) {
                fr_mul(&acc, &acc, &tau);
                fr_add(&acc, &acc, &q[k]);
            }
            fr_t kc;
            fr_to_canonical(&kc, &acc);
            g1_mul(&nat[a], &g, &kc);
        }
        proofs_to_bytes(proofs, nat);
        free(q);
    }
    free(f);
    return rc;
}

/* ======================================================================
 * Cells (2x RS extension): FFT_8192 of the zero-padded coefficients, written
 * in bit-reversed order (the same convention k_fr_to_cells.comp uses).
 * ====================================================================== */
static int cells_one(uint8_t *cells, const uint8_t *blob) {
    fr_t *f = (fr_t *)calloc(N_EXT, sizeof(fr_t));
    fr_t inv_blob;
    fr_from_u64(&inv_blob, N_BLOB);
    fr_inv(&inv_blob, &inv_blob);
    int rc = blob_to_coeffs(f, blob, &inv_blob);
    if (rc == ORC_OK) {
        fr_ntt(f, N_EXT, 0);
        for (int i = 0; i < N_EXT; i++) fr_to_be(cells + 32 * (size_t)brev((uint32_t)i, 13), &f[i]);
    }
    free(f);
    return rc;
}

int orc_compute_cells(uint8_t *cells, const uint8_t *blobs, size_t n, int nthreads) {
    if (!cells || !blobs) return ORC_BADARGS;
    if (n == 0) return ORC_OK;
    roots_ready();
    batch_job proto;
    memset(&proto, 0, sizeof proto);
    proto.cells = cells;
    proto.blobs = blobs;
    proto.kind = 2;
    return run_batch(proto, n, nthreads);
}

/* ======================================================================
 * Recovery, reference order (src/vkzg.cpp:1086-1164).
 * ====================================================================== */
static int recover_one(uint8_t *out, const uint8_t *cells, const uint8_t *present) {
    /* host-side missing list, src/vkzg.cpp:1093-1105 with brevCell at :1046-1050 */
    uint32_t missing[N_CIRC];
    uint32_t count = 0;
    for (uint32_t i = 0; i < N_CIRC; i++) {
        if (!present[i]) {
            if (count >= N_TERMS) return ORC_BADARGS;
            missing[count++] = brev(i, 7);
        }
    }
    fr_t *E = (fr_t *)malloc(sizeof(fr_t) * N_EXT);
    fr_t *Z = (fr_t *)calloc(N_EXT, sizeof(fr_t));
    fr_t *A = (fr_t *)malloc(sizeof(fr_t) * N_EXT);
    fr_t *B = (fr_t *)malloc(sizeof(fr_t) * N_EXT);
    fr_t *Zc = (fr_t *)malloc(sizeof(fr_t) * N_EXT);
    /* 1. cells -> Fr, brev13 (k_cells_to_fr.comp:25-35), no canonicity check */
    for (int i = 0; i < N_EXT; i++) {
        fr_t v;
        be32_to_limbs(v.l, cells + 32 * (size_t)i);
        fr_from_canonical(&E[brev((uint32_t)i, 13)], &v);
    }
    /* 2. Z_short by long multiplication of (x - w_8192^(64 m)) (k_vanishing_poly.comp:59-90) */
    if (count == 0) {
        Z[0] = FR_ONE;
    } else {
        fr_t sp[N_TERMS + 1];
        fr_neg(&sp[0], &g_roots_fwd[missing[0] * 64]);
        for (uint32_t i = 1; i < count; i++) {
            fr_t nr;
            fr_neg(&nr, &g_roots_fwd[missing[i] * 64]);
            fr_add(&sp[i], &nr, &sp[i - 1]);
            for (uint32_t j = i - 1; j > 0; j--) {
                fr_t pj;
                fr_mul(&pj, &sp[j], &nr);
                fr_add(&sp[j], &pj, &sp[j - 1]);
            }
            fr_mul(&sp[0], &sp[0], &nr);
        }
        sp[count] = FR_ONE;
        for (uint32_t i = 0; i <= count; i++) Z[i * N_TERMS] = sp[i];
    }
    memcpy(Zc, Z, sizeof(fr_t) * N_EXT);
    /* 3-4. Z -> eval; E*Z */
    fr_ntt(Z, N_EXT, 0);
    for (int i = 0; i < N_EXT; i++) fr_mul(&A[i], &E[i], &Z[i]);
    /* 5. -> coefficients, 1/8192 */
    fr_t inv_ext, seven, inv_seven;
    fr_from_u64(&inv_ext, N_EXT);
    fr_inv(&inv_ext, &inv_ext);
    fr_from_u64(&seven, 7);
    fr_inv(&inv_seven, &seven);
    fr_ntt(A, N_EXT, 1);
    for (int i = 0; i < N_EXT; i++) fr_mul(&A[i], &A[i], &inv_ext);
    /* 6. coset evaluations with shift 7 */
    fr_t sh = FR_ONE;
    for (int i = 0; i < N_EXT; i++) {
        fr_mul(&A[i], &A[i], &sh);
        fr_mul(&B[i], &Zc[i], &sh);
        fr_mul(&sh, &sh, &seven);
    }
    fr_ntt(A, N_EXT, 0);
    fr_ntt(B, N_EXT, 0);
    /* 7. division, per-element Fermat as in k_ew_div.comp:28 */
    for (int i = 0; i < N_EXT; i++) {
        fr_t bi;
        fr_inv(&bi, &B[i]);
        fr_mul(&A[i], &A[i], &bi);
    }
    /* 8. coset IFFT: unscaled inverse, 1/8192, times 7^-i */
    fr_ntt(A, N_EXT, 1);
    sh = FR_ONE;
    for (int i = 0; i < N_EXT; i++) {
        fr_mul(&A[i], &A[i], &inv_ext);
        fr_mul(&A[i], &A[i], &sh);
        fr_mul(&sh, &sh, &inv_seven);
    }
    /* 9-10. evaluate on the extended domain; bytes at brev13 (k_fr_to_cells.comp:27-35) */
    fr_ntt(A, N_EXT, 0);
    for (int i = 0; i < N_EXT; i++) fr_to_be(out + 32 * (size_t)brev((uint32_t)i, 13), &A[i]);
    free(E);
    free(Z);
    free(A);
    free(B);
    free(Zc);
    return ORC_OK;
}

int orc_recover_cells(uint8_t *cells_out, const uint8_t *cells, const uint8_t *present, size_t n, int nthreads) {
    if (!cells_out || !cells || !present) return ORC_BADARGS;
    if (n == 0) return ORC_OK;
    roots_ready();
    /* argument errors are reported before any work, like the reference's host loop */
    for (size_t b = 0; b < n; b++) {
        int miss = 0;
        for (int i = 0; i < N_CIRC; i++) miss += !present[b * N_CIRC + i];
        if (miss > N_TERMS) return ORC_BADARGS;
    }
    batch_job proto;
    memset(&proto, 0, sizeof proto);
    proto.cells = cells_out;
    proto.blobs = cells;
    proto.present = present;
    proto.kind = 1;
    return run_batch(proto, n, nthreads);
}

/* ======================================================================
 * Synthetic setup from a seed (SplitMix64 -> tau mod r).
 * ====================================================================== */
static uint64_t splitmix64(uint64_t *s) {
    uint64_t z = (*s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

int orc_synthetic_setup(uint64_t seed, uint8_t *tau_be, uint8_t *g1_monomial, uint8_t *g1_lagrange) {
    roots_ready();
    uint64_t s = seed;
    fr_t tau;
    do {
        for (int i = 0; i < 4; i++) tau.l[i] = splitmix64(&s);
        tau.l[3] &= 0x7fffffffffffffffULL;
    } while (!fr_is_canonical(&tau) || fr_is_zero(&tau));
    if (tau_be) limbs_to_be32(tau_be, tau.l);
    fr_t taum;
    fr_from_canonical(&taum, &tau);
    g1j_t g = g1_generator();
    g1j_t *pts = (g1j_t *)malloc(sizeof(g1j_t) * N_BLOB);
    g1a_t *aff = (g1a_t *)malloc(sizeof(g1a_t) * N_BLOB);
    if (g1_monomial) {
        fr_t pw = FR_ONE;
        for (int i = 0; i < N_BLOB; i++) {
            fr_t kc;
            fr_to_canonical(&kc, &pw);
            g1_mul(&pts[i], &g, &kc);
            fr_mul(&pw, &pw, &taum);
        }
        g1_batch_to_affine(aff, pts, N_BLOB);
        for (int i = 0; i < N_BLOB; i++) g1_compress(g1_monomial + 48 * i, &aff[i]);
    }
    if (g1_lagrange) {
        /* L_i(tau) = w^i (tau^n - 1) / (n (tau - w^i)), w = w_4096; stored bit-reversed */
        fr_t tn = taum, nfr, num;
        for (int k = 0; k < 12; k++) fr_mul(&tn, &tn, &tn);
        fr_sub(&num, &tn, &FR_ONE);
        fr_from_u64(&nfr, N_BLOB);
        for (int i = 0; i < N_BLOB; i++) {
            const fr_t *wi = &g_roots_fwd[i * 2];
            fr_t den, li, kc;
            fr_sub(&den, &taum, wi);
            fr_mul(&den, &den, &nfr);
            fr_inv(&den, &den);
            fr_mul(&li, &num, wi);
            fr_mul(&li, &li, &den);
            fr_to_canonical(&kc, &li);
            g1_mul(&pts[brev((uint32_t)i, 12)], &g, &kc);
        }
        g1_batch_to_affine(aff, pts, N_BLOB);
        for (int i = 0; i < N_BLOB; i++) g1_compress(g1_lagrange + 48 * i, &aff[i]);
    }
    free(pts);
    free(aff);
    return ORC_OK;
}

/* ======================================================================
 * Primitive exports.
 * ====================================================================== */
int orc_fp_mul_be(const uint8_t *a48, const uint8_t *b48, uint8_t *out48) {
    fp_t a, b, r;
    be48_to_limbs(a.l, a48);
    be48_to_limbs(b.l, b48);
    if (!limbs_lt(a.l, FP_P.l, 6) || !limbs_lt(b.l, FP_P.l, 6)) return ORC_BADARGS;
    fp_from_canonical(&a, &a);
    fp_from_canonical(&b, &b);
    fp_mul(&r, &a, &b);
    fp_to_canonical(&r, &r);
    limbs_to_be48(out48, r.l);
    return ORC_OK;
}

int orc_fr_mul_be(const uint8_t *a32, const uint8_t *b32, uint8_t *out32) {
    fr_t a, b, r;
    be32_to_limbs(a.l, a32);
    be32_to_limbs(b.l, b32);
    if (!fr_is_canonical(&a) || !fr_is_canonical(&b)) return ORC_BADARGS;
    fr_from_canonical(&a, &a);
    fr_from_canonical(&b, &b);
    fr_mul(&r, &a, &b);
    fr_to_canonical(&r, &r);
    limbs_to_be32(out32, r.l);
    return ORC_OK;
}

int orc_fr_inv_be(const uint8_t *a32, uint8_t *out32) {
    fr_t a, r;
    be32_to_limbs(a.l, a32);
    if (!fr_is_canonical(&a)) return ORC_BADARGS;
    fr_from_canonical(&a, &a);
    fr_inv(&r, &a);
    fr_to_canonical(&r, &r);
    limbs_to_be32(out32, r.l);
    return ORC_OK;
}

void orc_fp_to_mont(const uint8_t *a48, uint32_t *mont12) {
    fp_t a;
    be48_to_limbs(a.l, a48);
    fp_from_canonical(&a, &a);
    memcpy(mont12, a.l, 48);
}

void orc_fp_from_mont(const uint32_t *mont12, uint8_t *a48) {
    fp_t a;
    memcpy(a.l, mont12, 48);
    fp_to_canonical(&a, &a);
    limbs_to_be48(a48, a.l);
}

void orc_fr_to_mont(const uint8_t *a32, uint32_t *mont8) {
    fr_t a;
    be32_to_limbs(a.l, a32);
    fr_from_canonical(&a, &a);
    memcpy(mont8, a.l, 32);
}

void orc_fr_from_mont(const uint32_t *mont8, uint8_t *a32) {
    fr_t a;
    memcpy(a.l, mont8, 32);
    fr_to_canonical(&a, &a);
    limbs_to_be32(a32, a.l);
}

int orc_g1_decompress(const uint8_t *in48, uint8_t *xy96) {
    g1a_t a;
    if (g1_decompress(&a, in48) != 0) return ORC_BADARGS;
    g1_to_xy(xy96, &a);
    return ORC_OK;
}

int orc_g1_compress(const uint8_t *xy96, uint8_t *out48) {
    g1a_t a;
    fp_t x, y;
    be48_to_limbs(x.l, xy96);
    be48_to_limbs(y.l, xy96 + 48);
    if (limbs_is_zero(x.l, 6) && limbs_is_zero(y.l, 6)) {
        memset(&a, 0, sizeof a);
    } else {
        fp_from_canonical(&a.x, &x);
        fp_from_canonical(&a.y, &y);
    }
    g1_compress(out48, &a);
    return ORC_OK;
}

int orc_g1_mul(const uint8_t *p48, const uint8_t *k32, uint8_t *out48) {
    g1a_t a;
    if (g1_decompress(&a, p48) != 0) return ORC_BADARGS;
    fr_t k;
    be32_to_limbs(k.l, k32);
    g1j_t pj = g1_from_affine(&a), r;
    g1_mul(&r, &pj, &k);
    g1a_t o = g1_to_affine(&r);
    g1_compress(out48, &o);
    return ORC_OK;
}

int orc_g1_add(const uint8_t *p48, const uint8_t *q48, uint8_t *out48) {
    g1a_t a, b;
    if (g1_decompress(&a, p48) != 0 || g1_decompress(&b, q48) != 0) return ORC_BADARGS;
    g1j_t aj = g1_from_affine(&a), r;
    g1_madd(&r, &aj, &b);
    g1a_t o = g1_to_affine(&r);
    g1_compress(out48, &o);
    return ORC_OK;
}
