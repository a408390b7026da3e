// Host build of the device arithmetic headers (the PTX carry chains run on the
// host through their emulated carry flag), exposed to tests/test_host_arith.py.
#include "../vkzg_b200/csrc/curve.cuh"

#include <string.h>

using namespace vkzg;

extern "C" {
void shim_fp_mul(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    Fp x, y;
    memcpy(x.v, a, 48);
    memcpy(y.v, b, 48);
    memcpy(r, fp_mul(x, y).v, 48);
}
void shim_fp_mul_ks(const uint32_t *a, const uint32_t *b, uint32_t *r) { mont_mul_ks<12>(r, a, b); }
void shim_fr_mul_ks(const uint32_t *a, const uint32_t *b, uint32_t *r) { mont_mul_ks<8>(r, a, b); }
void shim_fp_mul_ks2(const uint32_t *a, const uint32_t *b, uint32_t *r) { mont_mul_ks<12, 2>(r, a, b); }
void shim_fr_mul_ks2(const uint32_t *a, const uint32_t *b, uint32_t *r) { mont_mul_ks<8, 2>(r, a, b); }
void shim_fp_sqr_ks(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    (void)b;
    mont_sqr_ks<12>(r, a);
}
void shim_fr_sqr_ks(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    (void)b;
    mont_sqr_ks<8>(r, a);
}
void shim_fp_sqr(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    (void)b;
    Fp x;
    memcpy(x.v, a, 48);
    memcpy(r, fp_sqr(x).v, 48);
}
void shim_fr_sqr(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    (void)b;
    mont_sqr<8>(r, a);
}
void shim_fp_add(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    Fp x, y;
    memcpy(x.v, a, 48);
    memcpy(y.v, b, 48);
    memcpy(r, fp_add(x, y).v, 48);
}
void shim_fp_sub(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    Fp x, y;
    memcpy(x.v, a, 48);
    memcpy(y.v, b, 48);
    memcpy(r, fp_sub(x, y).v, 48);
}
void shim_fr_mul(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    Fr x, y;
    memcpy(x.v, a, 32);
    memcpy(y.v, b, 32);
    memcpy(r, fr_mul(x, y).v, 32);
}
void shim_fr_add(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    Fr x, y;
    memcpy(x.v, a, 32);
    memcpy(y.v, b, 32);
    memcpy(r, fr_add(x, y).v, 32);
}
void shim_fr_sub(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    Fr x, y;
    memcpy(x.v, a, 32);
    memcpy(y.v, b, 32);
    memcpy(r, fr_sub(x, y).v, 32);
}
void shim_fr_from_raw(const uint32_t *a, uint32_t *r) {
    Fr x;
    memcpy(x.v, a, 32);
    memcpy(r, fr_from_canonical(x).v, 32);
}
void shim_fp_inv(const uint32_t *a, uint32_t *r) {
    Fp x;
    memcpy(x.v, a, 48);
    memcpy(r, fp_inv(x).v, 48);
}
void shim_fr_inv(const uint32_t *a, uint32_t *r) {
    Fr x;
    memcpy(x.v, a, 32);
    memcpy(r, fr_inv(x).v, 32);
}
// compressed in -> (2 P + Q) compressed out, through dbl / add / madd
int shim_g1_ops(const uint8_t *p48, const uint8_t *q48, uint8_t *out_dbl_add, uint8_t *out_madd) {
    G1A p, q;
    if (!g1_decompress(p, p48) || !g1_decompress(q, q48)) return -1;
    const G1J pj = g1_from_affine(p);
    const G1J r1 = g1_add(g1_dbl(pj), g1_from_affine(q));
    const G1J r2 = g1_madd(g1_add(pj, pj), q);
    const G1J rs[2] = {r1, r2};
    uint8_t *outs[2] = {out_dbl_add, out_madd};
    for (int k = 0; k < 2; k++) {
        G1A a;
        if (fp_is_zero(rs[k].z)) {
            a.x = fp_zero();
            a.y = fp_zero();
        } else {
            const Fp zi = fp_inv(rs[k].z), z2 = fp_sqr(zi);
            a.x = fp_mul(rs[k].x, z2);
            a.y = fp_mul(rs[k].y, fp_mul(z2, zi));
        }
        g1_compress(outs[k], a);
    }
    return 0;
}
// k * P (canonical scalar as 8 LE words)
int shim_g1_mul(const uint8_t *p48, const uint32_t *k, uint8_t *out48) {
    G1A p;
    if (!g1_decompress(p, p48)) return -1;
    Fr s;
    memcpy(s.v, k, 32);
    const G1J r = g1_mul_scalar(g1_from_affine(p), s);
    G1A a;
    if (fp_is_zero(r.z)) {
        a.x = fp_zero();
        a.y = fp_zero();
    } else {
        const Fp zi = fp_inv(r.z), z2 = fp_sqr(zi);
        a.x = fp_mul(r.x, z2);
        a.y = fp_mul(r.y, fp_mul(z2, zi));
    }
    g1_compress(out48, a);
    return 0;
}
}

#include "../vkzg_b200/csrc/comb_windows.h"
#include "../vkzg_b200/csrc/glv.h"
#include "../vkzg_b200/csrc/inverse.cuh"
extern "C" {
// compressed P -> compressed phi(P)
int shim_g1_phi(const uint8_t *p48, uint8_t *out48) {
    G1A p;
    if (!g1_decompress(p, p48)) return -1;
    g1_compress(out48, g1_phi(p));
    return 0;
}
// k (8 LE words, < r) -> the two halves as 4 LE words each, signs, and their
// 16 signed digits each; returns 0 when the digits hold both halves
int shim_glv_split(const uint32_t *k, uint32_t *mag8, int *neg2, int *dig32) {
    const GlvSplit s = glv_split(k);
    for (int h = 0; h < 2; h++) {
        for (int i = 0; i < 4; i++) mag8[4 * h + i] = (uint32_t)(s.mag[h] >> (32 * i));
        neg2[h] = s.neg[h];
        if (!glv_digits(s.mag[h], s.neg[h], dig32 + kGlvDigits * h)) return -1;
    }
    return 0;
}
void shim_fp_inv_fast(const uint32_t *a, uint32_t *r) {
    Fp x;
    memcpy(x.v, a, 48);
    memcpy(r, fp_inv_fast(x).v, 48);
}
void shim_fp_inv_var(const uint32_t *a, uint32_t *r) {
    Fp x;
    memcpy(x.v, a, 48);
    memcpy(r, fp_inv_fast<true>(x).v, 48);
}
// the digit table's layout for d windows: each window's width, bit and first
// entry within a base column, and the column's entry count
void shim_comb_windows(int d, int *width, int *bit, uint32_t *entry, uint32_t *entries) {
    const CombWindows w = comb_windows(d);
    for (int k = 0; k < d; k++) {
        width[k] = w.width(k);
        bit[k] = w.bit_off(k);
        entry[k] = w.entry_off(k);
    }
    *entries = w.entries();
}
// divsteps30 against its table-driven grouped form (seven groups of 4 and one
// of 2): 0 when delta and the matrix agree
int shim_divsteps_grouped_differs(int32_t delta, uint32_t f, uint32_t g) {
    static const DivstepTable<4> t4 = make_divstep_table<4>();
    static const DivstepTable<2> t2 = make_divstep_table<2>();
    int32_t d1 = delta, d2 = delta, a[4], b[4];
    divsteps30(d1, f, g, a[0], a[1], a[2], a[3]);
    divsteps30_grouped(t4.e, t2.e, d2, f, g, b[0], b[1], b[2], b[3]);
    return d1 != d2 || memcmp(a, b, sizeof a) != 0;
}
void shim_fr_inv_fast(const uint32_t *a, uint32_t *r) {
    Fr x;
    memcpy(x.v, a, 32);
    memcpy(r, fr_inv_fast(x).v, 32);
}
}

extern "C" {
// Fp products on the FP64 pipe (field_f64.cuh), host build with std::fma
void shim_fp_mul_f64(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    Fp x, y;
    memcpy(x.v, a, 48);
    memcpy(y.v, b, 48);
    memcpy(r, f64::mont_mul(x, y).v, 48);
}
void shim_fp_sqr_f64(const uint32_t *a, const uint32_t *b, uint32_t *r) {
    (void)b;
    Fp x;
    memcpy(x.v, a, 48);
    memcpy(r, f64::mont_sqr(x).v, 48);
}
}
