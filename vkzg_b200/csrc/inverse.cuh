// Modular inversion by batched divsteps (Bernstein & Yang, "Fast constant-time
// gcd computation and modular inversion", 2019), variable-time form.
//
// Fermat inversion (a^(m-2), what the reference uses: field.glsl.inc:257-275,
// 528-547) is ~570 dependent Fp multiplies; on one GPU thread that is close to a
// millisecond of latency, paid at the root of every batch inversion.  Divsteps
// instead work on 30-bit digits: 30 divsteps on the low words of (f, g) give a
// 2x2 integer matrix with entries below 2^30 in magnitude, which is then applied
// to the full-width (f, g) and to the cofactors (d, e) (the latter modulo m,
// divided by 2^30 with a Montgomery-style correction).  Invariants:
//   f == d * x (mod m),  g == e * x (mod m),  f odd,  d, e in (-2m, m).
// Starting from f = m, g = x, d = 0, e = 1, when g reaches 0, f = +-1 and
// x^-1 = +-d.  Numbers are signed radix-2^30 limbs: limbs 0..L-2 in [0, 2^30),
// the top limb signed.
#pragma once

#include "field.cuh"

namespace vkzg {

// m in radix 2^30 and m^-1 mod 2^30, for Fp (13 limbs) and Fr (9 limbs).
VK_HD constexpr int32_t fp_m30(int i) {
    return i == 0 ? 1073719979 : i == 1 ? 670826495 : i == 2 ? 356515835 : i == 3 ? 721420204
         : i == 4 ? 821437470 : i == 5 ? 55215066 : i == 6 ? 288093811 : i == 7 ? 316751073
         : i == 8 ? 752313463 : i == 9 ? 517541166 : i == 10 ? 698659258 : i == 11 ? 982409209 : 1704209;
}
VK_HD constexpr int32_t fr_m30(int i) {
    return i == 0 ? 1 : i == 1 ? 1073741820 : i == 2 ? 1072021487 : i == 3 ? 795410623
         : i == 4 ? 567805267 : i == 5 ? 660611110 : i == 6 ? 399803187 : i == 7 ? 701811303 : 29677;
}
template <int N>
VK_HD constexpr int32_t mod_m30(int i) {
    return N == 12 ? fp_m30(i) : fr_m30(i);
}
template <int N>
VK_HD constexpr uint32_t mod_minv30() {
    return N == 12 ? 196611u : 1u;
}

constexpr uint32_t kMask30 = (1u << 30) - 1;

// 30 divsteps on the low words.  delta as in the paper (starts at 1).  Returns
// the transition matrix scaled by 2^30: 2^30 [f', g'] = [[u, v], [q, r]] [f, g].
// A divstep is: with g odd and delta > 0, (delta, f, g) <- (1 - delta, g,
// (g - f) / 2); otherwise (1 + delta, f, (g + (g mod 2) f) / 2).  The candidate
// values of g (and of the cofactor rows) are formed from the old values in
// parallel and then selected, which keeps the step's dependency chain through
// g short: 31.8 against 41.1 us per launch of 2368 inversions (one per lane,
// averaged over 50 back-to-back launches) with the masked-arithmetic form of
// the same step.
VK_HD void divsteps30(int32_t &delta, uint32_t f, uint32_t g, int32_t &u_out, int32_t &v_out, int32_t &q_out,
                      int32_t &r_out) {
    uint32_t u = 1, v = 0, q = 0, r = 1;
#pragma unroll
    for (int i = 0; i < 30; i++) {
        const bool odd = g & 1u;
        const bool swap = odd && delta > 0;
        const uint32_t g2 = swap ? g - f : (odd ? g + f : g);  // only the low bits matter
        const uint32_t f2 = swap ? g : f;
        // cofactors: a swap gives (u, v, q, r) <- (2q, 2r, q - u, r - v); an odd g
        // without one q += u, r += v; then u and v double
        const uint32_t q2 = swap ? q - u : (odd ? q + u : q);
        const uint32_t r2 = swap ? r - v : (odd ? r + v : r);
        const uint32_t u2 = swap ? q : u, v2 = swap ? r : v;
        delta = swap ? 1 - delta : 1 + delta;
        f = f2;
        g = g2 >> 1;
        u = u2 << 1;
        v = v2 << 1;
        q = q2;
        r = r2;
    }
    u_out = (int32_t)u;
    v_out = (int32_t)v;
    q_out = (int32_t)q;
    r_out = (int32_t)r;
}

VK_HD int ctz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __ffs((int)x) - 1;
#else
    return __builtin_ctz(x);
#endif
}

// f^-1 mod 2^32 for odd f: 5 correct bits from (3f) ^ 2, then three Newton
// steps x <- x (2 - f x), each doubling them.
VK_HD uint32_t inv_mod_2_32(uint32_t f) {
    uint32_t x = (3u * f) ^ 2u;
    x *= 2u - f * x;
    x *= 2u - f * x;
    x *= 2u - f * x;
    return x;
}

// The transition matrix of divsteps30, in variable time (the multi-step form
// of Bernstein & Yang's divsteps used by libsecp256k1's modinv32 "var"
// routines, restated): a run of z even values of g is z divsteps at once
// (g >>= z, u, v <<= z, delta += z); with g odd and delta <= 0 the next
// k = min(1 - delta, steps left) divsteps never swap, and together they add
// w f to g with w = -g f^-1 mod 2^k, leaving k zero bits for the next run; with
// g odd and delta > 0 the divstep swaps: (f, g) <- (g, -f), delta <- -delta,
// after which the same cancellation applies.  Only f's low bits matter, so
// its inverse mod 2^32 is recomputed at a swap.
VK_HD void divsteps30_var(int32_t &delta, uint32_t f, uint32_t g, int32_t &u_out, int32_t &v_out, int32_t &q_out,
                          int32_t &r_out) {
    uint32_t u = 1, v = 0, q = 0, r = 1;
    uint32_t finv = inv_mod_2_32(f);
    int i = 30;
    for (;;) {
        const int z = ctz32(g | (0xffffffffu << i)); // bit i stops the count at the steps left
        g >>= z;
        u <<= z;
        v <<= z;
        delta += z;
        i -= z;
        if (i == 0) break;
        if (delta > 0) {
            delta = -delta;
            const uint32_t tf = f, tu = u, tv = v;
            f = g;
            g = 0u - tf;
            u = q;
            q = 0u - tu;
            v = r;
            r = 0u - tv;
            finv = inv_mod_2_32(f);
        }
        const int k = (1 - delta) < i ? (1 - delta) : i;
        const uint32_t w = (0u - g * finv) & (0xffffffffu >> (32 - k));
        g += f * w;
        q += u * w;
        r += v * w;
    }
    u_out = (int32_t)u;
    v_out = (int32_t)v;
    q_out = (int32_t)q;
    r_out = (int32_t)r;
}

// (f, g) <- ([[u, v], [q, r]] (f, g)) / 2^30, exact.
template <int L>
VK_HD void update_fg30(int32_t *f, int32_t *g, int32_t u, int32_t v, int32_t q, int32_t r) {
    int64_t cf = (int64_t)u * f[0] + (int64_t)v * g[0];
    int64_t cg = (int64_t)q * f[0] + (int64_t)r * g[0];
    cf >>= 30;
    cg >>= 30;
    for (int i = 1; i < L; i++) {
        cf += (int64_t)u * f[i] + (int64_t)v * g[i];
        cg += (int64_t)q * f[i] + (int64_t)r * g[i];
        f[i - 1] = (int32_t)((uint32_t)cf & kMask30);
        g[i - 1] = (int32_t)((uint32_t)cg & kMask30);
        cf >>= 30;
        cg >>= 30;
    }
    f[L - 1] = (int32_t)cf;
    g[L - 1] = (int32_t)cg;
}

// (d, e) <- ([[u, v], [q, r]] (d, e)) / 2^30 mod m, kept in (-2m, m): a
// multiple of m chosen from the signs of d, e plus a correction making the sum
// divisible by 2^30 is added before the shift.
template <int N, int L>
VK_HD void update_de30(int32_t *d, int32_t *e, int32_t u, int32_t v, int32_t q, int32_t r) {
    const int32_t sd = d[L - 1] >> 31, se = e[L - 1] >> 31;  // -1 when negative
    int32_t md = (u & sd) + (v & se);
    int32_t me = (q & sd) + (r & se);
    int64_t cd = (int64_t)u * d[0] + (int64_t)v * e[0];
    int64_t ce = (int64_t)q * d[0] + (int64_t)r * e[0];
    md -= (int32_t)((mod_minv30<N>() * (uint32_t)cd + (uint32_t)md) & kMask30);
    me -= (int32_t)((mod_minv30<N>() * (uint32_t)ce + (uint32_t)me) & kMask30);
    cd += (int64_t)mod_m30<N>(0) * md;
    ce += (int64_t)mod_m30<N>(0) * me;
    cd >>= 30;
    ce >>= 30;
    for (int i = 1; i < L; i++) {
        cd += (int64_t)u * d[i] + (int64_t)v * e[i] + (int64_t)mod_m30<N>(i) * md;
        ce += (int64_t)q * d[i] + (int64_t)r * e[i] + (int64_t)mod_m30<N>(i) * me;
        d[i - 1] = (int32_t)((uint32_t)cd & kMask30);
        e[i - 1] = (int32_t)((uint32_t)ce & kMask30);
        cd >>= 30;
        ce >>= 30;
    }
    d[L - 1] = (int32_t)cd;
    e[L - 1] = (int32_t)ce;
}

// Adds k*m to a signed radix-2^30 number (k small), renormalising limbs.
template <int N, int L>
VK_HD void add_m30(int32_t *a, int32_t k) {
    int64_t c = 0;
    for (int i = 0; i < L; i++) {
        c += (int64_t)a[i] + (int64_t)k * mod_m30<N>(i);
        if (i < L - 1) {
            a[i] = (int32_t)((uint32_t)c & kMask30);
            c >>= 30;
        } else {
            a[i] = (int32_t)c;
        }
    }
}

// sign of a normalised signed radix-2^30 number compared with m: returns true when a >= m
template <int N, int L>
VK_HD bool ge_m30(const int32_t *a) {
    for (int i = L - 1; i >= 0; i--) {
        if (a[i] != mod_m30<N>(i)) return a[i] > mod_m30<N>(i);
    }
    return true;
}

// x^-1 mod m for a plain integer x < m given as N 32-bit words (0 -> 0).
// VAR: the variable-time batch (divsteps30_var) instead of divsteps30.  On the
// GPU the fixed batches are faster: one launch of 16 inversions per SM, one
// per thread, took 44.6 us with them and 59.4 us in variable time (the lanes of
// a warp leave the variable-time loop at different iterations).
template <int N, bool VAR = false>
VK_HD void inverse_words(uint32_t *out, const uint32_t *x) {
    constexpr int L = N == 12 ? 13 : 9;
    int32_t f[L], g[L], d[L], e[L];
    // words -> radix 2^30
    {
        int acc_bits = 0, w = 0;
        uint64_t acc = 0;
        for (int i = 0; i < L; i++) {
            while (acc_bits < 30 && w < N) {
                acc |= (uint64_t)x[w++] << acc_bits;
                acc_bits += 32;
            }
            g[i] = (int32_t)((uint32_t)acc & kMask30);
            acc >>= 30;
            acc_bits -= 30;
            if (acc_bits < 0) acc_bits = 0;
            f[i] = mod_m30<N>(i);
            d[i] = 0;
            e[i] = 0;
        }
    }
    e[0] = 1;
    int32_t delta = 1;
    bool g_zero = true;
    for (int i = 0; i < L; i++) g_zero &= g[i] == 0;
    if (g_zero) {
        for (int i = 0; i < N; i++) out[i] = 0;
        return;
    }
    // 64 batches = 1920 divsteps, beyond the worst case for a 381-bit modulus
    for (int it = 0; it < 64 && !g_zero; it++) {
        int32_t u, v, q, r;
        if (VAR) divsteps30_var(delta, (uint32_t)f[0], (uint32_t)g[0], u, v, q, r);
        else divsteps30(delta, (uint32_t)f[0], (uint32_t)g[0], u, v, q, r);
        update_de30<N, L>(d, e, u, v, q, r);
        update_fg30<L>(f, g, u, v, q, r);
        g_zero = true;
        for (int i = 0; i < L; i++) g_zero &= g[i] == 0;
    }
    // f = +-1: x^-1 = f * d, then into [0, m)
    if (f[L - 1] < 0) {
        for (int i = 0; i < L; i++) d[i] = -d[i];
        add_m30<N, L>(d, 0); // renormalise limbs after negation
    }
    while (d[L - 1] < 0) add_m30<N, L>(d, 1);
    while (ge_m30<N, L>(d)) add_m30<N, L>(d, -1);
    // radix 2^30 -> words
    {
        uint64_t acc = 0;
        int acc_bits = 0, i = 0;
        for (int w = 0; w < N; w++) {
            while (acc_bits < 32 && i < L) {
                acc |= (uint64_t)(uint32_t)d[i++] << acc_bits;
                acc_bits += 30;
            }
            out[w] = (uint32_t)acc;
            acc >>= 32;
            acc_bits -= 32;
        }
    }
}

// Montgomery-form inverses: for a = x R, inverse_words gives (x R)^-1; one
// Montgomery product with R^3 gives x^-1 R.
template <bool VAR = false>
VK_HD Fp fp_inv_fast(const Fp &a) {
    Fp raw;
    inverse_words<12, VAR>(raw.v, a.v);
    const Fp r3 = Fp{{0xd94ca1e0u, 0xed48ac6bu, 0x03a7adf8u, 0x315f831eu, 0x615e29ddu, 0x9a53352au, 0x921e1761u,
                      0x34c04e5eu, 0x65724728u, 0x2512d435u, 0x91755d4du, 0x0aa63460u}};
    return fp_mul(r3, raw);
}
VK_HD Fr fr_inv_fast(const Fr &a) {
    Fr raw;
    inverse_words<8>(raw.v, a.v);
    const Fr r3 = Fr{{0x439b73afu, 0xc62c1807u, 0x8cf06990u, 0x1b3e0d18u, 0xc7b5f418u, 0x73d13c71u, 0xc8db33e9u,
                      0x6e2a5bb9u}};
    return fr_mul(r3, raw);
}

// ------------------------------------------ divsteps in groups from a table
// J divsteps depend only on the low J bits of f and g and on delta, and for
// delta outside [-(J-1), J-1] they act as at the nearer end of that range (so
// the table is indexed by delta clamped to it).  Their transition is a matrix
// M with 2^J (f', g') = M (f, g), entries at most 2^J in magnitude, and delta'
// = +-delta + c (the sign flips at each swap).  An entry packs the four matrix
// entries as signed bytes (bits 0-31), the sign flip (bit 32) and c (bits
// 40-47); entries are ordered by (clamped delta, (f mod 2^J) >> 1, g mod 2^J).
template <int J>
constexpr int kDivstepEntries = (2 * J - 1) << (2 * J - 1);

VK_HD constexpr uint64_t divstep_group_entry(int delta, int64_t f, int64_t g, int J) {
    int64_t u = 1, v = 0, q = 0, r = 1;
    const int d0 = delta;
    int flips = 0;
    for (int i = 0; i < J; i++) {
        if ((g & 1) && delta > 0) {
            const int64_t nf = g, ng = (g - f) / 2, nu = 2 * q, nv = 2 * r, nq = q - u, nr = r - v;
            delta = 1 - delta;
            f = nf;
            g = ng;
            u = nu;
            v = nv;
            q = nq;
            r = nr;
            flips++;
        } else if (g & 1) {
            g = (g + f) / 2;
            q += u;
            r += v;
            u *= 2;
            v *= 2;
            delta++;
        } else {
            g /= 2;
            u *= 2;
            v *= 2;
            delta++;
        }
    }
    const int sign = (flips & 1) ? -1 : 1;
    const int c = delta - sign * d0;
    return (uint64_t)(uint8_t)(int8_t)u | (uint64_t)(uint8_t)(int8_t)v << 8 | (uint64_t)(uint8_t)(int8_t)q << 16 |
           (uint64_t)(uint8_t)(int8_t)r << 24 | (uint64_t)(sign < 0) << 32 | (uint64_t)(uint8_t)(int8_t)c << 40;
}

template <int J>
struct DivstepTable {
    uint64_t e[kDivstepEntries<J>];
};
template <int J>
VK_HD constexpr DivstepTable<J> make_divstep_table() {
    DivstepTable<J> t{};
    for (int d = -(J - 1); d <= J - 1; d++)
        for (int fo = 0; fo < (1 << (J - 1)); fo++)
            for (int g = 0; g < (1 << J); g++)
                t.e[((d + J - 1) * (1 << (J - 1)) + fo) * (1 << J) + g] = divstep_group_entry(d, 2 * fo + 1, g, J);
    return t;
}

// J divsteps on (delta, f, g) from table tbl, accumulated into (u, v, q, r)
template <int J>
VK_HD void divstep_group(const uint64_t *tbl, int32_t &delta, uint32_t &f, uint32_t &g, int32_t &u, int32_t &v,
                         int32_t &q, int32_t &r) {
    const int dc = delta < -(J - 1) ? -(J - 1) : (delta > J - 1 ? J - 1 : delta);
    const uint32_t idx = ((uint32_t)(dc + J - 1) * (1u << (J - 1)) + ((f >> 1) & ((1u << (J - 1)) - 1))) * (1u << J) +
                         (g & ((1u << J) - 1));
    const uint64_t e = tbl[idx];
    const uint32_t lo = (uint32_t)e, hi = (uint32_t)(e >> 32);
    const int32_t m00 = (int8_t)lo, m01 = (int8_t)(lo >> 8), m10 = (int8_t)(lo >> 16), m11 = (int8_t)(lo >> 24);
    const int32_t c = (int8_t)(hi >> 8);
    delta = (hi & 1u) ? c - delta : c + delta;
    const uint32_t f2 = ((uint32_t)m00 * f + (uint32_t)m01 * g) >> J;
    const uint32_t g2 = ((uint32_t)m10 * f + (uint32_t)m11 * g) >> J;
    f = f2;
    g = g2;
    const int32_t u2 = m00 * u + m01 * q, v2 = m00 * v + m01 * r;
    const int32_t q2 = m10 * u + m11 * q, r2 = m10 * v + m11 * r;
    u = u2;
    v = v2;
    q = q2;
    r = r2;
}

// divsteps30 as seven groups of 4 and one of 2 (t4, t2: the J = 4 and J = 2 tables)
VK_HD void divsteps30_grouped(const uint64_t *t4, const uint64_t *t2, int32_t &delta, uint32_t f, uint32_t g,
                              int32_t &u, int32_t &v, int32_t &q, int32_t &r) {
    u = 1;
    v = 0;
    q = 0;
    r = 1;
#pragma unroll
    for (int k = 0; k < 7; k++) divstep_group<4>(t4, delta, f, g, u, v, q, r);
    divstep_group<2>(t2, delta, f, g, u, v, q, r);
}

#if defined(__CUDACC__)
static __device__ const DivstepTable<4> kDivstepTable4 = make_divstep_table<4>();
static __device__ const DivstepTable<2> kDivstepTable2 = make_divstep_table<2>();

// x^-1 for an Fp value in Montgomery form, computed by the four lanes 4k..4k+3
// of a warp together (every lane passes the same a; the result is valid on the
// lane with lane % 4 == 2).  Each lane keeps one pair -- (f, g) on lanes 0 and 1,
// (d, e) on lanes 2 and 3 -- runs the batch's divsteps itself (t4, t2 in shared
// memory), and computes one row of the batch's update (lane 0 f', 1 g', 2 d',
// 3 e'), which the pair's two lanes then exchange.  A batch thus costs one row
// of 13-limb products per lane instead of four; the same batches as
// inverse_words, so the same result.  The quad's four lanes must run this
// together (they shuffle among themselves only).  Measured per launch of 2368
// inversions, averaged over 50 back-to-back launches: 24.7 us, against 31.8 us
// at one inversion per lane.
static __device__ __noinline__ Fp fp_inv_quad(const uint64_t *t4, const uint64_t *t2, const Fp &a) {
    constexpr int N = 12, L = 13;
    const int lane = threadIdx.x & 31, role = lane & 3, base = lane & ~3;
    const bool odd_role = role & 1, modular = role >= 2;
    const unsigned qm = 0xFu << base;
    int32_t x[L], y[L];
    {
        int32_t gl[L];
        int acc_bits = 0, w = 0;
        uint64_t acc = 0;
#pragma unroll
        for (int i = 0; i < L; i++) {
            while (acc_bits < 30 && w < N) {
                acc |= (uint64_t)a.v[w++] << acc_bits;
                acc_bits += 32;
            }
            gl[i] = (int32_t)((uint32_t)acc & kMask30);
            acc >>= 30;
            acc_bits -= 30;
            if (acc_bits < 0) acc_bits = 0;
        }
#pragma unroll
        for (int i = 0; i < L; i++) {
            x[i] = modular ? 0 : mod_m30<N>(i);         // f = m, d = 0
            y[i] = modular ? (i == 0 ? 1 : 0) : gl[i];  // g = x, e = 1
        }
    }
    bool gz = true;
#pragma unroll
    for (int i = 0; i < L; i++) gz &= y[i] == 0;
    bool g_zero = __shfl_sync(qm, gz, base);
    if (g_zero) return Fp{};
    int32_t delta = 1;
    uint32_t f0 = (uint32_t)__shfl_sync(qm, x[0], base), g0 = (uint32_t)__shfl_sync(qm, y[0], base);
    // 64 batches = 1920 divsteps, beyond the worst case for a 381-bit modulus
    for (int it = 0; it < 64 && !g_zero; it++) {
        int32_t u, v, q, r;
        divsteps30_grouped(t4, t2, delta, f0, g0, u, v, q, r);
        const int32_t ca = odd_role ? q : u, cb = odd_role ? r : v;
        // this lane's row, (ca x + cb y + m md) / 2^30, with md = 0 for (f, g)
        // and for (d, e) the multiple of m of update_de30
        const int32_t sx = x[L - 1] >> 31, sy = y[L - 1] >> 31;
        int32_t md = (ca & sx) + (cb & sy);
        int64_t c = (int64_t)ca * x[0] + (int64_t)cb * y[0];
        md -= (int32_t)((mod_minv30<N>() * (uint32_t)c + (uint32_t)md) & kMask30);
        if (!modular) md = 0;
        c += (int64_t)mod_m30<N>(0) * md;
        c >>= 30;
        int32_t out[L];
#pragma unroll
        for (int i = 1; i < L; i++) {
            c += (int64_t)ca * x[i] + (int64_t)cb * y[i] + (int64_t)mod_m30<N>(i) * md;
            out[i - 1] = (int32_t)((uint32_t)c & kMask30);
            c >>= 30;
        }
        out[L - 1] = (int32_t)c;
#pragma unroll
        for (int i = 0; i < L; i++) {
            const int32_t other = __shfl_xor_sync(qm, out[i], 1);
            x[i] = odd_role ? other : out[i];
            y[i] = odd_role ? out[i] : other;
        }
        gz = true;
#pragma unroll
        for (int i = 0; i < L; i++) gz &= y[i] == 0;
        g_zero = __shfl_sync(qm, gz, base);
        f0 = (uint32_t)__shfl_sync(qm, x[0], base);
        g0 = (uint32_t)__shfl_sync(qm, y[0], base);
    }
    // f = +-1 (lanes 0, 1): x^-1 = f d (lanes 2, 3), then into [0, m)
    const int32_t f_top = __shfl_sync(qm, x[L - 1], base);
    int32_t *d = x;
    if (f_top < 0) {
#pragma unroll
        for (int i = 0; i < L; i++) d[i] = -d[i];
        add_m30<N, L>(d, 0);
    }
    while (d[L - 1] < 0) add_m30<N, L>(d, 1);
    while (ge_m30<N, L>(d)) add_m30<N, L>(d, -1);
    Fp raw;
    {
        uint64_t acc = 0;
        int acc_bits = 0, i = 0;
#pragma unroll
        for (int w = 0; w < N; w++) {
            while (acc_bits < 32 && i < L) {
                acc |= (uint64_t)(uint32_t)d[i++] << acc_bits;
                acc_bits += 30;
            }
            raw.v[w] = (uint32_t)acc;
            acc >>= 32;
            acc_bits -= 32;
        }
    }
    const Fp r3 = Fp{{0xd94ca1e0u, 0xed48ac6bu, 0x03a7adf8u, 0x315f831eu, 0x615e29ddu, 0x9a53352au, 0x921e1761u,
                      0x34c04e5eu, 0x65724728u, 0x2512d435u, 0x91755d4du, 0x0aa63460u}};
    return fp_mul(r3, raw);
}
#endif

} // namespace vkzg
