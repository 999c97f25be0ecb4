// Optimal-ate Miller loop over the M-type twist E'(Fp2): y^2 = x^3 + 4(1+u),
// split final exponentiation, and the decomposed GT exponentiation.
//
// Lines.  For T on E' and P = (xP, yP) in G1 the line through the untwisted
// points, scaled by w^3 and by an Fp2 factor (both killed by the easy part
// of the final exponentiation), is  c0 + (c1 xP) v + (c2 yP) v w  with
//   doubling (T = (X:Y:Z) homogeneous):  c0 = 3b'Z^2 - Y^2, c1 = 3X^2, c2 = -2YZ
//   addition (T + Q, Q affine):          c0 = u xQ - v yQ,  c1 = -u,   c2 = v
// where u = yQ Z - Y, v = xQ Z - X.  Only final-exponentiated values are
// canonical, so this scaling is free to differ from any other implementation.
//
// The hard part follows the addition chain of the reference,
// btx/src/final_exponentiation.rs:255-283 (with raise_to_z at :399-413),
// which computes f^(3 (p^4 - p^2 + 1) / r).
#pragma once
#include "curves.cuh"

namespace wbte {

constexpr int MILLER_LINES = 68;  // 63 doublings + 5 additions for |x|

struct Line { Fp2 c0, c1, c2; };
struct G2Proj { Fp2 X, Y, Z; };

WBTE_INL Fp2 fp2_mul3(const Fp2& a) { return fp2_add(fp2_dbl(a), a); }
WBTE_INL Fp2 fp2_mul4(const Fp2& a) { return fp2_dbl(fp2_dbl(a)); }

// T <- 2T, returns the tangent line.
static __device__ __noinline__ Line line_double(G2Proj& T) {
    Fp2 t0 = fp2_sqr(T.Y);
    Fp2 t1 = fp2_sqr(T.Z);
    Fp2 t2 = fp2_mul4(fp2_mul3(fp2_mul_xi(t1)));  // 3 b' Z^2, b' = 4 (1 + u)
    Fp2 X2 = fp2_sqr(T.X);
    Fp2 YZ = fp2_mul(T.Y, T.Z);
    Fp2 XY = fp2_mul(T.X, T.Y);
    Line l;
    l.c0 = fp2_sub(t2, t0);
    l.c1 = fp2_mul3(X2);
    l.c2 = fp2_neg(fp2_dbl(YZ));
    Fp2 t23 = fp2_mul3(t2);
    T.X = fp2_dbl(fp2_mul(XY, fp2_sub(t0, t23)));
    T.Y = fp2_sub(fp2_sqr(fp2_add(t0, t23)), fp2_mul4(fp2_mul3(fp2_sqr(t2))));
    T.Z = fp2_mul4(fp2_dbl(fp2_mul(t0, YZ)));
    return l;
}

// T <- T + Q, returns the chord.
static __device__ __noinline__ Line line_add(G2Proj& T, const G2A& Q) {
    Fp2 u = fp2_sub(fp2_mul(Q.y, T.Z), T.Y);
    Fp2 v = fp2_sub(fp2_mul(Q.x, T.Z), T.X);
    Line l;
    l.c0 = fp2_sub(fp2_mul(u, Q.x), fp2_mul(v, Q.y));
    l.c1 = fp2_neg(u);
    l.c2 = v;
    Fp2 v2 = fp2_sqr(v);
    Fp2 v3 = fp2_mul(v2, v);
    Fp2 v2X = fp2_mul(v2, T.X);
    Fp2 A = fp2_sub(fp2_sub(fp2_mul(fp2_sqr(u), T.Z), v3), fp2_dbl(v2X));
    T.X = fp2_mul(v, A);
    T.Y = fp2_sub(fp2_mul(u, fp2_sub(v2X, A)), fp2_mul(v3, T.Y));
    T.Z = fp2_mul(v3, T.Z);
    return l;
}

WBTE_INL void mul_by_line(Fp12& f, const Line& l, const G1A& P) {
    fp12_mul_line(f, f, l.c0, fp2_mul_fp(l.c1, P.x), fp2_mul_fp(l.c2, P.y));
}

WBTE_INL G2Proj g2proj_from_affine(const G2A& q) { return G2Proj{q.x, q.y, fp2_one()}; }

// Miller loop computing lines on the fly; identities give 1.
static __device__ __noinline__ void miller_loop(Fp12& f, const G1A& P, const G2A& Q) {
    f = fp12_one();
    if (is_inf(P) || is_inf(Q)) return;
    G2Proj T = g2proj_from_affine(Q);
    for (int i = 62; i >= 0; i--) {
        if (i != 62) fp12_sqr(f, f);
        Line l = line_double(T);
        mul_by_line(f, l, P);
        if ((X_ABS >> i) & 1) {
            l = line_add(T, Q);
            mul_by_line(f, l, P);
        }
    }
    fp12_conj(f, f);  // the BLS12-381 parameter is negative
}

// Miller loop over precomputed lines.  `lines` points at this pair's first
// line; consecutive lines of one pair are `stride` Line records apart.
static __device__ __noinline__ void miller_loop_lines(Fp12& f, const Line* lines, size_t stride, const G1A& P) {
    f = fp12_one();
    if (is_inf(P)) return;
    int idx = 0;
    for (int i = 62; i >= 0; i--) {
        if (i != 62) fp12_sqr(f, f);
        Line l = load_vec(lines + stride * idx++);
        mul_by_line(f, l, P);
        if ((X_ABS >> i) & 1) {
            l = load_vec(lines + stride * idx++);
            mul_by_line(f, l, P);
        }
    }
    fp12_conj(f, f);
}

// Product of T <= MULTI_MILLER_MAX Miller loops over precomputed lines
// sharing one accumulator, so the 62 Fp12 squarings are paid once for all T
// pairs.  Pair t uses the G1 point at points[t] (device memory) and the line
// table at lines + t * pair_stride (lines of one table `stride` apart);
// identities contribute 1.
constexpr int MULTI_MILLER_MAX = 8;
static __device__ __noinline__ void multi_miller_loop_lines(Fp12& f, const Line* lines, size_t stride,
                                                            size_t pair_stride, const G1A* points, int T) {
    G1A P[MULTI_MILLER_MAX];
    for (int t = 0; t < T; t++) P[t] = load_affine(points + t);
    f = fp12_one();
    int idx = 0;
    for (int i = 62; i >= 0; i--) {
        if (i != 62) fp12_sqr(f, f);
        for (int t = 0; t < T; t++) {
            if (is_inf(P[t])) continue;
            Line l = load_vec(lines + t * pair_stride + stride * idx);
            mul_by_line(f, l, P[t]);
        }
        idx++;
        if ((X_ABS >> i) & 1) {
            for (int t = 0; t < T; t++) {
                if (is_inf(P[t])) continue;
                Line l = load_vec(lines + t * pair_stride + stride * idx);
                mul_by_line(f, l, P[t]);
            }
            idx++;
        }
    }
    fp12_conj(f, f);
}

// Product of C <= MULTI_MILLER_MAX Miller loops with lines computed on the
// fly (unprepared_multi_miller_loop, weighted_btx/src/final_exponentiation.rs:
// 229-274): pairs (P[t], Q[t]) share one accumulator, so the 62 Fp12
// squarings are paid once for all C pairs; identities contribute 1.
static __device__ __noinline__ void multi_miller_loop(Fp12& f, const G1A* P, const G2A* Q, int C) {
    G2Proj T[MULTI_MILLER_MAX];
    bool live[MULTI_MILLER_MAX];
    for (int t = 0; t < C; t++) {
        live[t] = !is_inf(P[t]) && !is_inf(Q[t]);
        if (live[t]) T[t] = g2proj_from_affine(Q[t]);
    }
    f = fp12_one();
    for (int i = 62; i >= 0; i--) {
        if (i != 62) fp12_sqr(f, f);
        for (int t = 0; t < C; t++) {
            if (!live[t]) continue;
            Line l = line_double(T[t]);
            mul_by_line(f, l, P[t]);
        }
        if ((X_ABS >> i) & 1) {
            for (int t = 0; t < C; t++) {
                if (!live[t]) continue;
                Line l = line_add(T[t], Q[t]);
                mul_by_line(f, l, P[t]);
            }
        }
    }
    fp12_conj(f, f);
}

// ------------------------------------------------- final exponentiation
// f^((p^6 - 1)(p^2 + 1))
static __device__ __noinline__ void final_exp_easy(Fp12& r, const Fp12& f) {
    Fp12 inv, t, u;
    fp12_inv(inv, f);
    fp12_conj(t, f);
    fp12_mul(t, t, inv);
    fp12_frobenius(u, t, 2);
    fp12_mul(r, t, u);
}

WBTE_INL void mul_then_square(Fp12& acc, const Fp12& m, int n) {
    fp12_mul(acc, acc, m);
    for (int i = 0; i < n; i++) fp12_cyclotomic_sqr(acc, acc);
}
// x^(|z|/2) followed by conjugation, i.e. x^(z/2) for the negative parameter
static __device__ __noinline__ void raise_to_z_div_by_2(Fp12& r, const Fp12& x) {
    Fp12 acc;
    fp12_cyclotomic_sqr(acc, x);
    mul_then_square(acc, x, 2);
    mul_then_square(acc, x, 3);
    mul_then_square(acc, x, 9);
    mul_then_square(acc, x, 32);
    mul_then_square(acc, x, 15);
    fp12_conj(r, acc);
}
WBTE_INL void raise_to_z(Fp12& r, const Fp12& x) {
    Fp12 t;
    raise_to_z_div_by_2(t, x);
    fp12_cyclotomic_sqr(r, t);
}

static __device__ __noinline__ void final_exp_hard(Fp12& out, const Fp12& in) {
    Fp12 result = in, y0, y1, y2, y3;
    fp12_cyclotomic_sqr(y0, result);
    raise_to_z(y1, y0);
    raise_to_z_div_by_2(y2, y1);
    fp12_conj(y3, result);
    fp12_mul(y1, y1, y3);
    fp12_conj(y1, y1);
    fp12_mul(y1, y1, y2);
    raise_to_z(y2, y1);
    raise_to_z(y3, y2);
    fp12_conj(y1, y1);
    fp12_mul(y3, y3, y1);
    fp12_conj(y1, y1);
    fp12_frobenius(y1, y1, 3);
    fp12_frobenius(y2, y2, 2);
    fp12_mul(y1, y1, y2);
    raise_to_z(y2, y3);
    fp12_mul(y2, y2, y0);
    fp12_mul(y2, y2, result);
    fp12_mul(y1, y1, y2);
    fp12_frobenius(y2, y3, 1);
    fp12_mul(out, y1, y2);
}

// ------------------------------------------ decomposed GT exponentiation
// A canonical scalar s < r is written s = d0 + d1|x| + d2|x|^2 + d3|x|^3
// with 0 <= di < |x|; on GT, Frobenius^i followed by conjugation for odd i
// acts as exponentiation by |x|^i.  Each digit is recoded in width-4 NAF
// and the four recodings share one run of at most 65 cyclotomic squarings.
// On cyclotomic elements outside GT the result agrees with x^s after the
// hard part of the final exponentiation.
struct CycPlan {
    int8_t naf[4][65];
    int digits;
};

// |x| = 2^16 * X_ODD with X_ODD < 2^48
constexpr uint64_t X_ODD = X_ABS >> 16;

WBTE_INL void make_cyc_plan(CycPlan& pl, const uint32_t s_in[8]) {
    uint32_t s[8];
    _Pragma("unroll") for (int i = 0; i < 8; i++) s[i] = s_in[i];
    pl.digits = 0;
    for (int c = 0; c < 4; c++) {
        // s = q |x| + rem:  q = (s >> 16) div X_ODD, rem = ((s >> 16) mod X_ODD) 2^16 + (s & 0xffff)
        uint32_t lo16 = s[0] & 0xffffu;
        uint16_t chunks[15];
        for (int j = 0; j < 15; j++) {
            int bit = 16 + 16 * j;
            chunks[j] = (uint16_t)(s[bit >> 5] >> (bit & 31));
        }
        uint64_t rem = 0;
        uint16_t q[15];
        for (int j = 14; j >= 0; j--) {
            uint64_t cur = (rem << 16) | chunks[j];
            q[j] = (uint16_t)(cur / X_ODD);
            rem = cur % X_ODD;
        }
        uint64_t comp = (rem << 16) | lo16;
        for (int i = 0; i < 8; i++) s[i] = 0;
        for (int j = 0; j < 15; j++) s[j >> 1] |= (uint32_t)q[j] << (16 * (j & 1));
        // width-4 NAF of comp; a negative digit may carry into bit 64
        uint64_t v = comp;
        uint32_t carry_bit = 0;  // bit 64 of the running value
        int pos = 0;
        for (int i = 0; i < 65; i++) pl.naf[c][i] = 0;
        while (v != 0 || carry_bit) {
            if (v & 1) {
                int d = (int)(v & 15);
                if (d >= 8) d -= 16;
                pl.naf[c][pos] = (int8_t)d;
                if (d > 0) {
                    v -= (uint64_t)d;
                } else {
                    uint64_t nv = v + (uint64_t)(-d);
                    if (nv < v) carry_bit = 1;
                    v = nv;
                }
            }
            v = (v >> 1) | ((uint64_t)carry_bit << 63);
            carry_bit = 0;
            pos++;
        }
        if (pos > pl.digits) pl.digits = pos;
    }
}

static __device__ __noinline__ void cyc_pow_plan(Fp12& out, const Fp12& value, const CycPlan& pl) {
    if (pl.digits == 0) { out = fp12_one(); return; }
    Fp12 tab[4][4], two;
    fp12_cyclotomic_sqr(two, value);
    tab[0][0] = value;
    for (int i = 1; i < 4; i++) fp12_mul(tab[0][i], tab[0][i - 1], two);
    for (int pw = 1; pw < 4; pw++)
        for (int i = 0; i < 4; i++) {
            fp12_frobenius(tab[pw][i], tab[0][i], pw);
            if (pw & 1) fp12_conj(tab[pw][i], tab[pw][i]);
        }
    Fp12 acc = fp12_one();
    bool started = false;
    for (int pos = pl.digits - 1; pos >= 0; pos--) {
        if (started) fp12_cyclotomic_sqr(acc, acc);
        for (int c = 0; c < 4; c++) {
            int d = pl.naf[c][pos];
            if (!d) continue;
            int ad = d < 0 ? -d : d;
            if (started) {
                if (d < 0) {
                    Fp12 m;
                    fp12_conj(m, tab[c][(ad - 1) >> 1]);
                    fp12_mul(acc, acc, m);
                } else {
                    fp12_mul(acc, acc, tab[c][(ad - 1) >> 1]);
                }
            } else {
                if (d < 0) fp12_conj(acc, tab[c][(ad - 1) >> 1]);
                else acc = tab[c][(ad - 1) >> 1];
                started = true;
            }
        }
    }
    out = acc;
}

WBTE_INL void gt_pow(Fp12& out, const Fp12& value, const uint32_t s[8]) {
    CycPlan pl;
    make_cyc_plan(pl, s);
    cyc_pow_plan(out, value, pl);
}

// ------------------------------------------------ lane-split exponentiation
// The transforms split one exponentiation across a few threads of a warp, one
// base-|x| digit each, so that every thread of the warp runs the same fixed
// schedule of squarings (data-dependent NAF lengths otherwise diverge).

// s = d0 + d1|x| + d2|x|^2 + d3|x|^3 with 0 <= dc < |x| (s < r < |x|^4)
WBTE_INL void decompose_base_x(uint64_t d[4], const uint32_t s_in[8]) {
    uint32_t s[8];
    _Pragma("unroll") for (int i = 0; i < 8; i++) s[i] = s_in[i];
    for (int c = 0; c < 4; c++) {
        uint32_t lo16 = s[0] & 0xffffu;
        uint16_t chunks[15];
        for (int j = 0; j < 15; j++) {
            int bit = 16 + 16 * j;
            chunks[j] = (uint16_t)(s[bit >> 5] >> (bit & 31));
        }
        uint64_t rem = 0;
        uint16_t q[15];
        for (int j = 14; j >= 0; j--) {
            uint64_t cur = (rem << 16) | chunks[j];
            q[j] = (uint16_t)(cur / X_ODD);
            rem = cur % X_ODD;
        }
        d[c] = (rem << 16) | lo16;
        for (int i = 0; i < 8; i++) s[i] = 0;
        for (int j = 0; j < 15; j++) s[j >> 1] |= (uint32_t)q[j] << (16 * (j & 1));
    }
}

// Signed radix-16 recoding of v = hi 2^64 + lo with `top` nibbles (16 or 32):
// v = sum_{k=0..top} digit_k 16^k with digits in [-7, 8].  Rounding a nibble
// above 8 down by 16 carries one into the next digit, and the carry into
// digit k is set exactly when the low k nibbles of v exceed 0x88...8 (k
// eights), so each digit is computed on its own, without a digit array.
WBTE_INL int r16_carry(uint64_t lo, uint64_t hi, int k) {
    constexpr uint64_t E = 0x8888888888888888ull;
    if (k <= 16) {
        uint64_t m = k == 16 ? ~0ull : ((1ull << (4 * k)) - 1);
        return (lo & m) > (E & m);
    }
    int kh = k - 16;
    uint64_t m = kh == 16 ? ~0ull : ((1ull << (4 * kh)) - 1);
    uint64_t h = hi & m, e = E & m;
    return h > e || (h == e && lo > E);
}
WBTE_INL int r16_digit(uint64_t lo, uint64_t hi, int k, int top) {
    int nib = 0;
    if (k < top) nib = (int)(((k < 16) ? (lo >> (4 * k)) : (hi >> (4 * (k - 16)))) & 15u);
    int cout = k < top ? r16_carry(lo, hi, k + 1) : 0;
    return nib + r16_carry(lo, hi, k) - 16 * cout;
}

// out = (+-Frobenius^c(v))^d for one base-|x| digit d (conjugated for odd
// c), i.e. v^(d |x|^c) on GT; v must be cyclotomic.
static __device__ __noinline__ void gt_pow_lane(Fp12& out, const Fp12& v, uint64_t d, int c) {
    Fp12 tab[8];  // base^1 .. base^8
    if (c == 0) {
        tab[0] = v;
    } else {
        fp12_frobenius(tab[0], v, c);
        if (c & 1) fp12_conj(tab[0], tab[0]);
    }
    fp12_cyclotomic_sqr(tab[1], tab[0]);
    for (int k = 2; k < 8; k++) fp12_mul(tab[k], tab[k - 1], tab[0]);
    Fp12 acc = fp12_one();
    for (int k = 16; k >= 0; k--) {
        if (k != 16) {
            fp12_cyclotomic_sqr(acc, acc);
            fp12_cyclotomic_sqr(acc, acc);
            fp12_cyclotomic_sqr(acc, acc);
            fp12_cyclotomic_sqr(acc, acc);
        }
        int dd = r16_digit(d, 0, k, 16);
        int ad = dd < 0 ? -dd : dd;
        if (ad) {
            Fp12 m = tab[ad - 1];
            if (dd < 0) fp12_conj(m, m);
            fp12_mul(acc, acc, m);
        }
    }
    out = acc;
}

// out = prod over the digits c = c0, c0 + step, ... < 4 of v^(d_c |x|^c):
// one run of 64 cyclotomic squarings shared by the selected digits (Straus),
// over one table of powers of phi^c0(v), phi = conj o Frobenius acting as
// |x|; a later digit c applies phi^(c - c0) to the entry it multiplies in.
// step 4 is gt_pow_lane (one digit); step 1 is the whole exponentiation.
static __device__ __noinline__ void gt_pow_digits(Fp12& out, const Fp12& v, const uint64_t d[4], int c0, int step) {
    Fp12 tab[8];  // phi^c0(v)^1 .. ^8
    if (c0 == 0) {
        tab[0] = v;
    } else {
        fp12_frobenius(tab[0], v, c0);
        if (c0 & 1) fp12_conj(tab[0], tab[0]);
    }
    fp12_cyclotomic_sqr(tab[1], tab[0]);
    for (int k = 2; k < 8; k++) fp12_mul(tab[k], tab[k - 1], tab[0]);
    Fp12 acc = fp12_one();
    for (int k = 16; k >= 0; k--) {
        if (k != 16) {
            fp12_cyclotomic_sqr(acc, acc);
            fp12_cyclotomic_sqr(acc, acc);
            fp12_cyclotomic_sqr(acc, acc);
            fp12_cyclotomic_sqr(acc, acc);
        }
        for (int c = c0; c < 4; c += step) {
            const int dd = r16_digit(d[c], 0, k, 16);
            const int ad = dd < 0 ? -dd : dd;
            if (!ad) continue;
            const int rel = c - c0;
            Fp12 m;
            if (rel == 0) m = tab[ad - 1];
            else fp12_frobenius(m, tab[ad - 1], rel);
            if (((rel & 1) != 0) != (dd < 0)) fp12_conj(m, m);
            fp12_mul(acc, acc, m);
        }
    }
    out = acc;
}

// out = [w]p for w = hi 2^64 + lo < 16^top, over the signed radix-16 digits
template <class F>
static __device__ __noinline__ void xyzz_mul_r16(Xyzz<F>& out, const Xyzz<F>& p, uint64_t lo, uint64_t hi, int top) {
    Xyzz<F> tab[8];  // [1]p .. [8]p
    tab[0] = p;
    tab[1] = xyzz_dbl(tab[0]);
    for (int k = 2; k < 8; k++) tab[k] = xyzz_add(tab[k - 1], tab[0]);
    Xyzz<F> acc;
    set_inf(acc);
    for (int k = top; k >= 0; k--) {
        acc = xyzz_dbl(acc);
        acc = xyzz_dbl(acc);
        acc = xyzz_dbl(acc);
        acc = xyzz_dbl(acc);
        int dd = r16_digit(lo, hi, k, top);
        int ad = dd < 0 ? -dd : dd;
        if (ad) {
            Xyzz<F> m = tab[ad - 1];
            if (dd < 0) m = neg(m);
            acc = xyzz_add(acc, m);
        }
    }
    out = acc;
}

// psi (untwist-Frobenius-twist) on G2 in XYZZ coordinates; acts as [x]
WBTE_INL G2X g2_psi(const G2X& p) {
    G2X r;
    r.X = fp2_mul(fp2_conj(p.X), fp2_from_const(C_PSI_CX));
    r.Y = fp2_mul(fp2_conj(p.Y), fp2_from_const(C_PSI_CY));
    r.ZZ = fp2_conj(p.ZZ);
    r.ZZZ = fp2_conj(p.ZZZ);
    return r;
}
// phi (x, y) -> (beta x, y) on G1 in XYZZ coordinates; acts as [x^2 - 1]
WBTE_INL G1X g1_phi(const G1X& p) {
    G1X r = p;
    r.X = fp_mul(p.X, fp_from_const(C_GLV_BETA));
    return r;
}

// Lane c (0..3) of [s]v on G2 for s = sum_c d_c |x|^c:
// out = [d_c]((-1)^c psi^c(v)) = [d_c |x|^c]v.
WBTE_INL void g2_mul_lane(G2X& out, const G2X& v, const uint64_t d[4], int c) {
    G2X base = v;
    for (int i = 0; i < c; i++) base = g2_psi(base);
    if (c & 1) base = neg(base);
    xyzz_mul_r16(out, base, d[c], 0, 16);
}

// Lane c (0 or 1) of [s]v on G1 for s = a + b |x|^2 with a = d0 + d1|x| and
// b = d2 + d3|x| (both below |x|^2 < 2^128): [a]v, or [b](phi(v) + v) since
// phi(v) + v = [x^2]v.
WBTE_INL void g1_mul_lane(G1X& out, const G1X& v, const uint64_t d[4], int c) {
    G1X base = v;
    if (c) base = xyzz_add(g1_phi(v), v);
    uint64_t lo = d[2 * c], hi = d[2 * c + 1];
    // w = lo + hi |x| as a 128-bit integer
    uint64_t plo = hi * X_ABS, phi = __umul64hi(hi, X_ABS);
    uint64_t wlo = plo + lo;
    uint64_t whi = phi + (wlo < plo ? 1 : 0);
    xyzz_mul_r16(out, base, wlo, whi, 32);
}

}  // namespace wbte
