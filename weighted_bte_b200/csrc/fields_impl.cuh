// Out-of-line tower arithmetic.  Included once by fields.cuh; every function
// has internal linkage, so each translation unit carries its own copy.
#pragma once

namespace wbte {

// a^(p-2) with a 4-bit fixed window over the constant exponent.
WBTE_NOINL Fp fp_inv(Fp a) {
    Fp tab[16];
    tab[0] = fp_one();
    tab[1] = a;
    for (int i = 2; i < 16; i++) tab[i] = fp_mul(tab[i - 1], a);
    Fp r = fp_one();
    bool started = false;
    for (int w = 95; w >= 0; w--) {
        if (started) {
            r = fp_sqr(r);
            r = fp_sqr(r);
            r = fp_sqr(r);
            r = fp_sqr(r);
        }
        uint32_t d = (C_P_MINUS_2[w / 8] >> (4 * (w % 8))) & 15u;
        if (d) {
            r = started ? fp_mul(r, tab[d]) : tab[d];
            started = true;
        }
    }
    return r;
}

WBTE_NOINL Fr fr_inv(Fr a) {
    Fr tab[16];
    tab[0] = fr_one();
    tab[1] = a;
    for (int i = 2; i < 16; i++) tab[i] = fr_mul(tab[i - 1], a);
    Fr r = fr_one();
    bool started = false;
    for (int w = 63; w >= 0; w--) {
        if (started) {
            r = fr_mul(r, r);
            r = fr_mul(r, r);
            r = fr_mul(r, r);
            r = fr_mul(r, r);
        }
        uint32_t d = (C_R_MINUS_2[w / 8] >> (4 * (w % 8))) & 15u;
        if (d) {
            r = started ? fr_mul(r, tab[d]) : tab[d];
            started = true;
        }
    }
    return r;
}

WBTE_NOINL Fp2 fp2_inv(Fp2 a) {
    Fp n = fp_add(fp_sqr(a.c0), fp_sqr(a.c1));
    n = fp_inv(n);
    return Fp2{fp_mul(a.c0, n), fp_neg(fp_mul(a.c1, n))};
}

// Karatsuba over Fp2: 6 Fp2 products.
WBTE_NOINL void fp6_mul(Fp6& r, const Fp6& a, const Fp6& b) {
    Fp2 t0 = fp2_mul(a.c0, b.c0);
    Fp2 t1 = fp2_mul(a.c1, b.c1);
    Fp2 t2 = fp2_mul(a.c2, b.c2);
    Fp2 s12 = fp2_mul(fp2_add(a.c1, a.c2), fp2_add(b.c1, b.c2));
    Fp2 s01 = fp2_mul(fp2_add(a.c0, a.c1), fp2_add(b.c0, b.c1));
    Fp2 s02 = fp2_mul(fp2_add(a.c0, a.c2), fp2_add(b.c0, b.c2));
    Fp2 c0 = fp2_add(t0, fp2_mul_xi(fp2_sub(fp2_sub(s12, t1), t2)));
    Fp2 c1 = fp2_add(fp2_sub(fp2_sub(s01, t0), t1), fp2_mul_xi(t2));
    Fp2 c2 = fp2_add(fp2_sub(fp2_sub(s02, t0), t2), t1);
    r.c0 = c0;
    r.c1 = c1;
    r.c2 = c2;
}

// a * (b0 + b1 v): 5 Fp2 products.
WBTE_NOINL void fp6_mul_01(Fp6& r, const Fp6& a, const Fp2& b0, const Fp2& b1) {
    Fp2 t0 = fp2_mul(a.c0, b0);
    Fp2 t1 = fp2_mul(a.c1, b1);
    Fp2 c0 = fp2_add(fp2_mul_xi(fp2_mul(a.c2, b1)), t0);
    Fp2 c1 = fp2_sub(fp2_sub(fp2_mul(fp2_add(a.c0, a.c1), fp2_add(b0, b1)), t0), t1);
    Fp2 c2 = fp2_add(fp2_mul(a.c2, b0), t1);
    r.c0 = c0;
    r.c1 = c1;
    r.c2 = c2;
}

// a * (b1 v): 3 Fp2 products.
WBTE_NOINL void fp6_mul_1(Fp6& r, const Fp6& a, const Fp2& b1) {
    Fp2 c0 = fp2_mul_xi(fp2_mul(a.c2, b1));
    Fp2 c1 = fp2_mul(a.c0, b1);
    Fp2 c2 = fp2_mul(a.c1, b1);
    r.c0 = c0;
    r.c1 = c1;
    r.c2 = c2;
}

WBTE_NOINL void fp6_inv(Fp6& r, const Fp6& a) {
    Fp2 A = fp2_sub(fp2_sqr(a.c0), fp2_mul_xi(fp2_mul(a.c1, a.c2)));
    Fp2 B = fp2_sub(fp2_mul_xi(fp2_sqr(a.c2)), fp2_mul(a.c0, a.c1));
    Fp2 C = fp2_sub(fp2_sqr(a.c1), fp2_mul(a.c0, a.c2));
    Fp2 F = fp2_add(fp2_mul_xi(fp2_add(fp2_mul(a.c2, B), fp2_mul(a.c1, C))), fp2_mul(a.c0, A));
    F = fp2_inv(F);
    r.c0 = fp2_mul(A, F);
    r.c1 = fp2_mul(B, F);
    r.c2 = fp2_mul(C, F);
}

// Karatsuba over Fp6: 3 Fp6 products.
WBTE_NOINL void fp12_mul(Fp12& r, const Fp12& a, const Fp12& b) {
    Fp6 t0, t1, s;
    fp6_mul(t0, a.c0, b.c0);
    fp6_mul(t1, a.c1, b.c1);
    Fp6 sa = fp6_add(a.c0, a.c1);
    Fp6 sb = fp6_add(b.c0, b.c1);
    fp6_mul(s, sa, sb);
    r.c1 = fp6_sub(fp6_sub(s, t0), t1);
    r.c0 = fp6_add(t0, fp6_mul_v(t1));
}

// (a + b w)^2 = (a + b)(a + b v) - ab - ab v + 2ab w: 2 Fp6 products.
WBTE_NOINL void fp12_sqr(Fp12& r, const Fp12& x) {
    Fp6 ab, s;
    fp6_mul(ab, x.c0, x.c1);
    Fp6 l = fp6_add(x.c0, x.c1);
    Fp6 m = fp6_add(x.c0, fp6_mul_v(x.c1));
    fp6_mul(s, l, m);
    r.c0 = fp6_sub(fp6_sub(s, ab), fp6_mul_v(ab));
    r.c1 = fp6_add(ab, ab);
}

// x * ((a0 + a1 v) + (b1 v) w): 13 Fp2 products.
WBTE_NOINL void fp12_mul_line(Fp12& r, const Fp12& x, const Fp2& a0, const Fp2& a1, const Fp2& b1) {
    Fp6 t0, t1, s;
    fp6_mul_01(t0, x.c0, a0, a1);
    fp6_mul_1(t1, x.c1, b1);
    Fp6 sx = fp6_add(x.c0, x.c1);
    fp6_mul_01(s, sx, a0, fp2_add(a1, b1));
    r.c1 = fp6_sub(fp6_sub(s, t0), t1);
    r.c0 = fp6_add(t0, fp6_mul_v(t1));
}

// Squaring in Fp4 = Fp2[t]/(t^2 - xi): (a + b t)^2 = (a^2 + xi b^2) + 2ab t.
WBTE_INL void fp4_sqr(Fp2& c0, Fp2& c1, const Fp2& a, const Fp2& b) {
    Fp2 t0 = fp2_sqr(a);
    Fp2 t1 = fp2_sqr(b);
    c0 = fp2_add(fp2_mul_xi(t1), t0);
    c1 = fp2_sub(fp2_sub(fp2_sqr(fp2_add(a, b)), t0), t1);
}

// Granger-Scott squaring, valid for elements of the cyclotomic subgroup
// (where it equals the ordinary square exactly).  The three Fp4 squarings
// act on the coefficient pairs (w^0, w^3), (w^1, w^4), (w^2, w^5).
WBTE_NOINL void fp12_cyclotomic_sqr(Fp12& r, const Fp12& f) {
    Fp2 z0 = f.c0.c0, z4 = f.c0.c1, z3 = f.c0.c2;
    Fp2 z2 = f.c1.c0, z1 = f.c1.c1, z5 = f.c1.c2;
    Fp2 t0, t1, t2, t3;
    fp4_sqr(t0, t1, z0, z1);
    // 3 t0 - 2 z0, 3 t1 + 2 z1
    z0 = fp2_sub(t0, z0);
    z0 = fp2_add(fp2_dbl(z0), t0);
    z1 = fp2_add(t1, z1);
    z1 = fp2_add(fp2_dbl(z1), t1);
    fp4_sqr(t0, t1, z2, z3);
    fp4_sqr(t2, t3, z4, z5);
    z4 = fp2_sub(t0, z4);
    z4 = fp2_add(fp2_dbl(z4), t0);
    z5 = fp2_add(t1, z5);
    z5 = fp2_add(fp2_dbl(z5), t1);
    t0 = fp2_mul_xi(t3);
    z2 = fp2_add(t0, z2);
    z2 = fp2_add(fp2_dbl(z2), t0);
    z3 = fp2_sub(t2, z3);
    z3 = fp2_add(fp2_dbl(z3), t2);
    r.c0.c0 = z0;
    r.c0.c1 = z4;
    r.c0.c2 = z3;
    r.c1.c0 = z2;
    r.c1.c1 = z1;
    r.c1.c2 = z5;
}

// x^(p^k), k in 1..3: conjugate every Fp2 coefficient for odd k, then scale
// the coefficient of w^i by xi^{i (p^k - 1)/6}.
WBTE_NOINL void fp12_frobenius(Fp12& r, const Fp12& x, int k) {
    Fp2 c[6] = {x.c0.c0, x.c1.c0, x.c0.c1, x.c1.c1, x.c0.c2, x.c1.c2};  // w^0..w^5
    for (int i = 0; i < 6; i++) {
        if (k & 1) c[i] = fp2_conj(c[i]);
        if (i) c[i] = fp2_mul(c[i], fp2_from_const(C_FROB[k - 1][i]));
    }
    r.c0.c0 = c[0];
    r.c1.c0 = c[1];
    r.c0.c1 = c[2];
    r.c1.c1 = c[3];
    r.c0.c2 = c[4];
    r.c1.c2 = c[5];
}

// (a + b w)^{-1} = (a - b w) / (a^2 - b^2 v)
WBTE_NOINL void fp12_inv(Fp12& r, const Fp12& x) {
    Fp6 t0, t1;
    fp6_mul(t0, x.c0, x.c0);
    fp6_mul(t1, x.c1, x.c1);
    t0 = fp6_sub(t0, fp6_mul_v(t1));
    fp6_inv(t1, t0);
    Fp6 c0, c1;
    fp6_mul(c0, x.c0, t1);
    fp6_mul(c1, x.c1, t1);
    r.c0 = c0;
    r.c1 = fp6_neg(c1);
}

}  // namespace wbte
