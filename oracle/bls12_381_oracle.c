/*
 * CPU oracle for the batched threshold-decryption path over BLS12-381.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C restatement of the
 * arithmetic the reference crates obtain from blst 0.3.17 / blstrs 0.7.1
 * (an un-vendored dependency) and of the algorithms the reference writes
 * itself.  Only tests/, the smoke check and the CPU-baseline leg of the
 * benchmark load it, always as the checker.  The product library never links
 * or calls it.
 *
 * Memory layout follows blst (which is what the reference hands across its
 * C ABI): Fp is 6 little-endian 64-bit limbs in Montgomery form with
 * R = 2^384; Fp2/Fp6/Fp12 are nested coefficient arrays (c0 before c1);
 * affine G1 = (x, y) 96 bytes, affine G2 = (x.c0, x.c1, y.c0, y.c1)
 * 192 bytes, the point at infinity is all zero bytes.  Scalars cross the
 * boundary as canonical 32-byte little-endian integers (blst's
 * `p{1,2}s_mult_pippenger` scalar format).
 *
 * Algorithms restated from the reference (paths inside the reference project):
  *   - hard part of the final exponentiation: btx/src/final_exponentiation.rs:255-283
  *     (raise_to_z / raise_to_z_div_by_2 at :399-413)
 *   - easy part and batched easy part: btx/src/final_exponentiation.rs:276-305,356-371
 *   - Radix-2 DIT transform with bit reversal: btx/src/fft.rs:357-411,584-595
 *   - truncated cyclotomic inverse transform: btx/src/fft.rs:284-350
 *   - four-way base-|x| GT exponent decomposition and width-4 NAF:
 *     btx/src/fft.rs:73-154,543-594
 *   - Lagrange coefficients at zero: weighted_btx/src/interpolation.rs:67-98
 * The Miller loop here is the textbook affine optimal-ate loop over the
 * M-type sextic twist; it deliberately differs from any GPU formulation so
 * that only final-exponentiated values (which are canonical) can agree.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint64_t u64;
typedef unsigned __int128 u128;
typedef uint8_t u8;

typedef struct { u64 l[6]; } fp;
typedef struct { fp c0, c1; } fp2;
typedef struct { fp2 c0, c1, c2; } fp6;
typedef struct { fp6 c0, c1; } fp12;
typedef struct { u64 l[4]; } fr;

/* ------------------------------------------------------------------ */
/* Multi-precision helpers                                            */
/* ------------------------------------------------------------------ */
static const u64 P_L[6] = {0xb9feffffffffaaabULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL,
                           0x64774b84f38512bfULL, 0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL};
static const u64 R_L[4] = {0xffffffff00000001ULL, 0x53bda402fffe5bfeULL, 0x3339d80809a1d805ULL,
                           0x73eda753299d7d48ULL};
static const u64 X_ABS = 0xd201000000010000ULL;

static u64 P_INV, R_INV;           /* -m^{-1} mod 2^64 */
static fp FP_ONE, FP_R2;            /* Montgomery 1 and R^2 mod p */
static fr FR_ONE, FR_R2;
static u64 P_MINUS_2[6], P_PLUS_1_DIV_4[6], P_MINUS_1_DIV_2[6];
static u64 R_MINUS_2[4];

static u64 neg_inv64(u64 m0) {
    u64 x = 1;
    for (int i = 0; i < 7; i++) x *= 2 - m0 * x; /* Newton: x = m0^{-1} */
    return (u64)0 - x;
}

static int geq_n(const u64 *a, const u64 *b, int n) {
    for (int i = n - 1; i >= 0; i--) {
        if (a[i] != b[i]) return a[i] > b[i];
    }
    return 1;
}
static u64 sub_n(u64 *o, const u64 *a, const u64 *b, int n) {
    u64 borrow = 0;
    for (int i = 0; i < n; i++) {
        u128 d = (u128)a[i] - b[i] - borrow;
        o[i] = (u64)d;
        borrow = (u64)(d >> 64) & 1;
    }
    return borrow;
}
static u64 add_n(u64 *o, const u64 *a, const u64 *b, int n) {
    u64 carry = 0;
    for (int i = 0; i < n; i++) {
        u128 s = (u128)a[i] + b[i] + carry;
        o[i] = (u64)s;
        carry = (u64)(s >> 64);
    }
    return carry;
}

/* CIOS Montgomery multiplication, n <= 6. */
static void mont_mul_n(u64 *out, const u64 *a, const u64 *b, const u64 *m, u64 minv, int n) {
    u64 t[8] = {0};
    for (int i = 0; i < n; i++) {
        u64 c = 0;
        for (int j = 0; j < n; j++) {
            u128 s = (u128)a[j] * b[i] + t[j] + c;
            t[j] = (u64)s;
            c = (u64)(s >> 64);
        }
        u128 s = (u128)t[n] + c;
        t[n] = (u64)s;
        t[n + 1] = (u64)(s >> 64);
        u64 mm = t[0] * minv;
        s = (u128)mm * m[0] + t[0];
        c = (u64)(s >> 64);
        for (int j = 1; j < n; j++) {
            s = (u128)mm * m[j] + t[j] + c;
            t[j - 1] = (u64)s;
            c = (u64)(s >> 64);
        }
        s = (u128)t[n] + c;
        t[n - 1] = (u64)s;
        t[n] = t[n + 1] + (u64)(s >> 64);
    }
    if (t[n] || geq_n(t, m, n)) sub_n(t, t, m, n);
    memcpy(out, t, 8 * n);
}

/* ------------------------------------------------------------------ */
/* Fp                                                                 */
/* ------------------------------------------------------------------ */
/* Work counting (built only into the counting library, single-threaded, see
 * the Makefile): every Fp Montgomery product or square counts once. */
#ifdef ORC_COUNT_MULS
static unsigned long long g_fp_products;
#define ORC_COUNT_FP() (g_fp_products++)
#else
#define ORC_COUNT_FP() ((void)0)
#endif
unsigned long long orc_fp_product_count(void) {
#ifdef ORC_COUNT_MULS
    return g_fp_products;
#else
    return 0;
#endif
}
void orc_fp_product_count_reset(void) {
#ifdef ORC_COUNT_MULS
    g_fp_products = 0;
#endif
}
static inline void fp_mul(fp *o, const fp *a, const fp *b) {
    ORC_COUNT_FP();
    mont_mul_n(o->l, a->l, b->l, P_L, P_INV, 6);
}
static inline void fp_sqr(fp *o, const fp *a) { fp_mul(o, a, a); }
static inline void fp_add(fp *o, const fp *a, const fp *b) {
    u64 c = add_n(o->l, a->l, b->l, 6);
    if (c || geq_n(o->l, P_L, 6)) sub_n(o->l, o->l, P_L, 6);
}
static inline void fp_sub(fp *o, const fp *a, const fp *b) {
    if (sub_n(o->l, a->l, b->l, 6)) add_n(o->l, o->l, P_L, 6);
}
static inline int fp_is_zero(const fp *a) {
    u64 x = 0;
    for (int i = 0; i < 6; i++) x |= a->l[i];
    return x == 0;
}
static inline void fp_neg(fp *o, const fp *a) {
    if (fp_is_zero(a)) { *o = *a; return; }
    sub_n(o->l, P_L, a->l, 6);
}
static inline int fp_eq(const fp *a, const fp *b) { return memcmp(a, b, sizeof(fp)) == 0; }
static void fp_pow(fp *o, const fp *a, const u64 *e, int nlimbs) {
    fp r = FP_ONE, b = *a;
    for (int i = 0; i < nlimbs * 64; i++) {
        if ((e[i / 64] >> (i % 64)) & 1) fp_mul(&r, &r, &b);
        fp_sqr(&b, &b);
    }
    *o = r;
}
static void fp_inv(fp *o, const fp *a) { fp_pow(o, a, P_MINUS_2, 6); }
static void fp_from_mont(u64 out[6], const fp *a) {
    u64 one[6] = {1, 0, 0, 0, 0, 0};
    mont_mul_n(out, a->l, one, P_L, P_INV, 6);
}
static void fp_to_mont(fp *o, const u64 in[6]) { mont_mul_n(o->l, in, FP_R2.l, P_L, P_INV, 6); }
static void fp_from_u64(fp *o, u64 v) {
    u64 t[6] = {v, 0, 0, 0, 0, 0};
    fp_to_mont(o, t);
}
/* returns 1 if canonical(a) > (p-1)/2 */
static int fp_lexicographically_largest(const fp *a) {
    u64 c[6];
    fp_from_mont(c, a);
    for (int i = 5; i >= 0; i--) {
        if (c[i] != P_MINUS_1_DIV_2[i]) return c[i] > P_MINUS_1_DIV_2[i];
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Fr                                                                 */
/* ------------------------------------------------------------------ */
static inline void fr_mul(fr *o, const fr *a, const fr *b) { mont_mul_n(o->l, a->l, b->l, R_L, R_INV, 4); }
static inline void fr_add(fr *o, const fr *a, const fr *b) {
    u64 c = add_n(o->l, a->l, b->l, 4);
    if (c || geq_n(o->l, R_L, 4)) sub_n(o->l, o->l, R_L, 4);
}
static inline void fr_sub(fr *o, const fr *a, const fr *b) {
    if (sub_n(o->l, a->l, b->l, 4)) add_n(o->l, o->l, R_L, 4);
}
static inline int fr_is_zero(const fr *a) { return (a->l[0] | a->l[1] | a->l[2] | a->l[3]) == 0; }
static inline void fr_neg(fr *o, const fr *a) {
    if (fr_is_zero(a)) { *o = *a; return; }
    sub_n(o->l, R_L, a->l, 4);
}
static void fr_inv(fr *o, const fr *a) {
    fr r = FR_ONE, b = *a;
    for (int i = 0; i < 256; i++) {
        if ((R_MINUS_2[i / 64] >> (i % 64)) & 1) fr_mul(&r, &r, &b);
        fr_mul(&b, &b, &b);
    }
    *o = r;
}
static void fr_to_mont(fr *o, const u64 in[4]) { mont_mul_n(o->l, in, FR_R2.l, R_L, R_INV, 4); }
static void fr_from_mont(u64 out[4], const fr *a) {
    u64 one[4] = {1, 0, 0, 0};
    mont_mul_n(out, a->l, one, R_L, R_INV, 4);
}
static void fr_load(fr *o, const u8 *bytes32) {
    u64 t[4];
    memcpy(t, bytes32, 32);
    fr_to_mont(o, t);
}
static void fr_store(u8 *bytes32, const fr *a) {
    u64 t[4];
    fr_from_mont(t, a);
    memcpy(bytes32, t, 32);
}

/* ------------------------------------------------------------------ */
/* Fp2 = Fp[u]/(u^2+1)                                                 */
/* ------------------------------------------------------------------ */
static inline void fp2_add(fp2 *o, const fp2 *a, const fp2 *b) { fp_add(&o->c0, &a->c0, &b->c0); fp_add(&o->c1, &a->c1, &b->c1); }
static inline void fp2_sub(fp2 *o, const fp2 *a, const fp2 *b) { fp_sub(&o->c0, &a->c0, &b->c0); fp_sub(&o->c1, &a->c1, &b->c1); }
static inline void fp2_neg(fp2 *o, const fp2 *a) { fp_neg(&o->c0, &a->c0); fp_neg(&o->c1, &a->c1); }
static inline void fp2_conj(fp2 *o, const fp2 *a) { o->c0 = a->c0; fp_neg(&o->c1, &a->c1); }
static void fp2_mul(fp2 *o, const fp2 *a, const fp2 *b) {
    fp t0, t1, t2, s0, s1;
    fp_mul(&t0, &a->c0, &b->c0);
    fp_mul(&t1, &a->c1, &b->c1);
    fp_add(&s0, &a->c0, &a->c1);
    fp_add(&s1, &b->c0, &b->c1);
    fp_mul(&t2, &s0, &s1);
    fp_sub(&o->c0, &t0, &t1);
    fp_sub(&t2, &t2, &t0);
    fp_sub(&o->c1, &t2, &t1);
}
static inline void fp2_sqr(fp2 *o, const fp2 *a) { fp2_mul(o, a, a); }
static inline void fp2_mul_fp(fp2 *o, const fp2 *a, const fp *b) { fp_mul(&o->c0, &a->c0, b); fp_mul(&o->c1, &a->c1, b); }
/* multiply by xi = 1 + u */
static inline void fp2_mul_xi(fp2 *o, const fp2 *a) {
    fp t0, t1;
    fp_sub(&t0, &a->c0, &a->c1);
    fp_add(&t1, &a->c0, &a->c1);
    o->c0 = t0;
    o->c1 = t1;
}
static inline int fp2_is_zero(const fp2 *a) { return fp_is_zero(&a->c0) && fp_is_zero(&a->c1); }
static inline int fp2_eq(const fp2 *a, const fp2 *b) { return fp_eq(&a->c0, &b->c0) && fp_eq(&a->c1, &b->c1); }
static void fp2_inv(fp2 *o, const fp2 *a) {
    fp t0, t1, n;
    fp_sqr(&t0, &a->c0);
    fp_sqr(&t1, &a->c1);
    fp_add(&n, &t0, &t1);
    fp_inv(&n, &n);
    fp_mul(&o->c0, &a->c0, &n);
    fp_mul(&t1, &a->c1, &n);
    fp_neg(&o->c1, &t1);
}
static fp2 FP2_ZERO, FP2_ONE;

/* ------------------------------------------------------------------ */
/* Fp6 = Fp2[v]/(v^3 - xi)                                             */
/* ------------------------------------------------------------------ */
static void fp6_add(fp6 *o, const fp6 *a, const fp6 *b) { fp2_add(&o->c0, &a->c0, &b->c0); fp2_add(&o->c1, &a->c1, &b->c1); fp2_add(&o->c2, &a->c2, &b->c2); }
static void fp6_sub(fp6 *o, const fp6 *a, const fp6 *b) { fp2_sub(&o->c0, &a->c0, &b->c0); fp2_sub(&o->c1, &a->c1, &b->c1); fp2_sub(&o->c2, &a->c2, &b->c2); }
static void fp6_neg(fp6 *o, const fp6 *a) { fp2_neg(&o->c0, &a->c0); fp2_neg(&o->c1, &a->c1); fp2_neg(&o->c2, &a->c2); }
/* schoolbook product: a deliberately simple formulation */
static void fp6_mul(fp6 *o, const fp6 *a, const fp6 *b) {
    fp2 t, r0, r1, r2, s;
    /* r0 = a0b0 + xi(a1b2 + a2b1) */
    fp2_mul(&r0, &a->c0, &b->c0);
    fp2_mul(&t, &a->c1, &b->c2);
    fp2_mul(&s, &a->c2, &b->c1);
    fp2_add(&t, &t, &s);
    fp2_mul_xi(&t, &t);
    fp2_add(&r0, &r0, &t);
    /* r1 = a0b1 + a1b0 + xi a2b2 */
    fp2_mul(&r1, &a->c0, &b->c1);
    fp2_mul(&t, &a->c1, &b->c0);
    fp2_add(&r1, &r1, &t);
    fp2_mul(&t, &a->c2, &b->c2);
    fp2_mul_xi(&t, &t);
    fp2_add(&r1, &r1, &t);
    /* r2 = a0b2 + a1b1 + a2b0 */
    fp2_mul(&r2, &a->c0, &b->c2);
    fp2_mul(&t, &a->c1, &b->c1);
    fp2_add(&r2, &r2, &t);
    fp2_mul(&t, &a->c2, &b->c0);
    fp2_add(&r2, &r2, &t);
    o->c0 = r0;
    o->c1 = r1;
    o->c2 = r2;
}
static void fp6_mul_v(fp6 *o, const fp6 *a) {
    fp2 t;
    fp2_mul_xi(&t, &a->c2);
    o->c2 = a->c1;
    o->c1 = a->c0;
    o->c0 = t;
}
static void fp6_inv(fp6 *o, const fp6 *a) {
    fp2 A, B, C, t, F;
    fp2_sqr(&A, &a->c0);
    fp2_mul(&t, &a->c1, &a->c2);
    fp2_mul_xi(&t, &t);
    fp2_sub(&A, &A, &t);
    fp2_sqr(&B, &a->c2);
    fp2_mul_xi(&B, &B);
    fp2_mul(&t, &a->c0, &a->c1);
    fp2_sub(&B, &B, &t);
    fp2_sqr(&C, &a->c1);
    fp2_mul(&t, &a->c0, &a->c2);
    fp2_sub(&C, &C, &t);
    fp2_mul(&F, &a->c2, &B);
    fp2_mul(&t, &a->c1, &C);
    fp2_add(&F, &F, &t);
    fp2_mul_xi(&F, &F);
    fp2_mul(&t, &a->c0, &A);
    fp2_add(&F, &F, &t);
    fp2_inv(&F, &F);
    fp2_mul(&o->c0, &A, &F);
    fp2_mul(&o->c1, &B, &F);
    fp2_mul(&o->c2, &C, &F);
}
static int fp6_is_zero(const fp6 *a) { return fp2_is_zero(&a->c0) && fp2_is_zero(&a->c1) && fp2_is_zero(&a->c2); }

/* ------------------------------------------------------------------ */
/* Fp12 = Fp6[w]/(w^2 - v)                                             */
/* ------------------------------------------------------------------ */
static fp12 FP12_ONE;
static fp2 FROB[4][6]; /* FROB[k][i] = xi^{i (p^k - 1)/6} */

static void fp12_mul(fp12 *o, const fp12 *a, const fp12 *b) {
    fp6 t0, t1, t2, r0, r1;
    fp6_mul(&t0, &a->c0, &b->c0);
    fp6_mul(&t1, &a->c1, &b->c1);
    fp6_mul_v(&t2, &t1);
    fp6_add(&r0, &t0, &t2);
    fp6_mul(&t0, &a->c0, &b->c1);
    fp6_mul(&t1, &a->c1, &b->c0);
    fp6_add(&r1, &t0, &t1);
    o->c0 = r0;
    o->c1 = r1;
}
static inline void fp12_sqr(fp12 *o, const fp12 *a) { fp12_mul(o, a, a); }
static void fp12_conj(fp12 *o, const fp12 *a) { o->c0 = a->c0; fp6_neg(&o->c1, &a->c1); }
static void fp12_inv(fp12 *o, const fp12 *a) {
    fp6 t0, t1;
    fp6_mul(&t0, &a->c0, &a->c0);
    fp6_mul(&t1, &a->c1, &a->c1);
    fp6_mul_v(&t1, &t1);
    fp6_sub(&t0, &t0, &t1);
    fp6_inv(&t0, &t0);
    fp6_mul(&o->c0, &a->c0, &t0);
    fp6_mul(&t1, &a->c1, &t0);
    fp6_neg(&o->c1, &t1);
}
static int fp12_eq(const fp12 *a, const fp12 *b) { return memcmp(a, b, sizeof(fp12)) == 0; }
/* coefficient of w^i: i even -> c0.c(i/2), i odd -> c1.c(i/2) */
static fp2 *fp12_coeff(fp12 *a, int i) {
    fp6 *h = (i & 1) ? &a->c1 : &a->c0;
    int j = i >> 1;
    return j == 0 ? &h->c0 : (j == 1 ? &h->c1 : &h->c2);
}
static void fp12_frobenius(fp12 *o, const fp12 *a, int k) {
    fp12 t = *a;
    for (int i = 0; i < 6; i++) {
        fp2 *c = fp12_coeff(&t, i);
        if (k & 1) fp2_conj(c, c);
        fp2_mul(c, c, &FROB[k][i]);
    }
    *o = t;
}

/* ------------------------------------------------------------------ */
/* Curves.  G1: y^2 = x^3 + 4 over Fp.  G2: y^2 = x^3 + 4(1+u) over Fp2 */
/* Jacobian coordinates, Z == 0 is the point at infinity.             */
/* ------------------------------------------------------------------ */
typedef struct { fp X, Y, Z; } g1j;
typedef struct { fp2 X, Y, Z; } g2j;
typedef struct { fp x, y; } g1a;
typedef struct { fp2 x, y; } g2a;

static fp B1;   /* 4 */
static fp2 B2;  /* 4(1+u) */
static g1a G1_GEN;
static g2a G2_GEN;

#define DEFINE_CURVE(NAME, F, J, A, F_ADD, F_SUB, F_MUL, F_SQR, F_INV, F_ISZ, F_EQ, F_NEG, F_ONE)  \
    static void NAME##_dbl(J *o, const J *p) {                                                 \
        if (F_ISZ(&p->Z)) { *o = *p; return; }                                                 \
        F A_, B_, C_, D_, E_, Fv, t;                                                           \
        F_SQR(&A_, &p->X);                                                                     \
        F_SQR(&B_, &p->Y);                                                                     \
        F_SQR(&C_, &B_);                                                                       \
        F_ADD(&t, &p->X, &B_);                                                                 \
        F_SQR(&t, &t);                                                                         \
        F_SUB(&t, &t, &A_);                                                                    \
        F_SUB(&t, &t, &C_);                                                                    \
        F_ADD(&D_, &t, &t);                                                                    \
        F_ADD(&E_, &A_, &A_);                                                                  \
        F_ADD(&E_, &E_, &A_);                                                                  \
        F_SQR(&Fv, &E_);                                                                       \
        J r;                                                                                   \
        F_SUB(&r.X, &Fv, &D_);                                                                 \
        F_SUB(&r.X, &r.X, &D_);                                                                \
        F_MUL(&r.Z, &p->Y, &p->Z);                                                             \
        F_ADD(&r.Z, &r.Z, &r.Z);                                                               \
        F_SUB(&t, &D_, &r.X);                                                                  \
        F_MUL(&r.Y, &E_, &t);                                                                  \
        F_ADD(&C_, &C_, &C_);                                                                  \
        F_ADD(&C_, &C_, &C_);                                                                  \
        F_ADD(&C_, &C_, &C_);                                                                  \
        F_SUB(&r.Y, &r.Y, &C_);                                                                \
        *o = r;                                                                                \
    }                                                                                          \
    static void NAME##_add(J *o, const J *p, const J *q) {                                     \
        if (F_ISZ(&p->Z)) { *o = *q; return; }                                                 \
        if (F_ISZ(&q->Z)) { *o = *p; return; }                                                 \
        F z1z1, z2z2, u1, u2, s1, s2, h, rr, t;                                                \
        F_SQR(&z1z1, &p->Z);                                                                   \
        F_SQR(&z2z2, &q->Z);                                                                   \
        F_MUL(&u1, &p->X, &z2z2);                                                              \
        F_MUL(&u2, &q->X, &z1z1);                                                              \
        F_MUL(&s1, &p->Y, &q->Z);                                                              \
        F_MUL(&s1, &s1, &z2z2);                                                                \
        F_MUL(&s2, &q->Y, &p->Z);                                                              \
        F_MUL(&s2, &s2, &z1z1);                                                                \
        F_SUB(&h, &u2, &u1);                                                                   \
        F_SUB(&rr, &s2, &s1);                                                                  \
        if (F_ISZ(&h)) {                                                                       \
            if (F_ISZ(&rr)) { NAME##_dbl(o, p); return; }                                      \
            memset(o, 0, sizeof(J));                                                           \
            return;                                                                            \
        }                                                                                      \
        F hh, hhh, v;                                                                          \
        F_SQR(&hh, &h);                                                                        \
        F_MUL(&hhh, &hh, &h);                                                                  \
        F_MUL(&v, &u1, &hh);                                                                   \
        J r;                                                                                   \
        F_SQR(&r.X, &rr);                                                                      \
        F_SUB(&r.X, &r.X, &hhh);                                                               \
        F_SUB(&r.X, &r.X, &v);                                                                 \
        F_SUB(&r.X, &r.X, &v);                                                                 \
        F_SUB(&t, &v, &r.X);                                                                   \
        F_MUL(&r.Y, &rr, &t);                                                                  \
        F_MUL(&t, &s1, &hhh);                                                                  \
        F_SUB(&r.Y, &r.Y, &t);                                                                 \
        F_MUL(&r.Z, &p->Z, &q->Z);                                                             \
        F_MUL(&r.Z, &r.Z, &h);                                                                 \
        *o = r;                                                                                \
    }                                                                                          \
    static void NAME##_neg(J *o, const J *p) { o->X = p->X; F_NEG(&o->Y, &p->Y); o->Z = p->Z; } \
    static void NAME##_from_affine(J *o, const A *a) {                                         \
        if (F_ISZ(&a->x) && F_ISZ(&a->y)) { memset(o, 0, sizeof(J)); return; }                 \
        o->X = a->x; o->Y = a->y; o->Z = F_ONE;                                                \
    }                                                                                          \
    static void NAME##_to_affine(A *o, const J *p) {                                           \
        if (F_ISZ(&p->Z)) { memset(o, 0, sizeof(A)); return; }                                 \
        F zi, zi2, zi3;                                                                        \
        F_INV(&zi, &p->Z);                                                                     \
        F_SQR(&zi2, &zi);                                                                      \
        F_MUL(&zi3, &zi2, &zi);                                                                \
        F_MUL(&o->x, &p->X, &zi2);                                                             \
        F_MUL(&o->y, &p->Y, &zi3);                                                             \
    }                                                                                          \
    /* double-and-add over a canonical little-endian scalar */                                 \
    static void NAME##_mul(J *o, const J *p, const u64 *k, int nlimbs) {                       \
        J acc;                                                                                 \
        memset(&acc, 0, sizeof(J));                                                            \
        for (int i = nlimbs * 64 - 1; i >= 0; i--) {                                           \
            NAME##_dbl(&acc, &acc);                                                            \
            if ((k[i / 64] >> (i % 64)) & 1) NAME##_add(&acc, &acc, p);                         \
        }                                                                                      \
        *o = acc;                                                                              \
    }

static fp FP_ONE_V; /* copy used by macro (needs an lvalue) */
static fp2 FP2_ONE_V;
DEFINE_CURVE(g1, fp, g1j, g1a, fp_add, fp_sub, fp_mul, fp_sqr, fp_inv, fp_is_zero, fp_eq, fp_neg, FP_ONE_V)
DEFINE_CURVE(g2, fp2, g2j, g2a, fp2_add, fp2_sub, fp2_mul, fp2_sqr, fp2_inv, fp2_is_zero, fp2_eq, fp2_neg, FP2_ONE_V)

static int g1a_is_inf(const g1a *a) { return fp_is_zero(&a->x) && fp_is_zero(&a->y); }
static int g2a_is_inf(const g2a *a) { return fp2_is_zero(&a->x) && fp2_is_zero(&a->y); }

static int g1a_on_curve(const g1a *a) {
    if (g1a_is_inf(a)) return 1;
    fp l, r;
    fp_sqr(&l, &a->y);
    fp_sqr(&r, &a->x);
    fp_mul(&r, &r, &a->x);
    fp_add(&r, &r, &B1);
    return fp_eq(&l, &r);
}
static int g2a_on_curve(const g2a *a) {
    if (g2a_is_inf(a)) return 1;
    fp2 l, r;
    fp2_sqr(&l, &a->y);
    fp2_sqr(&r, &a->x);
    fp2_mul(&r, &r, &a->x);
    fp2_add(&r, &r, &B2);
    return fp2_eq(&l, &r);
}

/* ------------------------------------------------------------------ */
/* Initialisation                                                     */
/* ------------------------------------------------------------------ */
static void mod_double(u64 *a, const u64 *m, int n) {
    u64 c = add_n(a, a, a, n);
    if (c || geq_n(a, m, n)) sub_n(a, a, m, n);
}
static void fp_from_hex_be(fp *o, const char *hex) {
    u64 t[6] = {0};
    int len = (int)strlen(hex);
    for (int i = 0; i < len; i++) {
        char ch = hex[len - 1 - i];
        u64 v = (ch >= '0' && ch <= '9') ? (u64)(ch - '0') : (u64)((ch | 32) - 'a' + 10);
        t[i / 16] |= v << (4 * (i % 16));
    }
    fp_to_mont(o, t);
}
static void fp2_pow_limbs(fp2 *o, const fp2 *a, const u64 *e, int nlimbs) {
    fp2 r = FP2_ONE, b = *a;
    for (int i = 0; i < nlimbs * 64; i++) {
        if ((e[i / 64] >> (i % 64)) & 1) fp2_mul(&r, &r, &b);
        fp2_sqr(&b, &b);
    }
    *o = r;
}

static int g_initialised = 0;
static fr FR_ROOT_OF_UNITY; /* 7^((r-1)/2^32) */

void orc_init(void) {
    if (g_initialised) return;
    P_INV = neg_inv64(P_L[0]);
    R_INV = neg_inv64(R_L[0]);
    /* R mod m and R^2 mod m by repeated doubling */
    u64 t[6] = {1, 0, 0, 0, 0, 0};
    for (int i = 0; i < 384; i++) mod_double(t, P_L, 6);
    memcpy(FP_ONE.l, t, 48);
    for (int i = 0; i < 384; i++) mod_double(t, P_L, 6);
    memcpy(FP_R2.l, t, 48);
    u64 s[4] = {1, 0, 0, 0};
    for (int i = 0; i < 256; i++) mod_double(s, R_L, 4);
    memcpy(FR_ONE.l, s, 32);
    for (int i = 0; i < 256; i++) mod_double(s, R_L, 4);
    memcpy(FR_R2.l, s, 32);
    /* exponents */
    u64 two[6] = {2, 0, 0, 0, 0, 0}, one[6] = {1, 0, 0, 0, 0, 0};
    sub_n(P_MINUS_2, P_L, two, 6);
    add_n(P_PLUS_1_DIV_4, P_L, one, 6);
    for (int i = 0; i < 6; i++) P_PLUS_1_DIV_4[i] = (P_PLUS_1_DIV_4[i] >> 2) | (i < 5 ? P_PLUS_1_DIV_4[i + 1] << 62 : 0);
    sub_n(P_MINUS_1_DIV_2, P_L, one, 6);
    for (int i = 0; i < 6; i++) P_MINUS_1_DIV_2[i] = (P_MINUS_1_DIV_2[i] >> 1) | (i < 5 ? P_MINUS_1_DIV_2[i + 1] << 63 : 0);
    sub_n(R_MINUS_2, R_L, two, 4);

    FP_ONE_V = FP_ONE;
    memset(&FP2_ZERO, 0, sizeof(fp2));
    FP2_ONE = FP2_ZERO;
    FP2_ONE.c0 = FP_ONE;
    FP2_ONE_V = FP2_ONE;
    memset(&FP12_ONE, 0, sizeof(fp12));
    FP12_ONE.c0.c0 = FP2_ONE;

    fp_from_u64(&B1, 4);
    B2.c0 = B1;
    B2.c1 = B1;

    fp_from_hex_be(&G1_GEN.x, "17f1d3a73197d7942695638c4fa9ac0fc3688c4f9774b905a14e3a3f171bac586c55e83ff97a1aeffb3af00adb22c6bb");
    fp_from_hex_be(&G1_GEN.y, "08b3f481e3aaa0f1a09e30ed741d8ae4fcf5e095d5d00af600db18cb2c04b3edd03cc744a2888ae40caa232946c5e7e1");
    fp_from_hex_be(&G2_GEN.x.c0, "024aa2b2f08f0a91260805272dc51051c6e47ad4fa403b02b4510b647ae3d1770bac0326a805bbefd48056c8c121bdb8");
    fp_from_hex_be(&G2_GEN.x.c1, "13e02b6052719f607dacd3a088274f65596bd0d09920b61ab5da61bbdc7f5049334cf11213945d57e5ac7d055d042b7e");
    fp_from_hex_be(&G2_GEN.y.c0, "0ce5d527727d6e118cc9cdc6da2e351aadfd9baa8cbdd3a76d429a695160d12c923ac9cc3baca289e193548608b82801");
    fp_from_hex_be(&G2_GEN.y.c1, "0606c4a02ea734cc32acd2b02bc28b99cb3e287e85a763af267492ab572e99ab3f370d275cec1da1aaa9075ff05f79be");

    /* Frobenius coefficients: gamma = xi^{(p-1)/6}; FROB[1][i] = gamma^i,
     * FROB[2][i] = (gamma * conj(gamma))^i, FROB[3][i] = (gamma^2 conj(gamma))^i. */
    u64 e[6];
    sub_n(e, P_L, one, 6);
    {
        /* divide by 6 */
        u128 rem = 0;
        for (int i = 5; i >= 0; i--) {
            u128 cur = (rem << 64) | e[i];
            e[i] = (u64)(cur / 6);
            rem = cur % 6;
        }
    }
    fp2 xi = FP2_ONE, gam, gc, g2v, g3v;
    xi.c1 = FP_ONE;
    fp2_pow_limbs(&gam, &xi, e, 6);
    fp2_conj(&gc, &gam);
    fp2_mul(&g2v, &gam, &gc);
    fp2_mul(&g3v, &g2v, &gam);
    fp2 base[4] = {FP2_ONE, gam, g2v, g3v};
    for (int k = 0; k < 4; k++) {
        FROB[k][0] = FP2_ONE;
        for (int i = 1; i < 6; i++) fp2_mul(&FROB[k][i], &FROB[k][i - 1], &base[k]);
    }
    /* Fr two-adic root of unity from the multiplicative generator 7 */
    u64 tt[4];
    memcpy(tt, R_L, 32);
    tt[0] -= 1;
    for (int i = 0; i < 4; i++) tt[i] = (tt[i] >> 32) | (i < 3 ? tt[i + 1] << 32 : 0);
    fr seven, rr = FR_ONE;
    u64 sv[4] = {7, 0, 0, 0};
    fr_to_mont(&seven, sv);
    for (int i = 0; i < 256; i++) {
        if ((tt[i / 64] >> (i % 64)) & 1) fr_mul(&rr, &rr, &seven);
        fr_mul(&seven, &seven, &seven);
    }
    FR_ROOT_OF_UNITY = rr;
    g_initialised = 1;
}

/* ------------------------------------------------------------------ */
/* Pairing: affine Miller loop, split final exponentiation             */
/* ------------------------------------------------------------------ */
/* Multiply f by the sparse line value a0 + a1 v + b1 v w (b1 in Fp). */
static void mul_by_line(fp12 *f, const fp2 *a0, const fp2 *a1, const fp *b1) {
    fp12 l;
    memset(&l, 0, sizeof(l));
    l.c0.c0 = *a0;
    l.c0.c1 = *a1;
    l.c1.c1.c0 = *b1;
    fp12_mul(f, f, &l);
}

static void miller_loop_affine(fp12 *out, const g1a *P, const g2a *Q) {
    if (g1a_is_inf(P) || g2a_is_inf(Q)) { *out = FP12_ONE; return; }
    fp12 f = FP12_ONE;
    g2a T = *Q;
    fp2 lam, t, a0, a1, x3, y3;
    for (int i = 62; i >= 0; i--) {
        fp12_sqr(&f, &f);
        /* tangent: lambda = 3x^2 / 2y */
        fp2_sqr(&t, &T.x);
        fp2_add(&lam, &t, &t);
        fp2_add(&lam, &lam, &t);
        fp2_add(&t, &T.y, &T.y);
        fp2_inv(&t, &t);
        fp2_mul(&lam, &lam, &t);
        fp2_mul(&a0, &lam, &T.x);
        fp2_sub(&a0, &a0, &T.y);
        fp2_mul_fp(&a1, &lam, &P->x);
        fp2_neg(&a1, &a1);
        mul_by_line(&f, &a0, &a1, &P->y);
        fp2_sqr(&x3, &lam);
        fp2_sub(&x3, &x3, &T.x);
        fp2_sub(&x3, &x3, &T.x);
        fp2_sub(&t, &T.x, &x3);
        fp2_mul(&y3, &lam, &t);
        fp2_sub(&y3, &y3, &T.y);
        T.x = x3;
        T.y = y3;
        if ((X_ABS >> i) & 1) {
            fp2_sub(&lam, &Q->y, &T.y);
            fp2_sub(&t, &Q->x, &T.x);
            fp2_inv(&t, &t);
            fp2_mul(&lam, &lam, &t);
            fp2_mul(&a0, &lam, &T.x);
            fp2_sub(&a0, &a0, &T.y);
            fp2_mul_fp(&a1, &lam, &P->x);
            fp2_neg(&a1, &a1);
            mul_by_line(&f, &a0, &a1, &P->y);
            fp2_sqr(&x3, &lam);
            fp2_sub(&x3, &x3, &T.x);
            fp2_sub(&x3, &x3, &Q->x);
            fp2_sub(&t, &T.x, &x3);
            fp2_mul(&y3, &lam, &t);
            fp2_sub(&y3, &y3, &T.y);
            T.x = x3;
            T.y = y3;
        }
    }
    /* the BLS12-381 parameter is negative */
    fp12_conj(out, &f);
}

static void easy_part_with_inverse(fp12 *o, const fp12 *f, const fp12 *finv) {
    fp12 t, u;
    fp12_conj(&t, f);
    fp12_mul(&t, &t, finv);
    fp12_frobenius(&u, &t, 2);
    fp12_mul(o, &t, &u);
}
static void easy_part(fp12 *o, const fp12 *f) {
    fp12 inv;
    fp12_inv(&inv, f);
    easy_part_with_inverse(o, f, &inv);
}
static void cyc_sqr(fp12 *o, const fp12 *a) { fp12_sqr(o, a); }
static void mul_then_square(fp12 *acc, const fp12 *m, int n) {
    fp12_mul(acc, acc, m);
    for (int i = 0; i < n; i++) cyc_sqr(acc, acc);
}
static void raise_to_z_div_by_2(fp12 *o, const fp12 *in) {
    fp12 r;
    cyc_sqr(&r, in);
    mul_then_square(&r, in, 2);
    mul_then_square(&r, in, 3);
    mul_then_square(&r, in, 9);
    mul_then_square(&r, in, 32);
    mul_then_square(&r, in, 15);
    fp12_conj(o, &r);
}
static void raise_to_z(fp12 *o, const fp12 *in) {
    fp12 t;
    raise_to_z_div_by_2(&t, in);
    cyc_sqr(o, &t);
}
static void hard_part(fp12 *out, const fp12 *in) {
    fp12 result = *in, y0, y1, y2, y3;
    cyc_sqr(&y0, &result);
    raise_to_z(&y1, &y0);
    raise_to_z_div_by_2(&y2, &y1);
    fp12_conj(&y3, &result);
    fp12_mul(&y1, &y1, &y3);
    fp12_conj(&y1, &y1);
    fp12_mul(&y1, &y1, &y2);
    raise_to_z(&y2, &y1);
    raise_to_z(&y3, &y2);
    fp12_conj(&y1, &y1);
    fp12_mul(&y3, &y3, &y1);
    fp12_conj(&y1, &y1);
    fp12_frobenius(&y1, &y1, 3);
    fp12_frobenius(&y2, &y2, 2);
    fp12_mul(&y1, &y1, &y2);
    raise_to_z(&y2, &y3);
    fp12_mul(&y2, &y2, &y0);
    fp12_mul(&y2, &y2, &result);
    fp12_mul(&y1, &y1, &y2);
    fp12_frobenius(&y2, &y3, 1);
    fp12_mul(out, &y1, &y2);
}
static void final_exp(fp12 *o, const fp12 *f) {
    fp12 t;
    easy_part(&t, f);
    hard_part(o, &t);
}

/* ------------------------------------------------------------------ */
/* GT exponentiation                                                  */
/* ------------------------------------------------------------------ */
static void fp12_pow_limbs(fp12 *o, const fp12 *a, const u64 *e, int nlimbs) {
    fp12 r = FP12_ONE;
    for (int i = nlimbs * 64 - 1; i >= 0; i--) {
        fp12_sqr(&r, &r);
        if ((e[i / 64] >> (i % 64)) & 1) fp12_mul(&r, &r, a);
    }
    *o = r;
}

/* Four-way base-|x| decomposition (btx/src/fft.rs:543-567). */
static void decompose_base_x(u64 comp[4], const u64 scalar[4]) {
    u64 l[4] = {scalar[0], scalar[1], scalar[2], scalar[3]};
    for (int c = 0; c < 4; c++) {
        u128 rem = 0;
        for (int i = 3; i >= 0; i--) {
            u128 cur = (rem << 64) | l[i];
            l[i] = (u64)(cur / X_ABS);
            rem = cur % X_ABS;
        }
        comp[c] = (u64)rem;
    }
}
/* Width-4 NAF of a 64-bit value, up to 65 digits (btx/src/fft.rs:569-594). */
static int wnaf4(int8_t d[65], u64 v64) {
    u128 v = v64;
    int pos = 0;
    memset(d, 0, 65);
    while (v) {
        if (v & 1) {
            int digit = (int)(v & 15);
            if (digit >= 8) digit -= 16;
            d[pos] = (int8_t)digit;
            if (digit > 0) v -= (u128)digit;
            else v += (u128)(-digit);
        }
        v >>= 1;
        pos++;
    }
    return pos;
}
typedef struct { int8_t naf[4][65]; int digits; } cyc_plan;
static void make_plan(cyc_plan *pl, const u64 scalar[4]) {
    u64 comp[4];
    decompose_base_x(comp, scalar);
    pl->digits = 0;
    for (int c = 0; c < 4; c++) {
        int n = wnaf4(pl->naf[c], comp[c]);
        if (n > pl->digits) pl->digits = n;
    }
}
/* Decomposed cyclotomic action (btx/src/fft.rs:73-154). */
static void cyc_pow_plan(fp12 *o, const fp12 *value, const cyc_plan *pl) {
    if (pl->digits == 0) { *o = FP12_ONE; return; }
    fp12 tab[4][4], two;
    cyc_sqr(&two, value);
    tab[0][0] = *value;
    for (int i = 1; i < 4; i++) fp12_mul(&tab[0][i], &tab[0][i - 1], &two);
    for (int pw = 1; pw < 4; pw++)
        for (int i = 0; i < 4; i++) {
            fp12_frobenius(&tab[pw][i], &tab[0][i], pw);
            if (pw & 1) fp12_conj(&tab[pw][i], &tab[pw][i]);
        }
    fp12 acc = FP12_ONE;
    int started = 0;
    for (int pos = pl->digits - 1; pos >= 0; pos--) {
        if (started) cyc_sqr(&acc, &acc);
        for (int c = 0; c < 4; c++) {
            int dg = pl->naf[c][pos];
            if (!dg) continue;
            fp12 m = tab[c][((dg < 0 ? -dg : dg) - 1) / 2];
            if (dg < 0) fp12_conj(&m, &m);
            if (started) fp12_mul(&acc, &acc, &m);
            else { acc = m; started = 1; }
        }
    }
    *o = acc;
}

/* ------------------------------------------------------------------ */
/* Exported API                                                        */
/* ------------------------------------------------------------------ */
#define G1A(ptr) ((g1a *)(ptr))
#define G2A(ptr) ((g2a *)(ptr))

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

void orc_g1_generator(u8 *out) { memcpy(out, &G1_GEN, 96); }
void orc_g2_generator(u8 *out) { memcpy(out, &G2_GEN, 192); }
void orc_fr_root_of_unity(u8 *out32) { fr_store(out32, &FR_ROOT_OF_UNITY); }
int orc_g1_on_curve(const u8 *a) { return g1a_on_curve(G1A(a)); }
int orc_g2_on_curve(const u8 *a) { return g2a_on_curve(G2A(a)); }

/* field element conversions: canonical little-endian 48 bytes <-> Montgomery */
void orc_fp_to_mont(u8 *out48, const u8 *in48) {
    u64 t[6];
    memcpy(t, in48, 48);
    fp o;
    fp_to_mont(&o, t);
    memcpy(out48, &o, 48);
}
void orc_fp_from_mont(u8 *out48, const u8 *in48) {
    fp a;
    memcpy(&a, in48, 48);
    u64 t[6];
    fp_from_mont(t, &a);
    memcpy(out48, t, 48);
}

void orc_g1_add(u8 *out, const u8 *a, const u8 *b) {
    g1j x, y;
    g1_from_affine(&x, G1A(a));
    g1_from_affine(&y, G1A(b));
    g1_add(&x, &x, &y);
    g1_to_affine(G1A(out), &x);
}
void orc_g2_add(u8 *out, const u8 *a, const u8 *b) {
    g2j x, y;
    g2_from_affine(&x, G2A(a));
    g2_from_affine(&y, G2A(b));
    g2_add(&x, &x, &y);
    g2_to_affine(G2A(out), &x);
}
void orc_g1_neg(u8 *out, const u8 *a) {
    g1a r = *G1A(a);
    fp_neg(&r.y, &r.y);
    memcpy(out, &r, 96);
}
void orc_g2_neg(u8 *out, const u8 *a) {
    g2a r = *G2A(a);
    fp2_neg(&r.y, &r.y);
    memcpy(out, &r, 192);
}
/* out[i] = scalars[i] * points[i]  (points stride 0 => one fixed base) */
void orc_g1_mul_batch(u8 *out, const u8 *points, int64_t point_stride, const u8 *scalars, int64_t n) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < n; i++) {
        g1j p, r;
        u64 k[4];
        memcpy(k, scalars + 32 * i, 32);
        g1_from_affine(&p, G1A(points + point_stride * i));
        g1_mul(&r, &p, k, 4);
        g1_to_affine(G1A(out + 96 * i), &r);
    }
}
void orc_g2_mul_batch(u8 *out, const u8 *points, int64_t point_stride, const u8 *scalars, int64_t n) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < n; i++) {
        g2j p, r;
        u64 k[4];
        memcpy(k, scalars + 32 * i, 32);
        g2_from_affine(&p, G2A(points + point_stride * i));
        g2_mul(&r, &p, k, 4);
        g2_to_affine(G2A(out + 192 * i), &r);
    }
}

/* ZCash / IETF compressed serialisation */
static void fp_to_be48(u8 *out, const fp *a) {
    u64 t[6];
    fp_from_mont(t, a);
    for (int i = 0; i < 48; i++) out[47 - i] = (u8)(t[i / 8] >> (8 * (i % 8)));
}
void orc_g1_compress(u8 *out48, const u8 *in96) {
    const g1a *a = G1A(in96);
    if (g1a_is_inf(a)) {
        memset(out48, 0, 48);
        out48[0] = 0xc0;
        return;
    }
    fp_to_be48(out48, &a->x);
    out48[0] |= 0x80;
    if (fp_lexicographically_largest(&a->y)) out48[0] |= 0x20;
}
void orc_g2_compress(u8 *out96, const u8 *in192) {
    const g2a *a = G2A(in192);
    if (g2a_is_inf(a)) {
        memset(out96, 0, 96);
        out96[0] = 0xc0;
        return;
    }
    fp_to_be48(out96, &a->x.c1);
    fp_to_be48(out96 + 48, &a->x.c0);
    out96[0] |= 0x80;
    int largest = fp_is_zero(&a->y.c1) ? fp_lexicographically_largest(&a->y.c0)
                                       : fp_lexicographically_largest(&a->y.c1);
    if (largest) out96[0] |= 0x20;
}
/* 12 coefficients, c0.c0.c0 first, each 48-byte big-endian canonical */
void orc_fp12_to_bytes(u8 *out576, const u8 *in576) {
    const fp *c = (const fp *)in576;
    for (int i = 0; i < 12; i++) fp_to_be48(out576 + 48 * i, &c[i]);
}

/* ---------------- MSM (Pippenger, unsigned windows) ---------------- */
static int msm_window(int64_t n) {
    if (n < 32) return 3;
    int lg = 0;
    while ((1LL << (lg + 1)) <= n) lg++;
    int c = lg - 2;
    if (c < 4) c = 4;
    if (c > 16) c = 16;
    return c;
}
static inline u64 scalar_window(const u8 *s, int bit, int c) {
    u64 v = 0;
    for (int b = 0; b < c; b++) {
        int pos = bit + b;
        if (pos >= 256) break;
        v |= (u64)((s[pos >> 3] >> (pos & 7)) & 1) << b;
    }
    return v;
}
#define DEFINE_MSM(NAME, J, A, ASZ)                                                            \
    static void NAME##_msm_core(J *out, const u8 *bases, const int64_t *pidx, const u8 *scal,  \
                                const int64_t *sidx, int64_t n) {                              \
        memset(out, 0, sizeof(J));                                                             \
        if (n == 0) return;                                                                    \
        if (n < 8) {                                                                           \
            for (int64_t i = 0; i < n; i++) {                                                  \
                J p, r;                                                                        \
                u64 k[4];                                                                      \
                memcpy(k, scal + 32 * (sidx ? sidx[i] : i), 32);                               \
                NAME##_from_affine(&p, (const A *)(bases + ASZ * (pidx ? pidx[i] : i)));       \
                NAME##_mul(&r, &p, k, 4);                                                      \
                NAME##_add(out, out, &r);                                                      \
            }                                                                                  \
            return;                                                                            \
        }                                                                                      \
        int c = msm_window(n);                                                                 \
        int nb = 1 << c;                                                                       \
        J *buckets = (J *)malloc(sizeof(J) * nb);                                              \
        J acc;                                                                                 \
        memset(&acc, 0, sizeof(J));                                                            \
        int top = ((255 + c - 1) / c) * c;                                                     \
        for (int bit = top - c; bit >= 0; bit -= c) {                                          \
            for (int i = 0; i < c; i++) NAME##_dbl(&acc, &acc);                                 \
            memset(buckets, 0, sizeof(J) * nb);                                                \
            for (int64_t i = 0; i < n; i++) {                                                  \
                u64 w = scalar_window(scal + 32 * (sidx ? sidx[i] : i), bit, c);               \
                if (!w) continue;                                                              \
                J p;                                                                           \
                NAME##_from_affine(&p, (const A *)(bases + ASZ * (pidx ? pidx[i] : i)));       \
                NAME##_add(&buckets[w], &buckets[w], &p);                                      \
            }                                                                                  \
            J run, sum;                                                                        \
            memset(&run, 0, sizeof(J));                                                        \
            memset(&sum, 0, sizeof(J));                                                        \
            for (int b = nb - 1; b >= 1; b--) {                                                \
                NAME##_add(&run, &run, &buckets[b]);                                           \
                NAME##_add(&sum, &sum, &run);                                                  \
            }                                                                                  \
            NAME##_add(&acc, &acc, &sum);                                                      \
        }                                                                                      \
        free(buckets);                                                                         \
        *out = acc;                                                                            \
    }
DEFINE_MSM(g1, g1j, g1a, 96)
DEFINE_MSM(g2, g2j, g2a, 192)

void orc_g1_msm(u8 *out, const u8 *points, const u8 *scalars, int64_t n) {
    g1j r;
    g1_msm_core(&r, points, NULL, scalars, NULL, n);
    g1_to_affine(G1A(out), &r);
}
void orc_g2_msm(u8 *out, const u8 *points, const u8 *scalars, int64_t n) {
    g2j r;
    g2_msm_core(&r, points, NULL, scalars, NULL, n);
    g2_to_affine(G2A(out), &r);
}
/* k gathered MSMs: MSM j sums over t in [offsets[j], offsets[j+1]) of
 * scalars[sidx[t]] * bases[pidx[t]].  Runs the MSMs in parallel. */
void orc_g1_msm_gather(u8 *out, const u8 *bases, const int64_t *pidx, const u8 *scalars,
                       const int64_t *sidx, const int64_t *offsets, int64_t k) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t j = 0; j < k; j++) {
        g1j r;
        g1_msm_core(&r, bases, pidx + offsets[j], scalars, sidx + offsets[j], offsets[j + 1] - offsets[j]);
        g1_to_affine(G1A(out + 96 * j), &r);
    }
}
void orc_g2_msm_gather(u8 *out, const u8 *bases, const int64_t *pidx, const u8 *scalars,
                       const int64_t *sidx, const int64_t *offsets, int64_t k) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t j = 0; j < k; j++) {
        g2j r;
        g2_msm_core(&r, bases, pidx + offsets[j], scalars, sidx + offsets[j], offsets[j + 1] - offsets[j]);
        g2_to_affine(G2A(out + 192 * j), &r);
    }
}

/* ---------------- Radix-2 transforms (btx/src/fft.rs:357-411) ---------------- */
static int64_t bitrev(int64_t i, int bits) {
    int64_t r = 0;
    for (int b = 0; b < bits; b++) r |= ((i >> b) & 1) << (bits - 1 - b);
    return r;
}
static void fr_pow_u64(fr *o, const fr *a, u64 e) {
    fr r = FR_ONE, b = *a;
    while (e) {
        if (e & 1) fr_mul(&r, &r, &b);
        fr_mul(&b, &b, &b);
        e >>= 1;
    }
    *o = r;
}
static int log2_exact(int64_t n) {
    int lg = 0;
    while ((1LL << lg) < n) lg++;
    return lg;
}
/* generator of the size-n subgroup, or its inverse */
static void domain_generator(fr *g, int64_t n, int inverse) {
    int lg = log2_exact(n);
    fr x = FR_ROOT_OF_UNITY;
    for (int i = lg; i < 32; i++) fr_mul(&x, &x, &x);
    if (inverse) fr_inv(&x, &x);
    *g = x;
}
/* twiddle powers for one stage: tw[j] = step^j (canonical u64[4]) */
static void stage_twiddles(u64 (*tw)[4], const fr *step, int64_t half) {
    fr t = FR_ONE;
    for (int64_t j = 0; j < half; j++) {
        fr_from_mont(tw[j], &t);
        fr_mul(&t, &t, step);
    }
}
#define DEFINE_GROUP_NTT(NAME, J, A)                                                           \
    void orc_##NAME##_ntt(u8 *io, int64_t n, int inverse) {                                    \
        A *a = (A *)io;                                                                        \
        J *v = (J *)malloc(sizeof(J) * n);                                                     \
        int bits = log2_exact(n);                                                              \
        for (int64_t i = 0; i < n; i++) NAME##_from_affine(&v[bitrev(i, bits)], &a[i]);        \
        fr g;                                                                                  \
        domain_generator(&g, n, inverse);                                                      \
        u64(*tw)[4] = malloc(sizeof(u64[4]) * (n > 1 ? n / 2 : 1));                            \
        for (int64_t size = 2; size <= n; size *= 2) {                                         \
            int64_t half = size / 2;                                                           \
            fr step;                                                                           \
            fr_pow_u64(&step, &g, (u64)(n / size));                                            \
            stage_twiddles(tw, &step, half);                                                   \
            _Pragma("omp parallel for schedule(dynamic, 1)")                                   \
            for (int64_t idx = 0; idx < n / 2; idx++) {                                        \
                int64_t chunk = idx / half, j = idx % half;                                    \
                J *u = &v[chunk * size + j], *w = &v[chunk * size + j + half];                 \
                J t, un;                                                                       \
                if (j == 0) t = *w;                                                            \
                else NAME##_mul(&t, w, tw[j], 4);                                              \
                NAME##_neg(&un, &t);                                                           \
                NAME##_add(&un, u, &un);                                                       \
                NAME##_add(u, u, &t);                                                          \
                *w = un;                                                                       \
            }                                                                                  \
        }                                                                                      \
        free(tw);                                                                              \
        for (int64_t i = 0; i < n; i++) NAME##_to_affine(&a[i], &v[i]);                        \
        free(v);                                                                               \
    }
DEFINE_GROUP_NTT(g1, g1j, g1a)
DEFINE_GROUP_NTT(g2, g2j, g2a)

/* Fr transform on canonical 32-byte scalars */
void orc_fr_ntt(u8 *io, int64_t n, int inverse) {
    fr *v = (fr *)malloc(sizeof(fr) * n);
    int bits = log2_exact(n);
    for (int64_t i = 0; i < n; i++) fr_load(&v[bitrev(i, bits)], io + 32 * i);
    fr g;
    domain_generator(&g, n, inverse);
    for (int64_t size = 2; size <= n; size *= 2) {
        int64_t half = size / 2;
        fr step, w;
        fr_pow_u64(&step, &g, (u64)(n / size));
        for (int64_t c = 0; c < n; c += size) {
            w = FR_ONE;
            for (int64_t j = 0; j < half; j++) {
                fr t, u = v[c + j];
                fr_mul(&t, &v[c + j + half], &w);
                fr_add(&v[c + j], &u, &t);
                fr_sub(&v[c + j + half], &u, &t);
                fr_mul(&w, &w, &step);
            }
        }
    }
    for (int64_t i = 0; i < n; i++) fr_store(io + 32 * i, &v[i]);
    free(v);
}

/* GT transform by ordinary exponentiation (the generic group transform). */
void orc_gt_ntt(u8 *io, int64_t n, int inverse) {
    fp12 *a = (fp12 *)io;
    fp12 *v = (fp12 *)malloc(sizeof(fp12) * n);
    int bits = log2_exact(n);
    for (int64_t i = 0; i < n; i++) v[bitrev(i, bits)] = a[i];
    fr g;
    domain_generator(&g, n, inverse);
    u64(*tw)[4] = malloc(sizeof(u64[4]) * (n > 1 ? n / 2 : 1));
    for (int64_t size = 2; size <= n; size *= 2) {
        int64_t half = size / 2;
        fr step;
        fr_pow_u64(&step, &g, (u64)(n / size));
        stage_twiddles(tw, &step, half);
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t idx = 0; idx < n / 2; idx++) {
            int64_t chunk = idx / half, j = idx % half;
            fp12 *u = &v[chunk * size + j], *w = &v[chunk * size + j + half];
            fp12 t, ti, un;
            if (j == 0) t = *w;
            else fp12_pow_limbs(&t, w, tw[j], 4);
            fp12_inv(&ti, &t);
            fp12_mul(&un, u, &ti);
            fp12_mul(u, u, &t);
            *w = un;
        }
    }
    free(tw);
    memcpy(io, v, sizeof(fp12) * n);
    free(v);
}

/* Truncated, unscaled inverse transform over cyclotomic values with the
 * decomposed twiddle action (btx/src/fft.rs:284-350).  Only the first
 * out_count outputs are meaningful afterwards. */
void orc_cyclotomic_prefix_ifft(u8 *io, int64_t n, int64_t out_count) {
    fp12 *v = (fp12 *)malloc(sizeof(fp12) * n);
    int bits = log2_exact(n);
    fp12 *a = (fp12 *)io;
    for (int64_t i = 0; i < n; i++) v[bitrev(i, bits)] = a[i];
    fr g;
    domain_generator(&g, n, 1);
    cyc_plan *plans = malloc(sizeof(cyc_plan) * (n > 1 ? n / 2 : 1));
    u64(*tw)[4] = malloc(sizeof(u64[4]) * (n > 1 ? n / 2 : 1));
    for (int64_t size = 2; size < n; size *= 2) {
        int64_t half = size / 2;
        fr step;
        fr_pow_u64(&step, &g, (u64)(n / size));
        stage_twiddles(tw, &step, half);
        for (int64_t j = 1; j < half; j++) make_plan(&plans[j], tw[j]);
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t idx = 0; idx < n / 2; idx++) {
            int64_t chunk = idx / half, j = idx % half;
            fp12 *u = &v[chunk * size + j], *w = &v[chunk * size + j + half];
            fp12 t, ti, un;
            if (j == 0) t = *w;
            else cyc_pow_plan(&t, w, &plans[j]);
            fp12_conj(&ti, &t);
            fp12_mul(&un, u, &ti);
            fp12_mul(u, u, &t);
            *w = un;
        }
    }
    if (out_count > 0 && n >= 2) {
        int64_t half = n / 2;
        stage_twiddles(tw, &g, half);
        fp12 *left = v, *right = v + half;
        fp12_mul(&left[0], &left[0], &right[0]);
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t j = 1; j < out_count; j++) {
            cyc_plan pl;
            make_plan(&pl, tw[j]);
            fp12 t;
            cyc_pow_plan(&t, &right[j], &pl);
            fp12_mul(&left[j], &left[j], &t);
        }
    }
    free(tw);
    free(plans);
    memcpy(io, v, sizeof(fp12) * n);
    free(v);
}

/* ---------------- pairing exports ---------------- */
void orc_miller_loop(u8 *out, const u8 *g1, const u8 *g2) {
    miller_loop_affine((fp12 *)out, G1A(g1), G2A(g2));
}
void orc_final_exp(u8 *out, const u8 *in) { final_exp((fp12 *)out, (const fp12 *)in); }
void orc_easy_final_exp(u8 *out, const u8 *in) { easy_part((fp12 *)out, (const fp12 *)in); }
void orc_hard_final_exp(u8 *out, const u8 *in) { hard_part((fp12 *)out, (const fp12 *)in); }
void orc_hard_final_exp_batch(u8 *out, const u8 *in, int64_t n) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < n; i++) hard_part((fp12 *)(out + 576 * i), (const fp12 *)(in + 576 * i));
}
/* Batched easy part sharing one inversion (btx/src/final_exponentiation.rs:281-305). */
void orc_batch_easy_final_exp(u8 *out, const u8 *in, int64_t n) {
    if (n <= 0) return;
    const fp12 *x = (const fp12 *)in;
    fp12 *pre = malloc(sizeof(fp12) * n);
    fp12 prod = FP12_ONE;
    for (int64_t i = 0; i < n; i++) {
        pre[i] = prod;
        fp12_mul(&prod, &prod, &x[i]);
    }
    fp12 pinv;
    fp12_inv(&pinv, &prod);
    for (int64_t i = n - 1; i >= 0; i--) {
        fp12 inv;
        fp12_mul(&inv, &pinv, &pre[i]);
        fp12_mul(&pinv, &pinv, &x[i]);
        easy_part_with_inverse((fp12 *)(out + 576 * i), &x[i], &inv);
    }
    free(pre);
}
void orc_pairing(u8 *out, const u8 *g1, const u8 *g2) {
    fp12 f;
    miller_loop_affine(&f, G1A(g1), G2A(g2));
    final_exp((fp12 *)out, &f);
}
/* out[j] = raw product of Miller loops over pairs [offsets[j], offsets[j+1]);
 * identities contribute 1 (weighted_btx/src/final_exponentiation.rs:229-274). */
void orc_multi_miller_batch(u8 *out, const u8 *g1s, const u8 *g2s, const int64_t *offsets, int64_t k) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t j = 0; j < k; j++) {
        fp12 acc = FP12_ONE, f;
        for (int64_t t = offsets[j]; t < offsets[j + 1]; t++) {
            miller_loop_affine(&f, G1A(g1s + 96 * t), G2A(g2s + 192 * t));
            fp12_mul(&acc, &acc, &f);
        }
        memcpy(out + 576 * j, &acc, 576);
    }
}
void orc_miller_loop_batch(u8 *out, const u8 *g1s, const u8 *g2s, int64_t n) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < n; i++)
        miller_loop_affine((fp12 *)(out + 576 * i), G1A(g1s + 96 * i), G2A(g2s + 192 * i));
}
void orc_final_exp_batch(u8 *out, const u8 *in, int64_t n) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < n; i++) final_exp((fp12 *)(out + 576 * i), (const fp12 *)(in + 576 * i));
}

/* ---------------- Fp12 exports ---------------- */
void orc_fp12_one(u8 *out) { memcpy(out, &FP12_ONE, 576); }
int orc_fp12_is_one(const u8 *a) { return fp12_eq((const fp12 *)a, &FP12_ONE); }
void orc_fp12_mul(u8 *out, const u8 *a, const u8 *b) { fp12_mul((fp12 *)out, (const fp12 *)a, (const fp12 *)b); }
void orc_fp12_inv(u8 *out, const u8 *a) { fp12_inv((fp12 *)out, (const fp12 *)a); }
void orc_fp12_conj(u8 *out, const u8 *a) { fp12_conj((fp12 *)out, (const fp12 *)a); }
void orc_fp12_frobenius(u8 *out, const u8 *a, int k) { fp12_frobenius((fp12 *)out, (const fp12 *)a, k); }
void orc_fp12_pow(u8 *out, const u8 *a, const u8 *exp_le, int nbytes) {
    int nl = (nbytes + 7) / 8;
    u64 *e = calloc(nl, 8);
    memcpy(e, exp_le, nbytes);
    fp12_pow_limbs((fp12 *)out, (const fp12 *)a, e, nl);
    free(e);
}
/* out[i] = in[i]^scalars[i]; base stride 0 => one fixed base */
void orc_gt_pow_batch(u8 *out, const u8 *in, int64_t stride, const u8 *scalars, int64_t n) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < n; i++) {
        u64 e[4];
        memcpy(e, scalars + 32 * i, 32);
        fp12_pow_limbs((fp12 *)(out + 576 * i), (const fp12 *)(in + stride * i), e, 4);
    }
}
void orc_gt_pow_decomposed(u8 *out, const u8 *a, const u8 *scalar32) {
    u64 s[4];
    memcpy(s, scalar32, 32);
    cyc_plan pl;
    make_plan(&pl, s);
    cyc_pow_plan((fp12 *)out, (const fp12 *)a, &pl);
}
void orc_base_x_decompose(u64 *out4, const u8 *scalar32) {
    u64 s[4];
    memcpy(s, scalar32, 32);
    decompose_base_x(out4, s);
}
int orc_wnaf4(int8_t *out65, u64 v) { return wnaf4(out65, v); }

/* ---------------- Lagrange coefficients at zero ---------------- */
/* Direct formula with one batch inversion (weighted_btx/src/interpolation.rs:67-98). */
int orc_lagrange_at_zero(u8 *out, const u8 *points, int64_t n) {
    fr *x = malloc(sizeof(fr) * n), *num = malloc(sizeof(fr) * n), *den = malloc(sizeof(fr) * n);
    for (int64_t i = 0; i < n; i++) fr_load(&x[i], points + 32 * i);
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(| : bad)
    for (int64_t i = 0; i < n; i++) {
        fr a = FR_ONE, b = FR_ONE, t;
        for (int64_t k = 0; k < n; k++) {
            if (k == i) continue;
            fr_neg(&t, &x[k]);
            fr_mul(&a, &a, &t);
            fr_sub(&t, &x[i], &x[k]);
            fr_mul(&b, &b, &t);
        }
        num[i] = a;
        den[i] = b;
        if (fr_is_zero(&b)) bad = 1;
    }
    if (!bad) {
        for (int64_t i = 0; i < n; i++) {
            fr inv;
            fr_inv(&inv, &den[i]);
            fr_mul(&num[i], &num[i], &inv);
            fr_store(out + 32 * i, &num[i]);
        }
    }
    free(x);
    free(num);
    free(den);
    return bad ? -1 : 0;
}

/* ---------------- formula checks ---------------- */
/* Granger-Scott cyclotomic squaring, restated so that the CPU suite can check
 * the formula against the ordinary square on cyclotomic elements. */
static void fp4_sqr_chk(fp2 *c0, fp2 *c1, const fp2 *a, const fp2 *b) {
    fp2 t0, t1, t2;
    fp2_sqr(&t0, a);
    fp2_sqr(&t1, b);
    fp2_mul_xi(&t2, &t1);
    fp2_add(c0, &t2, &t0);
    fp2_add(&t2, a, b);
    fp2_sqr(&t2, &t2);
    fp2_sub(&t2, &t2, &t0);
    fp2_sub(c1, &t2, &t1);
}
void orc_cyclotomic_sqr_gs(u8 *out, const u8 *in) {
    const fp12 *f = (const fp12 *)in;
    fp2 z0 = f->c0.c0, z4 = f->c0.c1, z3 = f->c0.c2, z2 = f->c1.c0, z1 = f->c1.c1, z5 = f->c1.c2;
    fp2 t0, t1, t2, t3;
    fp4_sqr_chk(&t0, &t1, &z0, &z1);
    fp2_sub(&z0, &t0, &z0); fp2_add(&z0, &z0, &z0); fp2_add(&z0, &z0, &t0);
    fp2_add(&z1, &t1, &z1); fp2_add(&z1, &z1, &z1); fp2_add(&z1, &z1, &t1);
    fp4_sqr_chk(&t0, &t1, &z2, &z3);
    fp4_sqr_chk(&t2, &t3, &z4, &z5);
    fp2_sub(&z4, &t0, &z4); fp2_add(&z4, &z4, &z4); fp2_add(&z4, &z4, &t0);
    fp2_add(&z5, &t1, &z5); fp2_add(&z5, &z5, &z5); fp2_add(&z5, &z5, &t1);
    fp2_mul_xi(&t0, &t3);
    fp2_add(&z2, &t0, &z2); fp2_add(&z2, &z2, &z2); fp2_add(&z2, &z2, &t0);
    fp2_sub(&z3, &t2, &z3); fp2_add(&z3, &z3, &z3); fp2_add(&z3, &z3, &t2);
    fp12 r;
    r.c0.c0 = z0; r.c0.c1 = z4; r.c0.c2 = z3; r.c1.c0 = z2; r.c1.c1 = z1; r.c1.c2 = z5;
    memcpy(out, &r, 576);
}

/* Homogeneous-projective line formulas (the shape the GPU kernels use),
 * restated so the CPU suite can check that their final-exponentiated
 * Miller value equals the affine loop's. */
static void fp2_small(fp2 *o, const fp2 *a, int k) {
    fp2 r = FP2_ZERO;
    for (int i = 0; i < k; i++) fp2_add(&r, &r, a);
    *o = r;
}
void orc_miller_loop_projective_check(u8 *out, const u8 *g1, const u8 *g2) {
    const g1a *P = G1A(g1);
    const g2a *Q = G2A(g2);
    fp12 f = FP12_ONE;
    if (g1a_is_inf(P) || g2a_is_inf(Q)) { memcpy(out, &f, 576); return; }
    fp2 X = Q->x, Y = Q->y, Z = FP2_ONE;
    fp2 a0, a1, b1, t0, t1, t2, X2, YZ, XY, t, t23;
    for (int i = 62; i >= 0; i--) {
        if (i != 62) fp12_sqr(&f, &f);
        fp2_sqr(&t0, &Y);
        fp2_sqr(&t1, &Z);
        fp2_mul_xi(&t2, &t1);
        fp2_small(&t2, &t2, 12);
        fp2_sqr(&X2, &X);
        fp2_mul(&YZ, &Y, &Z);
        fp2_mul(&XY, &X, &Y);
        fp2_sub(&a0, &t2, &t0);
        fp2_small(&t, &X2, 3);
        fp2_mul_fp(&a1, &t, &P->x);
        fp2_small(&t, &YZ, 2);
        fp2_neg(&t, &t);
        fp2_mul_fp(&b1, &t, &P->y);
        { fp12 l; memset(&l, 0, sizeof l); l.c0.c0 = a0; l.c0.c1 = a1; l.c1.c1 = b1; fp12_mul(&f, &f, &l); }
        fp2_small(&t23, &t2, 3);
        fp2_sub(&t, &t0, &t23);
        fp2_mul(&t, &XY, &t);
        fp2_small(&X, &t, 2);
        fp2_add(&t, &t0, &t23);
        fp2_sqr(&t, &t);
        fp2 s;
        fp2_sqr(&s, &t2);
        fp2_small(&s, &s, 12);
        fp2_sub(&Y, &t, &s);
        fp2_mul(&t, &t0, &YZ);
        fp2_small(&Z, &t, 8);
        if ((X_ABS >> i) & 1) {
            fp2 u, v, v2, v3, v2X, A;
            fp2_mul(&u, &Q->y, &Z); fp2_sub(&u, &u, &Y);
            fp2_mul(&v, &Q->x, &Z); fp2_sub(&v, &v, &X);
            fp2_mul(&a0, &u, &Q->x); fp2_mul(&t, &v, &Q->y); fp2_sub(&a0, &a0, &t);
            fp2_neg(&t, &u); fp2_mul_fp(&a1, &t, &P->x);
            fp2_mul_fp(&b1, &v, &P->y);
            { fp12 l; memset(&l, 0, sizeof l); l.c0.c0 = a0; l.c0.c1 = a1; l.c1.c1 = b1; fp12_mul(&f, &f, &l); }
            fp2_sqr(&v2, &v); fp2_mul(&v3, &v2, &v); fp2_mul(&v2X, &v2, &X);
            fp2_sqr(&A, &u); fp2_mul(&A, &A, &Z); fp2_sub(&A, &A, &v3); fp2_sub(&A, &A, &v2X); fp2_sub(&A, &A, &v2X);
            fp2_mul(&X, &v, &A);
            fp2_sub(&t, &v2X, &A); fp2_mul(&t, &u, &t); fp2 w3; fp2_mul(&w3, &v3, &Y); fp2_sub(&Y, &t, &w3);
            fp2_mul(&Z, &v3, &Z);
        }
    }
    fp12_conj((fp12 *)out, &f);
}

/* Tagged torus encoding of GT (append_gt, weighted_btx/src/encoding.rs:11-19):
 * identity -> 0 followed by zeros; else 1 followed by the Fp2 coefficients of
 * (c0 + 1) / c1, each Fp as 48 big-endian bytes (289 bytes in total). */
void orc_gt_compress(u8 *out289, const u8 *in576) {
    const fp12 *f = (const fp12 *)in576;
    memset(out289, 0, 289);
    if (fp12_eq(f, &FP12_ONE)) return;
    fp6 c0 = f->c0, inv, b;
    fp2_add(&c0.c0, &c0.c0, &FP2_ONE);
    fp6_inv(&inv, &f->c1);
    fp6_mul(&b, &c0, &inv);
    out289[0] = 1;
    const fp2 *cs[3] = {&b.c0, &b.c1, &b.c2};
    for (int k = 0; k < 3; k++) {
        fp_to_be48(out289 + 1 + 96 * k, &cs[k]->c0);
        fp_to_be48(out289 + 1 + 96 * k + 48, &cs[k]->c1);
    }
}

/* Fixed-base multiples of the generators with an 8-bit comb:
 * T[w][d] = d * 2^(8w) * G, so [s]G is the sum of T[w][byte w of s]. */
static g1j *G1_TAB = NULL;
static g2j *G2_TAB = NULL;
static void build_tables(void) {
#pragma omp critical(orc_tables)
    {
        if (!G1_TAB) {
            g1j *t1 = malloc(sizeof(g1j) * 32 * 256);
            g2j *t2 = malloc(sizeof(g2j) * 32 * 256);
            g1j b1;
            g2j b2;
            g1_from_affine(&b1, &G1_GEN);
            g2_from_affine(&b2, &G2_GEN);
            for (int w = 0; w < 32; w++) {
                memset(&t1[256 * w], 0, sizeof(g1j));
                memset(&t2[256 * w], 0, sizeof(g2j));
                for (int d = 1; d < 256; d++) {
                    g1_add(&t1[256 * w + d], &t1[256 * w + d - 1], &b1);
                    g2_add(&t2[256 * w + d], &t2[256 * w + d - 1], &b2);
                }
                for (int i = 0; i < 8; i++) {
                    g1_dbl(&b1, &b1);
                    g2_dbl(&b2, &b2);
                }
            }
            G2_TAB = t2;
            G1_TAB = t1;
        }
    }
}
void orc_g1_mul_generator_batch(u8 *out, const u8 *scalars, int64_t n) {
    build_tables();
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; i++) {
        g1j acc;
        memset(&acc, 0, sizeof acc);
        const u8 *s = scalars + 32 * i;
        for (int w = 0; w < 32; w++)
            if (s[w]) g1_add(&acc, &acc, &G1_TAB[256 * w + s[w]]);
        g1_to_affine(G1A(out + 96 * i), &acc);
    }
}
void orc_g2_mul_generator_batch(u8 *out, const u8 *scalars, int64_t n) {
    build_tables();
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; i++) {
        g2j acc;
        memset(&acc, 0, sizeof acc);
        const u8 *s = scalars + 32 * i;
        for (int w = 0; w < 32; w++)
            if (s[w]) g2_add(&acc, &acc, &G2_TAB[256 * w + s[w]]);
        g2_to_affine(G2A(out + 192 * i), &acc);
    }
}
