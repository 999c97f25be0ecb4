// G1 (y^2 = x^3 + 4 over Fp) and G2 (y^2 = x^3 + 4(1+u) over Fp2) in
// extended Jacobian "XYZZ" coordinates: x = X/ZZ, y = Y/ZZZ, ZZ^3 = ZZZ^2,
// ZZ = 0 for the point at infinity.  Affine points use blst's layout and the
// all-zero encoding for infinity.  Formulas (a = 0): dbl-2008-s-1,
// madd-2008-s, add-2008-s of the Explicit-Formulas Database.
#pragma once
#include "fields.cuh"

namespace wbte {

// ------------------------------------------------------- field overloads
WBTE_INL Fp f_add(const Fp& a, const Fp& b) { return fp_add(a, b); }
WBTE_INL Fp f_sub(const Fp& a, const Fp& b) { return fp_sub(a, b); }
WBTE_INL Fp f_mul(const Fp& a, const Fp& b) { return fp_mul(a, b); }
WBTE_INL Fp f_sqr(const Fp& a) { return fp_sqr(a); }
WBTE_INL Fp f_dbl(const Fp& a) { return fp_dbl(a); }
WBTE_INL Fp f_neg(const Fp& a) { return fp_neg(a); }
WBTE_INL bool f_is_zero(const Fp& a) { return fp_is_zero(a); }
WBTE_INL Fp f_inv(const Fp& a) { return fp_inv(a); }
WBTE_INL void f_set_zero(Fp& a) { a = fp_zero(); }
WBTE_INL void f_set_one(Fp& a) { a = fp_one(); }
WBTE_INL Fp2 f_add(const Fp2& a, const Fp2& b) { return fp2_add(a, b); }
WBTE_INL Fp2 f_sub(const Fp2& a, const Fp2& b) { return fp2_sub(a, b); }
WBTE_INL Fp2 f_mul(const Fp2& a, const Fp2& b) { return fp2_mul(a, b); }
WBTE_INL Fp2 f_sqr(const Fp2& a) { return fp2_sqr(a); }
WBTE_INL Fp2 f_dbl(const Fp2& a) { return fp2_dbl(a); }
WBTE_INL Fp2 f_neg(const Fp2& a) { return fp2_neg(a); }
WBTE_INL bool f_is_zero(const Fp2& a) { return fp2_is_zero(a); }
WBTE_INL Fp2 f_inv(const Fp2& a) { return fp2_inv(a); }
WBTE_INL void f_set_zero(Fp2& a) { a = fp2_zero(); }
WBTE_INL void f_set_one(Fp2& a) { a = fp2_one(); }

template <class F> struct Affine { F x, y; };
template <class F> struct Xyzz { F X, Y, ZZ, ZZZ; };

using G1A = Affine<Fp>;
using G2A = Affine<Fp2>;
using G1X = Xyzz<Fp>;
using G2X = Xyzz<Fp2>;

template <class F> WBTE_INL bool is_inf(const Affine<F>& a) { return f_is_zero(a.x) && f_is_zero(a.y); }
template <class F> WBTE_INL bool is_inf(const Xyzz<F>& a) { return f_is_zero(a.ZZ); }
template <class F> WBTE_INL void set_inf(Xyzz<F>& a) { f_set_zero(a.X); f_set_one(a.Y); f_set_zero(a.ZZ); f_set_zero(a.ZZZ); }
template <class F> WBTE_INL void set_inf(Affine<F>& a) { f_set_zero(a.x); f_set_zero(a.y); }
template <class F> WBTE_INL Xyzz<F> from_affine(const Affine<F>& a) {
    Xyzz<F> r;
    if (is_inf(a)) { set_inf(r); return r; }
    r.X = a.x; r.Y = a.y; f_set_one(r.ZZ); f_set_one(r.ZZZ);
    return r;
}
template <class F> WBTE_INL Affine<F> neg(const Affine<F>& a) {
    Affine<F> r = a;
    if (!is_inf(a)) r.y = f_neg(a.y);
    return r;
}
template <class F> WBTE_INL Xyzz<F> neg(const Xyzz<F>& a) {
    Xyzz<F> r = a;
    r.Y = f_neg(a.Y);
    return r;
}

// 2P
template <class F> static __device__ __noinline__ Xyzz<F> xyzz_dbl(const Xyzz<F> p) {
    if (is_inf(p)) return p;
    F U = f_dbl(p.Y);
    F V = f_sqr(U);
    F W = f_mul(U, V);
    F S = f_mul(p.X, V);
    F X2 = f_sqr(p.X);
    F M = f_add(f_dbl(X2), X2);
    Xyzz<F> r;
    r.X = f_sub(f_sub(f_sqr(M), S), S);
    r.Y = f_sub(f_mul(M, f_sub(S, r.X)), f_mul(W, p.Y));
    r.ZZ = f_mul(V, p.ZZ);
    r.ZZZ = f_mul(W, p.ZZZ);
    return r;
}

// 2Q for affine Q (ZZ = ZZZ = 1)
template <class F> WBTE_INL Xyzz<F> xyzz_mdbl(const Affine<F>& q) {
    Xyzz<F> r;
    if (is_inf(q)) { set_inf(r); return r; }
    F U = f_dbl(q.y);
    F V = f_sqr(U);
    F W = f_mul(U, V);
    F S = f_mul(q.x, V);
    F X2 = f_sqr(q.x);
    F M = f_add(f_dbl(X2), X2);
    r.X = f_sub(f_sub(f_sqr(M), S), S);
    r.Y = f_sub(f_mul(M, f_sub(S, r.X)), f_mul(W, q.y));
    r.ZZ = V;
    r.ZZZ = W;
    return r;
}

// P + Q for affine Q
template <class F> static __device__ __noinline__ Xyzz<F> xyzz_madd(const Xyzz<F> p, const Affine<F> q) {
    if (is_inf(q)) return p;
    if (is_inf(p)) return from_affine(q);
    F U2 = f_mul(q.x, p.ZZ);
    F S2 = f_mul(q.y, p.ZZZ);
    F P = f_sub(U2, p.X);
    F R = f_sub(S2, p.Y);
    if (f_is_zero(P)) {
        if (f_is_zero(R)) return xyzz_mdbl(q);
        Xyzz<F> r;
        set_inf(r);
        return r;
    }
    F PP = f_sqr(P);
    F PPP = f_mul(P, PP);
    F Q = f_mul(p.X, PP);
    Xyzz<F> r;
    r.X = f_sub(f_sub(f_sub(f_sqr(R), PPP), Q), Q);
    r.Y = f_sub(f_mul(R, f_sub(Q, r.X)), f_mul(p.Y, PPP));
    r.ZZ = f_mul(p.ZZ, PP);
    r.ZZZ = f_mul(p.ZZZ, PPP);
    return r;
}

// P + Q
template <class F> static __device__ __noinline__ Xyzz<F> xyzz_add(const Xyzz<F> p, const Xyzz<F> q) {
    if (is_inf(q)) return p;
    if (is_inf(p)) return q;
    F U1 = f_mul(p.X, q.ZZ);
    F U2 = f_mul(q.X, p.ZZ);
    F S1 = f_mul(p.Y, q.ZZZ);
    F S2 = f_mul(q.Y, p.ZZZ);
    F P = f_sub(U2, U1);
    F R = f_sub(S2, S1);
    if (f_is_zero(P)) {
        if (f_is_zero(R)) return xyzz_dbl(p);
        Xyzz<F> r;
        set_inf(r);
        return r;
    }
    F PP = f_sqr(P);
    F PPP = f_mul(P, PP);
    F Q = f_mul(U1, PP);
    Xyzz<F> r;
    r.X = f_sub(f_sub(f_sub(f_sqr(R), PPP), Q), Q);
    r.Y = f_sub(f_mul(R, f_sub(Q, r.X)), f_mul(S1, PPP));
    r.ZZ = f_mul(f_mul(p.ZZ, q.ZZ), PP);
    r.ZZZ = f_mul(f_mul(p.ZZZ, q.ZZZ), PPP);
    return r;
}

template <class F> static __device__ __noinline__ Affine<F> to_affine(const Xyzz<F> p) {
    Affine<F> r;
    if (is_inf(p)) { set_inf(r); return r; }
    F t = f_inv(f_mul(p.ZZ, p.ZZZ));
    r.x = f_mul(p.X, f_mul(t, p.ZZZ));
    r.y = f_mul(p.Y, f_mul(t, p.ZZ));
    return r;
}

// [k]P for a canonical scalar given as 8 little-endian 32-bit words, with a
// 4-bit fixed window over an XYZZ table.
template <class F> static __device__ __noinline__ Xyzz<F> xyzz_mul(const Xyzz<F> p, const uint32_t k[8]) {
    Xyzz<F> tab[16];
    set_inf(tab[0]);
    tab[1] = p;
    tab[2] = xyzz_dbl(p);
    for (int i = 3; i < 16; i++) tab[i] = xyzz_add(tab[i - 1], p);
    Xyzz<F> acc;
    set_inf(acc);
    for (int w = 63; w >= 0; w--) {
        acc = xyzz_dbl(acc);
        acc = xyzz_dbl(acc);
        acc = xyzz_dbl(acc);
        acc = xyzz_dbl(acc);
        uint32_t d = (k[w >> 3] >> (4 * (w & 7))) & 15u;
        if (d) acc = xyzz_add(acc, tab[d]);
    }
    return acc;
}

// [k]P for a scalar of at most 64 bits
template <class F> static __device__ __noinline__ Xyzz<F> xyzz_mul_u64(const Xyzz<F> p, uint64_t k) {
    Xyzz<F> acc;
    set_inf(acc);
    for (int i = 63; i >= 0; i--) {
        acc = xyzz_dbl(acc);
        if ((k >> i) & 1) acc = xyzz_add(acc, p);
    }
    return acc;
}

// Point loads and stores in blst's affine layout (16-byte vector accesses).
template <class A> WBTE_INL A load_affine(const A* ptr) {
    A r;
    const uint4* s = reinterpret_cast<const uint4*>(ptr);
    uint4* d = reinterpret_cast<uint4*>(&r);
    _Pragma("unroll") for (int i = 0; i < (int)(sizeof(A) / 16); i++) d[i] = __ldg(s + i);
    return r;
}
template <class A> WBTE_INL void store_affine(A* ptr, const A& v) {
    uint4* d = reinterpret_cast<uint4*>(ptr);
    const uint4* s = reinterpret_cast<const uint4*>(&v);
    _Pragma("unroll") for (int i = 0; i < (int)(sizeof(A) / 16); i++) d[i] = s[i];
}
template <class T> WBTE_INL T load_vec(const T* ptr) {
    T r;
    const uint4* s = reinterpret_cast<const uint4*>(ptr);
    uint4* d = reinterpret_cast<uint4*>(&r);
    _Pragma("unroll") for (int i = 0; i < (int)(sizeof(T) / 16); i++) d[i] = s[i];
    return r;
}
template <class T> WBTE_INL void store_vec(T* ptr, const T& v) {
    uint4* d = reinterpret_cast<uint4*>(ptr);
    const uint4* s = reinterpret_cast<const uint4*>(&v);
    _Pragma("unroll") for (int i = 0; i < (int)(sizeof(T) / 16); i++) d[i] = s[i];
}

WBTE_INL G1A g1_generator() {
    G1A g;
    g.x = fp_from_const(C_G1_GEN[0]);
    g.y = fp_from_const(C_G1_GEN[1]);
    return g;
}
WBTE_INL G2A g2_generator() {
    G2A g;
    g.x = Fp2{fp_from_const(C_G2_GEN[0]), fp_from_const(C_G2_GEN[1])};
    g.y = Fp2{fp_from_const(C_G2_GEN[2]), fp_from_const(C_G2_GEN[3])};
    return g;
}

// canonical scalar words from a 32-byte little-endian encoding
WBTE_INL void load_scalar(uint32_t k[8], const uint8_t* bytes) {
    const uint4* s = reinterpret_cast<const uint4*>(bytes);
    uint4 a = s[0], b = s[1];
    k[0] = a.x; k[1] = a.y; k[2] = a.z; k[3] = a.w;
    k[4] = b.x; k[5] = b.y; k[6] = b.z; k[7] = b.w;
}

}  // namespace wbte
