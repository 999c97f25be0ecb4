// BLS12-381 field tower for sm_100a: Fp (12 x 32-bit Montgomery limbs,
// R = 2^384, byte-identical to blst's blst_fp), Fr (8 x 32-bit limbs),
// Fp2 = Fp[u]/(u^2+1), Fp6 = Fp2[v]/(v^3-(1+u)), Fp12 = Fp6[w]/(w^2-v).
//
// Fp operations are inlined single PTX blocks (field_asm.cuh).  Fp2 products
// are inlined; Fp6/Fp12 products are out-of-line so that kernels built from
// them stay within the instruction cache.
#pragma once
#include <cstdint>
#include "field_asm.cuh"
#include "constants.cuh"

#define WBTE_INL __device__ __forceinline__
#define WBTE_NOINL static __device__ __noinline__

namespace wbte {

struct Fp { uint32_t v[12]; };
struct Fr { uint32_t v[8]; };
struct Fp2 { Fp c0, c1; };
struct Fp6 { Fp2 c0, c1, c2; };
struct Fp12 { Fp6 c0, c1; };

// ------------------------------------------------------------------ Fp
WBTE_INL Fp fp_zero() { Fp r; _Pragma("unroll") for (int i = 0; i < 12; i++) r.v[i] = 0; return r; }
WBTE_INL Fp fp_one() { Fp r; _Pragma("unroll") for (int i = 0; i < 12; i++) r.v[i] = C_FP_ONE[i]; return r; }
#if defined(WBTE_FP_NOINLINE)
// One out-of-line copy of the 12-limb product keeps every kernel's hot loop
// inside the instruction cache.
#if defined(WBTE_FP_ROLLED) && WBTE_FP_ROLLED == 4
// the same product as a loop of rows, WBTE_FP_ROLLED rows per iteration:
// less code per product for kernels bound by instruction fetch
static __device__ __noinline__ Fp fp_mul_ool(Fp a, Fp b) { Fp r; fp_mont_mul_r4(r.v, a.v, b.v); return r; }
#elif defined(WBTE_FP_ROLLED) && WBTE_FP_ROLLED == 6
static __device__ __noinline__ Fp fp_mul_ool(Fp a, Fp b) { Fp r; fp_mont_mul_r6(r.v, a.v, b.v); return r; }
#else
static __device__ __noinline__ Fp fp_mul_ool(Fp a, Fp b) { Fp r; fp_mont_mul(r.v, a.v, b.v); return r; }
#endif
WBTE_INL Fp fp_mul(const Fp& a, const Fp& b) { return fp_mul_ool(a, b); }
WBTE_INL Fp fp_sqr(const Fp& a) { return fp_mul_ool(a, a); }
#else
WBTE_INL Fp fp_mul(const Fp& a, const Fp& b) { Fp r; fp_mont_mul(r.v, a.v, b.v); return r; }
WBTE_INL Fp fp_sqr(const Fp& a) { Fp r; fp_mont_mul(r.v, a.v, a.v); return r; }
#endif
#if defined(WBTE_FPADD_NOINLINE)
// out-of-line sums: smaller code for kernels bound by instruction fetch
static __device__ __noinline__ Fp fp_add_ool(Fp a, Fp b) { Fp r; fp_add_raw(r.v, a.v, b.v); return r; }
static __device__ __noinline__ Fp fp_sub_ool(Fp a, Fp b) { Fp r; fp_sub_raw(r.v, a.v, b.v); return r; }
WBTE_INL Fp fp_add(const Fp& a, const Fp& b) { return fp_add_ool(a, b); }
WBTE_INL Fp fp_sub(const Fp& a, const Fp& b) { return fp_sub_ool(a, b); }
#else
WBTE_INL Fp fp_add(const Fp& a, const Fp& b) { Fp r; fp_add_raw(r.v, a.v, b.v); return r; }
WBTE_INL Fp fp_sub(const Fp& a, const Fp& b) { Fp r; fp_sub_raw(r.v, a.v, b.v); return r; }
#endif
// a + b without reduction: only valid as a multiplication input (< 2p).
WBTE_INL Fp fp_add_lazy(const Fp& a, const Fp& b) { Fp r; fp_add_nored(r.v, a.v, b.v); return r; }
WBTE_INL Fp fp_dbl(const Fp& a) { return fp_add(a, a); }
WBTE_INL Fp fp_neg(const Fp& a) { return fp_sub(fp_zero(), a); }
WBTE_INL bool fp_is_zero(const Fp& a) {
    uint32_t x = 0;
    _Pragma("unroll") for (int i = 0; i < 12; i++) x |= a.v[i];
    return x == 0;
}
WBTE_INL bool fp_eq(const Fp& a, const Fp& b) {
    uint32_t x = 0;
    _Pragma("unroll") for (int i = 0; i < 12; i++) x |= a.v[i] ^ b.v[i];
    return x == 0;
}
WBTE_INL Fp fp_from_const(const uint32_t (&c)[12]) {
    Fp r;
    _Pragma("unroll") for (int i = 0; i < 12; i++) r.v[i] = c[i];
    return r;
}
// canonical (non-Montgomery) value of a
WBTE_INL Fp fp_from_mont(const Fp& a) {
    Fp one = fp_zero();
    one.v[0] = 1;
    return fp_mul(a, one);
}
WBTE_INL Fp fp_to_mont(const Fp& a) { return fp_mul(a, fp_from_const(C_FP_R2)); }

// ------------------------------------------------------------------ Fr
WBTE_INL Fr fr_zero() { Fr r; _Pragma("unroll") for (int i = 0; i < 8; i++) r.v[i] = 0; return r; }
WBTE_INL Fr fr_one() { Fr r; _Pragma("unroll") for (int i = 0; i < 8; i++) r.v[i] = C_FR_ONE[i]; return r; }
WBTE_INL Fr fr_mul(const Fr& a, const Fr& b) { Fr r; fr_mont_mul(r.v, a.v, b.v); return r; }
WBTE_INL Fr fr_add(const Fr& a, const Fr& b) { Fr r; fr_add_raw(r.v, a.v, b.v); return r; }
WBTE_INL Fr fr_sub(const Fr& a, const Fr& b) { Fr r; fr_sub_raw(r.v, a.v, b.v); return r; }
WBTE_INL Fr fr_neg(const Fr& a) { return fr_sub(fr_zero(), a); }
WBTE_INL bool fr_is_zero(const Fr& a) {
    uint32_t x = 0;
    _Pragma("unroll") for (int i = 0; i < 8; i++) x |= a.v[i];
    return x == 0;
}
WBTE_INL Fr fr_to_mont(const Fr& a) {
    Fr r2;
    _Pragma("unroll") for (int i = 0; i < 8; i++) r2.v[i] = C_FR_R2[i];
    return fr_mul(a, r2);
}
WBTE_INL Fr fr_from_mont(const Fr& a) {
    Fr one = fr_zero();
    one.v[0] = 1;
    return fr_mul(a, one);
}
// Montgomery-form power by a small exponent
WBTE_INL Fr fr_pow_u64(Fr base, uint64_t e) {
    Fr r = fr_one();
    while (e) {
        if (e & 1) r = fr_mul(r, base);
        base = fr_mul(base, base);
        e >>= 1;
    }
    return r;
}

// ----------------------------------------------------------------- Fp2
WBTE_INL Fp2 fp2_zero() { return Fp2{fp_zero(), fp_zero()}; }
WBTE_INL Fp2 fp2_one() { return Fp2{fp_one(), fp_zero()}; }
WBTE_INL Fp2 fp2_add(const Fp2& a, const Fp2& b) { return Fp2{fp_add(a.c0, b.c0), fp_add(a.c1, b.c1)}; }
WBTE_INL Fp2 fp2_sub(const Fp2& a, const Fp2& b) { return Fp2{fp_sub(a.c0, b.c0), fp_sub(a.c1, b.c1)}; }
WBTE_INL Fp2 fp2_dbl(const Fp2& a) { return Fp2{fp_dbl(a.c0), fp_dbl(a.c1)}; }
WBTE_INL Fp2 fp2_neg(const Fp2& a) { return Fp2{fp_neg(a.c0), fp_neg(a.c1)}; }
WBTE_INL Fp2 fp2_conj(const Fp2& a) { return Fp2{a.c0, fp_neg(a.c1)}; }
WBTE_INL bool fp2_is_zero(const Fp2& a) { return fp_is_zero(a.c0) && fp_is_zero(a.c1); }
WBTE_INL bool fp2_eq(const Fp2& a, const Fp2& b) { return fp_eq(a.c0, b.c0) && fp_eq(a.c1, b.c1); }
#if defined(WBTE_FP2_NOINLINE) || defined(WBTE_FP2_LAZY)
#define WBTE_FP2_MUL static __device__ __noinline__
#else
#define WBTE_FP2_MUL WBTE_INL
#endif
#if defined(WBTE_FP2_LAZY)
// Karatsuba with lazy reduction (field_asm.cuh): three double-width products
// and two Montgomery reductions, 1,464 multiply-adds instead of 1,764.  One
// out-of-line copy: the block is about 1,800 instructions.
WBTE_FP2_MUL Fp2 fp2_mul(const Fp2& a, const Fp2& b) {
    Fp2 r;
    fp2_mont_mul_lazy(r.c0.v, r.c1.v, a.c0.v, a.c1.v, b.c0.v, b.c1.v);
    return r;
}
#else
// Karatsuba: 3 Fp products; the operand sums stay unreduced (< 2p).
WBTE_FP2_MUL Fp2 fp2_mul(const Fp2& a, const Fp2& b) {
    Fp t0 = fp_mul(a.c0, b.c0);
    Fp t1 = fp_mul(a.c1, b.c1);
    Fp t2 = fp_mul(fp_add_lazy(a.c0, a.c1), fp_add_lazy(b.c0, b.c1));
    return Fp2{fp_sub(t0, t1), fp_sub(fp_sub(t2, t0), t1)};
}
#endif
// (a0 + a1 u)^2 = (a0 + a1)(a0 - a1) + 2 a0 a1 u
WBTE_FP2_MUL Fp2 fp2_sqr(const Fp2& a) {
    Fp t = fp_mul(a.c0, a.c1);
    Fp c0 = fp_mul(fp_add_lazy(a.c0, a.c1), fp_sub(a.c0, a.c1));
    return Fp2{c0, fp_dbl(t)};
}
WBTE_INL Fp2 fp2_mul_fp(const Fp2& a, const Fp& b) { return Fp2{fp_mul(a.c0, b), fp_mul(a.c1, b)}; }
// multiply by xi = 1 + u
WBTE_INL Fp2 fp2_mul_xi(const Fp2& a) { return Fp2{fp_sub(a.c0, a.c1), fp_add(a.c0, a.c1)}; }
WBTE_INL Fp2 fp2_from_const(const uint32_t (&c)[2][12]) { return Fp2{fp_from_const(c[0]), fp_from_const(c[1])}; }

// ----------------------------------------------------------------- Fp6
WBTE_INL Fp6 fp6_zero() { return Fp6{fp2_zero(), fp2_zero(), fp2_zero()}; }
WBTE_INL Fp6 fp6_one() { return Fp6{fp2_one(), fp2_zero(), fp2_zero()}; }
WBTE_INL Fp6 fp6_add(const Fp6& a, const Fp6& b) { return Fp6{fp2_add(a.c0, b.c0), fp2_add(a.c1, b.c1), fp2_add(a.c2, b.c2)}; }
WBTE_INL Fp6 fp6_sub(const Fp6& a, const Fp6& b) { return Fp6{fp2_sub(a.c0, b.c0), fp2_sub(a.c1, b.c1), fp2_sub(a.c2, b.c2)}; }
WBTE_INL Fp6 fp6_neg(const Fp6& a) { return Fp6{fp2_neg(a.c0), fp2_neg(a.c1), fp2_neg(a.c2)}; }
// (c0 + c1 v + c2 v^2) v = xi c2 + c0 v + c1 v^2
WBTE_INL Fp6 fp6_mul_v(const Fp6& a) { return Fp6{fp2_mul_xi(a.c2), a.c0, a.c1}; }

// ---------------------------------------------------------------- Fp12
WBTE_INL Fp12 fp12_one() { return Fp12{fp6_one(), fp6_zero()}; }
WBTE_INL void fp12_conj(Fp12& r, const Fp12& a) { r.c0 = a.c0; r.c1 = fp6_neg(a.c1); }
WBTE_INL bool fp12_is_one(const Fp12& a) {
    Fp12 one = fp12_one();
    const uint32_t* x = reinterpret_cast<const uint32_t*>(&a);
    const uint32_t* y = reinterpret_cast<const uint32_t*>(&one);
    uint32_t d = 0;
    for (int i = 0; i < 144; i++) d |= x[i] ^ y[i];
    return d == 0;
}

}  // namespace wbte

#include "fields_impl.cuh"
