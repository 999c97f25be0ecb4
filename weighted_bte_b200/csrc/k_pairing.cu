// Pairing-side kernels: G2 line tables, Miller loops, split final
// exponentiation and the GT element kernels (products, masks, encodings).
// The GT transforms live in k_gt.cu.
#include <algorithm>
#include <cstdlib>

#include "launch.h"
#include "pairing.cuh"

namespace wbte {

namespace {
constexpr int TPB = 64;
inline unsigned blocks_for(int64_t n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

WBTE_INL Fp12* as_gt(uint8_t* p) { return reinterpret_cast<Fp12*>(p); }
WBTE_INL const Fp12* as_gt(const uint8_t* p) { return reinterpret_cast<const Fp12*>(p); }

// resident 64-thread blocks per SM the Miller-loop and final-exponentiation
// kernels are compiled for (0: no bound, the compiler's 255 registers)
#ifndef WBTE_PAIR_MINBLOCKS
#define WBTE_PAIR_MINBLOCKS 0
#endif
#if WBTE_PAIR_MINBLOCKS > 0
#define WBTE_PAIR_BOUNDS __launch_bounds__(TPB, WBTE_PAIR_MINBLOCKS)
#else
#define WBTE_PAIR_BOUNDS
#endif

__global__ void k_prepare_lines(uint8_t* lines, const uint8_t* q, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Line* L = reinterpret_cast<Line*>(lines);
    G2A Q = load_affine(reinterpret_cast<const G2A*>(q + G2_AFF * i));
    if (is_inf(Q)) {
        // identity lines: every line value is 1, so the loop returns 1
        Line one{fp2_one(), fp2_zero(), fp2_zero()};
        for (int s = 0; s < MILLER_LINES; s++) store_vec(L + (int64_t)s * n + i, one);
        return;
    }
    G2Proj T = g2proj_from_affine(Q);
    int idx = 0;
    for (int b = 62; b >= 0; b--) {
        store_vec(L + (int64_t)(idx++) * n + i, line_double(T));
        if ((X_ABS >> b) & 1) store_vec(L + (int64_t)(idx++) * n + i, line_add(T, Q));
    }
}

// pair i uses line table i % lines_n (tables stored line-major, stride lines_n)
__global__ void WBTE_PAIR_BOUNDS k_miller_lines(uint8_t* out, const uint8_t* lines, const uint8_t* p, int64_t n, int64_t lines_n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    G1A P = load_affine(reinterpret_cast<const G1A*>(p + G1_AFF * i));
    Fp12 f;
    miller_loop_lines(f, reinterpret_cast<const Line*>(lines) + i % lines_n, (size_t)lines_n, P);
    store_vec(as_gt(out) + i, f);
}

__global__ void WBTE_PAIR_BOUNDS k_miller(uint8_t* out, const uint8_t* p, const uint8_t* q, int64_t n, int64_t p_mod, int64_t q_mod) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    G1A P = load_affine(reinterpret_cast<const G1A*>(p + G1_AFF * (p_mod ? i % p_mod : i)));
    G2A Q = load_affine(reinterpret_cast<const G2A*>(q + G2_AFF * (q_mod ? i % q_mod : i)));
    Fp12 f;
    miller_loop(f, P, Q);
    store_vec(as_gt(out) + i, f);
}

__global__ void k_fp12_segment_product(uint8_t* out, const uint8_t* in, const int64_t* offsets, int64_t k) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= k) return;
    Fp12 acc = fp12_one();
    for (int64_t t = offsets[j]; t < offsets[j + 1]; t++) {
        Fp12 x = load_vec(as_gt(in) + t);
        fp12_mul(acc, acc, x);
    }
    store_vec(as_gt(out) + j, acc);
}

__global__ void WBTE_PAIR_BOUNDS k_final_exp(uint8_t* out, const uint8_t* in, int64_t n, int mode) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fp12 f = load_vec(as_gt(in) + i), r;
    if (mode == FE_EASY) {
        final_exp_easy(r, f);
    } else if (mode == FE_HARD) {
        final_exp_hard(r, f);
    } else {
        final_exp_easy(r, f);
        final_exp_hard(r, r);
    }
    store_vec(as_gt(out) + i, r);
}

__global__ void k_fp12_mul(uint8_t* out, const uint8_t* a, int64_t sa, const uint8_t* b, int64_t sb, bool conj_b, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fp12 x = load_vec(as_gt(a) + sa * i), y = load_vec(as_gt(b) + sb * i), r;
    if (conj_b) fp12_conj(y, y);
    fp12_mul(r, x, y);
    store_vec(as_gt(out) + i, r);
}

__global__ void k_unmask(uint8_t* out, const uint8_t* second, const uint8_t* alpha, const uint8_t* beta,
                         const uint8_t* valid, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fp12 r;
    if (valid[i]) {
        Fp12 c2 = load_vec(as_gt(second) + i), al = load_vec(as_gt(alpha) + i), be = load_vec(as_gt(beta) + i);
        fp12_conj(al, al);
        fp12_mul(r, c2, al);
        fp12_mul(r, r, be);
    } else {
        r = fp12_one();
    }
    store_vec(as_gt(out) + i, r);
}

WBTE_INL void fp_store_be48(uint8_t* out, const Fp& m) {
    Fp c = fp_from_mont(m);
    for (int i = 0; i < 48; i++) out[47 - i] = (uint8_t)(c.v[i >> 2] >> (8 * (i & 3)));
}

// Tagged torus compression of GT: identity -> 0; otherwise 1 followed by the
// six Fp2 coefficients of (c0 + 1) / c1, each Fp as 48 big-endian bytes.
__global__ void k_gt_compress(uint8_t* out, const uint8_t* in, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fp12 f = load_vec(as_gt(in) + i);
    uint8_t* o = out + 289 * i;
    if (fp12_is_one(f)) {
        for (int b = 0; b < 289; b++) o[b] = 0;
        return;
    }
    Fp6 c0 = f.c0, inv, b;
    c0.c0 = fp2_add(c0.c0, fp2_one());
    fp6_inv(inv, f.c1);
    fp6_mul(b, c0, inv);
    o[0] = 1;
    const Fp2* cs[3] = {&b.c0, &b.c1, &b.c2};
    for (int k = 0; k < 3; k++) {
        fp_store_be48(o + 1 + 96 * k, cs[k]->c0);
        fp_store_be48(o + 1 + 96 * k + 48, cs[k]->c1);
    }
}

__global__ void k_fp12_conj(uint8_t* out, const uint8_t* in, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fp12 x = load_vec(as_gt(in) + i);
    fp12_conj(x, x);
    store_vec(as_gt(out) + i, x);
}

__global__ void k_fp12_mask(uint8_t* io, const uint8_t* valid, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!valid[i]) store_vec(as_gt(io) + i, fp12_one());
}

__global__ void k_fp12_is_one(uint8_t* flags, const uint8_t* in, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = fp12_is_one(load_vec(as_gt(in) + i)) ? 1 : 0;
}
}  // namespace

// ============================================================ launchers
void launch_prepare_lines(uint8_t* lines, const uint8_t* q, int64_t n, cudaStream_t s) {
    ProfScope prof_("prepare_lines", s);
    if (n <= 0) return;
    note_launch();
    k_prepare_lines<<<blocks_for(n), TPB, 0, s>>>(lines, q, n);
}
void launch_miller_lines(uint8_t* out, const uint8_t* lines, const uint8_t* p, int64_t n, cudaStream_t s,
                         int64_t lines_n) {
    ProfScope prof_("miller_lines", s);
    if (n <= 0) return;
    note_launch();
    k_miller_lines<<<blocks_for(n), TPB, 0, s>>>(out, lines, p, n, lines_n > 0 ? lines_n : n);
}
void launch_miller(uint8_t* out, const uint8_t* p, const uint8_t* q, int64_t n, cudaStream_t s, int64_t p_mod,
                   int64_t q_mod) {
    ProfScope prof_("miller", s);
    if (n <= 0) return;
    note_launch();
    k_miller<<<blocks_for(n), TPB, 0, s>>>(out, p, q, n, p_mod, q_mod);
}
void launch_fp12_mask(uint8_t* io, const uint8_t* valid, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    note_launch();
    k_fp12_mask<<<blocks_for(n), TPB, 0, s>>>(io, valid, n);
}
void launch_fp12_segment_product(uint8_t* out, const uint8_t* in, const int64_t* offsets, int64_t k, cudaStream_t s) {
    ProfScope prof_("fp12_product", s);
    if (k <= 0) return;
    note_launch();
    k_fp12_segment_product<<<blocks_for(k), TPB, 0, s>>>(out, in, offsets, k);
}
void launch_final_exp(uint8_t* out, const uint8_t* in, int64_t n, FinalExpMode mode, cudaStream_t s) {
    ProfScope prof_(mode == FE_EASY ? "final_exp_easy" : (mode == FE_HARD ? "final_exp_hard" : "final_exp"), s);
    if (n <= 0) return;
    note_launch();
    k_final_exp<<<blocks_for(n), TPB, 0, s>>>(out, in, n, (int)mode);
}

void launch_fp12_mul(uint8_t* out, const uint8_t* a, int64_t sa, const uint8_t* b, int64_t sb, bool conj_b, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    note_launch();
    k_fp12_mul<<<blocks_for(n), TPB, 0, s>>>(out, a, sa, b, sb, conj_b, n);
}
void launch_unmask(uint8_t* out, const uint8_t* second, const uint8_t* alpha, const uint8_t* beta, const uint8_t* valid,
                   int64_t n, cudaStream_t s) {
    ProfScope prof_("unmask", s);
    if (n <= 0) return;
    note_launch();
    k_unmask<<<blocks_for(n), TPB, 0, s>>>(out, second, alpha, beta, valid, n);
}
void launch_gt_compress(uint8_t* out, const uint8_t* in, int64_t n, cudaStream_t s) {
    ProfScope prof_("gt_compress", s);
    if (n <= 0) return;
    note_launch();
    k_gt_compress<<<blocks_for(n), TPB, 0, s>>>(out, in, n);
}
void launch_fp12_conj(uint8_t* out, const uint8_t* in, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    note_launch();
    k_fp12_conj<<<blocks_for(n), TPB, 0, s>>>(out, in, n);
}
void launch_fp12_is_one(uint8_t* flags, const uint8_t* in, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    note_launch();
    k_fp12_is_one<<<blocks_for(n), TPB, 0, s>>>(flags, in, n);
}

}  // namespace wbte
