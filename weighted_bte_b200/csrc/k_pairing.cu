// Pairing-side kernels: G2 line tables, Miller loops, split final
// exponentiation and the GT element kernels (products, masks, encodings).
// The GT transforms live in k_gt.cu.
#include <algorithm>
#include <atomic>
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

// Segment s of `per` consecutive pairs is split into `chunks` runs of at most
// C pairs; thread (s, ch) writes the product of its run's Miller loops, one
// multi-Miller loop sharing the squarings.
__global__ void WBTE_PAIR_BOUNDS k_miller_chunks(uint8_t* out, const uint8_t* p, const uint8_t* q, int64_t per,
                                                 int64_t K, int C, int64_t chunks) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= K * chunks) return;
    const int64_t s = g / chunks, lo = (g % chunks) * C;
    const int cnt = (int)(per - lo < C ? per - lo : C);
    G1A P[MULTI_MILLER_MAX];
    G2A Q[MULTI_MILLER_MAX];
    for (int t = 0; t < cnt; t++) {
        P[t] = load_affine(reinterpret_cast<const G1A*>(p + G1_AFF * (s * per + lo + t)));
        Q[t] = load_affine(reinterpret_cast<const G2A*>(q + G2_AFF * (s * per + lo + t)));
    }
    Fp12 f;
    multi_miller_loop(f, P, Q, cnt);
    store_vec(as_gt(out) + g, f);
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

WBTE_INL bool fp12_is_zero(const Fp12& a) {
    const uint32_t* x = reinterpret_cast<const uint32_t*>(&a);
    uint32_t d = 0;
    for (int i = 0; i < 144; i++) d |= x[i];
    return d == 0;
}

// The easy part f^((p^6 - 1)(p^2 + 1)) of C consecutive values per thread
// sharing one Fp12 inversion (batch_easy_final_exponentiation,
// btx/src/final_exponentiation.rs:228-252): the forward pass keeps the prefix
// products in `pre`, one inversion of the chunk's product, and each value's
// inverse falls out on the way back.  A zero value (no inverse) is left out
// of the product and gives zero, as the per-value kernel does.  full: the
// hard part follows.  in may equal out.
__global__ void WBTE_PAIR_BOUNDS k_final_exp_easy_batch(uint8_t* out, const uint8_t* in, uint8_t* pre, int64_t n,
                                                        int64_t C, int full) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t lo = t * C, hi = lo + C < n ? lo + C : n;
    if (lo >= n) return;
    Fp12 acc = fp12_one();
    for (int64_t i = lo; i < hi; i++) {
        const Fp12 f = load_vec(as_gt(in) + i);
        store_vec(as_gt(pre) + i, acc);
        if (!fp12_is_zero(f)) fp12_mul(acc, acc, f);
    }
    Fp12 inv;
    fp12_inv(inv, acc);
    for (int64_t i = hi - 1; i >= lo; i--) {
        const Fp12 f = load_vec(as_gt(in) + i);
        Fp12 r;
        if (fp12_is_zero(f)) {
            r = f;
        } else {
            Fp12 fi, u;
            fp12_mul(fi, inv, load_vec(as_gt(pre) + i));  // 1 / f_i
            fp12_mul(inv, inv, f);
            fp12_conj(r, f);
            fp12_mul(r, r, fi);  // f^(p^6 - 1)
            fp12_frobenius(u, r, 2);
            fp12_mul(r, r, u);  // ^(p^2 + 1)
            if (full) final_exp_hard(r, r);
        }
        store_vec(as_gt(out) + i, r);
    }
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
// Pairs per thread of the chunked unprepared Miller loops: sharing the 62
// squarings over C pairs saves 2,232 Fp products per extra pair (about a
// third of a loop), but a launch of fewer threads than the device holds
// takes as long as the longest thread, so chunks grow only while the launch
// still fills the resident threads.
int miller_chunk(int64_t pairs) {
    if (g_tune.miller_chunk > 0) return g_tune.miller_chunk;
    static std::atomic<int64_t> resident{0};
    int64_t r = resident.load();
    if (r == 0) {
        int dev = 0, sms = 0, blocks = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_miller_chunks, TPB, 0);
        r = (int64_t)(sms > 0 ? sms : 148) * (blocks > 0 ? blocks : 1) * TPB;
        resident.store(r);
    }
    const int64_t C = pairs / r;
    return (int)(C < 1 ? 1 : (C > MULTI_MILLER_MAX ? MULTI_MILLER_MAX : C));
}
int64_t launch_miller_chunks(uint8_t* out, const uint8_t* p, const uint8_t* q, int64_t per, int64_t K, int C,
                             cudaStream_t s) {
    if (per <= 0 || K <= 0) return 0;
    if (C < 1) C = 1;
    if (C > MULTI_MILLER_MAX) C = MULTI_MILLER_MAX;
    // the profile tag names the run length, which fixes the product count
    static const char* const tags[MULTI_MILLER_MAX + 1] = {"", "miller_c1", "miller_c2", "miller_c3", "miller_c4",
                                                          "miller_c5", "miller_c6", "miller_c7", "miller_c8"};
    ProfScope prof_(tags[C], s);
    const int64_t chunks = (per + C - 1) / C;
    note_launch();
    k_miller_chunks<<<blocks_for(K * chunks), TPB, 0, s>>>(out, p, q, per, K, C, chunks);
    return chunks;
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
// Values per thread of the batched easy part: one Fp12 inversion (about 600
// Fp products) per chunk against three products per value, so chunks grow
// only while the launch still fills the resident threads.
static int64_t easy_chunk(int64_t n) {
    static std::atomic<int64_t> resident{0};
    int64_t r = resident.load();
    if (r == 0) {
        int dev = 0, sms = 0, blocks = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_final_exp_easy_batch, TPB, 0);
        r = (int64_t)(sms > 0 ? sms : 148) * (blocks > 0 ? blocks : 1) * TPB;
        resident.store(r);
    }
    const int64_t C = n / r;
    return C < 1 ? 1 : (C > 8 ? 8 : C);
}

void launch_final_exp(uint8_t* out, const uint8_t* in, int64_t n, FinalExpMode mode, cudaStream_t s) {
    ProfScope prof_(mode == FE_EASY ? "final_exp_easy" : (mode == FE_HARD ? "final_exp_hard" : "final_exp"), s);
    if (n <= 0) return;
    const int64_t C = mode == FE_HARD ? 1 : easy_chunk(n);
    uint8_t* pre = nullptr;
    if (C > 1 && cudaMallocAsync(&pre, GT_SZ * (size_t)n, s) == cudaSuccess) {
        const int64_t threads = (n + C - 1) / C;
        note_launch();
        k_final_exp_easy_batch<<<blocks_for(threads), TPB, 0, s>>>(out, in, pre, n, C, mode == FE_FULL ? 1 : 0);
        cudaFreeAsync(pre, s);
        return;
    }
    cudaGetLastError();
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
