// GT transforms and GT exponentiation: the radix-2 and radix-4 stages of the
// (truncated) cyclotomic transforms, their lane-split, joint and warp-uniform
// exponentiation kernels, and batched GT powers.  Built with out-of-line Fp2
// products and Fp sums: these kernels are bound by instruction fetch, and the
// smaller code runs faster here (the Miller-loop and final-exponentiation
// kernels of k_pairing.cu keep them inline).
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

__device__ __forceinline__ int64_t bitrev64(int64_t i, int bits) {
    return bits ? (int64_t)(__brevll((unsigned long long)i) >> (64 - bits)) : 0;
}

__global__ void k_gt_bitrev(uint8_t* dst, const uint8_t* src, int64_t n, int bits, int64_t count) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n * count) return;
    const int64_t q = i / n, j = i % n;
    store_vec(as_gt(dst) + q * n + bitrev64(j, bits), load_vec(as_gt(src) + i));
}

// The GT transforms and GT exponentiation split each exponentiation v^s over
// GT_LANES = 4 consecutive threads, one base-|x| digit of s each
// (gt_pow_lane); the four parts meet in shared memory.  Blocks are one warp.
constexpr int GT_LANES = 4;
constexpr int WARP = 32;
// resident blocks per SM the GT kernels are compiled for (register budget)
#ifndef WBTE_GT_MINBLOCKS
#define WBTE_GT_MINBLOCKS 1
#endif
// k_gt_radix4_pows_plan: 12 one-warp blocks per SM (170 registers) hide more
// latency than 8 blocks at 255 registers, in spite of the spills
#ifndef WBTE_PLAN_MINBLOCKS
#define WBTE_PLAN_MINBLOCKS 12
#endif

// parts of v^s for the butterfly or element this lane belongs to
WBTE_INL void gt_pow_part(Fp12& part, const Fp12& v, const uint8_t* scalar, int c) {
    uint32_t s[8];
    load_scalar(s, scalar);
    uint64_t d[4];
    decompose_base_x(d, s);
    gt_pow_lane(part, v, d[c], c);
}

// sh[lane - c] <- product of the four parts of its group
WBTE_INL void gt_combine(Fp12* sh, int lane, int c) {
    __syncwarp();
    if ((c & 1) == 0) {
        Fp12 x = load_vec(sh + lane), y = load_vec(sh + lane + 1);
        fp12_mul(x, x, y);
        store_vec(sh + lane, x);
    }
    __syncwarp();
    if (c == 0) {
        Fp12 x = load_vec(sh + lane), y = load_vec(sh + lane + 2);
        fp12_mul(x, x, y);
        store_vec(sh + lane, x);
    }
    __syncwarp();
}

// One butterfly per group of lanes: u' = u t, v' = u t^-1 with t = v^tw
// (inverse by conjugation in the cyclotomic subgroup).
__global__ void __launch_bounds__(WARP, WBTE_GT_MINBLOCKS) k_gt_stage(uint8_t* io, const uint8_t* tw, int64_t n, int64_t half,
                                                  int64_t count) {
    __shared__ Fp12 sh[WARP];
    const int lane = threadIdx.x, c = lane % GT_LANES;
    const int64_t t = ((int64_t)blockIdx.x * WARP + lane) / GT_LANES;
    const bool active = t < (n / 2) * count;
    const int64_t q = active ? t / (n / 2) : 0, tt = active ? t % (n / 2) : 0;
    const int64_t chunk = tt / half, j = tt % half;
    const int64_t a = q * n + chunk * 2 * half + j, b = a + half;
    Fp12 part = fp12_one();
    if (active) {
        Fp12 v = load_vec(as_gt(io) + b);
        if (j != 0) gt_pow_part(part, v, tw + FR_SZ * (j * (n / (2 * half))), c);
        else if (c == 0) part = v;
    }
    store_vec(sh + lane, part);
    gt_combine(sh, lane, c);
    // lanes 0 and 1 both read u before either output is written
    Fp12 u;
    if (active && c < 2) u = load_vec(as_gt(io) + a);
    __syncwarp();
    if (active && c < 2) {
        Fp12 tv = load_vec(sh + (lane - c)), r;
        if (c == 1) fp12_conj(tv, tv);
        fp12_mul(r, u, tv);
        store_vec(as_gt(io) + (c == 0 ? a : b), r);
    }
}

// x^(omega_4) under the decomposed action.  The forward domain's primitive
// 4th root of unity is omega_4 = |x|^3 (its base-|x| digits are 0, 0, 0, 1),
// which acts as conj(Frobenius^3(x)); the inverse domain's omega_4^-1 acts as
// its inverse, Frobenius^3(x).  (Agrees with the plain power after the hard
// part, like every decomposed action.)
WBTE_INL void gt_omega4(Fp12& r, const Fp12& x, bool inverse) {
    fp12_frobenius(r, x, 3);
    if (!inverse) fp12_conj(r, r);
}

// One radix-4 DIT stage merging the radix-2 stages of half sizes h and 2h:
// per block of 4h and offset j < h, with a, b, c, d at j, j+h, j+2h, j+3h and
// w1 = w^(2j s), w2 = w^(j s), w3 = w1 w2 (s = n / 4h):
//   t1 = b^w1, u = c^w2, v = d^w3, cw = u v, dw = (u / v)^omega_4
//   j: a t1 cw   j+h: a/t1 dw   j+2h: a t1 / cw   j+3h: a/t1 / dw
// Three exponentiations per four outputs instead of the radix-2 pair's four.
// Each exponentiation is split over the group's 4 lanes (one base-|x| digit
// each) and combined in shared memory.  prefix: write only the first two
// outputs (the last stage of the truncated inverse transform).
__global__ void __launch_bounds__(WARP, WBTE_GT_MINBLOCKS) k_gt_radix4(uint8_t* io, const uint8_t* tw, int64_t n, int64_t h,
                                                   int64_t count, int inverse, int prefix) {
    __shared__ Fp12 sh[WARP];
    const int lane = threadIdx.x, c = lane % GT_LANES;
    const int64_t t = ((int64_t)blockIdx.x * WARP + lane) / GT_LANES;
    const bool active = t < (n / 4) * count;
    const int64_t q = active ? t / (n / 4) : 0, tt = active ? t % (n / 4) : 0;
    const int64_t blk = tt / h, j = tt % h;
    Fp12* base = as_gt(io) + q * n + blk * 4 * h + j;
    const int64_t s = n / (4 * h);
    Fp12 a, ex[3];
    if (active) a = load_vec(base);  // read before any output of the group is written
    for (int e = 0; e < 3; e++) {
        int64_t idx = (e == 0 ? 2 * j : (e == 1 ? j : 3 * j)) * s;
        const bool neg = idx >= n / 2;  // w^(k + n/2) = -w^k: the inverse
        if (neg) idx -= n / 2;
        Fp12 part = fp12_one();
        if (active) {
            Fp12 x = load_vec(base + (int64_t)(e + 1) * h);
            if (idx != 0) gt_pow_part(part, x, tw + FR_SZ * idx, c);
            else if (c == 0) part = x;
        }
        __syncwarp();  // the previous exponentiation's result has been read
        store_vec(sh + lane, part);
        gt_combine(sh, lane, c);
        ex[e] = load_vec(sh + (lane - c));
        if (neg) fp12_conj(ex[e], ex[e]);
    }
    if (!active || (prefix && c >= 2)) return;
    Fp12 r, m;
    if (c == 0 || c == 2) {
        fp12_mul(m, ex[1], ex[2]);  // cw
    } else {
        fp12_conj(m, ex[2]);
        fp12_mul(m, ex[1], m);
        gt_omega4(m, m, inverse != 0);  // dw
    }
    if (c >= 2) fp12_conj(m, m);
    Fp12 t1 = ex[0];
    if (c & 1) fp12_conj(t1, t1);
    fp12_mul(r, a, t1);
    fp12_mul(r, r, m);
    const int64_t pos = c == 0 ? 0 : (c == 1 ? h : (c == 2 ? 2 * h : 3 * h));
    store_vec(base + pos, r);
}

// The radix-4 stage as two launches for large batches of transforms: the
// three twiddle powers of every butterfly, each exponentiation over L lanes
// (L = 1: one thread runs all four base-|x| digits with shared squarings,
// about 40% fewer Fp products than four one-digit lanes), into ex[3 t + e];
// then the four outputs of each butterfly from a and its three powers.
template <int L>
__global__ void __launch_bounds__(WARP, WBTE_GT_MINBLOCKS) k_gt_radix4_pows(uint8_t* ex, const uint8_t* io, const uint8_t* tw,
                                                        int64_t n, int64_t h, int64_t count) {
    __shared__ Fp12 sh[L > 1 ? WARP : 1];
    const int lane = threadIdx.x, sub = lane % L;
    const int64_t g = ((int64_t)blockIdx.x * WARP + lane) / L;
    const bool active = g < 3 * (n / 4) * count;
    Fp12 part = fp12_one();
    bool neg = false;
    if (active) {
        const int64_t t = g / 3;
        const int e = (int)(g % 3);
        const int64_t q = t / (n / 4), tt = t % (n / 4), blk = tt / h, j = tt % h;
        int64_t idx = (e == 0 ? 2 * j : (e == 1 ? j : 3 * j)) * (n / (4 * h));
        neg = idx >= n / 2;  // w^(k + n/2) = -w^k: the inverse
        if (neg) idx -= n / 2;
        const Fp12 x = load_vec(as_gt(io) + q * n + blk * 4 * h + j + (int64_t)(e + 1) * h);
        if (idx != 0) {
            uint32_t sc[8];
            load_scalar(sc, tw + FR_SZ * idx);
            uint64_t d[4];
            decompose_base_x(d, sc);
            gt_pow_digits(part, x, d, sub, L);
        } else if (sub == 0) {
            part = x;
        }
    }
    if (L > 1) {
        store_vec(sh + lane, part);
        for (int w = 1; w < L; w *= 2) {
            __syncwarp();
            if (sub % (2 * w) == 0) {
                Fp12 a = load_vec(sh + lane), b = load_vec(sh + lane + w);
                fp12_mul(a, a, b);
                store_vec(sh + lane, a);
            }
        }
        __syncwarp();
        part = load_vec(sh + lane);
    }
    if (active && sub == 0) {
        if (neg) fp12_conj(part, part);
        store_vec(as_gt(ex) + g, part);
    }
}

// The twiddle powers of a radix-4 stage for batches of at least 32
// transforms: a warp takes one twiddle power across 32 transforms, so its
// exponent is warp-uniform and the data-dependent plan (width-4 NAF of the
// four base-|x| digits over one shared run of squarings, zero digits skipped,
// cyc_pow_plan) runs without divergence: about 4.3 k Fp products per power
// against 5.8 k for the fixed radix-16 schedule.  Same ex layout as
// k_gt_radix4_pows.
__global__ void __launch_bounds__(WARP, WBTE_PLAN_MINBLOCKS) k_gt_radix4_pows_plan(uint8_t* ex, const uint8_t* io,
                                                             const uint8_t* tw, int64_t n, int64_t h,
                                                             int64_t count, int64_t pad) {
    // threads take the transforms fastest over `pad` >= count slots (a
    // multiple of 32), so every warp shares one twiddle; slots past count idle
    const int64_t g = (int64_t)blockIdx.x * WARP + threadIdx.x;
    if (g >= 3 * (n / 4) * pad) return;
    const int64_t q = g % pad, rest = g / pad;
    if (q >= count) return;
    const int e = (int)(rest % 3);
    const int64_t tt = rest / 3, blk = tt / h, j = tt % h;
    int64_t idx = (e == 0 ? 2 * j : (e == 1 ? j : 3 * j)) * (n / (4 * h));
    const bool neg = idx >= n / 2;  // w^(k + n/2) = -w^k: the inverse
    if (neg) idx -= n / 2;
    const Fp12 x = load_vec(as_gt(io) + q * n + blk * 4 * h + j + (int64_t)(e + 1) * h);
    Fp12 part;
    if (idx != 0) {
        uint32_t sc[8];
        load_scalar(sc, tw + FR_SZ * idx);
        CycPlan pl;
        make_cyc_plan(pl, sc);
        cyc_pow_plan(part, x, pl);
    } else {
        part = x;
    }
    if (neg) fp12_conj(part, part);
    store_vec(as_gt(ex) + (q * (n / 4) + tt) * 3 + e, part);
}

// outputs of the radix-4 butterflies from their twiddle powers (the formulas
// of k_gt_radix4); one thread per output, four (two with prefix) per
// butterfly in one warp, every read done before the warp's first write
__global__ void k_gt_radix4_outputs(uint8_t* io, const uint8_t* ex, int64_t n, int64_t h, int64_t count, int inverse,
                                    int prefix) {
    const int outs = prefix ? 2 : 4;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool active = i < (n / 4) * count * outs;
    const int64_t t = active ? i / outs : 0;
    const int c = (int)(i % outs);
    const int64_t q = t / (n / 4), tt = t % (n / 4), blk = tt / h, j = tt % h;
    Fp12* base = as_gt(io) + q * n + blk * 4 * h + j;
    Fp12 a, t1, e1, e2;
    if (active) {
        a = load_vec(base);
        t1 = load_vec(as_gt(ex) + 3 * t);
        e1 = load_vec(as_gt(ex) + 3 * t + 1);
        e2 = load_vec(as_gt(ex) + 3 * t + 2);
    }
    __syncwarp();
    if (!active) return;
    Fp12 r, m;
    if (c == 0 || c == 2) {
        fp12_mul(m, e1, e2);  // cw
    } else {
        fp12_conj(m, e2);
        fp12_mul(m, e1, m);
        gt_omega4(m, m, inverse != 0);  // dw
    }
    if (c >= 2) fp12_conj(m, m);
    if (c & 1) fp12_conj(t1, t1);
    fp12_mul(r, a, t1);
    fp12_mul(r, r, m);
    store_vec(base + (int64_t)c * h, r);
}

// last stage keeping only the first out_count outputs
__global__ void __launch_bounds__(WARP, WBTE_GT_MINBLOCKS) k_gt_last_prefix(uint8_t* io, const uint8_t* tw, int64_t n, int64_t out_count,
                                                        int64_t count) {
    __shared__ Fp12 sh[WARP];
    const int lane = threadIdx.x, c = lane % GT_LANES;
    const int64_t jj = ((int64_t)blockIdx.x * WARP + lane) / GT_LANES;
    const bool active = jj < out_count * count;
    const int64_t q = active ? jj / out_count : 0, j = active ? jj % out_count : 0;
    const int64_t half = n / 2;
    Fp12* base = as_gt(io) + q * n;
    Fp12 part = fp12_one();
    if (active) {
        Fp12 v = load_vec(base + half + j);
        if (j != 0) gt_pow_part(part, v, tw + FR_SZ * j, c);
        else if (c == 0) part = v;
    }
    store_vec(sh + lane, part);
    gt_combine(sh, lane, c);
    if (active && c == 0) {
        Fp12 u = load_vec(base + j), tv = load_vec(sh + lane);
        fp12_mul(u, u, tv);
        store_vec(base + j, u);
    }
}

__global__ void __launch_bounds__(WARP, WBTE_GT_MINBLOCKS) k_gt_pow(uint8_t* out, const uint8_t* base, int64_t stride, const uint8_t* scalars, int64_t n) {
    __shared__ Fp12 sh[WARP];
    const int lane = threadIdx.x, c = lane % GT_LANES;
    const int64_t i = ((int64_t)blockIdx.x * WARP + lane) / GT_LANES;
    const bool active = i < n;
    Fp12 part = fp12_one();
    if (active) gt_pow_part(part, load_vec(as_gt(base) + stride * i), scalars + FR_SZ * i, c);
    store_vec(sh + lane, part);
    gt_combine(sh, lane, c);
    if (active && c == 0) store_vec(as_gt(out) + i, load_vec(sh + lane));
}

// out[q B + i] = base[q B + i]^(scalars[i]) for K arrays of B values sharing
// the B exponents (a slot's exponent is the same in every array): threads
// take the arrays fastest over `pad` >= K slots (a multiple of 32), so every
// warp shares one exponent and runs its width-4 NAF plan without divergence;
// slots past K idle.
__global__ void __launch_bounds__(WARP, WBTE_PLAN_MINBLOCKS) k_gt_pow_shared_plan(uint8_t* out, const uint8_t* base,
                                                                                   const uint8_t* scalars, int64_t B,
                                                                                   int64_t K, int64_t pad) {
    const int64_t g = (int64_t)blockIdx.x * WARP + threadIdx.x;
    if (g >= B * pad) return;
    const int64_t q = g % pad, i = g / pad;
    if (q >= K) return;
    const Fp12 x = load_vec(as_gt(base) + q * B + i);
    uint32_t sc[8];
    load_scalar(sc, scalars + FR_SZ * i);
    CycPlan pl;
    make_cyc_plan(pl, sc);
    Fp12 r;
    cyc_pow_plan(r, x, pl);
    store_vec(as_gt(out) + q * B + i, r);
}

// out[i] = base[i stride]^c_i for small signed c_i on cyclotomic values:
// square-and-multiply over the bits of |c_i| with cyclotomic squarings, then
// the inverse (conjugation) for negative c_i -- mul_cyclotomic_signed_small of
// weighted_pfe/src/fft.rs:671-699.  c_i = 0 gives one.
__global__ void k_gt_pow_small(uint8_t* out, const uint8_t* base, int64_t stride, const int32_t* coeffs, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t c = coeffs[i];
    uint32_t mag = c < 0 ? (uint32_t)(-(int64_t)c) : (uint32_t)c;
    Fp12 acc = fp12_one();
    if (mag) {
        const Fp12 x = load_vec(as_gt(base) + stride * i);
        acc = x;
        for (int b = 30 - __clz(mag); b >= 0; b--) {
            fp12_cyclotomic_sqr(acc, acc);
            if ((mag >> b) & 1) fp12_mul(acc, acc, x);
        }
        if (c < 0) fp12_conj(acc, acc);
    }
    store_vec(as_gt(out) + i, acc);
}

}  // namespace

bool launch_gt_pow_shared(uint8_t* out, const uint8_t* base, const uint8_t* scalars, int64_t B, int64_t K,
                          cudaStream_t s) {
    const int64_t pad = K % WARP == 0 ? K : (K >= 24 && K < WARP ? (int64_t)WARP : 0);
    if (pad == 0 || B <= 0) return false;
    ProfScope prof_("gt_pow", s);
    note_launch();
    k_gt_pow_shared_plan<<<blocks_for(B * pad, WARP), WARP, 0, s>>>(out, base, scalars, B, K, pad);
    return true;
}

void launch_gt_pow_small(uint8_t* out, const uint8_t* base, int64_t stride, const int32_t* coeffs, int64_t n,
                         cudaStream_t s) {
    ProfScope prof_("gt_pow_small", s);
    if (n <= 0) return;
    note_launch();
    k_gt_pow_small<<<blocks_for(n), TPB, 0, s>>>(out, base, stride, coeffs, n);
}

// Lanes per exponentiation for a radix-4 stage of E twiddle powers, from a
// cost model: one lane's work in Fp products (65 squarings and 74 products
// for all four digits on one lane, about 52 with the warp-uniform NAF plan
// of k_gt_radix4_pows_plan; 65 and 40 on each of two; 65 and 25 on each of
// four, with the Frobenius maps and the lane combine) times
// max(1, E L / resident threads).  WBTE_GT_LANES = 1, 2 or 4 overrides it, and
// so does the calling context's tuning knob.
static int gt_pow_lanes(int64_t E, bool shared_plan) {
    static std::atomic<int64_t> cap{0};
    if (const char* env = getenv("WBTE_GT_LANES")) {
        const int v = atoi(env);
        if (v == 1 || v == 2 || v == 4) return v;
    }
    if (g_tune.gt_lanes == 1 || g_tune.gt_lanes == 2 || g_tune.gt_lanes == 4) return g_tune.gt_lanes;
    int64_t c = cap.load();
    if (c == 0) {
        int dev = 0, sms = 0, blocks = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_gt_radix4_pows<1>, WARP, 0);
        c = (int64_t)(blocks > 0 ? blocks : 1) * WARP * (sms > 0 ? sms : 1);
        cap.store(c);
    }
    const double work[3] = {shared_plan ? 4300.0 : 5829.0, 3560.0, 2533.0};
    int best = 1;
    double best_t = 0;
    for (int i = 0, L = 1; L <= GT_LANES; i++, L *= 2) {
        const double t = std::max(1.0, (double)(E * L) / (double)c) * work[i];
        if (L == 1 || t < best_t) best = L, best_t = t;
    }
    return best;
}

static void gt_transform(uint8_t* io, const uint8_t* tw, int64_t n, int64_t out_count, bool prefix, cudaStream_t s,
                         int64_t count, bool inverse) {
    if (n <= 1 || count <= 0) return;
    if (count > WARP && count % WARP != 0) {
        // the largest multiple of 32 transforms takes the warp-uniform plan
        // kernels; the rest runs on its own
        const int64_t a = count - count % WARP;
        gt_transform(io, tw, n, out_count, prefix, s, a, inverse);
        gt_transform(io + GT_SZ * (size_t)(n * a), tw, n, out_count, prefix, s, count - a, inverse);
        return;
    }
    ProfScope prof_("gt_ifft", s);
    int bits = 0;
    while ((int64_t(1) << bits) < n) bits++;
    uint8_t* tmp = nullptr;
    if (cudaMallocAsync(&tmp, GT_SZ * (size_t)(n * count), s) != cudaSuccess) return;
    note_launch();
    k_gt_bitrev<<<blocks_for(n * count), TPB, 0, s>>>(tmp, io, n, bits, count);
    if (n < 4 || (prefix && out_count != n / 2)) {
        // radix-2 throughout (tiny transforms, or a prefix other than the first half)
        int64_t last_half = prefix ? n / 4 : n / 2;
        for (int64_t half = 1; half <= last_half; half *= 2) {
            note_launch();
            k_gt_stage<<<blocks_for(GT_LANES * (n / 2) * count, WARP), WARP, 0, s>>>(tmp, tw, n, half, count);
        }
        if (prefix && out_count > 0) {
            note_launch();
            k_gt_last_prefix<<<blocks_for(GT_LANES * out_count * count, WARP), WARP, 0, s>>>(tmp, tw, n, out_count,
                                                                                             count);
        }
    } else {
        // an odd number of stages starts with one radix-2 stage, the rest pair up
        int64_t half = 1;
        if (bits & 1) {
            note_launch();
            k_gt_stage<<<blocks_for(GT_LANES * (n / 2) * count, WARP), WARP, 0, s>>>(tmp, tw, n, 1, count);
            half = 2;
        }
        const int64_t E = 3 * (n / 4) * count;  // twiddle powers per radix-4 stage
        // warp-uniform plans for multiples of 32 transforms, and for 24..31
        // transforms padded to 32 (at most a quarter of the lanes idle, against
        // about 35 % more Fp products per power on the fixed schedule)
        const int64_t pad = count % WARP == 0 ? count : (count >= 24 && count < WARP ? (int64_t)WARP : 0);
        const bool shared_plan = pad >= WARP;
        const int L = gt_pow_lanes(E, shared_plan);
        uint8_t* ex = nullptr;
        if (L < GT_LANES && cudaMallocAsync(&ex, GT_SZ * (size_t)E, s) != cudaSuccess) {
            cudaFreeAsync(tmp, s);
            return;
        }
        for (; half < n; half *= 4) {
            const int pre = (prefix && 4 * half == n) ? 1 : 0;
            if (L == GT_LANES) {
                note_launch();
                k_gt_radix4<<<blocks_for(GT_LANES * (n / 4) * count, WARP), WARP, 0, s>>>(
                    tmp, tw, n, half, count, inverse ? 1 : 0, pre);
                continue;
            }
            note_launch(2);
            if (L == 1 && shared_plan)
                k_gt_radix4_pows_plan<<<blocks_for(3 * (n / 4) * pad, WARP), WARP, 0, s>>>(ex, tmp, tw, n, half,
                                                                                            count, pad);
            else if (L == 1)
                k_gt_radix4_pows<1><<<blocks_for(E, WARP), WARP, 0, s>>>(ex, tmp, tw, n, half, count);
            else
                k_gt_radix4_pows<2><<<blocks_for(2 * E, WARP), WARP, 0, s>>>(ex, tmp, tw, n, half, count);
            k_gt_radix4_outputs<<<blocks_for((n / 4) * count * (pre ? 2 : 4)), TPB, 0, s>>>(
                tmp, ex, n, half, count, inverse ? 1 : 0, pre);
        }
        if (ex) cudaFreeAsync(ex, s);
    }
    cudaMemcpyAsync(io, tmp, GT_SZ * (size_t)(n * count), cudaMemcpyDeviceToDevice, s);
    cudaFreeAsync(tmp, s);
}
void launch_cyclotomic_prefix_ifft(uint8_t* io, const uint8_t* tw_inv, int64_t n, int64_t out_count, cudaStream_t s,
                                   int64_t count) {
    gt_transform(io, tw_inv, n, out_count, true, s, count, true);
}
void launch_gt_ntt(uint8_t* io, const uint8_t* tw, int64_t n, cudaStream_t s, int64_t count, bool inverse) {
    gt_transform(io, tw, n, n, false, s, count, inverse);
}

void launch_gt_pow(uint8_t* out, const uint8_t* base, int64_t stride, const uint8_t* scalars, int64_t n, cudaStream_t s) {
    ProfScope prof_("gt_pow", s);
    if (n <= 0) return;
    note_launch();
    k_gt_pow<<<blocks_for(GT_LANES * n, WARP), WARP, 0, s>>>(out, base, stride, scalars, n);
}

}  // namespace wbte
