// Scalar-field kernels, batched point multiplication, radix-2 group
// transforms, compressed encodings and Schnorr checks.
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <type_traits>

#include "launch.h"
#include "pairing.cuh"

namespace wbte {

namespace {
constexpr int TPB = 128;
inline unsigned blocks_for(int64_t n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

WBTE_INL Fr load_fr_mont(const uint8_t* p) {
    Fr a;
    load_scalar(a.v, p);
    return fr_to_mont(a);
}
WBTE_INL void store_fr_canonical(uint8_t* p, const Fr& m) {
    Fr a = fr_from_mont(m);
    uint4* d = reinterpret_cast<uint4*>(p);
    d[0] = make_uint4(a.v[0], a.v[1], a.v[2], a.v[3]);
    d[1] = make_uint4(a.v[4], a.v[5], a.v[6], a.v[7]);
}

template <class F> struct GroupOf;
template <> struct GroupOf<Fp> { static constexpr size_t AFF = G1_AFF; };
template <> struct GroupOf<Fp2> { static constexpr size_t AFF = G2_AFF; };

// ------------------------------------------------------------- scalars
__global__ void k_fr_powers(uint8_t* out, const uint8_t* base, int64_t n, int64_t first) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fr b = load_fr_mont(base);
    // base^(first + i) by square-and-multiply
    uint64_t e = (uint64_t)(first + i);
    Fr r = fr_pow_u64(b, e);
    store_fr_canonical(out + FR_SZ * i, r);
}

__global__ void k_fr_mul_gather(uint8_t* out, const uint8_t* a, const uint8_t* b, const int32_t* bidx, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fr x = load_fr_mont(a + FR_SZ * i);
    Fr y = load_fr_mont(b + FR_SZ * (bidx ? (int64_t)bidx[i] : i));
    store_fr_canonical(out + FR_SZ * i, fr_mul(x, y));
}

__global__ void k_fr_scale(uint8_t* out, const uint8_t* a, const uint8_t* c, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    store_fr_canonical(out + FR_SZ * i, fr_mul(load_fr_mont(a + FR_SZ * i), load_fr_mont(c)));
}

__global__ void k_fr_scale_size_inv(uint8_t* out, const uint8_t* a, int log_m, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fr c;
    _Pragma("unroll") for (int t = 0; t < 8; t++) c.v[t] = C_DOMAIN_SIZE_INV[log_m][t];
    store_fr_canonical(out + FR_SZ * i, fr_mul(load_fr_mont(a + FR_SZ * i), c));
}

__global__ void k_material_scalars(uint8_t* out, const uint8_t* z, const int32_t* owner, const uint8_t* qp,
                                   int64_t W, int64_t N, int64_t rows) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= rows * W) return;
    int64_t r = i / W, w = i % W;
    Fr x = load_fr_mont(z + FR_SZ * w);
    Fr y = load_fr_mont(qp + FR_SZ * (r * N + owner[w]));
    store_fr_canonical(out + FR_SZ * i, fr_mul(x, y));
}

// Partial-fraction party keys of weighted_pfe (setup.rs:223-247):
//   g = 1 / (rho_j + alpha_i),  u = g^2 + beta_{-1} / (alpha_i + 1) + beta_0 / alpha_i
// stored at i * N + j (slot-major) or j * B + i (party-major); u may be null.
__global__ void k_wpfe_fractions(uint8_t* g, uint8_t* u, const uint8_t* rho, const uint8_t* alpha,
                                 const uint8_t* masks, int64_t N, int64_t B, int party_major) {
    int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (x >= N * B) return;
    int64_t i = x / N, j = x % N;
    int64_t o = party_major ? j * B + i : x;
    Fr a = load_fr_mont(alpha + FR_SZ * i);
    Fr gi = fr_inv(fr_add(load_fr_mont(rho + FR_SZ * j), a));
    store_fr_canonical(g + FR_SZ * o, gi);
    if (u) {
        Fr bm1 = load_fr_mont(masks), b0 = load_fr_mont(masks + FR_SZ);
        Fr t = fr_mul(gi, gi);
        t = fr_add(t, fr_mul(bm1, fr_inv(fr_add(a, fr_one()))));
        t = fr_add(t, fr_mul(b0, fr_inv(a)));
        store_fr_canonical(u + FR_SZ * o, t);
    }
}

__global__ void k_gather(uint8_t* out, const uint8_t* in, const int32_t* idx, int64_t n, int64_t record) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t* src = in + record * (int64_t)idx[i];
    uint8_t* dst = out + record * i;
    if ((record & 15) == 0) {
        for (int64_t b = 0; b < record; b += 16)
            *reinterpret_cast<uint4*>(dst + b) = *reinterpret_cast<const uint4*>(src + b);
    } else {
        for (int64_t b = 0; b < record; b++) dst[b] = src[b];
    }
}

// L_i(0) = prod_{k != i} (-x_k) / (x_i - x_k)
__global__ void k_lagrange(uint8_t* out, const uint8_t* x, int64_t n, int32_t* status) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fr xi = load_fr_mont(x + FR_SZ * i);
    Fr num = fr_one(), den = fr_one();
    for (int64_t k = 0; k < n; k++) {
        if (k == i) continue;
        Fr xk = load_fr_mont(x + FR_SZ * k);
        num = fr_mul(num, fr_neg(xk));
        den = fr_mul(den, fr_sub(xi, xk));
    }
    if (fr_is_zero(den)) {
        atomicExch(status, 1);
        return;
    }
    store_fr_canonical(out + FR_SZ * i, fr_mul(num, fr_inv(den)));
}

__global__ void k_domain_twiddles(uint8_t* tw, int log_n, int64_t count, bool inverse) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= count) return;
    Fr g;
    _Pragma("unroll") for (int i = 0; i < 8; i++) g.v[i] = inverse ? C_DOMAIN_GEN_INV[log_n][i] : C_DOMAIN_GEN[log_n][i];
    store_fr_canonical(tw + FR_SZ * j, fr_pow_u64(g, (uint64_t)j));
}

// -------------------------------------------------------------- points
template <class F>
__global__ void k_mul_batch(uint8_t* out, const uint8_t* pts, int64_t stride, const uint8_t* scalars, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    using A = Affine<F>;
    A p = load_affine(reinterpret_cast<const A*>(pts + stride * i * GroupOf<F>::AFF));
    uint32_t k[8];
    load_scalar(k, scalars + FR_SZ * i);
    Xyzz<F> r = xyzz_mul(from_affine(p), k);
    store_affine(reinterpret_cast<A*>(out + GroupOf<F>::AFF * i), to_affine(r));
}

template <class F> WBTE_INL Affine<F> generator_of();
template <> WBTE_INL Affine<Fp> generator_of<Fp>() { return g1_generator(); }
template <> WBTE_INL Affine<Fp2> generator_of<Fp2>() { return g2_generator(); }

// Fixed-base multiplication by the generator with a table of
// T[w][d] = d * 2^(8w) * G (w < 32, d < 256), one mixed addition per window.
template <class F>
__global__ void k_build_gen_table(uint8_t* table) {
    int w = blockIdx.x;  // 0..31
    int d = threadIdx.x; // 0..255
    using A = Affine<F>;
    Xyzz<F> base = from_affine(generator_of<F>());
    for (int i = 0; i < 8 * w; i++) base = xyzz_dbl(base);
    Xyzz<F> r = xyzz_mul_u64(base, (uint64_t)d);
    store_affine(reinterpret_cast<A*>(table + GroupOf<F>::AFF * (256 * w + d)), to_affine(r));
}

template <class F>
__global__ void k_mul_generator(uint8_t* out, const uint8_t* table, const uint8_t* scalars, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    using A = Affine<F>;
    const A* T = reinterpret_cast<const A*>(table);
    const uint8_t* s = scalars + FR_SZ * i;
    Xyzz<F> acc;
    set_inf(acc);
    for (int w = 0; w < 32; w++) {
        uint32_t d = s[w];
        if (d) acc = xyzz_madd(acc, load_affine(T + 256 * w + d));
    }
    store_affine(reinterpret_cast<A*>(out + GroupOf<F>::AFF * i), to_affine(acc));
}

template <class F>
__global__ void k_mul_pow2(uint8_t* out, const uint8_t* in, int64_t n, int k) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    using A = Affine<F>;
    Xyzz<F> r = from_affine(load_affine(reinterpret_cast<const A*>(in + GroupOf<F>::AFF * i)));
    for (int t = 0; t < k; t++) r = xyzz_dbl(r);
    store_affine(reinterpret_cast<A*>(out + GroupOf<F>::AFF * i), to_affine(r));
}

template <class F>
__global__ void k_segment_sum(uint8_t* out, const uint8_t* in, const int64_t* offsets, int64_t k) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= k) return;
    using A = Affine<F>;
    Xyzz<F> acc;
    set_inf(acc);
    for (int64_t t = offsets[j]; t < offsets[j + 1]; t++)
        acc = xyzz_madd(acc, load_affine(reinterpret_cast<const A*>(in + GroupOf<F>::AFF * t)));
    store_affine(reinterpret_cast<A*>(out + GroupOf<F>::AFF * j), to_affine(acc));
}

template <class F>
__global__ void k_negate(uint8_t* out, const uint8_t* in, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    using A = Affine<F>;
    A p = load_affine(reinterpret_cast<const A*>(in + GroupOf<F>::AFF * i));
    store_affine(reinterpret_cast<A*>(out + GroupOf<F>::AFF * i), neg(p));
}

// ----------------------------------------------------- group transforms
__device__ __forceinline__ int64_t bitrev64(int64_t i, int bits) {
    return bits ? (int64_t)(__brevll((unsigned long long)i) >> (64 - bits)) : 0;
}

// count transforms of size n, stored one after another
template <class F>
__global__ void k_ntt_load(uint8_t* work, const uint8_t* in, int64_t n, int bits, int64_t count) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n * count) return;
    using A = Affine<F>;
    const int64_t q = i / n, j = i % n;
    Xyzz<F> p = from_affine(load_affine(reinterpret_cast<const A*>(in + GroupOf<F>::AFF * i)));
    store_vec(reinterpret_cast<Xyzz<F>*>(work) + q * n + bitrev64(j, bits), p);
}

// One radix-2 butterfly per group of L lanes (blocks of one warp); twiddle
// index j * (n / size).  The twiddle multiplication is split along the
// base-|x| digits of the twiddle: four lanes on G2 ([d_c] (-1)^c psi^c(v)),
// two lanes on G1 ([a]v and [b](phi(v) + v)); the parts are summed in shared
// memory before the butterfly.
template <class F> struct NttLanes;
template <> struct NttLanes<Fp> { static constexpr int L = 2; };
template <> struct NttLanes<Fp2> { static constexpr int L = 4; };
constexpr int WARP = 32;

WBTE_INL void ntt_part(G1X& out, const G1X& v, const uint64_t d[4], int c) { g1_mul_lane(out, v, d, c); }
WBTE_INL void ntt_part(G2X& out, const G2X& v, const uint64_t d[4], int c) { g2_mul_lane(out, v, d, c); }

template <class F>
__global__ void __launch_bounds__(WARP) k_ntt_stage(uint8_t* work, const uint8_t* tw, int64_t n, int64_t half,
                                                   int64_t count) {
    constexpr int L = NttLanes<F>::L;
    __shared__ Xyzz<F> sh[WARP];
    const int lane = threadIdx.x, c = lane % L;
    const int64_t t = ((int64_t)blockIdx.x * WARP + lane) / L;
    const bool active = t < (n / 2) * count;
    const int64_t q = active ? t / (n / 2) : 0, tt = active ? t % (n / 2) : 0;
    const int64_t chunk = tt / half, j = tt % half;
    const int64_t a = q * n + chunk * 2 * half + j, b = a + half;
    Xyzz<F>* w = reinterpret_cast<Xyzz<F>*>(work);
    Xyzz<F> part;
    set_inf(part);
    if (active) {
        Xyzz<F> v = load_vec(w + b);
        if (j != 0) {
            uint32_t s[8];
            load_scalar(s, tw + FR_SZ * (j * (n / (2 * half))));
            uint64_t d[4];
            decompose_base_x(d, s);
            ntt_part(part, v, d, c);
        } else if (c == 0) {
            part = v;
        }
    }
    store_vec(sh + lane, part);
    __syncwarp();
    for (int step = 1; step < L; step *= 2) {
        if (c % (2 * step) == 0) store_vec(sh + lane, xyzz_add(load_vec(sh + lane), load_vec(sh + lane + step)));
        __syncwarp();
    }
    // lanes 0 and 1 both read u before either output is written
    Xyzz<F> u;
    if (active && c < 2) u = load_vec(w + a);
    __syncwarp();
    if (active && c < 2) {
        Xyzz<F> tv = load_vec(sh + (lane - c));
        if (c == 1) tv = neg(tv);
        store_vec(w + (c == 0 ? a : b), xyzz_add(u, tv));
    }
}

// MSMs of a few terms (the share checks' per-slot aggregates): out[o] =
// sum_t scalars[vsel[o] n + t] points[pbase[o] + idx[t]].  Every scalar is
// split into base-|x| digit groups (G2: four 64-bit digits, digit c acting
// on (-1)^c psi^c(v); G1: two 128-bit digits acting on v and phi(v) + v), and
// the (term, digit) pairs of one output are spread over L lanes.  Each lane
// runs one signed radix-16 Straus loop over its pairs -- one run of
// doublings shared by all of them -- and the lanes' sums meet in shared
// memory.  L = 1 does the least work; more lanes cut the latency of small
// launches.  Pippenger's windows would cost more than the terms here.
template <class F> struct SmallMsmDigits;
template <> struct SmallMsmDigits<Fp2> { static constexpr int D = 4, TOP = 16, TABS = 1; };
template <> struct SmallMsmDigits<Fp> { static constexpr int D = 2, TOP = 32, TABS = 2; };

WBTE_INL void small_msm_digits(uint64_t lo[4], uint64_t hi[4], const uint64_t d[4], const G2X*) {
    for (int c = 0; c < 4; c++) {
        lo[c] = d[c];
        hi[c] = 0;
    }
}
// G1: w_c = d_{2c} + d_{2c+1} |x| as 128-bit integers (s = w_0 + w_1 |x|^2)
WBTE_INL void small_msm_digits(uint64_t lo[4], uint64_t hi[4], const uint64_t d[4], const G1X*) {
    for (int c = 0; c < 2; c++) {
        const uint64_t plo = d[2 * c + 1] * X_ABS, phi = __umul64hi(d[2 * c + 1], X_ABS);
        lo[c] = plo + d[2 * c];
        hi[c] = phi + (lo[c] < plo ? 1 : 0);
    }
}
template <class F>
WBTE_INL void small_msm_table(Xyzz<F>* tab, const Xyzz<F>& v) {  // tab[m] = [m + 1] v
    tab[0] = v;
    tab[1] = xyzz_dbl(v);
    for (int m = 2; m < 8; m++) tab[m] = xyzz_add(tab[m - 1], v);
}
WBTE_INL void small_msm_tables(G2X tab[1][8], const G2X& v) { small_msm_table(tab[0], v); }
WBTE_INL void small_msm_tables(G1X tab[2][8], const G1X& v) {
    small_msm_table(tab[0], v);
    small_msm_table(tab[1], xyzz_add(g1_phi(v), v));
}
// [dd] times the digit-c base, dd != 0
WBTE_INL G2X small_msm_entry(const G2X tab[1][8], int c, int dd) {
    G2X m = tab[0][(dd < 0 ? -dd : dd) - 1];
    for (int i = 0; i < c; i++) m = g2_psi(m);
    if (((c & 1) != 0) != (dd < 0)) m = neg(m);
    return m;
}
WBTE_INL G1X small_msm_entry(const G1X tab[2][8], int c, int dd) {
    G1X m = tab[c][(dd < 0 ? -dd : dd) - 1];
    if (dd < 0) m = neg(m);
    return m;
}

// [k]v for a canonical scalar k by one thread: all base-|x| digit groups of
// k (G1: two, G2: four) share one run of doublings (signed radix-16 Straus)
template <class F>
static __device__ __noinline__ Xyzz<F> mul_joint(const Xyzz<F> v, const uint8_t* scalar) {
    using S = SmallMsmDigits<F>;
    Xyzz<F> tab[S::TABS][8];
    small_msm_tables(tab, v);
    uint32_t sc[8];
    load_scalar(sc, scalar);
    uint64_t d[4], lo[4], hi[4];
    decompose_base_x(d, sc);
    small_msm_digits(lo, hi, d, (const Xyzz<F>*)nullptr);
    Xyzz<F> acc;
    set_inf(acc);
    for (int kk = S::TOP; kk >= 0; kk--) {
        if (kk != S::TOP) {
            acc = xyzz_dbl(acc);
            acc = xyzz_dbl(acc);
            acc = xyzz_dbl(acc);
            acc = xyzz_dbl(acc);
        }
        for (int c = 0; c < S::D; c++) {
            const int dd = r16_digit(lo[c], hi[c], kk, S::TOP);
            if (dd) acc = xyzz_add(acc, small_msm_entry(tab, c, dd));
        }
    }
    return acc;
}

// width-5 NAF of the 128-bit w = hi 2^64 + lo: digits in {0, +-1, +-3, .., +-15},
// least significant first; returns the length (at most 129)
WBTE_INL int wnaf5_128(int8_t* dig, uint64_t lo, uint64_t hi) {
    int len = 0;
    while (lo | hi) {
        int d = 0;
        if (lo & 1) {
            d = (int)(lo & 31);
            if (d >= 16) d -= 32;
            if (d > 0) {
                const uint64_t n = lo - (uint64_t)d;
                hi -= n > lo ? 1 : 0;
                lo = n;
            } else {
                const uint64_t n = lo + (uint64_t)(-d);
                hi += n < lo ? 1 : 0;
                lo = n;
            }
        }
        dig[len++] = (int8_t)d;
        lo = (lo >> 1) | (hi << 63);
        hi >>= 1;
    }
    return len;
}

// [k]v on G1 for a canonical scalar k by one thread: the two GLV digit groups
// w_0, w_1 (v and phi(v) + v) in width-5 NAF over one run of doublings,
// tables of odd multiples.  Control flow follows the digits, so it is meant
// for warps whose threads share the scalar (no divergence then).
static __device__ __noinline__ G1X g1_mul_joint_naf(const G1X v, const uint8_t* scalar) {
    G1X tab[2][8];  // odd multiples 1, 3, .., 15 of v and of phi(v) + v
    tab[0][0] = v;
    tab[1][0] = xyzz_add(g1_phi(v), v);
    for (int c = 0; c < 2; c++) {
        const G1X two = xyzz_dbl(tab[c][0]);
        for (int m = 1; m < 8; m++) tab[c][m] = xyzz_add(tab[c][m - 1], two);
    }
    uint32_t sc[8];
    load_scalar(sc, scalar);
    uint64_t d[4], lo[4], hi[4];
    decompose_base_x(d, sc);
    small_msm_digits(lo, hi, d, (const G1X*)nullptr);
    int8_t naf[2][130];
    const int l0 = wnaf5_128(naf[0], lo[0], hi[0]), l1 = wnaf5_128(naf[1], lo[1], hi[1]);
    G1X acc;
    set_inf(acc);
    bool started = false;
    for (int pos = (l0 > l1 ? l0 : l1) - 1; pos >= 0; pos--) {
        if (started) acc = xyzz_dbl(acc);
        for (int c = 0; c < 2; c++) {
            const int dd = pos < (c ? l1 : l0) ? naf[c][pos] : 0;
            if (!dd) continue;
            G1X m = tab[c][((dd < 0 ? -dd : dd) - 1) >> 1];
            if (dd < 0) m = neg(m);
            acc = started ? xyzz_add(acc, m) : m;
            started = true;
        }
    }
    return acc;
}

// One radix-2 butterfly per thread with the twiddle multiplication on one
// thread (mul_joint: the digit groups share their doublings), for batches of
// transforms large enough to fill the GPU without the lane split.  Threads
// take the transforms fastest, so a warp shares one twiddle.
template <class F>
__global__ void __launch_bounds__(WARP) k_ntt_stage_joint(uint8_t* work, const uint8_t* tw, int64_t n, int64_t half,
                                                         int64_t count, int64_t pad) {
    // threads take the transforms fastest over `pad` >= count slots; slots
    // past count idle (pad a multiple of 32: every warp shares one twiddle)
    const int64_t g = (int64_t)blockIdx.x * WARP + threadIdx.x;
    if (g >= (n / 2) * pad) return;
    const int64_t q = g % pad, tt = g / pad;
    if (q >= count) return;
    const int64_t chunk = tt / half, j = tt % half;
    const int64_t a = q * n + chunk * 2 * half + j, b = a + half;
    Xyzz<F>* w = reinterpret_cast<Xyzz<F>*>(work);
    Xyzz<F> t = load_vec(w + b);
    if (j != 0) {
        const uint8_t* sc = tw + FR_SZ * (j * (n / (2 * half)));
        if constexpr (std::is_same<F, Fp>::value) {
            // whole warps share the twiddle when the slots come in multiples of 32
            t = pad % WARP == 0 ? g1_mul_joint_naf(t, sc) : mul_joint(t, sc);
        } else {
            t = mul_joint(t, sc);
        }
    }
    const Xyzz<F> u = load_vec(w + a);
    store_vec(w + a, xyzz_add(u, t));
    store_vec(w + b, xyzz_add(u, neg(t)));
}

template <class F>
__global__ void __launch_bounds__(WARP) k_small_msm(uint8_t* out, const uint8_t* points, const int64_t* pbase,
                                                   const int32_t* idx, const uint8_t* scalars, const int32_t* vsel,
                                                   int64_t k, int64_t n, int L) {
    using S = SmallMsmDigits<F>;
    constexpr int D = S::D;
    using A = Affine<F>;
    __shared__ Xyzz<F> sh[WARP];
    const int lane = threadIdx.x, sub = lane % L;
    const int64_t o = ((int64_t)blockIdx.x * WARP + lane) / L;
    const bool active = o < k;
    Xyzz<F> acc;
    set_inf(acc);
    if (active) {
        const int64_t v = vsel ? (int64_t)vsel[o] : 0;
        const A* P = reinterpret_cast<const A*>(points) + pbase[o];
        Xyzz<F> tab[SMALL_MSM_MAX][S::TABS][8];
        uint64_t lo[SMALL_MSM_MAX][4], hi[SMALL_MSM_MAX][4];
        // this lane's pairs p = sub, sub + L, ... (term p / D, digit p % D):
        // every lane of a warp runs the same iterations, so the warp stays converged
        int prev = -1;
        for (int p = sub; p < n * D; p += L) {
            const int t = p / D;
            if (t == prev) continue;
            prev = t;
            small_msm_tables(tab[t], from_affine(load_affine(P + (idx ? (int64_t)idx[t] : t))));
            uint32_t sc[8];
            load_scalar(sc, scalars + FR_SZ * (v * n + t));
            uint64_t d[4];
            decompose_base_x(d, sc);
            small_msm_digits(lo[t], hi[t], d, (const Xyzz<F>*)nullptr);
        }
        for (int kk = S::TOP; kk >= 0; kk--) {
            if (kk != S::TOP) {
                acc = xyzz_dbl(acc);
                acc = xyzz_dbl(acc);
                acc = xyzz_dbl(acc);
                acc = xyzz_dbl(acc);
            }
            for (int p = sub; p < n * D; p += L) {
                const int t = p / D, c = p % D;
                const int dd = r16_digit(lo[t][c], hi[t][c], kk, S::TOP);
                if (dd) acc = xyzz_add(acc, small_msm_entry(tab[t], c, dd));
            }
        }
    }
    store_vec(sh + lane, acc);
    __syncwarp();
    for (int step = 1; step < L; step *= 2) {
        if (sub % (2 * step) == 0) store_vec(sh + lane, xyzz_add(load_vec(sh + lane), load_vec(sh + lane + step)));
        __syncwarp();
    }
    if (active && sub == 0)
        store_affine(reinterpret_cast<A*>(out + GroupOf<F>::AFF * o), to_affine(load_vec(sh + lane)));
}

// XYZZ to affine for n points sharing one field inversion per chunk of C
// consecutive points (Montgomery's trick): x = X / ZZ, y = Y / ZZZ with
// 1 / (ZZ ZZZ) from the chunk's prefix products, which the forward pass
// keeps in the x slots of the output.  The point at infinity (ZZ = 0)
// skips the products and is written as zero bytes.
template <class F>
__global__ void k_xyzz_to_affine_batch(uint8_t* out, const uint8_t* work, int64_t n, int64_t C) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t lo = t * C, hi = lo + C < n ? lo + C : n;
    if (lo >= n) return;
    using A = Affine<F>;
    const Xyzz<F>* in = reinterpret_cast<const Xyzz<F>*>(work);
    A* o = reinterpret_cast<A*>(out);
    F acc;
    f_set_one(acc);
    for (int64_t i = lo; i < hi; i++) {
        const Xyzz<F> p = load_vec(in + i);
        A pre;
        pre.x = acc;
        f_set_zero(pre.y);
        store_affine(o + i, pre);
        if (!is_inf(p)) acc = f_mul(acc, f_mul(p.ZZ, p.ZZZ));
    }
    F inv = f_inv(acc);
    for (int64_t i = hi - 1; i >= lo; i--) {
        const Xyzz<F> p = load_vec(in + i);
        A r;
        if (is_inf(p)) {
            set_inf(r);
        } else {
            const F w = f_mul(p.ZZ, p.ZZZ);
            const F t_i = f_mul(inv, load_vec(o + i).x);  // 1 / (ZZ_i ZZZ_i), written above (plain load)
            inv = f_mul(inv, w);
            r.x = f_mul(p.X, f_mul(t_i, p.ZZZ));
            r.y = f_mul(p.Y, f_mul(t_i, p.ZZ));
        }
        store_affine(o + i, r);
    }
}

// blst's projective points (Jacobian X, Y, Z: x = X / Z^2, y = Y / Z^3) to
// affine, one inversion per chunk of C points (blst_p{1,2}s_to_affine);
// Z = 0 gives the all-zero identity.
template <class F>
__global__ void k_jacobian_to_affine_batch(uint8_t* out, const uint8_t* in, int64_t n, int64_t C) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t lo = t * C, hi = lo + C < n ? lo + C : n;
    if (lo >= n) return;
    using A = Affine<F>;
    struct Jac { F X, Y, Z; };
    const Jac* P = reinterpret_cast<const Jac*>(in);
    A* o = reinterpret_cast<A*>(out);
    F acc;
    f_set_one(acc);
    for (int64_t i = lo; i < hi; i++) {
        const Jac p = load_vec(P + i);
        A pre;
        pre.x = acc;
        f_set_zero(pre.y);
        store_affine(o + i, pre);
        if (!f_is_zero(p.Z)) acc = f_mul(acc, p.Z);
    }
    F inv = f_inv(acc);
    for (int64_t i = hi - 1; i >= lo; i--) {
        const Jac p = load_vec(P + i);
        A r;
        if (f_is_zero(p.Z)) {
            set_inf(r);
        } else {
            const F zi = f_mul(inv, load_vec(o + i).x);  // 1 / Z_i, written above (plain load)
            inv = f_mul(inv, p.Z);
            const F z2 = f_sqr(zi);
            r.x = f_mul(p.X, z2);
            r.y = f_mul(p.Y, f_mul(z2, zi));
        }
        store_affine(o + i, r);
    }
}


// ------------------------------------------------------------ encodings
WBTE_INL void fp_store_be48(uint8_t* out, const Fp& m) {
    Fp c = fp_from_mont(m);
    for (int i = 0; i < 48; i++) out[47 - i] = (uint8_t)(c.v[i >> 2] >> (8 * (i & 3)));
}
WBTE_INL bool fp_largest(const Fp& m) {
    Fp c = fp_from_mont(m);
    for (int i = 11; i >= 0; i--) {
        if (c.v[i] != C_P_HALF[i]) return c.v[i] > C_P_HALF[i];
    }
    return false;
}
__global__ void k_g1_compress(uint8_t* out, const uint8_t* in, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    G1A p = load_affine(reinterpret_cast<const G1A*>(in + G1_AFF * i));
    uint8_t* o = out + 48 * i;
    if (is_inf(p)) {
        for (int b = 0; b < 48; b++) o[b] = 0;
        o[0] = 0xc0;
        return;
    }
    fp_store_be48(o, p.x);
    o[0] |= 0x80 | (fp_largest(p.y) ? 0x20 : 0);
}
__global__ void k_g2_compress(uint8_t* out, const uint8_t* in, int64_t n) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    G2A p = load_affine(reinterpret_cast<const G2A*>(in + G2_AFF * i));
    uint8_t* o = out + 96 * i;
    if (is_inf(p)) {
        for (int b = 0; b < 96; b++) o[b] = 0;
        o[0] = 0xc0;
        return;
    }
    fp_store_be48(o, p.x.c1);
    fp_store_be48(o + 48, p.x.c0);
    bool largest = fp_is_zero(p.y.c1) ? fp_largest(p.y.c0) : fp_largest(p.y.c1);
    o[0] |= 0x80 | (largest ? 0x20 : 0);
}

// ------------------------------------------------------- decompression
// ZCash-format decoding as blstrs' checked from_compressed: big-endian x with
// flags in the top bits of the first byte (0x80 compressed, 0x40 infinity,
// 0x20 y is the larger root); x must be canonical, the point on the curve and,
// when asked, in the prime-order subgroup ([r]P = O).
enum DecodeStatus : uint8_t { DECODE_OK = 0, DECODE_BAD_ENCODING = 1, DECODE_NOT_ON_CURVE = 2, DECODE_NOT_IN_GROUP = 3 };

// a^e for one of the square-root exponents (E = 0: (p + 1) / 4, 1: (p - 3) / 4),
// 4-bit fixed windows; F = Fp or Fp2
template <int E, class F>
static __device__ __noinline__ F pow_sqrt_exp(F a) {
    F tab[16];
    f_set_one(tab[0]);
    tab[1] = a;
    for (int i = 2; i < 16; i++) tab[i] = f_mul(tab[i - 1], a);
    F r;
    f_set_one(r);
    bool started = false;
    for (int w = 95; w >= 0; w--) {
        if (started) {
            r = f_sqr(r);
            r = f_sqr(r);
            r = f_sqr(r);
            r = f_sqr(r);
        }
        const uint32_t limb = E == 0 ? C_P_PLUS1_DIV4[w / 8] : C_P_MINUS3_DIV4[w / 8];
        const uint32_t d = (limb >> (4 * (w % 8))) & 15u;
        if (d) {
            r = started ? f_mul(r, tab[d]) : tab[d];
            started = true;
        }
    }
    return r;
}

// big-endian 48 bytes -> canonical limbs; false if the value is not below p
WBTE_INL bool fp_load_be48(Fp& canon, const uint8_t* in, uint8_t first_mask) {
    for (int i = 0; i < 12; i++) canon.v[i] = 0;
    for (int b = 0; b < 48; b++) {
        const uint32_t byte = b == 0 ? (in[0] & first_mask) : in[b];
        canon.v[(47 - b) >> 2] |= byte << (8 * ((47 - b) & 3));
    }
    for (int i = 11; i >= 0; i--)
        if (canon.v[i] != C_P[i]) return canon.v[i] < C_P[i];
    return false;
}

// sqrt in Fp (p = 3 mod 4): a^((p + 1) / 4), checked
WBTE_INL bool fp_sqrt(Fp& r, const Fp& a) {
    r = pow_sqrt_exp<0>(a);
    return fp_eq(fp_sqr(r), a);
}

// sqrt in Fp2 for p = 3 mod 4, the complex method (Adj and Rodriguez-
// Henriquez, "Square root computation over even extension fields",
// Algorithm 9): a1 = a^((p - 3) / 4), alpha = a1^2 a, x0 = a1 a; alpha = -1
// gives u x0, else (1 + alpha)^((p - 1) / 2) x0; the result is checked
WBTE_INL bool fp2_sqrt(Fp2& r, const Fp2& a) {
    const Fp2 a1 = pow_sqrt_exp<1>(a);
    const Fp2 alpha = fp2_mul(fp2_sqr(a1), a);
    const Fp2 x0 = fp2_mul(a1, a);
    const Fp2 minus_one = fp2_neg(fp2_one());
    if (fp2_eq(alpha, minus_one)) {
        r = Fp2{fp_neg(x0.c1), x0.c0};  // u x0
    } else {
        // (1 + alpha)^((p - 1) / 2) = (1 + alpha)^((p - 3) / 4 * 2 + 1)
        const Fp2 t = fp2_add(fp2_one(), alpha);
        const Fp2 h = pow_sqrt_exp<1>(t);
        r = fp2_mul(fp2_mul(fp2_sqr(h), t), x0);
    }
    return fp2_eq(fp2_sqr(r), a);
}

template <class F>
WBTE_INL bool in_prime_subgroup(const Affine<F>& p) {
    uint32_t r[8];
    for (int i = 0; i < 8; i++) r[i] = C_R[i];
    return is_inf(xyzz_mul(from_affine(p), r));
}

__global__ void k_g1_decompress(uint8_t* out, uint8_t* status, const uint8_t* in, int64_t n, int check_group) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t* c = in + 48 * i;
    G1A p;
    set_inf(p);
    uint8_t st = DECODE_OK;
    const uint8_t flags = c[0] & 0xe0;
    if (!(flags & 0x80)) {
        st = DECODE_BAD_ENCODING;
    } else if (flags & 0x40) {
        bool zero = (flags & 0x20) == 0 && (c[0] & 0x1f) == 0;
        for (int b = 1; b < 48; b++) zero = zero && c[b] == 0;
        if (!zero) st = DECODE_BAD_ENCODING;
    } else {
        Fp x;
        if (!fp_load_be48(x, c, 0x1f)) {
            st = DECODE_BAD_ENCODING;
        } else {
            x = fp_to_mont(x);
            const Fp rhs = fp_add(fp_mul(fp_sqr(x), x), fp_from_const(C_FP_B1));
            Fp y;
            if (!fp_sqrt(y, rhs)) {
                st = DECODE_NOT_ON_CURVE;
            } else {
                if (fp_largest(y) != ((flags & 0x20) != 0)) y = fp_neg(y);
                p.x = x;
                p.y = y;
                if (check_group && !in_prime_subgroup(p)) st = DECODE_NOT_IN_GROUP;
            }
        }
    }
    if (st != DECODE_OK) set_inf(p);
    store_affine(reinterpret_cast<G1A*>(out + G1_AFF * i), p);
    status[i] = st;
}

__global__ void k_g2_decompress(uint8_t* out, uint8_t* status, const uint8_t* in, int64_t n, int check_group) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint8_t* c = in + 96 * i;
    G2A p;
    set_inf(p);
    uint8_t st = DECODE_OK;
    const uint8_t flags = c[0] & 0xe0;
    if (!(flags & 0x80)) {
        st = DECODE_BAD_ENCODING;
    } else if (flags & 0x40) {
        bool zero = (flags & 0x20) == 0 && (c[0] & 0x1f) == 0;
        for (int b = 1; b < 96; b++) zero = zero && c[b] == 0;
        if (!zero) st = DECODE_BAD_ENCODING;
    } else {
        Fp x1, x0;  // x = x0 + x1 u, x1 first
        if (!fp_load_be48(x1, c, 0x1f) || !fp_load_be48(x0, c + 48, 0xff)) {
            st = DECODE_BAD_ENCODING;
        } else {
            const Fp2 x{fp_to_mont(x0), fp_to_mont(x1)};
            const Fp2 b{fp_from_const(C_FP_B1), fp_from_const(C_FP_B1)};  // 4 (1 + u)
            const Fp2 rhs = fp2_add(fp2_mul(fp2_sqr(x), x), b);
            Fp2 y;
            if (!fp2_sqrt(y, rhs)) {
                st = DECODE_NOT_ON_CURVE;
            } else {
                const bool largest = fp_is_zero(y.c1) ? fp_largest(y.c0) : fp_largest(y.c1);
                if (largest != ((flags & 0x20) != 0)) y = fp2_neg(y);
                p.x = x;
                p.y = y;
                if (check_group && !in_prime_subgroup(p)) st = DECODE_NOT_IN_GROUP;
            }
        }
    }
    if (st != DECODE_OK) set_inf(p);
    store_affine(reinterpret_cast<G2A*>(out + G2_AFF * i), p);
    status[i] = st;
}

// [s]G from the generator table (one mixed addition per byte of s) and [c]X
// by the joint base-|x| form (the two digit groups share their doublings)
__global__ void k_schnorr_verify(uint8_t* valid, const uint8_t* X, const uint8_t* R, const uint8_t* sresp,
                                 const uint8_t* c, int64_t n, const uint8_t* gen_table) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const G1A* T = reinterpret_cast<const G1A*>(gen_table);
    const uint8_t* sb = sresp + FR_SZ * i;
    G1X lhs;
    set_inf(lhs);
    for (int w = 0; w < 32; w++) {
        const uint32_t d = sb[w];
        if (d) lhs = xyzz_madd(lhs, load_affine(T + 256 * w + d));
    }
    G1X cx = mul_joint(from_affine(load_affine(reinterpret_cast<const G1A*>(X + G1_AFF * i))), c + FR_SZ * i);
    G1A r = load_affine(reinterpret_cast<const G1A*>(R + G1_AFF * i));
    G1X rhs = xyzz_madd(cx, r);
    G1X diff = xyzz_add(lhs, neg(rhs));
    valid[i] = is_inf(diff) ? 1 : 0;
}

// Integer-pipe calibration: eight independent chains of 32-bit multiply-adds
// per thread, half low and half high products (the mix of the CIOS kernel).
__global__ void k_imad_probe(uint32_t* sink, int iters) {
    uint32_t a[8], b = 0x9e3779b9u + threadIdx.x;
    for (int k = 0; k < 8; k++) a[k] = threadIdx.x * 7u + blockIdx.x + (uint32_t)k;
    for (int i = 0; i < iters; i++) {
        _Pragma("unroll") for (int k = 0; k < 8; k += 2) {
            asm volatile("mad.lo.u32 %0, %0, %1, %0;" : "+r"(a[k]) : "r"(b));
            asm volatile("mad.hi.u32 %0, %0, %1, %0;" : "+r"(a[k + 1]) : "r"(b));
        }
    }
    uint32_t x = 0;
    for (int k = 0; k < 8; k++) x ^= a[k];
    if (x == 0x12345678u) sink[0] = x;
}

}  // namespace

// IMAD instructions per second sustained by the integer pipe (measured).
double measure_imad_rate(cudaStream_t s) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint32_t* sink = nullptr;
    if (cudaMallocAsync(&sink, 16, s) != cudaSuccess) return 0.0;
    const int iters = 8192, threads = 256, blocks = sms * 8;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    note_launch();
    k_imad_probe<<<blocks, threads, 0, s>>>(sink, iters / 8);  // warm-up
    cudaEventRecord(a, s);
    note_launch();
    k_imad_probe<<<blocks, threads, 0, s>>>(sink, iters);
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFreeAsync(sink, s);
    double ops = (double)blocks * threads * iters * 8.0;
    return ms > 0 ? ops / (ms * 1e-3) : 0.0;
}

// ============================================================ launchers
void launch_fr_powers(uint8_t* out, const uint8_t* base, int64_t n, int64_t first, cudaStream_t s) {
    ProfScope prof_("fr_scalars", s);
    if (n <= 0) return;
    note_launch();
    k_fr_powers<<<blocks_for(n), TPB, 0, s>>>(out, base, n, first);
}
void launch_fr_mul_gather(uint8_t* out, const uint8_t* a, const uint8_t* b, const int32_t* bidx, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    note_launch();
    k_fr_mul_gather<<<blocks_for(n), TPB, 0, s>>>(out, a, b, bidx, n);
}
void launch_fr_scale(uint8_t* out, const uint8_t* a, const uint8_t* c, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    note_launch();
    k_fr_scale<<<blocks_for(n), TPB, 0, s>>>(out, a, c, n);
}
void launch_fr_scale_size_inv(uint8_t* out, const uint8_t* a, int log_m, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    note_launch();
    k_fr_scale_size_inv<<<blocks_for(n), TPB, 0, s>>>(out, a, log_m, n);
}
void launch_material_scalars(uint8_t* out, const uint8_t* z, const int32_t* owner, const uint8_t* qp, int64_t W,
                             int64_t N, int64_t rows, cudaStream_t s) {
    ProfScope prof_("fr_scalars", s);
    if (rows * W <= 0) return;
    note_launch();
    k_material_scalars<<<blocks_for(rows * W), TPB, 0, s>>>(out, z, owner, qp, W, N, rows);
}
void launch_wpfe_fractions(uint8_t* g, uint8_t* u, const uint8_t* rho, const uint8_t* alpha, const uint8_t* masks,
                           int64_t N, int64_t B, bool party_major, cudaStream_t s) {
    ProfScope prof_("fr_fractions", s);
    if (N * B <= 0) return;
    note_launch();
    k_wpfe_fractions<<<blocks_for(N * B), TPB, 0, s>>>(g, u, rho, alpha, masks, N, B, party_major ? 1 : 0);
}
void launch_gather(uint8_t* out, const uint8_t* in, const int32_t* idx, int64_t n, int64_t record, cudaStream_t s) {
    if (n <= 0) return;
    note_launch();
    k_gather<<<blocks_for(n), TPB, 0, s>>>(out, in, idx, n, record);
}
void launch_lagrange_at_zero(uint8_t* out, const uint8_t* x, int64_t n, int32_t* status, cudaStream_t s) {
    ProfScope prof_("lagrange", s);
    if (n <= 0) return;
    note_launch();
    k_lagrange<<<blocks_for(n, 64), 64, 0, s>>>(out, x, n, status);
}
void launch_domain_twiddles(uint8_t* tw, int64_t n, int64_t count, bool inverse, cudaStream_t s) {
    if (count <= 0) return;
    int lg = 0;
    while ((int64_t(1) << lg) < n) lg++;
    note_launch();
    k_domain_twiddles<<<blocks_for(count), TPB, 0, s>>>(tw, lg, count, inverse);
}

void launch_mul_batch(Group g, uint8_t* out, const uint8_t* pts, int64_t stride, const uint8_t* scalars, int64_t n, cudaStream_t s) {
    ProfScope prof_("mul_batch", s);
    if (n <= 0) return;
    note_launch();
    if (g == GROUP_G1) k_mul_batch<Fp><<<blocks_for(n), TPB, 0, s>>>(out, pts, stride, scalars, n);
    else k_mul_batch<Fp2><<<blocks_for(n), TPB, 0, s>>>(out, pts, stride, scalars, n);
}

// Generator tables are built once per device on first use.  The build is
// finished (stream synchronised) before the table is published, so callers
// on other streams never read a table still being written.
static uint8_t* g_gen_table[2][64] = {};
static std::mutex g_gen_mu;
// the generator table of group g on the current device (null on failure)
static const uint8_t* generator_table(Group g, cudaStream_t s) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return nullptr;
    int gi = g == GROUP_G1 ? 0 : 1;
    size_t aff = g == GROUP_G1 ? G1_AFF : G2_AFF;
    std::lock_guard<std::mutex> lock(g_gen_mu);
    if (!g_gen_table[gi][dev]) {
        uint8_t* t = nullptr;
        if (cudaMalloc(&t, aff * 256 * 32) != cudaSuccess) return nullptr;
        note_launch();
        if (g == GROUP_G1) k_build_gen_table<Fp><<<32, 256, 0, s>>>(t);
        else k_build_gen_table<Fp2><<<32, 256, 0, s>>>(t);
        if (cudaStreamSynchronize(s) != cudaSuccess) return nullptr;
        g_gen_table[gi][dev] = t;
    }
    return g_gen_table[gi][dev];
}
void launch_mul_generator(Group g, uint8_t* out, const uint8_t* scalars, int64_t n, cudaStream_t s) {
    ProfScope prof_("mul_generator", s);
    if (n <= 0) return;
    const uint8_t* table = generator_table(g, s);
    if (!table) return;
    note_launch();
    if (g == GROUP_G1) k_mul_generator<Fp><<<blocks_for(n), TPB, 0, s>>>(out, table, scalars, n);
    else k_mul_generator<Fp2><<<blocks_for(n), TPB, 0, s>>>(out, table, scalars, n);
}

void launch_mul_pow2(Group g, uint8_t* out, const uint8_t* in, int64_t n, int k, cudaStream_t s) {
    ProfScope prof_("mul_pow2", s);
    if (n <= 0) return;
    note_launch();
    if (g == GROUP_G1) k_mul_pow2<Fp><<<blocks_for(n), TPB, 0, s>>>(out, in, n, k);
    else k_mul_pow2<Fp2><<<blocks_for(n), TPB, 0, s>>>(out, in, n, k);
}
void launch_segment_sum(Group g, uint8_t* out, const uint8_t* in, const int64_t* offsets, int64_t k, cudaStream_t s) {
    ProfScope prof_("point_sum", s);
    if (k <= 0) return;
    note_launch();
    if (g == GROUP_G1) k_segment_sum<Fp><<<blocks_for(k), TPB, 0, s>>>(out, in, offsets, k);
    else k_segment_sum<Fp2><<<blocks_for(k), TPB, 0, s>>>(out, in, offsets, k);
}
void launch_negate(Group g, uint8_t* out, const uint8_t* in, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    note_launch();
    if (g == GROUP_G1) k_negate<Fp><<<blocks_for(n), TPB, 0, s>>>(out, in, n);
    else k_negate<Fp2><<<blocks_for(n), TPB, 0, s>>>(out, in, n);
}

// Whether a transform stage of `butterflies` butterflies runs one thread per
// butterfly (k_ntt_stage_joint) rather than the lane split: a cost model of one
// thread's Fp products (G1: 128 doublings and 66 additions joint, against 128
// and 33 per lane on 2 lanes; G2: 64 and 68 against 64 and 17 per lane on 4
// lanes) times max(1, threads / resident threads).  WBTE_NTT_JOINT = 0 or 1
// overrides the choice, and so does the calling context's tuning knob.
static bool ntt_joint(Group g, int64_t butterflies) {
    if (const char* env = getenv("WBTE_NTT_JOINT")) return atoi(env) != 0;
    if (g_tune.ntt_joint == 0 || g_tune.ntt_joint == 1) return g_tune.ntt_joint == 1;
    static std::atomic<int64_t> cap[2][2] = {{{0}, {0}}, {{0}, {0}}};
    const int gi = g == GROUP_G1 ? 0 : 1;
    int64_t c[2];
    for (int v = 0; v < 2; v++) {
        c[v] = cap[gi][v].load();
        if (c[v] == 0) {
            int dev = 0, sms = 0, blocks = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (g == GROUP_G1)
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &blocks, v ? (const void*)k_ntt_stage_joint<Fp> : (const void*)k_ntt_stage<Fp>, WARP, 0);
            else
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &blocks, v ? (const void*)k_ntt_stage_joint<Fp2> : (const void*)k_ntt_stage<Fp2>, WARP, 0);
            c[v] = (int64_t)(blocks > 0 ? blocks : 1) * WARP * (sms > 0 ? sms : 1);
            cap[gi][v].store(c[v]);
        }
    }
    const bool g1 = g == GROUP_G1;
    const int L = g1 ? NttLanes<Fp>::L : NttLanes<Fp2>::L;
    const double dbl = g1 ? 9.0 : 30.0, add = g1 ? 12.0 : 42.0, dbls = g1 ? 128.0 : 64.0;
    const double adds_joint = g1 ? 66.0 + 15.0 : 68.0 + 7.0, adds_lane = g1 ? 33.0 + 8.0 : 17.0 + 7.0;
    const double joint = std::max(1.0, (double)butterflies / (double)c[1]) * (dbls * dbl + adds_joint * add);
    const double lane = std::max(1.0, (double)(butterflies * L) / (double)c[0]) * (dbls * dbl + adds_lane * add);
    return joint < lane;
}

// work[i] = [c_i] in[i] for small signed c_i (XYZZ out): double-and-add over
// the bits of |c_i| with mixed additions of the affine input, negated for
// negative c_i -- mul_group_signed_small, weighted_pfe/src/decryption.rs:736-760.
template <class F>
__global__ void k_mul_small(uint8_t* work, const uint8_t* in, const int32_t* coeffs, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    using A = Affine<F>;
    const int32_t c = coeffs[i];
    const uint32_t mag = c < 0 ? (uint32_t)(-(int64_t)c) : (uint32_t)c;
    Xyzz<F> acc;
    set_inf(acc);
    if (mag) {
        const A p = load_affine(reinterpret_cast<const A*>(in + GroupOf<F>::AFF * i));
        for (int b = 31 - __clz(mag); b >= 0; b--) {
            acc = xyzz_dbl(acc);
            if ((mag >> b) & 1) acc = xyzz_madd(acc, p);
        }
        if (c < 0) acc = neg(acc);
    }
    store_vec(reinterpret_cast<Xyzz<F>*>(work) + i, acc);
}

// Points per thread of the batched conversions: one inversion (about 485
// Fp products) per chunk against about 7 products per point, so chunks grow
// only while the launch still fills the resident threads.
static int64_t normalize_chunk(int64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t resident = (int64_t)(sms > 0 ? sms : 148) * 256;
    int64_t C = n / resident;
    return C < 1 ? 1 : (C > 32 ? 32 : C);
}

void launch_xyzz_to_affine(Group g, uint8_t* out, const uint8_t* work, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    const int64_t C = normalize_chunk(n), threads = (n + C - 1) / C;
    note_launch();
    if (g == GROUP_G1) k_xyzz_to_affine_batch<Fp><<<blocks_for(threads), TPB, 0, s>>>(out, work, n, C);
    else k_xyzz_to_affine_batch<Fp2><<<blocks_for(threads), TPB, 0, s>>>(out, work, n, C);
}

void launch_mul_small(Group g, uint8_t* out, const uint8_t* in, const int32_t* coeffs, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    uint8_t* work = nullptr;
    if (cudaMallocAsync(&work, (g == GROUP_G1 ? G1_XYZZ : G2_XYZZ) * (size_t)n, s) != cudaSuccess) return;
    note_launch();
    if (g == GROUP_G1) k_mul_small<Fp><<<blocks_for(n), TPB, 0, s>>>(work, in, coeffs, n);
    else k_mul_small<Fp2><<<blocks_for(n), TPB, 0, s>>>(work, in, coeffs, n);
    launch_xyzz_to_affine(g, out, work, n, s);
    cudaFreeAsync(work, s);
}

void launch_batch_normalize(Group g, uint8_t* out, const uint8_t* in, int64_t n, cudaStream_t s) {
    if (n <= 0) return;
    const int64_t C = normalize_chunk(n), threads = (n + C - 1) / C;
    note_launch();
    if (g == GROUP_G1) k_jacobian_to_affine_batch<Fp><<<blocks_for(threads), TPB, 0, s>>>(out, in, n, C);
    else k_jacobian_to_affine_batch<Fp2><<<blocks_for(threads), TPB, 0, s>>>(out, in, n, C);
}

void launch_group_ntt(Group g, uint8_t* io, uint8_t* work, const uint8_t* tw, int64_t n, cudaStream_t s, int64_t count) {
    if (n <= 0 || count <= 0) return;
    if (g == GROUP_G1 && count > WARP && count % WARP != 0) {
        // the largest multiple of 32 transforms takes the warp-uniform NAF
        // twiddles of k_ntt_stage_joint; the rest runs on its own
        const int64_t a = count - count % WARP;
        launch_group_ntt(g, io, work, tw, n, s, a);
        launch_group_ntt(g, io + G1_AFF * (size_t)(n * a), work + G1_XYZZ * (size_t)(n * a), tw, n, s, count - a);
        return;
    }
    ProfScope prof_(g == GROUP_G1 ? "ntt_g1" : "ntt_g2", s);
    int bits = 0;
    while ((int64_t(1) << bits) < n) bits++;
    const int64_t total = n * count, butterflies = (n / 2) * count;
    if (g == GROUP_G1) {
        note_launch();
        k_ntt_load<Fp><<<blocks_for(total), TPB, 0, s>>>(work, io, n, bits, count);
        const bool joint = ntt_joint(g, butterflies);
        // 24..31 transforms run padded to 32 slots: warp-uniform NAF twiddles
        // with at most a quarter of the lanes idle
        const int64_t pad = count >= 24 && count < WARP ? (int64_t)WARP : count;
        for (int64_t half = 1; half < n; half *= 2) {
            note_launch();
            if (joint)
                k_ntt_stage_joint<Fp><<<blocks_for((n / 2) * pad, WARP), WARP, 0, s>>>(work, tw, n, half, count, pad);
            else
                k_ntt_stage<Fp><<<blocks_for(NttLanes<Fp>::L * butterflies, WARP), WARP, 0, s>>>(work, tw, n, half, count);
        }
        launch_xyzz_to_affine(GROUP_G1, io, work, total, s);
    } else {
        note_launch();
        k_ntt_load<Fp2><<<blocks_for(total), TPB, 0, s>>>(work, io, n, bits, count);
        const bool joint = ntt_joint(g, butterflies);
        for (int64_t half = 1; half < n; half *= 2) {
            note_launch();
            if (joint)
                k_ntt_stage_joint<Fp2><<<blocks_for(butterflies, WARP), WARP, 0, s>>>(work, tw, n, half, count, count);
            else
                k_ntt_stage<Fp2><<<blocks_for(NttLanes<Fp2>::L * butterflies, WARP), WARP, 0, s>>>(work, tw, n, half, count);
        }
        launch_xyzz_to_affine(GROUP_G2, io, work, total, s);
    }
}

// ------------------------------------------- fixed-base G2 MSMs of few terms
// For G2 points that stay fixed across many calls (a committee's verification
// keys), table[p][w][m - 1] = [m 64^w] P_p (w < FB_WINDOWS, 1 <= m <= 32,
// affine).  A term [s]P then costs one mixed addition per nonzero signed
// radix-64 digit of each base-|x| digit of s (digit c acting through
// (-1)^c psi^c, applied to the table entry), and no doublings.
constexpr int FB_WINDOWS = 11, FB_ENTRIES = 32;  // 64-bit digits, radix 64

// signed radix-64 digit k of d (d < 2^64): digits in [-31, 32], the carry
// into digit k set when the low k digits of d exceed 0x20..20 (32 in each)
WBTE_INL int r64_digit(uint64_t d, int k) {
    auto carry = [&](int j) -> int {
        if (j == 0 || 6 * j > 64) return 0;  // above bit 64 the bound exceeds any d < 2^64
        const uint64_t m = (1ull << (6 * j)) - 1;
        const uint64_t e = 0x820820820820820ull & m;  // 32 * 64^i summed over i < j
        return (d & m) > e;
    };
    const int nib = 6 * k < 64 ? (int)((d >> (6 * k)) & 63u) : 0;
    return nib + carry(k) - 64 * carry(k + 1);
}

__global__ void k_fixed_tables_g2(uint8_t* tables, const uint8_t* points, const int64_t* point_index, int64_t np) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= np * FB_WINDOWS) return;
    const int64_t p = g / FB_WINDOWS;
    const int w = (int)(g % FB_WINDOWS);
    G2X base = from_affine(load_affine(reinterpret_cast<const G2A*>(points) + point_index[p]));
    for (int i = 0; i < 6 * w; i++) base = xyzz_dbl(base);
    G2A* T = reinterpret_cast<G2A*>(tables) + (p * FB_WINDOWS + w) * FB_ENTRIES;
    G2X acc = base;
    for (int m = 1; m <= FB_ENTRIES; m++) {
        store_affine(T + m - 1, to_affine(acc));
        if (m < FB_ENTRIES) acc = xyzz_add(acc, base);
    }
}

// psi on an affine G2 point (the identity stays the identity)
WBTE_INL G2A g2a_psi(const G2A& a) {
    if (is_inf(a)) return a;
    return G2A{fp2_mul(fp2_conj(a.x), fp2_from_const(C_PSI_CX)), fp2_mul(fp2_conj(a.y), fp2_from_const(C_PSI_CY))};
}

// out[o] = sum_t scalars[vsel[o] n + t] * P(tbase[o] + tidx[t]), one thread per output
__global__ void __launch_bounds__(WARP) k_fixed_msm_g2(uint8_t* out, const uint8_t* tables, const int64_t* tbase,
                                                      const int32_t* tidx, const uint8_t* scalars,
                                                      const int32_t* vsel, int64_t k, int64_t n) {
    const int64_t o = (int64_t)blockIdx.x * WARP + threadIdx.x;
    if (o >= k) return;
    const int64_t v = vsel ? (int64_t)vsel[o] : 0;
    G2X acc;
    set_inf(acc);
    for (int64_t t = 0; t < n; t++) {
        const G2A* T = reinterpret_cast<const G2A*>(tables) +
                       (tbase[o] + (tidx ? (int64_t)tidx[t] : t)) * (FB_WINDOWS * FB_ENTRIES);
        uint32_t sc[8];
        load_scalar(sc, scalars + FR_SZ * (v * n + t));
        uint64_t d[4];
        decompose_base_x(d, sc);
        for (int c = 0; c < 4; c++)
            for (int w = 0; w < FB_WINDOWS; w++) {
                const int dd = r64_digit(d[c], w);
                if (!dd) continue;
                G2A m = load_affine(T + w * FB_ENTRIES + (dd < 0 ? -dd : dd) - 1);
                for (int i = 0; i < c; i++) m = g2a_psi(m);
                if (((c & 1) != 0) != (dd < 0)) m.y = fp2_neg(m.y);
                acc = xyzz_madd(acc, m);
            }
    }
    store_affine(reinterpret_cast<G2A*>(out + G2_AFF * o), to_affine(acc));
}

// Lanes per small-MSM output, from a cost model: a lane's work is its
// tables (7 additions per term it touches; 15 on G1, two tables), the shared
// doublings and one addition per window and pair it holds; the launch takes
// about max(1, k L / resident threads) times one lane's work.  The lanes run
// from 1 up to one per (term, digit) pair, rounded up to a power of two.
// WBTE_SMALL_MSM_LANES (a power of two up to 32) overrides the choice.
static int small_msm_lanes(Group g, int64_t k, int64_t n) {
    if (const char* env = getenv("WBTE_SMALL_MSM_LANES")) {
        const int v = atoi(env);
        if (v >= 1 && v <= WARP && (v & (v - 1)) == 0) return v;
    }
    static std::atomic<int64_t> cap[2] = {{0}, {0}};
    const int gi = g == GROUP_G1 ? 0 : 1;
    int64_t c = cap[gi].load();
    if (c == 0) {
        int dev = 0, sms = 0, blocks = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (g == GROUP_G1) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_small_msm<Fp>, WARP, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_small_msm<Fp2>, WARP, 0);
        c = (int64_t)(blocks > 0 ? blocks : 1) * WARP * (sms > 0 ? sms : 1);
        cap[gi].store(c);
    }
    const bool g1 = g == GROUP_G1;
    const int D = g1 ? SmallMsmDigits<Fp>::D : SmallMsmDigits<Fp2>::D;
    const int windows = (g1 ? SmallMsmDigits<Fp>::TOP : SmallMsmDigits<Fp2>::TOP) + 1;
    const double add = g1 ? 12.0 : 42.0, dbl = g1 ? 9.0 : 30.0, table = g1 ? 15.0 : 7.0;  // Fp products
    const int64_t pairs = n * D;
    int best = 1;
    double best_t = 0;
    for (int L = 1; L <= WARP; L *= 2) {
        int terms = 0, prev = -1;
        for (int64_t p = 0; p < pairs; p += L)
            if (p / D != prev) prev = (int)(p / D), terms++;
        const double lane = terms * table * add + 4.0 * (windows - 1) * dbl + (double)((pairs + L - 1) / L) * windows * add;
        const double t = std::max(1.0, (double)(k * L) / (double)c) * lane;
        if (L == 1 || t < best_t) best = L, best_t = t;
        if (L >= pairs) break;
    }
    return best;
}

void launch_small_msm(Group g, uint8_t* out, const uint8_t* points, const int64_t* pbase, const int32_t* idx,
                      const uint8_t* scalars, const int32_t* vsel, int64_t k, int64_t n, cudaStream_t s) {
    ProfScope prof_(g == GROUP_G1 ? "small_msm_g1" : "small_msm_g2", s);
    if (k <= 0) return;
    if (n < 1 || n > SMALL_MSM_MAX) return;
    const int L = small_msm_lanes(g, k, n);
    note_launch();
    if (g == GROUP_G1)
        k_small_msm<Fp><<<blocks_for(L * k, WARP), WARP, 0, s>>>(out, points, pbase, idx, scalars, vsel, k, n, L);
    else
        k_small_msm<Fp2><<<blocks_for(L * k, WARP), WARP, 0, s>>>(out, points, pbase, idx, scalars, vsel, k, n, L);
}

void launch_decompress(Group g, uint8_t* out, uint8_t* status, const uint8_t* in, int64_t n, bool check_group,
                       cudaStream_t s) {
    ProfScope prof_("decompress", s);
    if (n <= 0) return;
    note_launch();
    if (g == GROUP_G1) k_g1_decompress<<<blocks_for(n), TPB, 0, s>>>(out, status, in, n, check_group ? 1 : 0);
    else k_g2_decompress<<<blocks_for(n), TPB, 0, s>>>(out, status, in, n, check_group ? 1 : 0);
}

void launch_fixed_tables_g2(uint8_t* tables, const uint8_t* points, const int64_t* point_index, int64_t np,
                            cudaStream_t s) {
    ProfScope prof_("fixed_tables_g2", s);
    if (np <= 0) return;
    note_launch();
    k_fixed_tables_g2<<<blocks_for(np * FB_WINDOWS), TPB, 0, s>>>(tables, points, point_index, np);
}
void launch_fixed_msm_g2(uint8_t* out, const uint8_t* tables, const int64_t* tbase, const int32_t* tidx,
                         const uint8_t* scalars, const int32_t* vsel, int64_t k, int64_t n, cudaStream_t s) {
    ProfScope prof_("fixed_msm_g2", s);
    if (k <= 0) return;
    note_launch();
    k_fixed_msm_g2<<<blocks_for(k, WARP), WARP, 0, s>>>(out, tables, tbase, tidx, scalars, vsel, k, n);
}

void launch_compress(Group g, uint8_t* out, const uint8_t* in, int64_t n, cudaStream_t s) {
    ProfScope prof_("compress", s);
    if (n <= 0) return;
    note_launch();
    if (g == GROUP_G1) k_g1_compress<<<blocks_for(n), TPB, 0, s>>>(out, in, n);
    else k_g2_compress<<<blocks_for(n), TPB, 0, s>>>(out, in, n);
}

void launch_schnorr_verify(uint8_t* valid, const uint8_t* X, const uint8_t* R, const uint8_t* sresp, const uint8_t* c,
                           int64_t n, cudaStream_t st) {
    ProfScope prof_("schnorr_verify", st);
    if (n <= 0) return;
    note_launch();
    const uint8_t* table = generator_table(GROUP_G1, st);
    if (!table) return;
    k_schnorr_verify<<<blocks_for(n), TPB, 0, st>>>(valid, X, R, sresp, c, n, table);
}

}  // namespace wbte
