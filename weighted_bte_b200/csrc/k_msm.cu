// Pippenger multi-scalar multiplication for families of equal-length MSMs.
//
//   out[j] = sum_t scalars[v_j][t] * points[pbase[j] + idx[t]]
//
// This covers blst's contiguous `p{1,2}s_mult_pippenger` blocks (one MSM,
// idx = identity), the reference's sparse indexed G2 MSMs
// (weighted_btx/src/blst_utils.rs:106-125: idx = accepted virtual indices,
// one base block per kernel offset) and the per-slot party blocks of
// weighted_btx/src/decryption.rs:463-481 (one family per party).  Scalars are
// shared by every MSM using the same vector, so the signed-digit recoding and
// the per-window bucket sort are done once per (vector, window).
//
// Pipeline:
//  1. digits:  signed c-bit windows, digit in (-2^(c-1), 2^(c-1)]
//  2. sort:    one CTA per (vector, window) counting-sorts term indices by
//              |digit| in descending order (zero digits dropped)
//  3. segments: one thread per (MSM, window, segment of S sorted terms)
//              evaluates sum_e |d_e| * (+-P_e) over its segment with a running
//              sum (Abel summation) -- no bucket array is materialised
//  4. reduce:  tree sums over the segments of each (MSM, window)
//  5. combine: Horner over windows, then conversion to affine.
// Group addition is exact and commutative, so the result does not depend on
// the order that atomics give terms inside a bucket.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>

#include "launch.h"
#include "pairing.cuh"

namespace wbte {

namespace {
constexpr int TPB = 128;
constexpr int SEG_TPB = 64;  // threads per block of k_segments
inline unsigned blocks_for(int64_t n, int tpb = TPB) { return (unsigned)((n + tpb - 1) / tpb); }

template <class F> struct Aff;
template <> struct Aff<Fp> { static constexpr size_t SZ = G1_AFF; };
template <> struct Aff<Fp2> { static constexpr size_t SZ = G2_AFF; };

// entry packing: term index (32 bits) | bucket (16 bits) << 32 | sign << 63
WBTE_INL uint64_t pack_entry(uint32_t t, uint32_t b, bool negative) {
    return (uint64_t)t | ((uint64_t)b << 32) | ((uint64_t)(negative ? 1 : 0) << 63);
}

__global__ void k_digits(int16_t* digits, const uint8_t* scalars, int64_t total, int64_t n, int c, int windows) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // i = v * n + t
    if (i >= total) return;
    uint32_t k[8];
    load_scalar(k, scalars + FR_SZ * i);
    int64_t v = i / n, t = i % n;
    int carry = 0;
    const int full = 1 << c, half = 1 << (c - 1);
    for (int w = 0; w < windows; w++) {
        int bit = w * c;
        uint32_t val = 0;
        if (bit < 256) {
            int word = bit >> 5, off = bit & 31;
            uint64_t two = (uint64_t)k[word] | ((word + 1 < 8) ? ((uint64_t)k[word + 1] << 32) : 0ull);
            val = (uint32_t)(two >> off) & (uint32_t)(full - 1);
        }
        int d = (int)val + carry;
        if (d > half) {
            d -= full;
            carry = 1;
        } else {
            carry = 0;
        }
        digits[(v * windows + w) * n + t] = (int16_t)d;
    }
}

// One CTA per (vector, window).  counts lives in dynamic shared memory.
__global__ void k_sort(uint64_t* entries, int32_t* nnz, const int16_t* digits, int64_t n, int buckets) {
    extern __shared__ int32_t sh[];
    int32_t* cnt = sh;                // buckets + 1
    int32_t* cur = sh + buckets + 1;  // buckets + 1
    int64_t vw = blockIdx.x;
    const int16_t* d = digits + vw * n;
    for (int b = threadIdx.x; b <= buckets; b += blockDim.x) cnt[b] = 0;
    __syncthreads();
    for (int64_t t = threadIdx.x; t < n; t += blockDim.x) {
        int x = d[t];
        atomicAdd(&cnt[x < 0 ? -x : x], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // descending bucket order; bucket 0 is dropped
        int32_t run = 0;
        for (int b = buckets; b >= 1; b--) {
            cur[b] = run;
            run += cnt[b];
        }
        nnz[vw] = run;
    }
    __syncthreads();
    uint64_t* out = entries + vw * n;
    for (int64_t t = threadIdx.x; t < n; t += blockDim.x) {
        int x = d[t];
        int b = x < 0 ? -x : x;
        if (b == 0) continue;
        int32_t pos = atomicAdd(&cur[b], 1);
        out[pos] = pack_entry((uint32_t)t, (uint32_t)b, x < 0);
    }
}

// acc += g * run for a small positive g
template <class F> WBTE_INL Xyzz<F> add_small_multiple(const Xyzz<F>& acc, const Xyzz<F>& run, uint32_t g) {
    if (g == 1) return xyzz_add(acc, run);
    Xyzz<F> m;
    set_inf(m);
    int top = 31 - __clz(g);
    for (int b = top; b >= 0; b--) {
        m = xyzz_dbl(m);
        if ((g >> b) & 1) m = xyzz_add(m, run);
    }
    return xyzz_add(acc, m);
}

// One thread per segment of S sorted terms of one (MSM, window): the running
// sum `run` of the terms seen so far, and at each bucket transition (bucket
// cur_b to b < cur_b) acc += (cur_b - b) * run; at the end acc += cur_b * run
// (Abel summation: acc = sum over the segment of |d| * (+-P)).
// Adding at the transition itself would diverge: every lane reaches its own
// transitions at its own terms, and a warp runs the addition whenever any of
// its 32 lanes does, so every lane would pay an XYZZ addition per term besides
// its mixed addition.  Instead a lane stores a snapshot of run (and the gap)
// in a small per-lane queue in shared memory, and the queued additions run
// when every lane of the warp that still has terms holds one, all lanes
// together; a full queue adds its oldest entry on its own.  The sum is the
// same: the group is commutative and every snapshot is added exactly once.
// Measured on B200 against adding at the transition: G1 and G2 MSMs of 2^16
// to 2^18 points 15-18 % faster, 2^20 5-7 %, the batched partial decryptions
// (384 MSMs of 512 terms) 10 %.
template <class F> struct SegQueue;
template <> struct SegQueue<Fp> { static constexpr int Q = 4; };
template <> struct SegQueue<Fp2> { static constexpr int Q = 2; };
template <class F> constexpr size_t seg_queue_bytes() {
    return (sizeof(Xyzz<F>) + sizeof(uint32_t)) * SegQueue<F>::Q * SEG_TPB;
}

template <class F>
__global__ void __launch_bounds__(SEG_TPB) k_segments(uint8_t* seg_out, const uint8_t* points, const int64_t* pbase,
                                                        const int32_t* idx, const uint64_t* entries,
                                                        const int32_t* nnz, const int32_t* vsel, int64_t k, int64_t n,
                                                        int windows, int64_t S, int64_t nseg) {
    constexpr int Q = SegQueue<F>::Q;
    extern __shared__ __align__(16) uint8_t seg_sh[];
    Xyzz<F>* qv = reinterpret_cast<Xyzz<F>*>(seg_sh);
    uint32_t* qg = reinterpret_cast<uint32_t*>(seg_sh + sizeof(Xyzz<F>) * Q * SEG_TPB);
    const int tid = threadIdx.x;
    const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    // threads past the grid's work stay in the loop (the warp votes need
    // every lane) with an empty segment
    using A = Affine<F>;
    int64_t lo = 0, hi = 0;
    const uint64_t* e = entries;
    const A* P = reinterpret_cast<const A*>(points);
    if (gid < k * windows * nseg) {
        const int64_t seg = gid % nseg;
        const int64_t w = (gid / nseg) % windows;
        const int64_t j = gid / (nseg * windows);
        const int64_t v = vsel ? vsel[j] : 0;
        const int64_t vw = v * windows + w;
        lo = seg * S;
        hi = lo + S;
        const int64_t cnt = nnz[vw];
        if (hi > cnt) hi = cnt;
        if (lo > hi) lo = hi;
        e = entries + vw * n;
        P = reinterpret_cast<const A*>(points) + pbase[j];
    }
    Xyzz<F> run, acc;
    set_inf(run);
    set_inf(acc);
    uint32_t cur_b = lo < hi ? ((uint32_t)(e[lo] >> 32) & 0x7fffu) : 0u;
    int qh = 0, qn = 0;
    for (int64_t i = 0; i < S; i++) {
        const int64_t x = lo + i;
        if (x < hi) {
            const uint64_t en = e[x];
            const uint32_t b = (uint32_t)(en >> 32) & 0x7fffu;
            const uint32_t t = (uint32_t)en;
            if (b != cur_b) {
                if (qn == Q) {
                    acc = add_small_multiple(acc, qv[qh * SEG_TPB + tid], qg[qh * SEG_TPB + tid]);
                    qh = qh + 1 == Q ? 0 : qh + 1;
                    qn--;
                }
                const int slot = (qh + qn) % Q;
                qv[slot * SEG_TPB + tid] = run;
                qg[slot * SEG_TPB + tid] = cur_b - b;
                qn++;
                cur_b = b;
            }
            A p = load_affine(P + (idx ? (int64_t)idx[t] : (int64_t)t));
            if (en >> 63) p = neg(p);
            run = xyzz_madd(run, p);
        }
        // lanes without terms left never hold the warp back
        if (__all_sync(0xffffffffu, qn > 0 || x + 1 >= hi) && qn > 0) {
            acc = add_small_multiple(acc, qv[qh * SEG_TPB + tid], qg[qh * SEG_TPB + tid]);
            qh = qh + 1 == Q ? 0 : qh + 1;
            qn--;
        }
    }
    if (lo < hi) acc = add_small_multiple(acc, run, cur_b);
    while (qn > 0) {
        acc = add_small_multiple(acc, qv[qh * SEG_TPB + tid], qg[qh * SEG_TPB + tid]);
        qh = qh + 1 == Q ? 0 : qh + 1;
        qn--;
    }
    if (gid < k * windows * nseg) store_vec(reinterpret_cast<Xyzz<F>*>(seg_out) + gid, acc);
}

// out[i] = sum_{g < G, i*G+g < len} in[row * len + i*G + g] for each row
template <class F>
__global__ void k_reduce(uint8_t* out, const uint8_t* in, int64_t rows, int64_t len, int64_t G, int64_t out_len) {
    int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (gid >= rows * out_len) return;
    int64_t row = gid / out_len, i = gid % out_len;
    const Xyzz<F>* src = reinterpret_cast<const Xyzz<F>*>(in) + row * len;
    Xyzz<F> acc;
    set_inf(acc);
    for (int64_t g = 0; g < G; g++) {
        int64_t x = i * G + g;
        if (x < len) acc = xyzz_add(acc, load_vec(src + x));
    }
    store_vec(reinterpret_cast<Xyzz<F>*>(out) + gid, acc);
}

// out[row * out_len + i] = sum of in[row * len + 32 i .. 32 i + 31]: one warp
// per output, a shuffle tree of five additions (lanes past len hold the
// identity); every lane runs each level, so the warp never diverges around
// the shuffles.
template <class F>
__global__ void k_reduce_warp(uint8_t* out, const uint8_t* in, int64_t rows, int64_t len, int64_t out_len) {
    const int lane = threadIdx.x & 31;
    const int64_t wid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (wid >= rows * out_len) return;  // whole warps: rows * out_len warps are launched
    const int64_t row = wid / out_len, i = wid % out_len, x = i * 32 + lane;
    Xyzz<F> acc;
    if (x < len) {
        acc = load_vec(reinterpret_cast<const Xyzz<F>*>(in) + row * len + x);
    } else {
        set_inf(acc);
    }
    constexpr int WORDS = sizeof(Xyzz<F>) / 4;
    for (int off = 16; off > 0; off >>= 1) {
        Xyzz<F> other;
        uint32_t* dst = reinterpret_cast<uint32_t*>(&other);
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&acc);
#pragma unroll
        for (int w = 0; w < WORDS; w++) dst[w] = __shfl_down_sync(0xffffffffu, src[w], off);
        if (lane + off >= 32) set_inf(other);
        acc = xyzz_add(acc, other);
    }
    if (lane == 0) store_vec(reinterpret_cast<Xyzz<F>*>(out) + wid, acc);
}

template <class F>
__global__ void k_combine(uint8_t* out, const uint8_t* wins, int64_t k, int windows, int c) {
    int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= k) return;
    const Xyzz<F>* W = reinterpret_cast<const Xyzz<F>*>(wins) + j * windows;
    Xyzz<F> acc;
    set_inf(acc);
    for (int w = windows - 1; w >= 0; w--) {
        if (!is_inf(acc))
            for (int i = 0; i < c; i++) acc = xyzz_dbl(acc);
        acc = xyzz_add(acc, load_vec(W + w));
    }
    store_affine(reinterpret_cast<Affine<F>*>(out + Aff<F>::SZ * j), to_affine(acc));
}

struct ScratchLayout {
    size_t digits, entries, nnz, seg, red, total;
};
ScratchLayout layout_for(size_t xyzz, int32_t V, int64_t k, int64_t n, const MsmPlan& p) {
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    ScratchLayout L;
    size_t off = 0;
    L.digits = off;
    off += align(sizeof(int16_t) * (size_t)V * p.windows * n);
    L.entries = off;
    off += align(sizeof(uint64_t) * (size_t)V * p.windows * n);
    L.nnz = off;
    off += align(sizeof(int32_t) * (size_t)V * p.windows);
    L.seg = off;
    off += align(xyzz * (size_t)k * p.windows * p.segments);
    L.red = off;
    size_t red_len = (size_t)((p.segments + 7) / 8);
    off += align(xyzz * (size_t)k * p.windows * (red_len > 1 ? red_len : 1));
    L.total = off;
    return L;
}

template <class F>
void run_family(uint8_t* out, const uint8_t* points, const int64_t* pbase, const int32_t* idx, const uint8_t* scalars,
                const int32_t* vsel, int32_t V, int64_t k, int64_t n, const MsmPlan& p, uint8_t* scratch, cudaStream_t s) {
    const size_t XZ = sizeof(Xyzz<F>);
    ScratchLayout L = layout_for(XZ, V, k, n, p);
    int16_t* digits = reinterpret_cast<int16_t*>(scratch + L.digits);
    uint64_t* entries = reinterpret_cast<uint64_t*>(scratch + L.entries);
    int32_t* nnz = reinterpret_cast<int32_t*>(scratch + L.nnz);
    uint8_t* seg = scratch + L.seg;
    uint8_t* red = scratch + L.red;
    int64_t total = (int64_t)V * n;
    const bool g1 = sizeof(F) == sizeof(Fp);
    void* tok = nullptr;
    prof_begin(g1 ? "msm_sort_g1" : "msm_sort_g2", s, &tok);
    note_launch();
    k_digits<<<blocks_for(total), TPB, 0, s>>>(digits, scalars, total, n, p.c, p.windows);
    size_t shmem = sizeof(int32_t) * 2 * (p.buckets + 1);
    note_launch();
    k_sort<<<(unsigned)((int64_t)V * p.windows), 256, shmem, s>>>(entries, nnz, digits, n, p.buckets);
    prof_end(tok, s);
    prof_begin(g1 ? "msm_segments_g1" : "msm_segments_g2", s, &tok);
    int64_t segthreads = k * p.windows * p.segments;
    note_launch();
    // the queues take about 49 KB of shared memory per block, past the 48 KB
    // default, so the kernel opts in once
    static const bool smem_ok = cudaFuncSetAttribute(k_segments<F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)seg_queue_bytes<F>()) == cudaSuccess;
    (void)smem_ok;
    k_segments<F><<<blocks_for(segthreads, SEG_TPB), SEG_TPB, seg_queue_bytes<F>(), s>>>(
        seg, points, pbase, idx, entries, nnz, vsel, k, n, p.windows, p.segment, p.segments);
    prof_end(tok, s);
    prof_begin(g1 ? "msm_reduce_g1" : "msm_reduce_g2", s, &tok);
    // tree-reduce segments per (MSM, window)
    int64_t rows = k * p.windows, len = p.segments;
    uint8_t* src = seg;
    uint8_t* bufs[2] = {red, seg};
    int flip = 0;
    while (len > 1) {
        // long rows: warp-shuffle trees of 32; the last few per row: one thread
        const int64_t G = len > 8 ? 32 : len;
        const int64_t out_len = (len + G - 1) / G;
        uint8_t* dst = bufs[flip];
        note_launch();
        if (G == 32)
            k_reduce_warp<F><<<blocks_for(rows * out_len * 32, 64), 64, 0, s>>>(dst, src, rows, len, out_len);
        else
            k_reduce<F><<<blocks_for(rows * out_len, 64), 64, 0, s>>>(dst, src, rows, len, G, out_len);
        src = dst;
        flip ^= 1;
        len = out_len;
    }
    note_launch();
    k_combine<F><<<blocks_for(k, 64), 64, 0, s>>>(out, src, k, p.windows, p.c);
    prof_end(tok, s);
}
}  // namespace

// Threads of k_segments<F> resident on the whole device (one wave), from the
// occupancy of the compiled kernel; cached per device and group.
static int64_t segment_wave_threads(Group g) {
    static std::atomic<int64_t> cache[2][64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148 * 256;
    int gi = g == GROUP_G1 ? 0 : 1;
    int64_t v = cache[gi][dev].load();
    if (v > 0) return v;
    int sms = 0, blocks = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (g == GROUP_G1) {
        cudaFuncSetAttribute(k_segments<Fp>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)seg_queue_bytes<Fp>());
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_segments<Fp>, SEG_TPB, seg_queue_bytes<Fp>());
    } else {
        cudaFuncSetAttribute(k_segments<Fp2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)seg_queue_bytes<Fp2>());
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_segments<Fp2>, SEG_TPB, seg_queue_bytes<Fp2>());
    }
    v = (int64_t)(sms > 0 ? sms : 148) * (blocks > 0 ? blocks : 4) * SEG_TPB;
    cache[gi][dev].store(v);
    return v;
}

MsmPlan msm_plan(Group g, int64_t n, int64_t k) {
    MsmPlan p;
    int lg = 0;
    while ((int64_t(1) << (lg + 1)) <= n) lg++;
    int c = lg - 1;
    if (n >= (1 << 14)) c = lg - 2;
    if (c < 4) c = 4;
    if (c > 13) c = 13;
    if (g_tune.msm_window >= 4 && g_tune.msm_window <= 13) c = g_tune.msm_window;
    p.c = c;
    p.windows = (256 + c - 1) / c;
    p.buckets = 1 << (c - 1);
    // Segments per (MSM, window): every thread of k_segments walks one
    // segment, so the launch takes ceil(threads / wave) waves of the longest
    // segment.  Cost model in mixed additions: S terms plus one full addition
    // (~1.43 mixed additions) per bucket change, min(S, buckets), and the
    // tree reduction of the segment sums.
    const int64_t wave = segment_wave_threads(g);
    const int64_t rows = k * p.windows;
    const double nnz = (double)n * (1.0 - 1.0 / (double)(int64_t(1) << c));
    double best = 1e300;
    int64_t best_s = 1;
    for (int64_t s = 1; s <= 1024 && s <= n; s++) {
        double S = std::ceil(nnz / (double)s);
        double per_thread = S + 1.43 * std::min(S, (double)p.buckets);
        int64_t threads = rows * s;
        double waves = std::ceil((double)threads / (double)wave);
        double reduce = s > 1 ? 1.43 * 8.0 * std::ceil((double)threads / (8.0 * (double)wave)) : 0.0;
        double cost = waves * per_thread + reduce;
        if (cost < best * 0.999) {
            best = cost;
            best_s = s;
        }
    }
    if (g_tune.msm_segments > 0) best_s = std::min<int64_t>(std::min<int64_t>(g_tune.msm_segments, 1024), n);
    p.segment = (n + best_s - 1) / best_s;
    p.segments = (n + p.segment - 1) / p.segment;
    if (p.segments < 1) p.segments = 1;
    return p;
}

size_t msm_family_scratch_bytes(Group g, int32_t V, int64_t k, int64_t n, const MsmPlan& plan) {
    return layout_for(g == GROUP_G1 ? G1_XYZZ : G2_XYZZ, V, k, n, plan).total;
}

void launch_msm_family_scratch(Group g, uint8_t* out, const uint8_t* points, const int64_t* pbase, const int32_t* idx,
                               const uint8_t* scalars, const int32_t* vsel, int32_t V, int64_t k, int64_t n,
                               const MsmPlan& plan, void* scratch, cudaStream_t s) {
    if (k <= 0) return;
    if (g == GROUP_G1)
        run_family<Fp>(out, points, pbase, idx, scalars, vsel, V, k, n, plan, (uint8_t*)scratch, s);
    else
        run_family<Fp2>(out, points, pbase, idx, scalars, vsel, V, k, n, plan, (uint8_t*)scratch, s);
}

void launch_msm_family(Group g, uint8_t* out, const uint8_t* points, const int64_t* pbase, const int32_t* idx,
                       const uint8_t* scalars, const int32_t* vsel, int32_t V, int64_t k, int64_t n, cudaStream_t s,
                       const MsmPlan* forced) {
    if (k <= 0) return;
    if (n <= 0) {
        cudaMemsetAsync(out, 0, (g == GROUP_G1 ? G1_AFF : G2_AFF) * (size_t)k, s);
        return;
    }
    if (!forced && n <= SMALL_MSM_MAX) {
        launch_small_msm(g, out, points, pbase, idx, scalars, vsel, k, n, s);
        return;
    }
    MsmPlan p = forced ? *forced : msm_plan(g, n, k);
    size_t bytes = msm_family_scratch_bytes(g, V, k, n, p);
    void* scratch = nullptr;
    if (cudaMallocAsync(&scratch, bytes, s) != cudaSuccess) return;
    launch_msm_family_scratch(g, out, points, pbase, idx, scalars, vsel, V, k, n, p, scratch, s);
    cudaFreeAsync(scratch, s);
}

}  // namespace wbte

// ===================================================================
// Allocation-free G1 MSM.
//
// Some callers must not allocate device memory while they serve a request:
// a service that has reserved HBM up front for its resident key material
// and its request buffers cannot let the library take more, because an
// allocation can fail under memory pressure in the middle of a request,
// can stall on device-wide synchronisation, and fragments a carefully
// partitioned device.  For them, wbte_g1_msm_static runs the same Pippenger
// kernels as wbte_g1_msm but takes its working memory from one fixed array
// that is part of the library's device image (every GPU that loads the
// library holds it until the process exits).
namespace {
constexpr size_t STATIC_MSM_BYTES = size_t(8) << 20;        // 8 MiB of scratch
constexpr size_t STATIC_MSM_TAIL = 256;                     // holds the point-base entry
constexpr uint64_t STATIC_MSM_MAX_POINTS = 16384;
static __device__ __align__(256) uint8_t g_static_msm_scratch[STATIC_MSM_BYTES];

std::mutex g_static_mu;
uint8_t* g_static_addr[128] = {};

// Plain device memory of device `dev` only: host, managed and other GPUs'
// memory are rejected (a peer pointer would be read over the interconnect).
bool static_is_device(const void* p, int dev) {
    cudaPointerAttributes a;
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

// The plan of wbte_g1_msm with fewer, longer segments where its scratch would
// not fit the array: every n <= STATIC_MSM_MAX_POINTS fits (at n = 16384 the
// digits and sorted entries take 3.6 MB and at most about 1000 segments of
// the 22 windows fit the rest).
bool static_plan(wbte::MsmPlan& p, int64_t n, size_t avail) {
    using namespace wbte;
    const Tuning saved = g_tune;
    g_tune = Tuning();
    p = msm_plan(GROUP_G1, n, 1);
    g_tune = saved;
    while (msm_family_scratch_bytes(GROUP_G1, 1, 1, n, p) > avail) {
        if (p.segments <= 1) return false;
        p.segment += std::max<int64_t>(1, p.segment / 8);
        p.segments = (n + p.segment - 1) / p.segment;
    }
    return true;
}
}  // namespace

extern "C" int32_t wbte_g1_msm_static(void* out, const void* points, const void* scalars, uint64_t n, void* stream) {
    using namespace wbte;
    if (n > STATIC_MSM_MAX_POINTS) return -2;  // WBTE_ERR_SIZE
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return -5;  // WBTE_ERR_CUDA
    if (!static_is_device(out, dev) || (n > 0 && (!static_is_device(points, dev) || !static_is_device(scalars, dev))))
        return -1;  // WBTE_ERR_INVALID_ARG: device pointers of the current device only
    cudaStream_t s = (cudaStream_t)stream;
    // an error left pending by earlier, unrelated runtime calls on this
    // thread must not be reported as this call's failure
    cudaGetLastError();
    uint8_t* base = nullptr;
    {
        // one-time set-up per device, with that device current
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (!g_static_addr[dev]) {
            void* ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, g_static_msm_scratch) != cudaSuccess) {
                cudaGetLastError();
                return -5;
            }
            g_static_addr[dev] = static_cast<uint8_t*>(ptr);
        }
        base = g_static_addr[dev];
    }
    if (n == 0) return cudaMemsetAsync(out, 0, G1_AFF, s) == cudaSuccess ? 0 : -5;
    MsmPlan p;
    if (!static_plan(p, (int64_t)n, STATIC_MSM_BYTES - STATIC_MSM_TAIL)) return -2;
    // point base of the single MSM: zero (the tail of the array is reused by
    // every call, so it is cleared here; nothing else must start at zero)
    int64_t* pbase = reinterpret_cast<int64_t*>(base + STATIC_MSM_BYTES - STATIC_MSM_TAIL);
    if (cudaMemsetAsync(pbase, 0, sizeof(int64_t), s) != cudaSuccess) return -5;
    // the opt-in per-kernel profiler would create CUDA events; keep it out of this call
    g_prof_suppress = true;
    launch_msm_family_scratch(GROUP_G1, static_cast<uint8_t*>(out), static_cast<const uint8_t*>(points), pbase,
                              nullptr, static_cast<const uint8_t*>(scalars), nullptr, 1, 1, (int64_t)n, p, base, s);
    g_prof_suppress = false;
    return cudaGetLastError() == cudaSuccess ? 0 : -5;
}
