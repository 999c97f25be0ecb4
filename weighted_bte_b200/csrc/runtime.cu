// libwbte runtime: the C ABI of include/wbte.h on top of the kernel
// launchers.  Host or device buffers are accepted for every data pointer;
// host buffers are staged through stream-ordered device allocations.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "launch.h"
#include "wbte.h"

using namespace wbte;

namespace wbte {
std::atomic<uint64_t> g_launches{0};
thread_local uint64_t t_launches = 0;

namespace {
struct ProfRec {
    const char* tag;
    cudaEvent_t a, b;
};
std::mutex g_prof_mu;
std::vector<ProfRec> g_prof;
std::atomic<bool> g_prof_on{false};
}  // namespace

thread_local bool g_prof_suppress = false;
thread_local Tuning g_tune;

void prof_begin(const char* tag, cudaStream_t s, void** token) {
    *token = nullptr;
    if (g_prof_suppress || !g_prof_on.load(std::memory_order_relaxed)) return;
    ProfRec* r = new ProfRec{tag, nullptr, nullptr};
    cudaEventCreate(&r->a);
    cudaEventCreate(&r->b);
    cudaEventRecord(r->a, s);
    *token = r;
}

void prof_end(void* token, cudaStream_t s) {
    if (!token) return;
    ProfRec* r = static_cast<ProfRec*>(token);
    cudaEventRecord(r->b, s);
    std::lock_guard<std::mutex> lock(g_prof_mu);
    g_prof.push_back(*r);
    delete r;
}
}  // namespace wbte

struct wbte_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    uint64_t budget = 0;
    std::string err;
    std::map<std::pair<int64_t, int>, uint8_t*> twiddles;
    std::mutex mu;
    Tuning tune;
};

namespace {

bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int log2_exact(uint64_t n) {
    int lg = 0;
    while ((uint64_t(1) << lg) < n) lg++;
    return (uint64_t(1) << lg) == n ? lg : -1;
}

uint64_t next_pow2(uint64_t n) {
    uint64_t m = 1;
    while (m < n) m <<= 1;
    return m;
}

// One ABI call: staging buffers, pending host copies, first error.
struct Call {
    wbte_ctx* ctx;
    cudaStream_t s;
    std::vector<void*> temps;
    struct Pending {
        void* host;
        const void* dev;
        size_t bytes;
    };
    std::vector<Pending> outs;
    int32_t status = WBTE_OK;
    bool sync = false;

    Tuning saved_tune;

    explicit Call(wbte_ctx* c) : ctx(c), s(c->stream), saved_tune(g_tune) {
        cudaSetDevice(c->device);
        g_tune = c->tune;
    }
    ~Call() { g_tune = saved_tune; }
    Call(const Call&) = delete;
    Call& operator=(const Call&) = delete;

    int32_t fail(int32_t code, const std::string& msg) {
        if (status == WBTE_OK) {
            status = code;
            ctx->err = msg;
        }
        return code;
    }
    bool ok() const { return status == WBTE_OK; }
    uint8_t* alloc(size_t bytes) {
        void* p = nullptr;
        if (bytes == 0) bytes = 16;
        if (cudaMallocAsync(&p, bytes, s) != cudaSuccess) {
            cudaGetLastError();
            fail(WBTE_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed");
            return nullptr;
        }
        temps.push_back(p);
        return (uint8_t*)p;
    }
    uint8_t* zeros(size_t bytes) {
        uint8_t* p = alloc(bytes);
        if (p) cudaMemsetAsync(p, 0, bytes, s);
        return p;
    }
    const uint8_t* in(const void* p, size_t bytes) {
        if (!p || bytes == 0 || is_device_ptr(p)) return (const uint8_t*)p;
        uint8_t* d = alloc(bytes);
        if (d) cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, s);
        return d;
    }
    template <class T> const T* in_vec(const std::vector<T>& v) {
        return reinterpret_cast<const T*>(in(v.data(), v.size() * sizeof(T)));
    }
    uint8_t* out(void* p, size_t bytes) {
        if (!p) return nullptr;
        if (is_device_ptr(p)) return (uint8_t*)p;
        uint8_t* d = alloc(bytes);
        if (d) outs.push_back({p, d, bytes});
        return d;
    }
    uint8_t* inout(void* p, size_t bytes) {
        if (!p) return nullptr;
        if (is_device_ptr(p)) return (uint8_t*)p;
        uint8_t* d = alloc(bytes);
        if (d) {
            cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, s);
            outs.push_back({p, d, bytes});
        }
        return d;
    }
    // copy a small device or host buffer to host (synchronising)
    bool to_host(void* dst, const void* src, size_t bytes) {
        if (cudaMemcpyAsync(dst, src, bytes, is_device_ptr(src) ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            fail(WBTE_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
            return false;
        }
        return true;
    }
    int32_t finish() {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) fail(WBTE_ERR_CUDA, cudaGetErrorString(e));
        for (auto& o : outs) cudaMemcpyAsync(o.host, o.dev, o.bytes, cudaMemcpyDeviceToHost, s);
        for (void* p : temps) cudaFreeAsync(p, s);
        if (!outs.empty() || sync || status != WBTE_OK) {
            e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) fail(WBTE_ERR_CUDA, cudaGetErrorString(e));
        }
        return status;
    }
};

const uint8_t* twiddles(Call& c, int64_t n, bool inverse) {
    std::lock_guard<std::mutex> lock(c.ctx->mu);
    auto key = std::make_pair(n, inverse ? 1 : 0);
    auto it = c.ctx->twiddles.find(key);
    if (it != c.ctx->twiddles.end()) return it->second;
    int64_t count = n / 2 > 0 ? n / 2 : 1;
    uint8_t* t = nullptr;
    if (cudaMalloc(&t, FR_SZ * count) != cudaSuccess) {
        cudaGetLastError();
        c.fail(WBTE_ERR_OOM, "twiddle table allocation failed");
        return nullptr;
    }
    launch_domain_twiddles(t, n, count, inverse, c.s);
    c.ctx->twiddles[key] = t;
    return t;
}

// product of n Fp12 values on the device into out (one value)
void fp12_product(Call& c, uint8_t* out, const uint8_t* in, int64_t n) {
    if (n <= 0) {
        return;
    }
    const int64_t G = 16;
    const uint8_t* cur = in;
    while (true) {
        int64_t groups = (n + G - 1) / G;
        std::vector<int64_t> offs(groups + 1);
        for (int64_t j = 0; j <= groups; j++) offs[j] = std::min(n, j * G);
        uint8_t* dst = groups == 1 ? out : c.alloc(GT_SZ * groups);
        const int64_t* doffs = c.in_vec(offs);
        if (!c.ok()) return;
        launch_fp12_segment_product(dst, cur, doffs, groups, c.s);
        if (groups == 1) return;
        cur = dst;
        n = groups;
    }
}

// out[b] = product of in[b len .. (b + 1) len) for b < K, by levels of
// products of 16 so that long segments spread over many threads
void fp12_segments_product(Call& c, uint8_t* out, const uint8_t* in, int64_t len, int64_t K) {
    if (len <= 0 || K <= 0) return;
    const int64_t G = 16;
    const uint8_t* cur = in;
    while (true) {
        int64_t groups = (len + G - 1) / G;
        // group j of segment b spans [b len + j G, next group's start); the last
        // group of a segment ends where the next segment begins, so no group
        // crosses a segment boundary
        std::vector<int64_t> offs(K * groups + 1);
        for (int64_t b = 0; b < K; b++)
            for (int64_t j = 0; j < groups; j++) offs[b * groups + j] = b * len + j * G;
        offs[K * groups] = K * len;
        uint8_t* dst = groups == 1 ? out : c.alloc(GT_SZ * K * groups);
        const int64_t* doffs = c.in_vec(offs);
        if (!c.ok()) return;
        launch_fp12_segment_product(dst, cur, doffs, K * groups, c.s);
        if (groups == 1) return;
        cur = dst;
        len = groups;
    }
}

// out[j] = product of in[offs[j] .. offs[j+1]) for the k = offs.size() - 1
// segments of any lengths, by levels of products of at most 16 consecutive
// values inside each segment, so that long segments spread over many
// threads (doffs: offs already on the device)
void fp12_ragged_product(Call& c, uint8_t* out, const uint8_t* in, std::vector<int64_t> offs, const int64_t* doffs) {
    const int64_t G = 16;
    const size_t k = offs.size() - 1;
    const uint8_t* cur = in;
    while (true) {
        int64_t longest = 0;
        for (size_t j = 0; j < k; j++) longest = std::max(longest, offs[j + 1] - offs[j]);
        if (longest <= G) {
            launch_fp12_segment_product(out, cur, doffs, (int64_t)k, c.s);
            return;
        }
        // groups of G inside every segment; segment j keeps its groups
        std::vector<int64_t> goffs(1, 0), next(1, 0);
        for (size_t j = 0; j < k; j++) {
            for (int64_t x = offs[j]; x < offs[j + 1]; x += G) goffs.push_back(std::min(offs[j + 1], x + G));
            next.push_back((int64_t)goffs.size() - 1);
        }
        const int64_t groups = (int64_t)goffs.size() - 1;
        uint8_t* dst = c.alloc(GT_SZ * (size_t)std::max<int64_t>(groups, 1));
        const int64_t* dg = c.in_vec(goffs);
        const int64_t* dn = c.in_vec(next);
        if (!c.ok()) return;
        launch_fp12_segment_product(dst, cur, dg, groups, c.s);
        cur = dst;
        offs = next;
        doffs = dn;
    }
}

// G2 generator affine bytes on the device
uint8_t* g2_generator_dev(Call& c) {
    uint8_t one[32] = {1};
    const uint8_t* s = c.in(one, 32);
    uint8_t* g = c.alloc(G2_AFF);
    if (c.ok()) launch_mul_generator(GROUP_G2, g, s, 1, c.s);
    return g;
}

int32_t check_ctx(wbte_ctx* ctx) { return ctx ? WBTE_OK : WBTE_ERR_INVALID_ARG; }

int32_t msm_family_impl(wbte_ctx* ctx, Group g, void* out, const void* points, uint64_t n_points, const int64_t* pbase,
                        const int32_t* pidx, const void* scalars, const int32_t* vsel, int32_t V, uint64_t k, uint64_t n) {
    if (check_ctx(ctx)) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    size_t aff = g == GROUP_G1 ? G1_AFF : G2_AFF;
    if (k == 0) return c.finish();
    if (!out || !pbase || V < 1 || (n > 0 && (!points || !scalars))) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    if (n >= (uint64_t(1) << 31)) return c.fail(WBTE_ERR_SIZE, "MSM length must be below 2^31");
    // bounds: every addressed point must lie inside [0, n_points)
    int64_t max_idx = -1, min_idx = 0;
    if (pidx) {
        for (uint64_t t = 0; t < n; t++) {
            max_idx = std::max<int64_t>(max_idx, pidx[t]);
            min_idx = std::min<int64_t>(min_idx, pidx[t]);
        }
    } else {
        max_idx = (int64_t)n - 1;
    }
    for (uint64_t j = 0; j < k; j++) {
        if (pbase[j] < 0 || min_idx < 0 || (n > 0 && (uint64_t)(pbase[j] + max_idx) >= n_points))
            return c.fail(WBTE_ERR_SIZE, "MSM point index out of range");
        if (vsel && (vsel[j] < 0 || vsel[j] >= V)) return c.fail(WBTE_ERR_INVALID_ARG, "scalar vector index out of range");
    }
    uint8_t* dout = c.out(out, aff * k);
    const uint8_t* dpts = c.in(points, aff * n_points);
    const uint8_t* dsc = c.in(scalars, FR_SZ * (size_t)V * n);
    std::vector<int64_t> hb(pbase, pbase + k);
    const int64_t* db = c.in_vec(hb);
    const int32_t* di = nullptr;
    if (pidx) {
        std::vector<int32_t> hi(pidx, pidx + n);
        di = c.in_vec(hi);
    }
    const int32_t* dv = nullptr;
    if (vsel) {
        std::vector<int32_t> hv(vsel, vsel + k);
        dv = c.in_vec(hv);
    }
    if (!c.ok()) return c.finish();
    launch_msm_family(g, dout, dpts, db, di, dsc, dv, V, (int64_t)k, (int64_t)n, c.s);
    return c.finish();
}

int32_t msm_impl(wbte_ctx* ctx, Group g, void* out, const void* points, const void* scalars, uint64_t n) {
    int64_t zero = 0;
    return msm_family_impl(ctx, g, out, points, n, &zero, nullptr, scalars, nullptr, 1, 1, n);
}

}  // namespace

// ====================================================================== ABI
extern "C" {

int32_t wbte_version(void) { return 10000; }

int32_t wbte_ctx_create(int32_t device, uint64_t budget, wbte_ctx** out) {
    if (!out) return WBTE_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return WBTE_ERR_CUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess) return WBTE_ERR_CUDA;
    wbte_ctx* c = new wbte_ctx();
    c->device = device;
    c->budget = budget;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return WBTE_ERR_CUDA;
    }
    c->stream = c->own_stream;
    // keep freed pool memory cached between calls
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t threshold = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    *out = c;
    return WBTE_OK;
}

int32_t wbte_ctx_destroy(wbte_ctx* ctx) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto& kv : ctx->twiddles) cudaFree(kv.second);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return WBTE_OK;
}

int32_t wbte_ctx_set_stream(wbte_ctx* ctx, void* stream) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return WBTE_OK;
}

int32_t wbte_ctx_set_tuning(wbte_ctx* ctx, int32_t knob, int64_t value) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    switch (knob) {
    case WBTE_TUNE_GT_LANES:
        if (value != 0 && value != 1 && value != 2 && value != 4) break;
        ctx->tune.gt_lanes = (int)value;
        return WBTE_OK;
    case WBTE_TUNE_MSM_WINDOW:
        if (value != 0 && (value < 4 || value > 13)) break;
        ctx->tune.msm_window = (int)value;
        return WBTE_OK;
    case WBTE_TUNE_MSM_SEGMENTS:
        if (value < 0 || value > 1024) break;
        ctx->tune.msm_segments = (int)value;
        return WBTE_OK;
    case WBTE_TUNE_NTT_JOINT:
        if (value < -1 || value > 1) break;
        ctx->tune.ntt_joint = (int)value;
        return WBTE_OK;
    case WBTE_TUNE_MILLER_CHUNK:
        if (value < 0 || value > 8) break;
        ctx->tune.miller_chunk = (int)value;
        return WBTE_OK;
    default:
        break;
    }
    ctx->err = "unknown tuning knob or value out of range";
    return WBTE_ERR_INVALID_ARG;
}

int32_t wbte_ctx_synchronize(wbte_ctx* ctx) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        ctx->err = cudaGetErrorString(e);
        return WBTE_ERR_CUDA;
    }
    return WBTE_OK;
}

const char* wbte_ctx_last_error(const wbte_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

uint64_t wbte_ctx_launch_count(const wbte_ctx* ctx) {
    (void)ctx;
    return g_launches.load();
}

uint64_t wbte_thread_launch_count(void) { return t_launches; }

int32_t wbte_measure_imad_rate(wbte_ctx* ctx, double* imad_per_s) {
    if (!ctx || !imad_per_s) return WBTE_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    *imad_per_s = measure_imad_rate(ctx->stream);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ctx->err = cudaGetErrorString(e);
        return WBTE_ERR_CUDA;
    }
    return WBTE_OK;
}

int32_t wbte_profile_enable(int32_t on) {
    std::lock_guard<std::mutex> lock(g_prof_mu);
    for (auto& r : g_prof) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    g_prof.clear();
    g_prof_on.store(on != 0);
    return WBTE_OK;
}

int32_t wbte_profile_read(char* names, int32_t name_stride, double* ms, int64_t* counts, int32_t max_entries,
                          int32_t* n_out) {
    if (!n_out || name_stride < 2) return WBTE_ERR_INVALID_ARG;
    if (cudaDeviceSynchronize() != cudaSuccess) return WBTE_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_prof_mu);
    std::map<std::string, std::pair<double, int64_t>> agg;
    for (auto& r : g_prof) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        auto& e = agg[r.tag];
        e.first += t;
        e.second += 1;
    }
    int32_t i = 0;
    for (auto& kv : agg) {
        if (i >= max_entries) break;
        if (names) {
            std::strncpy(names + (size_t)i * name_stride, kv.first.c_str(), name_stride - 1);
            names[(size_t)i * name_stride + name_stride - 1] = 0;
        }
        if (ms) ms[i] = kv.second.first;
        if (counts) counts[i] = kv.second.second;
        i++;
    }
    *n_out = i;
    return WBTE_OK;
}

// ------------------------------------------------------------------ MSM
int32_t wbte_g1_msm(wbte_ctx* ctx, void* out, const void* points, const void* scalars, uint64_t n) {
    return msm_impl(ctx, GROUP_G1, out, points, scalars, n);
}
int32_t wbte_g2_msm(wbte_ctx* ctx, void* out, const void* points, const void* scalars, uint64_t n) {
    return msm_impl(ctx, GROUP_G2, out, points, scalars, n);
}
int32_t wbte_g1_msm_family(wbte_ctx* ctx, void* out, const void* points, uint64_t n_points, const int64_t* pbase,
                           const int32_t* pidx, const void* scalars, const int32_t* vsel, int32_t V, uint64_t k, uint64_t n) {
    return msm_family_impl(ctx, GROUP_G1, out, points, n_points, pbase, pidx, scalars, vsel, V, k, n);
}
int32_t wbte_g2_msm_family(wbte_ctx* ctx, void* out, const void* points, uint64_t n_points, const int64_t* pbase,
                           const int32_t* pidx, const void* scalars, const int32_t* vsel, int32_t V, uint64_t k, uint64_t n) {
    return msm_family_impl(ctx, GROUP_G2, out, points, n_points, pbase, pidx, scalars, vsel, V, k, n);
}

// ---------------------------------------------------------- point ops
static int32_t mul_impl(wbte_ctx* ctx, Group g, void* out, const void* points, int32_t fixed, const void* scalars, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !points || !scalars) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    size_t aff = g == GROUP_G1 ? G1_AFF : G2_AFF;
    uint8_t* d = c.out(out, aff * n);
    const uint8_t* p = c.in(points, aff * (fixed ? 1 : n));
    const uint8_t* sc = c.in(scalars, FR_SZ * n);
    if (c.ok()) launch_mul_batch(g, d, p, fixed ? 0 : 1, sc, (int64_t)n, c.s);
    return c.finish();
}
int32_t wbte_g1_mul(wbte_ctx* ctx, void* out, const void* points, int32_t fixed, const void* scalars, uint64_t n) {
    return mul_impl(ctx, GROUP_G1, out, points, fixed, scalars, n);
}
int32_t wbte_g2_mul(wbte_ctx* ctx, void* out, const void* points, int32_t fixed, const void* scalars, uint64_t n) {
    return mul_impl(ctx, GROUP_G2, out, points, fixed, scalars, n);
}
static int32_t mul_gen_impl(wbte_ctx* ctx, Group g, void* out, const void* scalars, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !scalars) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    size_t aff = g == GROUP_G1 ? G1_AFF : G2_AFF;
    uint8_t* d = c.out(out, aff * n);
    const uint8_t* sc = c.in(scalars, FR_SZ * n);
    if (c.ok()) launch_mul_generator(g, d, sc, (int64_t)n, c.s);
    return c.finish();
}
int32_t wbte_g1_mul_generator(wbte_ctx* ctx, void* out, const void* scalars, uint64_t n) {
    return mul_gen_impl(ctx, GROUP_G1, out, scalars, n);
}
int32_t wbte_g2_mul_generator(wbte_ctx* ctx, void* out, const void* scalars, uint64_t n) {
    return mul_gen_impl(ctx, GROUP_G2, out, scalars, n);
}
static int32_t sum_impl(wbte_ctx* ctx, Group g, void* out, const void* in, const int64_t* offsets, uint64_t k) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (k == 0) return c.finish();
    if (!out || !offsets) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    for (uint64_t j = 0; j < k; j++)
        if (offsets[j + 1] < offsets[j] || offsets[0] < 0) return c.fail(WBTE_ERR_INVALID_ARG, "offsets must be ascending");
    size_t aff = g == GROUP_G1 ? G1_AFF : G2_AFF;
    uint8_t* d = c.out(out, aff * k);
    const uint8_t* din = c.in(in, aff * (size_t)offsets[k]);
    std::vector<int64_t> ho(offsets, offsets + k + 1);
    const int64_t* doffs = c.in_vec(ho);
    if (c.ok()) launch_segment_sum(g, d, din, doffs, (int64_t)k, c.s);
    return c.finish();
}
int32_t wbte_g1_sum(wbte_ctx* ctx, void* out, const void* in, const int64_t* offsets, uint64_t k) {
    return sum_impl(ctx, GROUP_G1, out, in, offsets, k);
}
int32_t wbte_g2_sum(wbte_ctx* ctx, void* out, const void* in, const int64_t* offsets, uint64_t k) {
    return sum_impl(ctx, GROUP_G2, out, in, offsets, k);
}
static int32_t compress_impl(wbte_ctx* ctx, Group g, void* out, const void* in, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !in) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    size_t aff = g == GROUP_G1 ? G1_AFF : G2_AFF;
    uint8_t* d = c.out(out, (aff / 2) * n);
    const uint8_t* s = c.in(in, aff * n);
    if (c.ok()) launch_compress(g, d, s, (int64_t)n, c.s);
    return c.finish();
}
static int32_t decompress_impl(wbte_ctx* ctx, Group g, void* out, uint8_t* status, const void* in, uint64_t n,
                               int32_t check_group) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !in) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    const size_t aff = g == GROUP_G1 ? G1_AFF : G2_AFF;
    uint8_t* d = c.out(out, aff * n);
    const uint8_t* s = c.in(in, (aff / 2) * n);
    uint8_t* st = status ? c.out(status, n) : c.alloc(n);
    if (!c.ok()) return c.finish();
    launch_decompress(g, d, st, s, (int64_t)n, check_group != 0, c.s);
    std::vector<uint8_t> h(n);
    if (c.to_host(h.data(), st, n)) {
        uint64_t bad = 0, first = n;
        for (uint64_t i = 0; i < n; i++)
            if (h[i]) {
                bad++;
                if (first == n) first = i;
            }
        if (bad) {
            static const char* why[4] = {"", "bad encoding", "not on the curve", "not in the prime-order subgroup"};
            c.fail(WBTE_ERR_NOT_ON_CURVE, std::to_string(bad) + " of " + std::to_string(n) +
                                              " points rejected; first at " + std::to_string(first) + ": " +
                                              why[h[first] < 4 ? h[first] : 1]);
        }
    }
    return c.finish();
}
int32_t wbte_g1_decompress(wbte_ctx* ctx, void* out, uint8_t* status, const void* in, uint64_t n, int32_t check_group) {
    return decompress_impl(ctx, GROUP_G1, out, status, in, n, check_group);
}
int32_t wbte_g2_decompress(wbte_ctx* ctx, void* out, uint8_t* status, const void* in, uint64_t n, int32_t check_group) {
    return decompress_impl(ctx, GROUP_G2, out, status, in, n, check_group);
}
static int32_t normalize_impl(wbte_ctx* ctx, Group g, void* out, const void* in, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !in) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    const size_t aff = g == GROUP_G1 ? G1_AFF : G2_AFF;
    uint8_t* d = c.out(out, aff * n);
    const uint8_t* di = c.in(in, 3 * (aff / 2) * n);
    if (c.ok()) launch_batch_normalize(g, d, di, (int64_t)n, c.s);
    return c.finish();
}
int32_t wbte_g1_batch_normalize(wbte_ctx* ctx, void* out, const void* in, uint64_t n) {
    return normalize_impl(ctx, GROUP_G1, out, in, n);
}
int32_t wbte_g2_batch_normalize(wbte_ctx* ctx, void* out, const void* in, uint64_t n) {
    return normalize_impl(ctx, GROUP_G2, out, in, n);
}
int32_t wbte_g1_compress(wbte_ctx* ctx, void* out, const void* in, uint64_t n) { return compress_impl(ctx, GROUP_G1, out, in, n); }
int32_t wbte_g2_compress(wbte_ctx* ctx, void* out, const void* in, uint64_t n) { return compress_impl(ctx, GROUP_G2, out, in, n); }

// ----------------------------------------------------------- transforms
static int32_t ntt_impl(wbte_ctx* ctx, Group g, void* io, uint64_t n, int32_t inverse) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!io) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    int lg = log2_exact(n);
    if (n == 0 || lg < 0 || lg > 32) return c.fail(WBTE_ERR_SIZE, "transform size must be a power of two <= 2^32");
    if (n == 1) return c.finish();
    size_t aff = g == GROUP_G1 ? G1_AFF : G2_AFF;
    size_t xz = g == GROUP_G1 ? G1_XYZZ : G2_XYZZ;
    uint8_t* d = c.inout(io, aff * n);
    uint8_t* work = c.alloc(xz * n);
    const uint8_t* tw = twiddles(c, (int64_t)n, inverse != 0);
    if (c.ok()) launch_group_ntt(g, d, work, tw, (int64_t)n, c.s);
    return c.finish();
}
int32_t wbte_g1_ntt(wbte_ctx* ctx, void* io, uint64_t n, int32_t inverse) { return ntt_impl(ctx, GROUP_G1, io, n, inverse); }
int32_t wbte_g2_ntt(wbte_ctx* ctx, void* io, uint64_t n, int32_t inverse) { return ntt_impl(ctx, GROUP_G2, io, n, inverse); }

int32_t wbte_gt_ntt(wbte_ctx* ctx, void* io, uint64_t n, int32_t inverse) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!io) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    int lg = log2_exact(n);
    if (n == 0 || lg < 0 || lg > 32) return c.fail(WBTE_ERR_SIZE, "transform size must be a power of two <= 2^32");
    if (n == 1) return c.finish();
    uint8_t* d = c.inout(io, GT_SZ * n);
    const uint8_t* tw = twiddles(c, (int64_t)n, inverse != 0);
    if (c.ok()) launch_gt_ntt(d, tw, (int64_t)n, c.s, 1, inverse != 0);
    return c.finish();
}

int32_t wbte_gt_cyclotomic_prefix_ifft(wbte_ctx* ctx, void* io, uint64_t n, uint64_t out_count) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!io) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    int lg = log2_exact(n);
    if (n < 2 || lg < 0 || lg > 32) return c.fail(WBTE_ERR_SIZE, "transform size must be a power of two in [2, 2^32]");
    if (out_count > n / 2) return c.fail(WBTE_ERR_SIZE, "out_count must be at most n / 2");
    uint8_t* d = c.inout(io, GT_SZ * n);
    const uint8_t* tw = twiddles(c, (int64_t)n, true);
    if (c.ok()) launch_cyclotomic_prefix_ifft(d, tw, (int64_t)n, (int64_t)out_count, c.s);
    return c.finish();
}

int32_t wbte_gt_ntt_many(wbte_ctx* ctx, void* io, uint64_t n, uint64_t count, int32_t inverse) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (count == 0) return c.finish();
    if (!io) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    int lg = log2_exact(n);
    if (n == 0 || lg < 0 || lg > 32) return c.fail(WBTE_ERR_SIZE, "transform size must be a power of two <= 2^32");
    if (n == 1) return c.finish();
    uint8_t* d = c.inout(io, GT_SZ * n * count);
    const uint8_t* tw = twiddles(c, (int64_t)n, inverse != 0);
    if (c.ok()) launch_gt_ntt(d, tw, (int64_t)n, c.s, (int64_t)count, inverse != 0);
    return c.finish();
}

int32_t wbte_gt_cyclotomic_prefix_ifft_many(wbte_ctx* ctx, void* io, uint64_t n, uint64_t out_count, uint64_t count) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (count == 0) return c.finish();
    if (!io) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    int lg = log2_exact(n);
    if (n < 2 || lg < 0 || lg > 32) return c.fail(WBTE_ERR_SIZE, "transform size must be a power of two in [2, 2^32]");
    if (out_count > n / 2) return c.fail(WBTE_ERR_SIZE, "out_count must be at most n / 2");
    uint8_t* d = c.inout(io, GT_SZ * n * count);
    const uint8_t* tw = twiddles(c, (int64_t)n, true);
    if (c.ok()) launch_cyclotomic_prefix_ifft(d, tw, (int64_t)n, (int64_t)out_count, c.s, (int64_t)count);
    return c.finish();
}

// -------------------------------------------------------------- pairing
int32_t wbte_g2_prepare_lines(wbte_ctx* ctx, void* lines, const void* q, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!lines || !q) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    uint8_t* d = c.out(lines, LINE_SZ * LINES_PER_POINT * n);
    const uint8_t* dq = c.in(q, G2_AFF * n);
    if (c.ok()) launch_prepare_lines(d, dq, (int64_t)n, c.s);
    return c.finish();
}
int32_t wbte_miller_loop_lines(wbte_ctx* ctx, void* out, const void* lines, const void* p, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !lines || !p) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    uint8_t* d = c.out(out, GT_SZ * n);
    const uint8_t* dl = c.in(lines, LINE_SZ * LINES_PER_POINT * n);
    const uint8_t* dp = c.in(p, G1_AFF * n);
    if (c.ok()) launch_miller_lines(d, dl, dp, (int64_t)n, c.s);
    return c.finish();
}
int32_t wbte_miller_loop(wbte_ctx* ctx, void* out, const void* p, const void* q, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !p || !q) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    uint8_t* d = c.out(out, GT_SZ * n);
    const uint8_t* dp = c.in(p, G1_AFF * n);
    const uint8_t* dq = c.in(q, G2_AFF * n);
    if (c.ok()) launch_miller(d, dp, dq, (int64_t)n, c.s);
    return c.finish();
}
int32_t wbte_multi_miller_loop(wbte_ctx* ctx, void* out, const void* p, const void* q, const int64_t* offsets, uint64_t k) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (k == 0) return c.finish();
    if (!out || !offsets) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    if (offsets[0] != 0) return c.fail(WBTE_ERR_INVALID_ARG, "offsets must start at 0");
    for (uint64_t j = 0; j < k; j++)
        if (offsets[j + 1] < offsets[j]) return c.fail(WBTE_ERR_INVALID_ARG, "offsets must be ascending");
    int64_t n = offsets[k];
    uint8_t* d = c.out(out, GT_SZ * k);
    const uint8_t* dp = c.in(p, G1_AFF * n);
    const uint8_t* dq = c.in(q, G2_AFF * n);
    uint8_t* f = c.alloc(GT_SZ * (n > 0 ? n : 1));
    std::vector<int64_t> ho(offsets, offsets + k + 1);
    const int64_t* doffs = c.in_vec(ho);
    if (!c.ok()) return c.finish();
    launch_miller(f, dp, dq, n, c.s);
    fp12_ragged_product(c, d, f, ho, doffs);
    return c.finish();
}
int32_t wbte_final_exp(wbte_ctx* ctx, void* out, const void* in, uint64_t n, int32_t mode) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !in) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    if (mode < 0 || mode > 2) return c.fail(WBTE_ERR_INVALID_ARG, "unknown final exponentiation mode");
    uint8_t* d = c.out(out, GT_SZ * n);
    const uint8_t* s = c.in(in, GT_SZ * n);
    if (c.ok()) launch_final_exp(d, s, (int64_t)n, (FinalExpMode)mode, c.s);
    return c.finish();
}
int32_t wbte_gt_pow(wbte_ctx* ctx, void* out, const void* base, int32_t fixed, const void* scalars, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !base || !scalars) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    uint8_t* d = c.out(out, GT_SZ * n);
    const uint8_t* b = c.in(base, GT_SZ * (fixed ? 1 : n));
    const uint8_t* sc = c.in(scalars, FR_SZ * n);
    if (c.ok()) launch_gt_pow(d, b, fixed ? 0 : 1, sc, (int64_t)n, c.s);
    return c.finish();
}
int32_t wbte_fp12_mul(wbte_ctx* ctx, void* out, const void* a, const void* b, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !a || !b) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    uint8_t* d = c.out(out, GT_SZ * n);
    const uint8_t* da = c.in(a, GT_SZ * n);
    const uint8_t* db = c.in(b, GT_SZ * n);
    if (c.ok()) launch_fp12_mul(d, da, 1, db, 1, false, (int64_t)n, c.s);
    return c.finish();
}
int32_t wbte_gt_compress(wbte_ctx* ctx, void* out, const void* in, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !in) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    uint8_t* d = c.out(out, 289 * n);
    const uint8_t* s = c.in(in, GT_SZ * n);
    if (c.ok()) launch_gt_compress(d, s, (int64_t)n, c.s);
    return c.finish();
}

// -------------------------------------------------------------- scalars
int32_t wbte_lagrange_at_zero(wbte_ctx* ctx, void* out, const void* points, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.fail(WBTE_ERR_INTERPOLATION, "the interpolation points must be nonempty and distinct");
    if (!out || !points) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    uint8_t* d = c.out(out, FR_SZ * n);
    const uint8_t* x = c.in(points, FR_SZ * n);
    int32_t* status = (int32_t*)c.zeros(sizeof(int32_t));
    if (!c.ok()) return c.finish();
    launch_lagrange_at_zero(d, x, (int64_t)n, status, c.s);
    int32_t st = 0;
    if (c.to_host(&st, status, sizeof(st)) && st) c.fail(WBTE_ERR_INTERPOLATION, "the interpolation points must be nonempty and distinct");
    return c.finish();
}
int32_t wbte_transcript_challenges(wbte_ctx* ctx, void* out, const wbte_transcript_field* fields, uint32_t count,
                                   uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!out || !fields) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    if (count > (uint32_t)TRANSCRIPT_MAX_FIELDS) return c.fail(WBTE_ERR_SIZE, "at most 8 transcript fields");
    TranscriptSpec spec{};
    spec.count = (int32_t)count;
    for (uint32_t k = 0; k < count; k++) {
        const wbte_transcript_field& f = fields[k];
        if (f.kind > TRANSCRIPT_GT_VARIABLE || (f.kind == TRANSCRIPT_GT_VARIABLE && f.len != 289))
            return c.fail(WBTE_ERR_INVALID_ARG, "invalid transcript field kind");
        if (f.len > (1u << 20)) return c.fail(WBTE_ERR_SIZE, "transcript field longer than 1 MiB");
        if (f.len == 0) {
            spec.f[k] = TranscriptField{nullptr, 0, 0, TRANSCRIPT_BYTES};
            continue;
        }
        if (!f.data) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
        if (f.stride != 0 && f.stride < f.len) return c.fail(WBTE_ERR_INVALID_ARG, "transcript records overlap");
        const size_t extent = f.stride == 0 ? f.len : f.stride * (n - 1) + f.len;
        spec.f[k] = TranscriptField{c.in(f.data, extent), f.stride, f.len, f.kind};
    }
    uint8_t* d = c.out(out, FR_SZ * n);
    int32_t* status = (int32_t*)c.zeros(sizeof(int32_t));
    if (!c.ok()) return c.finish();
    launch_transcript_challenges(d, spec, (int64_t)n, status, c.s);
    int32_t st = 0;
    if (c.to_host(&st, status, sizeof(st)) && st) c.fail(WBTE_ERR_INTERNAL, "challenge rejection sampling ran out of counters");
    return c.finish();
}
int32_t wbte_schnorr_verify(wbte_ctx* ctx, uint8_t* valid, const void* X, const void* R, const void* s, const void* ch, uint64_t n) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (n == 0) return c.finish();
    if (!valid || !X || !R || !s || !ch) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    uint8_t* d = c.out(valid, n);
    const uint8_t* dx = c.in(X, G1_AFF * n);
    const uint8_t* dr = c.in(R, G1_AFF * n);
    const uint8_t* ds = c.in(s, FR_SZ * n);
    const uint8_t* dc = c.in(ch, FR_SZ * n);
    if (c.ok()) launch_schnorr_verify(d, dx, dr, ds, dc, (int64_t)n, c.s);
    return c.finish();
}

// --------------------------------------------------------- weighted_btx
static int32_t check_key(Call& c, const wbte_wbtx_key* key) {
    if (!key || !key->party_offsets || key->party_count == 0 || key->max_batch_size == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "invalid weighted-BTX key");
    if ((uint64_t)key->party_offsets[key->party_count] != key->total_weight)
        return c.fail(WBTE_ERR_INVALID_ARG, "party offsets do not sum to the total weight");
    return WBTE_OK;
}

int32_t wbte_wbtx_partial_decrypt(wbte_ctx* ctx, void* sigma, const void* first, uint64_t B, const void* q, uint64_t T) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (T == 0) return c.finish();
    if (!sigma || !first || !q || B == 0) return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    uint8_t* dsig = c.out(sigma, G1_AFF * T);
    const uint8_t* dfirst = c.in(first, G1_AFF * B);
    const uint8_t* dq = c.in(q, FR_SZ * T);
    uint8_t* scalars = c.alloc(FR_SZ * T * B);
    std::vector<int64_t> base(T, 0);
    std::vector<int32_t> vsel(T);
    for (uint64_t j = 0; j < T; j++) vsel[j] = (int32_t)j;
    const int64_t* db = c.in_vec(base);
    const int32_t* dv = c.in_vec(vsel);
    if (!c.ok()) return c.finish();
    for (uint64_t j = 0; j < T; j++) launch_fr_powers(scalars + FR_SZ * B * j, dq + FR_SZ * j, (int64_t)B, 1, c.s);
    launch_msm_family(GROUP_G1, dsig, dfirst, db, nullptr, scalars, dv, (int32_t)T, (int64_t)T, (int64_t)B, c.s);
    return c.finish();
}

int32_t wbte_wbtx_verify_shares(wbte_ctx* ctx, int32_t* ok, const wbte_wbtx_key* key, const void* first, const uint8_t* valid,
                                uint64_t B, const void* sigma, const int64_t* party_indices, const void* challenges, uint64_t T) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!ok) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    *ok = 0;
    if (check_key(c, key)) return c.finish();
    if (T == 0) {
        *ok = 1;
        return c.finish();
    }
    if (!first || !valid || !sigma || !party_indices || !challenges) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    if (B == 0 || B > key->max_batch_size) return c.fail(WBTE_ERR_SIZE, "batch size out of range");
    std::vector<uint8_t> hvalid(B);
    if (!c.to_host(hvalid.data(), valid, B)) return c.finish();
    std::vector<int32_t> slots, pidx(T);
    for (uint64_t i = 0; i < B; i++)
        if (hvalid[i]) slots.push_back((int32_t)i);
    for (uint64_t j = 0; j < T; j++) {
        if (party_indices[j] < 0 || (uint64_t)party_indices[j] >= key->party_count)
            return c.fail(WBTE_ERR_INVALID_ARG, "invalid party index");
        pidx[j] = (int32_t)party_indices[j];
    }
    int64_t nv = (int64_t)slots.size();
    const uint8_t* dfirst = c.in(first, G1_AFF * B);
    const uint8_t* dsig = c.in(sigma, G1_AFF * T);
    const uint8_t* dch = c.in(challenges, FR_SZ * T);
    const uint8_t* dvk = c.in(key->verification_keys, G2_AFF * key->max_batch_size * key->party_count);
    uint8_t* P = c.alloc(G1_AFF * (nv + 1));
    uint8_t* Q = c.alloc(G2_AFF * (nv + 1));
    uint8_t* f = c.alloc(GT_SZ * (nv + 1));
    uint8_t* prod = c.alloc(GT_SZ);
    uint8_t* flag = c.alloc(1);
    std::vector<int64_t> zero(1, 0);
    const int64_t* dzero = c.in_vec(zero);
    std::vector<int64_t> vbase(nv > 0 ? nv : 1);
    for (int64_t j = 0; j < nv; j++) vbase[j] = (int64_t)slots[j] * (int64_t)key->party_count;
    const int64_t* dvbase = c.in_vec(vbase);
    const int32_t* dpidx = c.in_vec(pidx);
    const int32_t* dslots = nv ? c.in_vec(slots) : nullptr;
    uint8_t* g2 = g2_generator_dev(c);
    if (!c.ok()) return c.finish();
    // aggregate sigma, negated, as the last left input
    launch_msm_family(GROUP_G1, P + G1_AFF * nv, dsig, dzero, nullptr, dch, nullptr, 1, 1, (int64_t)T, c.s);
    launch_negate(GROUP_G1, P + G1_AFF * nv, P + G1_AFF * nv, 1, c.s);
    if (nv > 0) {
        launch_gather(P, dfirst, dslots, nv, G1_AFF, c.s);
        launch_msm_family(GROUP_G2, Q, dvk, dvbase, dpidx, dch, nullptr, 1, nv, (int64_t)T, c.s);
    }
    cudaMemcpyAsync(Q + G2_AFF * nv, g2, G2_AFF, cudaMemcpyDeviceToDevice, c.s);
    const int64_t runs = launch_miller_chunks(f, P, Q, nv + 1, 1, miller_chunk(nv + 1), c.s);
    fp12_product(c, prod, f, runs);
    launch_final_exp(prod, prod, 1, FE_FULL, c.s);
    launch_fp12_is_one(flag, prod, 1, c.s);
    uint8_t h = 0;
    if (c.to_host(&h, flag, 1)) *ok = h ? 1 : 0;
    return c.finish();
}

int32_t wbte_wbtx_prepare(wbte_ctx* ctx, const wbte_wbtx_key* key, const int64_t* party_indices, uint64_t T, uint64_t B,
                          void* kernel_lines, void* opening_keys, void* kernel) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (check_key(c, key)) return c.finish();
    if (!party_indices || T == 0 || !kernel_lines || !opening_keys) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    if (B == 0 || B > key->max_batch_size) return c.fail(WBTE_ERR_SIZE, "batch size out of range");
    const uint64_t N = key->party_count, W = key->total_weight, L = key->max_batch_size;
    const uint64_t m = next_pow2(2 * B);
    const int lgm = log2_exact(m);
    // accepted virtual indices and per-party coefficient offsets
    std::vector<int32_t> sel;
    std::vector<int64_t> coef_off(1, 0), party_base(T);
    for (uint64_t k = 0; k < T; k++) {
        int64_t j = party_indices[k];
        if (j < 0 || (uint64_t)j >= N) return c.fail(WBTE_ERR_INVALID_ARG, "invalid party index");
        if (k && party_indices[k - 1] >= j) return c.fail(WBTE_ERR_INVALID_ARG, "party indices must be strictly ascending");
        for (int64_t w = key->party_offsets[j]; w < key->party_offsets[j + 1]; w++) sel.push_back((int32_t)w);
        coef_off.push_back((int64_t)sel.size());
        party_base[k] = key->party_offsets[j];
    }
    const int64_t WT = (int64_t)sel.size();
    uint8_t* dlines = c.out(kernel_lines, LINE_SZ * LINES_PER_POINT * m);
    uint8_t* dopen = c.out(opening_keys, G2_AFF * B * T);
    uint8_t* dkern_out = kernel ? c.out(kernel, G2_AFF * m) : nullptr;
    const uint8_t* ddom = c.in(key->domain_points, FR_SZ * W);
    const uint8_t* dneg = c.in(key->negative_material, G2_AFF * L * W);
    const uint8_t* dpos = L > 1 ? c.in(key->positive_material, G2_AFF * (L - 1) * W) : nullptr;
    const int32_t* dsel = c.in_vec(sel);
    uint8_t* x = c.alloc(FR_SZ * WT);
    uint8_t* lam = c.alloc(FR_SZ * WT);
    int32_t* status = (int32_t*)c.zeros(sizeof(int32_t));
    uint8_t* kern = c.zeros(G2_AFF * m);
    uint8_t* open_scaled = c.alloc(G2_AFF * B * T);
    uint8_t* tmp = c.alloc(G2_AFF * B);
    uint8_t* work = c.alloc(G2_XYZZ * m);
    if (!c.ok()) return c.finish();
    // Lagrange coefficients of the accepted virtual points, scaled by 1/m so
    // that every MSM below already carries the inverse-transform factor.
    launch_gather(x, ddom, dsel, WT, FR_SZ, c.s);
    launch_lagrange_at_zero(lam, x, WT, status, c.s);
    launch_fr_scale_size_inv(lam, lam, lgm, WT, c.s);
    // A'[slot, k] = sum_{w in party k} lam'_w * negative[slot][w]
    std::vector<int64_t> slot_base(B);
    for (uint64_t k = 0; k < T; k++) {
        for (uint64_t i = 0; i < B; i++) slot_base[i] = (int64_t)(i * W) + party_base[k];
        const int64_t* dbase = c.in_vec(slot_base);
        if (!c.ok()) return c.finish();
        int64_t wk = coef_off[k + 1] - coef_off[k];
        launch_msm_family(GROUP_G2, tmp, dneg, dbase, nullptr, lam + FR_SZ * coef_off[k], nullptr, 1, (int64_t)B, wk, c.s);
        cudaMemcpy2DAsync(open_scaled + G2_AFF * k, G2_AFF * T, tmp, G2_AFF, G2_AFF, B, cudaMemcpyDeviceToDevice, c.s);
    }
    // kernel[d] = sum_k A'[d - 1, k] for 1 <= d < B
    if (B > 1) {
        std::vector<int64_t> offs(B);
        for (uint64_t d = 0; d < B; d++) offs[d] = (int64_t)(d * T);
        const int64_t* doffs = c.in_vec(offs);
        if (!c.ok()) return c.finish();
        launch_segment_sum(GROUP_G2, kern + G2_AFF, open_scaled, doffs, (int64_t)B - 1, c.s);
        // kernel[m - d] = sum_w lam'_w positive[d - 1][sel[w]], written in ascending m - d order
        std::vector<int64_t> pbase(B - 1);
        for (uint64_t j = 0; j + 1 < B; j++) pbase[j] = (int64_t)((B - 2 - j) * W);
        const int64_t* dpb = c.in_vec(pbase);
        if (!c.ok()) return c.finish();
        launch_msm_family(GROUP_G2, kern + G2_AFF * (m - B + 1), dpos, dpb, dsel, lam, nullptr, 1, (int64_t)B - 1, WT, c.s);
    }
    const uint8_t* tw = twiddles(c, (int64_t)m, false);
    if (!c.ok()) return c.finish();
    launch_group_ntt(GROUP_G2, kern, work, tw, (int64_t)m, c.s);
    launch_prepare_lines(dlines, kern, (int64_t)m, c.s);
    if (dkern_out) cudaMemcpyAsync(dkern_out, kern, G2_AFF * m, cudaMemcpyDeviceToDevice, c.s);
    // opening keys A = m * A'
    launch_mul_pow2(GROUP_G2, dopen, open_scaled, (int64_t)(B * T), lgm, c.s);
    int32_t st = 0;
    if (c.to_host(&st, status, sizeof(st)) && st) c.fail(WBTE_ERR_INTERPOLATION, "the interpolation points must be nonempty and distinct");
    return c.finish();
}

int32_t wbte_wbtx_precompute(wbte_ctx* ctx, void* beta, const void* kernel_lines, const void* first, const uint8_t* valid, uint64_t B) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!beta || !kernel_lines || !first || !valid || B == 0) return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    const uint64_t m = next_pow2(2 * B);
    uint8_t* dbeta = c.out(beta, GT_SZ * B);
    const uint8_t* dl = c.in(kernel_lines, LINE_SZ * LINES_PER_POINT * m);
    const uint8_t* dfirst = c.in(first, G1_AFF * B);
    const uint8_t* dvalid = c.in(valid, B);
    uint8_t* x = c.zeros(G1_AFF * m);
    uint8_t* work = c.alloc(G1_XYZZ * m);
    uint8_t* f = c.alloc(GT_SZ * m);
    const uint8_t* tw = twiddles(c, (int64_t)m, false);
    const uint8_t* twi = twiddles(c, (int64_t)m, true);
    if (!c.ok()) return c.finish();
    cudaMemcpyAsync(x, dfirst, G1_AFF * B, cudaMemcpyDeviceToDevice, c.s);
    launch_group_ntt(GROUP_G1, x, work, tw, (int64_t)m, c.s);
    launch_miller_lines(f, dl, x, (int64_t)m, c.s);
    launch_final_exp(f, f, (int64_t)m, FE_EASY, c.s);
    launch_cyclotomic_prefix_ifft(f, twi, (int64_t)m, (int64_t)B, c.s);
    launch_final_exp(dbeta, f, (int64_t)B, FE_HARD, c.s);
    launch_fp12_mask(dbeta, dvalid, (int64_t)B, c.s);
    return c.finish();
}

int32_t wbte_wbtx_open(wbte_ctx* ctx, void* messages, const void* opening_keys, const void* sigma, uint64_t T,
                       const void* second, const void* beta, const uint8_t* valid, uint64_t B) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!messages || !opening_keys || !sigma || !second || !beta || !valid || B == 0 || T == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    uint8_t* dm = c.out(messages, GT_SZ * B);
    const uint8_t* dk = c.in(opening_keys, G2_AFF * B * T);
    const uint8_t* ds = c.in(sigma, G1_AFF * T);
    const uint8_t* d2 = c.in(second, GT_SZ * B);
    const uint8_t* db = c.in(beta, GT_SZ * B);
    const uint8_t* dv = c.in(valid, B);
    uint8_t* f = c.alloc(GT_SZ * B * T);
    uint8_t* alpha = c.alloc(GT_SZ * B);
    std::vector<int64_t> offs(B + 1);
    for (uint64_t i = 0; i <= B; i++) offs[i] = (int64_t)(i * T);
    const int64_t* doffs = c.in_vec(offs);
    if (!c.ok()) return c.finish();
    launch_miller(f, ds, dk, (int64_t)(B * T), c.s, (int64_t)T);
    launch_fp12_segment_product(alpha, f, doffs, (int64_t)B, c.s);
    launch_final_exp(alpha, alpha, (int64_t)B, FE_FULL, c.s);
    launch_unmask(dm, d2, alpha, db, dv, (int64_t)B, c.s);
    return c.finish();
}

int32_t wbte_wbtx_keygen_material(wbte_ctx* ctx, const void* z, const int32_t* owner, const void* q_pos, const void* q_neg,
                                  uint64_t W, uint64_t N, uint64_t L, void* vk, void* negative, void* positive) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!z || !owner || !q_pos || !q_neg || !vk || !negative || (L > 1 && !positive) || W == 0 || N == 0 || L == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty dimension");
    for (uint64_t w = 0; w < W; w++)
        if (owner[w] < 0 || (uint64_t)owner[w] >= N) return c.fail(WBTE_ERR_INVALID_ARG, "owner index out of range");
    uint8_t* dvk = c.out(vk, G2_AFF * L * N);
    uint8_t* dneg = c.out(negative, G2_AFF * L * W);
    uint8_t* dpos = L > 1 ? c.out(positive, G2_AFF * (L - 1) * W) : nullptr;
    const uint8_t* dz = c.in(z, FR_SZ * W);
    const uint8_t* dqp = c.in(q_pos, FR_SZ * L * N);
    const uint8_t* dqn = c.in(q_neg, FR_SZ * L * N);
    std::vector<int32_t> ho(owner, owner + W);
    const int32_t* downer = c.in_vec(ho);
    const uint64_t rows_per_chunk = std::max<uint64_t>(1, (uint64_t(1) << 20) / W);
    uint8_t* sc = c.alloc(FR_SZ * W * std::min<uint64_t>(rows_per_chunk, L));
    if (!c.ok()) return c.finish();
    launch_mul_generator(GROUP_G2, dvk, dqp, (int64_t)(L * N), c.s);
    for (int pass = 0; pass < 2; pass++) {
        uint64_t rows = pass == 0 ? L : L - 1;
        const uint8_t* qp = pass == 0 ? dqn : dqp;
        uint8_t* dst = pass == 0 ? dneg : dpos;
        for (uint64_t r0 = 0; r0 < rows; r0 += rows_per_chunk) {
            uint64_t nr = std::min(rows_per_chunk, rows - r0);
            launch_material_scalars(sc, dz, downer, qp + FR_SZ * r0 * N, (int64_t)W, (int64_t)N, (int64_t)nr, c.s);
            launch_mul_generator(GROUP_G2, dst + G2_AFF * r0 * W, sc, (int64_t)(nr * W), c.s);
        }
    }
    return c.finish();
}

// ------------------------------------------------------------------ btx
int32_t wbte_btx_kernel(wbte_ctx* ctx, const void* low_powers, const void* high_powers, uint64_t L, uint64_t B,
                        void* kernel_lines, void* opening_lines, void* kernel) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!low_powers || (L > 1 && !high_powers) || !kernel_lines || !opening_lines)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    if (B == 0 || B > L) return c.fail(WBTE_ERR_SIZE, "batch size out of range");
    const uint64_t m = next_pow2(2 * B);
    const int lgm = log2_exact(m);
    uint8_t* dlines = c.out(kernel_lines, LINE_SZ * LINES_PER_POINT * m);
    uint8_t* dopen = c.out(opening_lines, LINE_SZ * LINES_PER_POINT * B);
    uint8_t* dkern_out = kernel ? c.out(kernel, G2_AFF * m) : nullptr;
    const uint8_t* dlow = c.in(low_powers, G2_AFF * L);
    const uint8_t* dhigh = L > 1 ? c.in(high_powers, G2_AFF * (L - 1)) : nullptr;
    // centered powers h_e = power(L + 1 + e): h_{-d} = low[L - d], h_d = high[d - 1]
    std::vector<int32_t> neg_idx, pos_idx, open_idx(B);
    for (uint64_t d = 1; d < B; d++) neg_idx.push_back((int32_t)(L - d));
    for (int64_t d = (int64_t)B - 1; d >= 1; d--) pos_idx.push_back((int32_t)(d - 1));
    for (uint64_t slot = 0; slot < B; slot++) open_idx[slot] = (int32_t)(L - 1 - slot);  // h_{-(slot+1)}
    std::vector<uint8_t> ones(FR_SZ * m, 0);
    for (uint64_t i = 0; i < m; i++) ones[FR_SZ * i] = 1;
    uint8_t* kern = c.zeros(G2_AFF * m);
    uint8_t* work = c.alloc(G2_XYZZ * m);
    uint8_t* opening = c.alloc(G2_AFF * B);
    uint8_t* inv = const_cast<uint8_t*>(c.in_vec(ones));
    const int32_t* dneg = B > 1 ? c.in_vec(neg_idx) : nullptr;
    const int32_t* dpos = B > 1 ? c.in_vec(pos_idx) : nullptr;
    const int32_t* dopi = c.in_vec(open_idx);
    const uint8_t* tw = twiddles(c, (int64_t)m, false);
    if (!c.ok()) return c.finish();
    // K[0] = 0, K[d] = h_{-d}, K[m - d] = h_d (btx/src/decryption.rs:145-153)
    if (B > 1) {
        launch_gather(kern + G2_AFF, dlow, dneg, (int64_t)B - 1, G2_AFF, c.s);
        launch_gather(kern + G2_AFF * (m - B + 1), dhigh, dpos, (int64_t)B - 1, G2_AFF, c.s);
    }
    launch_group_ntt(GROUP_G2, kern, work, tw, (int64_t)m, c.s);
    // the inverse-transform factor 1/m moves into the kernel (:155-161)
    launch_fr_scale_size_inv(inv, inv, lgm, (int64_t)m, c.s);
    launch_mul_batch(GROUP_G2, kern, kern, 1, inv, (int64_t)m, c.s);
    launch_prepare_lines(dlines, kern, (int64_t)m, c.s);
    if (dkern_out) cudaMemcpyAsync(dkern_out, kern, G2_AFF * m, cudaMemcpyDeviceToDevice, c.s);
    launch_gather(opening, dlow, dopi, (int64_t)B, G2_AFF, c.s);
    launch_prepare_lines(dopen, opening, (int64_t)B, c.s);
    return c.finish();
}

int32_t wbte_btx_precompute(wbte_ctx* ctx, void* beta, const void* kernel_lines, const void* first, const uint8_t* valid,
                            uint64_t B) {
    // the same middle product as weighted_btx (btx/src/decryption.rs:201-246)
    return wbte_wbtx_precompute(ctx, beta, kernel_lines, first, valid, B);
}

int32_t wbte_btx_partial_decrypt(wbte_ctx* ctx, void* sigma, const void* first, const void* shares, uint64_t B) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    if (B == 0) {
        Call c(ctx);
        return c.fail(WBTE_ERR_INVALID_ARG, "empty batch");
    }
    // sigma_j = sum_i share_{j,i} first_i (btx/src/decryption.rs:248-264)
    return wbte_g1_msm(ctx, sigma, first, shares, B);
}

int32_t wbte_btx_combine(wbte_ctx* ctx, void* sigma, const void* sigmas, const void* points, uint64_t T) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!sigma || !sigmas || !points || T == 0) return c.fail(WBTE_ERR_INVALID_ARG, "null argument or no shares");
    uint8_t* dsig = c.out(sigma, G1_AFF);
    const uint8_t* ds = c.in(sigmas, G1_AFF * T);
    const uint8_t* dx = c.in(points, FR_SZ * T);
    uint8_t* lam = c.alloc(FR_SZ * T);
    int32_t* status = (int32_t*)c.zeros(sizeof(int32_t));
    std::vector<int64_t> zero(1, 0);
    const int64_t* dzero = c.in_vec(zero);
    if (!c.ok()) return c.finish();
    launch_lagrange_at_zero(lam, dx, (int64_t)T, status, c.s);
    launch_msm_family(GROUP_G1, dsig, ds, dzero, nullptr, lam, nullptr, 1, 1, (int64_t)T, c.s);
    int32_t st = 0;
    if (c.to_host(&st, status, sizeof(st)) && st) c.fail(WBTE_ERR_INTERPOLATION, "the interpolation points must be nonempty and distinct");
    return c.finish();
}

int32_t wbte_btx_verify(wbte_ctx* ctx, int32_t* ok, const void* first, const uint8_t* valid, uint64_t B,
                        const void* slot_points, uint64_t n_slot_points, const void* sigma) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!ok) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    *ok = 0;
    if (!first || !valid || !slot_points || !sigma || B == 0) return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    if (n_slot_points < B) return c.fail(WBTE_ERR_SIZE, "fewer slot points than slots");
    std::vector<uint8_t> hvalid(B);
    if (!c.to_host(hvalid.data(), valid, B)) return c.finish();
    std::vector<int32_t> slots;
    for (uint64_t i = 0; i < B; i++)
        if (hvalid[i]) slots.push_back((int32_t)i);
    const int64_t nv = (int64_t)slots.size();
    const uint8_t* dfirst = c.in(first, G1_AFF * B);
    const uint8_t* dq = c.in(slot_points, G2_AFF * n_slot_points);
    const uint8_t* dsig = c.in(sigma, G1_AFF);
    uint8_t* P = c.alloc(G1_AFF * (nv + 1));
    uint8_t* Q = c.alloc(G2_AFF * (nv + 1));
    uint8_t* f = c.alloc(GT_SZ * (nv + 1));
    uint8_t* prod = c.alloc(GT_SZ);
    uint8_t* flag = c.alloc(1);
    const int32_t* dslots = nv ? c.in_vec(slots) : nullptr;
    uint8_t* g2 = g2_generator_dev(c);
    if (!c.ok()) return c.finish();
    // prod_{valid i} e(first_i, Q_i) * e(-sigma, G2) == 1 (btx/src/decryption.rs:340-400)
    if (nv > 0) {
        launch_gather(P, dfirst, dslots, nv, G1_AFF, c.s);
        launch_gather(Q, dq, dslots, nv, G2_AFF, c.s);
    }
    launch_negate(GROUP_G1, P + G1_AFF * nv, dsig, 1, c.s);
    cudaMemcpyAsync(Q + G2_AFF * nv, g2, G2_AFF, cudaMemcpyDeviceToDevice, c.s);
    const int64_t runs = launch_miller_chunks(f, P, Q, nv + 1, 1, miller_chunk(nv + 1), c.s);
    fp12_product(c, prod, f, runs);
    launch_final_exp(prod, prod, 1, FE_FULL, c.s);
    launch_fp12_is_one(flag, prod, 1, c.s);
    uint8_t h = 0;
    if (c.to_host(&h, flag, 1)) *ok = h ? 1 : 0;
    return c.finish();
}

int32_t wbte_btx_open(wbte_ctx* ctx, void* messages, const void* opening_lines, const void* sigma, const void* second,
                      const void* beta, const uint8_t* valid, uint64_t B) {
    return wbte_btx_open_many(ctx, messages, opening_lines, sigma, second, beta, valid, B, 1);
}

// P[b B + i] = sigma[b]: each slot's G1 point of the opening pairing
// e(sigma_b, h_{-(i+1)}) (btx/src/decryption.rs:402-458)
static const uint8_t* btx_opening_points(Call& c, const uint8_t* dsig, uint64_t B, uint64_t K) {
    std::vector<int32_t> idx(B * K);
    for (uint64_t o = 0; o < B * K; o++) idx[o] = (int32_t)(o / B);
    const int32_t* di = c.in_vec(idx);
    uint8_t* P = c.alloc(G1_AFF * B * K);
    if (c.ok()) launch_gather(P, dsig, di, (int64_t)(B * K), G1_AFF, c.s);
    return P;
}

int32_t wbte_btx_open_many(wbte_ctx* ctx, void* messages, const void* opening_lines, const void* sigma,
                           const void* second, const void* beta, const uint8_t* valid, uint64_t B, uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!messages || !opening_lines || !sigma || !second || !beta || !valid || B == 0 || K == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    const uint64_t n = B * K;
    uint8_t* dm = c.out(messages, GT_SZ * n);
    const uint8_t* dl = c.in(opening_lines, LINE_SZ * LINES_PER_POINT * B);
    const uint8_t* dsig = c.in(sigma, G1_AFF * K);
    const uint8_t* d2 = c.in(second, GT_SZ * n);
    const uint8_t* db = c.in(beta, GT_SZ * n);
    const uint8_t* dv = c.in(valid, n);
    uint8_t* alpha = c.alloc(GT_SZ * n);
    const uint8_t* P = btx_opening_points(c, dsig, B, K);
    if (!c.ok()) return c.finish();
    launch_miller_lines(alpha, dl, P, (int64_t)n, c.s, (int64_t)B);
    launch_final_exp(alpha, alpha, (int64_t)n, FE_FULL, c.s);
    launch_unmask(dm, d2, alpha, db, dv, (int64_t)n, c.s);
    return c.finish();
}

int32_t wbte_btx_precompute_many(wbte_ctx* ctx, void* beta, const void* kernel_lines, const void* first,
                                 const uint8_t* valid, uint64_t B, uint64_t K) {
    // the same middle product as weighted_btx's (btx/src/decryption.rs:201-246)
    return wbte_wbtx_precompute_many(ctx, beta, kernel_lines, first, valid, B, K);
}

int32_t wbte_btx_decrypt_many(wbte_ctx* ctx, void* messages, const void* kernel_lines, const void* opening_lines,
                              const void* first, const void* second, const uint8_t* valid, const void* sigma,
                              uint64_t B, uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!messages || !kernel_lines || !opening_lines || !first || !second || !valid || !sigma || B == 0 || K == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    const uint64_t m = next_pow2(2 * B), n = B * K;
    uint8_t* dm = c.out(messages, GT_SZ * n);
    const uint8_t* dl = c.in(kernel_lines, LINE_SZ * LINES_PER_POINT * m);
    const uint8_t* dol = c.in(opening_lines, LINE_SZ * LINES_PER_POINT * B);
    const uint8_t* dfirst = c.in(first, G1_AFF * n);
    const uint8_t* d2 = c.in(second, GT_SZ * n);
    const uint8_t* dv = c.in(valid, n);
    const uint8_t* dsig = c.in(sigma, G1_AFF * K);
    uint8_t* x = c.zeros(G1_AFF * m * K);
    uint8_t* work = c.alloc(G1_XYZZ * m * K);
    uint8_t* f = c.alloc(GT_SZ * m * K);
    uint8_t* y = c.alloc(GT_SZ * n);
    uint8_t* alpha = c.alloc(GT_SZ * n);
    const uint8_t* tw = twiddles(c, (int64_t)m, false);
    const uint8_t* twi = twiddles(c, (int64_t)m, true);
    const uint8_t* P = btx_opening_points(c, dsig, B, K);
    if (!c.ok()) return c.finish();
    // cross terms up to the truncated cyclotomic transform, the opening
    // pairings up to their easy part, then one hard part per slot for
    // beta / alpha (the hard part is a homomorphism of the cyclotomic subgroup)
    cudaMemcpy2DAsync(x, G1_AFF * m, dfirst, G1_AFF * B, G1_AFF * B, K, cudaMemcpyDeviceToDevice, c.s);
    launch_group_ntt(GROUP_G1, x, work, tw, (int64_t)m, c.s, (int64_t)K);
    launch_miller_lines(f, dl, x, (int64_t)(m * K), c.s, (int64_t)m);
    launch_final_exp(f, f, (int64_t)(m * K), FE_EASY, c.s);
    launch_cyclotomic_prefix_ifft(f, twi, (int64_t)m, (int64_t)B, c.s, (int64_t)K);
    launch_miller_lines(alpha, dol, P, (int64_t)n, c.s, (int64_t)B);
    launch_final_exp(alpha, alpha, (int64_t)n, FE_EASY, c.s);
    cudaMemcpy2DAsync(y, GT_SZ * B, f, GT_SZ * m, GT_SZ * B, K, cudaMemcpyDeviceToDevice, c.s);
    launch_fp12_mul(y, y, 1, alpha, 1, true, (int64_t)n, c.s);
    launch_final_exp(y, y, (int64_t)n, FE_HARD, c.s);
    launch_fp12_mul(dm, d2, 1, y, 1, false, (int64_t)n, c.s);
    launch_fp12_mask(dm, dv, (int64_t)n, c.s);
    return c.finish();
}

// ---------------------------------------------------------- weighted_pfe
// canonical little-endian encoding of a small signed integer modulo r
static std::vector<uint8_t> fr_small_signed(const std::vector<int64_t>& c) {
    static const uint64_t R_LIMBS[4] = {0xffffffff00000001ull, 0x53bda402fffe5bfeull, 0x3339d80809a1d805ull,
                                        0x73eda753299d7d48ull};
    std::vector<uint8_t> out(FR_SZ * c.size(), 0);
    for (size_t i = 0; i < c.size(); i++) {
        uint64_t v[4] = {0, 0, 0, 0};
        if (c[i] >= 0) {
            v[0] = (uint64_t)c[i];
        } else {
            uint64_t mag = (uint64_t)(-(c[i] + 1)) + 1, borrow = 0;
            for (int k = 0; k < 4; k++) {
                uint64_t sub = (k == 0 ? mag : 0) + borrow;
                uint64_t nb = (R_LIMBS[k] < sub || (sub == 0 && borrow)) ? 1 : 0;
                v[k] = R_LIMBS[k] - sub;
                borrow = nb;
            }
        }
        memcpy(out.data() + FR_SZ * i, v, FR_SZ);
    }
    return out;
}

static int32_t check_wpfe_key(Call& c, const wbte_wpfe_key* key) {
    if (!key || !key->party_offsets || key->party_count == 0 || key->batch_size == 0 || key->total_weight == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "invalid weighted-PFE key");
    if ((uint64_t)key->party_offsets[key->party_count] != key->total_weight)
        return c.fail(WBTE_ERR_INVALID_ARG, "party offsets do not sum to the total weight");
    if (log2_exact(key->batch_size) < 0) return c.fail(WBTE_ERR_SIZE, "batch size must be a power of two");
    return WBTE_OK;
}

int32_t wbte_wpfe_fractions(wbte_ctx* ctx, void* g, void* u, const void* rho, const void* alpha, const void* masks,
                            uint64_t N, uint64_t B, int32_t party_major) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!g || !rho || !alpha || (u && !masks) || N == 0 || B == 0) return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty dimension");
    uint8_t* dg = c.out(g, FR_SZ * N * B);
    uint8_t* du = u ? c.out(u, FR_SZ * N * B) : nullptr;
    const uint8_t* dr = c.in(rho, FR_SZ * N);
    const uint8_t* da = c.in(alpha, FR_SZ * B);
    const uint8_t* dm = u ? c.in(masks, 2 * FR_SZ) : nullptr;
    if (c.ok()) launch_wpfe_fractions(dg, du, dr, da, dm, (int64_t)N, (int64_t)B, party_major != 0, c.s);
    return c.finish();
}

int32_t wbte_wpfe_keygen_material(wbte_ctx* ctx, const void* z, const int32_t* owner, const void* g, const void* u,
                                  uint64_t W, uint64_t N, uint64_t B, void* vk, void* d1, void* d2) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!z || !owner || !g || !u || !vk || !d1 || !d2 || W == 0 || N == 0 || B == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty dimension");
    for (uint64_t w = 0; w < W; w++)
        if (owner[w] < 0 || (uint64_t)owner[w] >= N) return c.fail(WBTE_ERR_INVALID_ARG, "owner index out of range");
    uint8_t* dvk = c.out(vk, G2_AFF * B * N);
    uint8_t* dd1 = c.out(d1, G2_AFF * B * W);
    uint8_t* dd2 = c.out(d2, G2_AFF * B * W);
    const uint8_t* dz = c.in(z, FR_SZ * W);
    const uint8_t* dg = c.in(g, FR_SZ * B * N);
    const uint8_t* du = c.in(u, FR_SZ * B * N);
    std::vector<int32_t> ho(owner, owner + W);
    const int32_t* downer = c.in_vec(ho);
    const uint64_t rows_per_chunk = std::max<uint64_t>(1, (uint64_t(1) << 20) / W);
    uint8_t* sc = c.alloc(FR_SZ * W * std::min<uint64_t>(rows_per_chunk, B));
    if (!c.ok()) return c.finish();
    // vk[i N + j] = [g_{j,i}] G2; D[i W + w] = [Z(w) g_{owner(w),i}] G2; U likewise with u
    launch_mul_generator(GROUP_G2, dvk, dg, (int64_t)(B * N), c.s);
    for (int pass = 0; pass < 2; pass++) {
        const uint8_t* q = pass == 0 ? dg : du;
        uint8_t* dst = pass == 0 ? dd1 : dd2;
        for (uint64_t r0 = 0; r0 < B; r0 += rows_per_chunk) {
            uint64_t nr = std::min(rows_per_chunk, B - r0);
            launch_material_scalars(sc, dz, downer, q + FR_SZ * r0 * N, (int64_t)W, (int64_t)N, (int64_t)nr, c.s);
            launch_mul_generator(GROUP_G2, dst + G2_AFF * r0 * W, sc, (int64_t)(nr * W), c.s);
        }
    }
    return c.finish();
}

int32_t wbte_wpfe_partial_decrypt(wbte_ctx* ctx, void* sigma, const void* first, const void* rho, const void* alpha,
                                  uint64_t T, uint64_t B) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (T == 0) return c.finish();
    if (!sigma || !first || !rho || !alpha || B == 0) return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    uint8_t* dsig = c.out(sigma, G1_AFF * T);
    const uint8_t* dfirst = c.in(first, G1_AFF * B);
    const uint8_t* dr = c.in(rho, FR_SZ * T);
    const uint8_t* da = c.in(alpha, FR_SZ * B);
    uint8_t* g = c.alloc(FR_SZ * T * B);
    std::vector<int64_t> base(T, 0);
    std::vector<int32_t> vsel(T);
    for (uint64_t j = 0; j < T; j++) vsel[j] = (int32_t)j;
    const int64_t* db = c.in_vec(base);
    const int32_t* dv = c.in_vec(vsel);
    if (!c.ok()) return c.finish();
    // sigma_j = sum_i g_{j,i} first_i (weighted_pfe/src/decryption.rs:231-252)
    launch_wpfe_fractions(g, nullptr, dr, da, nullptr, (int64_t)T, (int64_t)B, true, c.s);
    launch_msm_family(GROUP_G1, dsig, dfirst, db, nullptr, g, dv, (int32_t)T, (int64_t)T, (int64_t)B, c.s);
    return c.finish();
}

int32_t wbte_wpfe_verify_shares(wbte_ctx* ctx, int32_t* ok, const wbte_wpfe_key* key, const void* first,
                                const void* sigma, const int64_t* party_indices, const void* challenges, uint64_t T) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    {
        Call c(ctx);
        if (check_wpfe_key(c, key)) return c.finish();
        if (!ok) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    }
    // the weighted_btx aggregate check with every slot valid
    // (weighted_pfe/src/decryption.rs:367-419 and :254-275)
    wbte_wbtx_key wk;
    wk.domain_points = key->domain_points;
    wk.verification_keys = key->verification_keys;
    wk.negative_material = key->d1;
    wk.positive_material = key->d2;
    wk.party_offsets = key->party_offsets;
    wk.party_count = key->party_count;
    wk.total_weight = key->total_weight;
    wk.max_batch_size = key->batch_size;
    std::vector<uint8_t> valid(key->batch_size, 1);
    return wbte_wbtx_verify_shares(ctx, ok, &wk, first, valid.data(), key->batch_size, sigma, party_indices, challenges, T);
}

int32_t wbte_wpfe_prepare(wbte_ctx* ctx, const wbte_wpfe_key* key, const int64_t* party_indices, uint64_t T,
                          const void* mask_scalars, void* by_party, void* total_lines, void* mask_lines, void* total,
                          void* mask) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (check_wpfe_key(c, key)) return c.finish();
    if (!party_indices || T == 0 || !mask_scalars || !by_party || !total_lines || !mask_lines || !key->d1 || !key->d2 ||
        !key->global_key || !key->domain_points)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    const uint64_t N = key->party_count, W = key->total_weight, B = key->batch_size;
    const int lg2b = log2_exact(2 * B);
    std::vector<int32_t> sel;
    std::vector<int64_t> coef_off(1, 0), party_base(T);
    for (uint64_t k = 0; k < T; k++) {
        int64_t j = party_indices[k];
        if (j < 0 || (uint64_t)j >= N) return c.fail(WBTE_ERR_INVALID_ARG, "invalid party index");
        if (k && party_indices[k - 1] >= j) return c.fail(WBTE_ERR_INVALID_ARG, "party indices must be strictly ascending");
        for (int64_t w = key->party_offsets[j]; w < key->party_offsets[j + 1]; w++) sel.push_back((int32_t)w);
        coef_off.push_back((int64_t)sel.size());
        party_base[k] = key->party_offsets[j];
    }
    const int64_t WT = (int64_t)sel.size();
    uint8_t* dby = c.out(by_party, G2_AFF * B * T);
    uint8_t* dtl = c.out(total_lines, LINE_SZ * LINES_PER_POINT * B);
    uint8_t* dml = c.out(mask_lines, LINE_SZ * LINES_PER_POINT * B);
    uint8_t* dtot_out = total ? c.out(total, G2_AFF * B) : nullptr;
    uint8_t* dmask_out = mask ? c.out(mask, G2_AFF * B) : nullptr;
    const uint8_t* ddom = c.in(key->domain_points, FR_SZ * W);
    const uint8_t* dd1 = c.in(key->d1, G2_AFF * B * W);
    const uint8_t* dd2 = c.in(key->d2, G2_AFF * B * W);
    const uint8_t* dV = c.in(key->global_key, G2_AFF);
    const uint8_t* dms = c.in(mask_scalars, 2 * FR_SZ * B);
    const int32_t* dsel = c.in_vec(sel);
    uint8_t* x = c.alloc(FR_SZ * WT);
    uint8_t* lam = c.alloc(FR_SZ * WT);
    uint8_t* lam_s = c.alloc(FR_SZ * WT);
    int32_t* status = (int32_t*)c.zeros(sizeof(int32_t));
    uint8_t* tmp = c.alloc(G2_AFF * B);
    uint8_t* tot = c.alloc(G2_AFF * B);
    uint8_t* d2t = c.alloc(G2_AFF * B);
    uint8_t* pairs = c.alloc(2 * G2_AFF * B);
    uint8_t* msk = c.alloc(G2_AFF * B);
    // segment offsets carry k + 1 entries for k segments
    std::vector<int64_t> slot_base(B), offs_T(B + 1), offs_2(B + 1), d2base(B);
    for (uint64_t i = 0; i <= B; i++) {
        offs_T[i] = (int64_t)(i * T);
        offs_2[i] = (int64_t)(2 * i);
        if (i < B) d2base[i] = (int64_t)(i * W);
    }
    const int64_t* doffT = c.in_vec(offs_T);
    const int64_t* doff2 = c.in_vec(offs_2);
    const int64_t* dd2b = c.in_vec(d2base);
    if (!c.ok()) return c.finish();
    // Lagrange coefficients of the accepted virtual points; lambda / 2B for D
    launch_gather(x, ddom, dsel, WT, FR_SZ, c.s);
    launch_lagrange_at_zero(lam, x, WT, status, c.s);
    launch_fr_scale_size_inv(lam_s, lam, lg2b, WT, c.s);
    // scaled_d1_by_party[i T + k] = sum_{w in party k} lambda_w / 2B D[i W + w]
    for (uint64_t k = 0; k < T; k++) {
        for (uint64_t i = 0; i < B; i++) slot_base[i] = (int64_t)(i * W) + party_base[k];
        const int64_t* dbase = c.in_vec(slot_base);
        if (!c.ok()) return c.finish();
        int64_t wk = coef_off[k + 1] - coef_off[k];
        launch_msm_family(GROUP_G2, tmp, dd1, dbase, nullptr, lam_s + FR_SZ * coef_off[k], nullptr, 1, (int64_t)B, wk, c.s);
        cudaMemcpy2DAsync(dby + G2_AFF * k, G2_AFF * T, tmp, G2_AFF, G2_AFF, B, cudaMemcpyDeviceToDevice, c.s);
    }
    launch_segment_sum(GROUP_G2, tot, dby, doffT, (int64_t)B, c.s);
    // mask_i = alpha_i (alpha_i + 1) sum_w lambda_w U[i W + w] - alpha_i V
    launch_msm_family(GROUP_G2, d2t, dd2, dd2b, dsel, lam, nullptr, 1, (int64_t)B, WT, c.s);
    launch_mul_batch(GROUP_G2, tmp, d2t, 1, dms, (int64_t)B, c.s);
    cudaMemcpy2DAsync(pairs, 2 * G2_AFF, tmp, G2_AFF, G2_AFF, B, cudaMemcpyDeviceToDevice, c.s);
    launch_mul_batch(GROUP_G2, tmp, dV, 0, dms + FR_SZ * B, (int64_t)B, c.s);
    cudaMemcpy2DAsync(pairs + G2_AFF, 2 * G2_AFF, tmp, G2_AFF, G2_AFF, B, cudaMemcpyDeviceToDevice, c.s);
    launch_segment_sum(GROUP_G2, msk, pairs, doff2, (int64_t)B, c.s);
    launch_prepare_lines(dtl, tot, (int64_t)B, c.s);
    launch_prepare_lines(dml, msk, (int64_t)B, c.s);
    if (dtot_out) cudaMemcpyAsync(dtot_out, tot, G2_AFF * B, cudaMemcpyDeviceToDevice, c.s);
    if (dmask_out) cudaMemcpyAsync(dmask_out, msk, G2_AFF * B, cudaMemcpyDeviceToDevice, c.s);
    int32_t st = 0;
    if (c.to_host(&st, status, sizeof(st)) && st) c.fail(WBTE_ERR_INTERPOLATION, "the interpolation points must be nonempty and distinct");
    return c.finish();
}

// The Cauchy sums of K batches of one size B laid back to back
// (precompute_batch, weighted_pfe/src/decryption.rs:540-574, :683-734):
//   dfc[b B + i] = 2B sum_{k != i} first[b B + k] / (alpha_k - alpha_i)
//   dpc[b B + i] = the same sums over e(first[b B + k], total_k) on easy-final-
//                  exponentiated values (canonical after the hard part),
// with the closed-form spectrum B - 1 - 2k of the Cauchy kernel (:194-213):
// per batch a forward transform, the spectrum, a cyclic rotation by one and
// the inverse transform, every step one launch over all K batches.
static bool wpfe_precompute_core(Call& c, uint8_t* dfc, uint8_t* dpc, const uint8_t* dfirst, const uint8_t* dl,
                                 uint64_t B, uint64_t K) {
    const uint64_t n = B * K;
    std::vector<int32_t> coeff(n), rot(n);
    for (uint64_t b = 0; b < K; b++)
        for (uint64_t k = 0; k < B; k++) {
            coeff[b * B + k] = (int32_t)B - 1 - 2 * (int32_t)k;
            rot[b * B + k] = (int32_t)(b * B + (k + B - 1) % B);
        }
    // the spectrum's coefficients are small signed integers: double-and-add
    // and square-and-multiply over their bits (mul_group_signed_small,
    // mul_cyclotomic_signed_small), not full scalar multiplications
    const int32_t* dcoef = c.in_vec(coeff);
    const int32_t* drot = c.in_vec(rot);
    uint8_t* x = c.alloc(G1_AFF * n);
    uint8_t* y = c.alloc(G1_AFF * n);
    uint8_t* work = c.alloc(G1_XYZZ * n);
    uint8_t* f = c.alloc(GT_SZ * n);
    uint8_t* h = c.alloc(GT_SZ * n);
    const uint8_t* tw = B > 1 ? twiddles(c, (int64_t)B, false) : nullptr;
    const uint8_t* twi = B > 1 ? twiddles(c, (int64_t)B, true) : nullptr;
    if (!c.ok()) return false;
    // G1: 2B sum_{k != i} first_k / (alpha_k - alpha_i) (:683-708)
    cudaMemcpyAsync(x, dfirst, G1_AFF * n, cudaMemcpyDeviceToDevice, c.s);
    if (B > 1) launch_group_ntt(GROUP_G1, x, work, tw, (int64_t)B, c.s, (int64_t)K);
    launch_mul_small(GROUP_G1, y, x, dcoef, (int64_t)n, c.s);
    launch_gather(x, y, drot, (int64_t)n, G1_AFF, c.s);
    launch_negate(GROUP_G1, x, x, (int64_t)n, c.s);
    if (B > 1) launch_group_ntt(GROUP_G1, x, work, twi, (int64_t)B, c.s, (int64_t)K);
    cudaMemcpyAsync(dfc, x, G1_AFF * n, cudaMemcpyDeviceToDevice, c.s);
    // GT: the same sums over e(first_k, D1_k) on easy-final-exponentiated values (:710-734)
    launch_miller_lines(f, dl, dfirst, (int64_t)n, c.s, (int64_t)B);
    launch_final_exp(f, f, (int64_t)n, FE_EASY, c.s);
    if (B > 1) launch_gt_ntt(f, tw, (int64_t)B, c.s, (int64_t)K);
    launch_gt_pow_small(h, f, 1, dcoef, (int64_t)n, c.s);
    launch_gather(f, h, drot, (int64_t)n, GT_SZ, c.s);
    launch_fp12_conj(f, f, (int64_t)n, c.s);
    if (B > 1) launch_gt_ntt(f, twi, (int64_t)B, c.s, (int64_t)K, true);
    cudaMemcpyAsync(dpc, f, GT_SZ * n, cudaMemcpyDeviceToDevice, c.s);
    return true;
}

// The opening of K batches of one size B against one committee
// (open_batch, weighted_pfe/src/decryption.rs:576-644):
//   messages[b B + i] = second - hard(e(first_i, mask_i) /
//       (prod_k e(2B sigma_{b,k} - first_cauchy_i, by_party[i T + k]) pairing_cauchy_i)^(alpha_i (alpha_i + 1)))
// ds: K*T shares (batch-major); dby: B*T G2 (shared); by_lines: their line
// tables or NULL (then T unprepared loops per slot); dap: B Fr.
static bool wpfe_open_core(Call& c, uint8_t* dm, const uint8_t* ds, uint64_t T, const uint8_t* dby,
                           const void* by_lines, const uint8_t* dfirst, const uint8_t* dml, const uint8_t* dfc,
                           const uint8_t* dpc, const uint8_t* d2, const uint8_t* dap, uint64_t B, uint64_t K) {
    const uint64_t n = B * K, nt = n * T;
    const uint8_t* d2b = c.in_vec(fr_small_signed(std::vector<int64_t>(T * K, 2 * (int64_t)B)));
    std::vector<int32_t> idx_share(nt), idx_slot(nt), idx_ap(n);
    // segment offsets carry k + 1 entries for k segments
    std::vector<int64_t> offs_2(nt + 1);
    for (uint64_t o = 0; o < n; o++) {
        idx_ap[o] = (int32_t)(o % B);
        for (uint64_t k = 0; k < T; k++) {
            idx_share[o * T + k] = (int32_t)((o / B) * T + k);
            idx_slot[o * T + k] = (int32_t)o;
        }
    }
    for (uint64_t x = 0; x <= nt; x++) offs_2[x] = (int64_t)(2 * x);
    const int32_t* dis = c.in_vec(idx_share);
    const int32_t* dil = c.in_vec(idx_slot);
    const int32_t* dia = c.in_vec(idx_ap);
    const int64_t* do2 = c.in_vec(offs_2);
    uint8_t* scaled = c.alloc(G1_AFF * T * K);
    uint8_t* negfc = c.alloc(G1_AFF * n);
    uint8_t* g0 = c.alloc(G1_AFF * nt);
    uint8_t* g1 = c.alloc(G1_AFF * nt);
    uint8_t* pairs = c.alloc(2 * G1_AFF * nt);
    uint8_t* left = c.alloc(G1_AFF * nt);
    uint8_t* ft = c.alloc(GT_SZ * n);
    uint8_t* mp = c.alloc(GT_SZ * n);
    uint8_t* apr = c.alloc(FR_SZ * n);
    const bool prepared = by_lines != nullptr;
    const uint8_t* dbl = prepared ? c.in(by_lines, LINE_SZ * LINES_PER_POINT * B * T) : nullptr;
    uint8_t* f = c.alloc(GT_SZ * (prepared ? n : nt));
    if (!c.ok()) return false;
    // left[(b B + i) T + k] = 2B sigma_{b,k} - first_cauchy[b B + i] (:596-612)
    launch_mul_batch(GROUP_G1, scaled, ds, 1, d2b, (int64_t)(T * K), c.s);
    launch_negate(GROUP_G1, negfc, dfc, (int64_t)n, c.s);
    launch_gather(g0, scaled, dis, (int64_t)nt, G1_AFF, c.s);
    launch_gather(g1, negfc, dil, (int64_t)nt, G1_AFF, c.s);
    cudaMemcpy2DAsync(pairs, 2 * G1_AFF, g0, G1_AFF, G1_AFF, nt, cudaMemcpyDeviceToDevice, c.s);
    cudaMemcpy2DAsync(pairs + G1_AFF, 2 * G1_AFF, g1, G1_AFF, G1_AFF, nt, cudaMemcpyDeviceToDevice, c.s);
    launch_segment_sum(GROUP_G1, left, pairs, do2, (int64_t)nt, c.s);
    // first terms: per slot the T pairings with the committee's keys of that
    // slot, one multi-Miller loop over their line tables when given
    if (prepared) {
        launch_miller_lines_multi(ft, dbl, left, (int64_t)n, (int64_t)B, (int)T, c.s, 1);
    } else {
        std::vector<int64_t> offs_T(n + 1);
        for (uint64_t o = 0; o <= n; o++) offs_T[o] = (int64_t)(o * T);
        const int64_t* doT = c.in_vec(offs_T);
        if (!c.ok()) return false;
        launch_miller(f, left, dby, (int64_t)nt, c.s, 0, (int64_t)(B * T));
        launch_fp12_segment_product(ft, f, doT, (int64_t)n, c.s);
    }
    launch_miller_lines(mp, dml, dfirst, (int64_t)n, c.s, (int64_t)B);
    launch_final_exp(ft, ft, (int64_t)n, FE_EASY, c.s);
    launch_final_exp(mp, mp, (int64_t)n, FE_EASY, c.s);
    // mask = hard(mp / (ft pairing_cauchy)^(alpha (alpha + 1))); message = second / mask (:614-643)
    launch_fp12_mul(ft, ft, 1, dpc, 1, false, (int64_t)n, c.s);
    // the slot's exponent is shared by the K batches: warp-uniform plans when K allows
    if (!launch_gt_pow_shared(f, ft, dap, (int64_t)B, (int64_t)K, c.s)) {
        launch_gather(apr, dap, dia, (int64_t)n, FR_SZ, c.s);
        launch_gt_pow(f, ft, 1, apr, (int64_t)n, c.s);
    }
    launch_fp12_mul(mp, mp, 1, f, 1, true, (int64_t)n, c.s);
    launch_final_exp(mp, mp, (int64_t)n, FE_HARD, c.s);
    launch_fp12_mul(dm, d2, 1, mp, 1, true, (int64_t)n, c.s);
    return true;
}

int32_t wbte_wpfe_precompute(wbte_ctx* ctx, void* first_cauchy, void* pairing_cauchy, const void* first,
                             const void* total_lines, uint64_t B) {
    return wbte_wpfe_precompute_many(ctx, first_cauchy, pairing_cauchy, first, total_lines, B, 1);
}

int32_t wbte_wpfe_open(wbte_ctx* ctx, void* messages, const void* sigmas, uint64_t T, const void* by_party,
                       const void* first, const void* mask_lines, const void* first_cauchy, const void* pairing_cauchy,
                       const void* second, const void* alpha_products, uint64_t B) {
    return wbte_wpfe_open_many(ctx, messages, sigmas, T, by_party, nullptr, first, mask_lines, first_cauchy,
                               pairing_cauchy, second, alpha_products, B, 1);
}

// ------------------------------------------- weighted_pfe, K batches per call
int32_t wbte_wpfe_partial_decrypt_many(wbte_ctx* ctx, void* sigma, const void* first, const void* rho,
                                       const void* alpha, uint64_t T, uint64_t B, uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (T == 0 || K == 0) return c.finish();
    if (!sigma || !first || !rho || !alpha || B == 0) return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    uint8_t* dsig = c.out(sigma, G1_AFF * T * K);
    const uint8_t* dfirst = c.in(first, G1_AFF * B * K);
    const uint8_t* dr = c.in(rho, FR_SZ * T);
    const uint8_t* da = c.in(alpha, FR_SZ * B);
    uint8_t* g = c.alloc(FR_SZ * T * B);
    std::vector<int64_t> base(T * K);
    std::vector<int32_t> vsel(T * K);
    for (uint64_t b = 0; b < K; b++)
        for (uint64_t j = 0; j < T; j++) {
            base[b * T + j] = (int64_t)(b * B);
            vsel[b * T + j] = (int32_t)j;
        }
    const int64_t* db = c.in_vec(base);
    const int32_t* dv = c.in_vec(vsel);
    if (!c.ok()) return c.finish();
    // sigma[b T + j] = sum_i g_{j,i} first[b B + i] (weighted_pfe/src/decryption.rs:231-252):
    // the T fraction vectors are shared by the K batches' MSMs
    launch_wpfe_fractions(g, nullptr, dr, da, nullptr, (int64_t)T, (int64_t)B, true, c.s);
    launch_msm_family(GROUP_G1, dsig, dfirst, db, nullptr, g, dv, (int32_t)T, (int64_t)(T * K), (int64_t)B, c.s);
    return c.finish();
}

static wbte_wbtx_key wpfe_as_wbtx_key(const wbte_wpfe_key* key) {
    wbte_wbtx_key wk;
    wk.domain_points = key->domain_points;
    wk.verification_keys = key->verification_keys;
    wk.negative_material = key->d1;
    wk.positive_material = key->d2;
    wk.party_offsets = key->party_offsets;
    wk.party_count = key->party_count;
    wk.total_weight = key->total_weight;
    wk.max_batch_size = key->batch_size;
    return wk;
}

int32_t wbte_wpfe_vk_tables(wbte_ctx* ctx, void* tables, const wbte_wpfe_key* key, const int64_t* party_indices,
                            uint64_t T) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    {
        Call c(ctx);
        if (check_wpfe_key(c, key)) return c.finish();
    }
    wbte_wbtx_key wk = wpfe_as_wbtx_key(key);
    return wbte_wbtx_vk_tables(ctx, tables, &wk, party_indices, T, key->batch_size);
}

int32_t wbte_wpfe_verify_shares_many(wbte_ctx* ctx, int32_t* ok, const wbte_wpfe_key* key, const void* first,
                                     const void* sigma, const int64_t* party_indices, const void* challenges,
                                     uint64_t T, uint64_t K, const void* vk_tables) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    {
        Call c(ctx);
        if (check_wpfe_key(c, key)) return c.finish();
    }
    // the aggregate check of verify_decryption_shares_batched
    // (weighted_pfe/src/decryption.rs:367-419) per batch: weighted_pfe
    // accepts a batch only when every proof holds, so every slot enters
    wbte_wbtx_key wk = wpfe_as_wbtx_key(key);
    return wbte_wbtx_verify_shares_many(ctx, ok, &wk, first, key->batch_size, sigma, party_indices, challenges, T, K,
                                        vk_tables);
}

int32_t wbte_wpfe_precompute_many(wbte_ctx* ctx, void* first_cauchy, void* pairing_cauchy, const void* first,
                                  const void* total_lines, uint64_t B, uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!first_cauchy || !pairing_cauchy || !first || !total_lines || B == 0 || K == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    if (log2_exact(B) < 0) return c.fail(WBTE_ERR_SIZE, "batch size must be a power of two");
    uint8_t* dfc = c.out(first_cauchy, G1_AFF * B * K);
    uint8_t* dpc = c.out(pairing_cauchy, GT_SZ * B * K);
    const uint8_t* dfirst = c.in(first, G1_AFF * B * K);
    const uint8_t* dl = c.in(total_lines, LINE_SZ * LINES_PER_POINT * B);
    if (c.ok()) wpfe_precompute_core(c, dfc, dpc, dfirst, dl, B, K);
    return c.finish();
}

int32_t wbte_wpfe_open_many(wbte_ctx* ctx, void* messages, const void* sigmas, uint64_t T, const void* by_party,
                            const void* by_party_lines, const void* first, const void* mask_lines,
                            const void* first_cauchy, const void* pairing_cauchy, const void* second,
                            const void* alpha_products, uint64_t B, uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!messages || !sigmas || T == 0 || !by_party || !first || !mask_lines || !first_cauchy || !pairing_cauchy ||
        !second || !alpha_products || B == 0 || K == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    const uint64_t n = B * K;
    uint8_t* dm = c.out(messages, GT_SZ * n);
    const uint8_t* ds = c.in(sigmas, G1_AFF * T * K);
    const uint8_t* dby = c.in(by_party, G2_AFF * B * T);
    const uint8_t* dfirst = c.in(first, G1_AFF * n);
    const uint8_t* dml = c.in(mask_lines, LINE_SZ * LINES_PER_POINT * B);
    const uint8_t* dfc = c.in(first_cauchy, G1_AFF * n);
    const uint8_t* dpc = c.in(pairing_cauchy, GT_SZ * n);
    const uint8_t* d2 = c.in(second, GT_SZ * n);
    const uint8_t* dap = c.in(alpha_products, FR_SZ * B);
    if (c.ok()) wpfe_open_core(c, dm, ds, T, dby, by_party_lines, dfirst, dml, dfc, dpc, d2, dap, B, K);
    return c.finish();
}

int32_t wbte_wpfe_decrypt_many(wbte_ctx* ctx, void* messages, const void* sigmas, uint64_t T, const void* by_party,
                               const void* by_party_lines, const void* total_lines, const void* mask_lines,
                               const void* first, const void* second, const void* alpha_products, uint64_t B,
                               uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!messages || !sigmas || T == 0 || !by_party || !total_lines || !mask_lines || !first || !second ||
        !alpha_products || B == 0 || K == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    if (log2_exact(B) < 0) return c.fail(WBTE_ERR_SIZE, "batch size must be a power of two");
    const uint64_t n = B * K;
    uint8_t* dm = c.out(messages, GT_SZ * n);
    const uint8_t* ds = c.in(sigmas, G1_AFF * T * K);
    const uint8_t* dby = c.in(by_party, G2_AFF * B * T);
    const uint8_t* dtl = c.in(total_lines, LINE_SZ * LINES_PER_POINT * B);
    const uint8_t* dml = c.in(mask_lines, LINE_SZ * LINES_PER_POINT * B);
    const uint8_t* dfirst = c.in(first, G1_AFF * n);
    const uint8_t* d2 = c.in(second, GT_SZ * n);
    const uint8_t* dap = c.in(alpha_products, FR_SZ * B);
    uint8_t* fc = c.alloc(G1_AFF * n);
    uint8_t* pc = c.alloc(GT_SZ * n);
    if (c.ok() && wpfe_precompute_core(c, fc, pc, dfirst, dtl, B, K))
        wpfe_open_core(c, dm, ds, T, dby, by_party_lines, dfirst, dml, fc, pc, d2, dap, B, K);
    return c.finish();
}

// ------------------------------------------------------------------ pfe
// Gamma-weighted cyclic convolution of pfe/src/decryption.rs:471-526 on B
// elements in place: io <- INTT(rem) with rem[i] = c spec[i+1] - spec[i] and
// spec = NTT(io) * E.  E and cvec hold B Fr each (E[k] = B - 1 - 2k mod r,
// cvec = B copies of c).  Group elements in affine form; GT in Fp12.
static void pfe_conv_group(Call& c, Group g, uint8_t* io, const uint8_t* E, const uint8_t* cvec, const int32_t* rot,
                           const int64_t* offs2, uint64_t B, const uint8_t* tw, const uint8_t* twi, uint64_t K = 1) {
    // K transforms of B elements back to back; E, cvec, rot and offs2 cover all K B
    const size_t aff = g == GROUP_G1 ? G1_AFF : G2_AFF, xz = g == GROUP_G1 ? G1_XYZZ : G2_XYZZ;
    const uint64_t n = B * K;
    uint8_t* work = c.alloc(xz * n);
    uint8_t* a = c.alloc(aff * n);
    uint8_t* b = c.alloc(aff * n);
    uint8_t* pairs = c.alloc(2 * aff * n);
    if (!c.ok()) return;
    if (B > 1) launch_group_ntt(g, io, work, tw, (int64_t)B, c.s, (int64_t)K);
    launch_mul_batch(g, a, io, 1, E, (int64_t)n, c.s);
    launch_gather(b, a, rot, (int64_t)n, aff, c.s);
    launch_mul_batch(g, b, b, 1, cvec, (int64_t)n, c.s);
    launch_negate(g, a, a, (int64_t)n, c.s);
    cudaMemcpy2DAsync(pairs, 2 * aff, b, aff, aff, n, cudaMemcpyDeviceToDevice, c.s);
    cudaMemcpy2DAsync(pairs + aff, 2 * aff, a, aff, aff, n, cudaMemcpyDeviceToDevice, c.s);
    launch_segment_sum(g, io, pairs, offs2, (int64_t)n, c.s);
    if (B > 1) launch_group_ntt(g, io, work, twi, (int64_t)B, c.s, (int64_t)K);
}
static void pfe_conv_gt(Call& c, uint8_t* io, const uint8_t* E, const uint8_t* cvec, const int32_t* rot, uint64_t B,
                        const uint8_t* tw, const uint8_t* twi, uint64_t K = 1) {
    const uint64_t n = B * K;
    uint8_t* a = c.alloc(GT_SZ * n);
    uint8_t* b = c.alloc(GT_SZ * n);
    uint8_t* h = c.alloc(GT_SZ * n);
    if (!c.ok()) return;
    if (B > 1) launch_gt_ntt(io, tw, (int64_t)B, c.s, (int64_t)K);
    launch_gt_pow(a, io, 1, E, (int64_t)n, c.s);
    launch_gather(h, a, rot, (int64_t)n, GT_SZ, c.s);
    launch_gt_pow(b, h, 1, cvec, (int64_t)n, c.s);
    launch_fp12_mul(io, b, 1, a, 1, true, (int64_t)n, c.s);
    if (B > 1) launch_gt_ntt(io, twi, (int64_t)B, c.s, (int64_t)K, true);
}

// index tables of the convolution over K batches of B: rot[b B + i] = b B +
// (i + 1) mod B, slot[b B + i] = i, batch[b B + i] = b, offs2 = 0, 2, 4, ..
struct PfeConvTables {
    std::vector<int32_t> rot, slot, batch;
    std::vector<int64_t> offs2;
    explicit PfeConvTables(uint64_t B, uint64_t K = 1) : rot(B * K), slot(B * K), batch(B * K), offs2(B * K + 1) {
        for (uint64_t b = 0; b < K; b++)
            for (uint64_t i = 0; i < B; i++) {
                rot[b * B + i] = (int32_t)(b * B + (i + 1) % B);
                slot[b * B + i] = (int32_t)i;
                batch[b * B + i] = (int32_t)b;
            }
        for (uint64_t i = 0; i <= B * K; i++) offs2[i] = (int64_t)(2 * i);
    }
};

int32_t wbte_pfe_kernel(wbte_ctx* ctx, const void* fraction_keys, const void* key_sum, uint64_t B, const void* scalars,
                        void* key_lines, void* generator_lines, void* mix_lines, void* scaled_keys, void* generators,
                        void* mixes) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!fraction_keys || !key_sum || !scalars || !key_lines || !generator_lines || !mix_lines || B == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    if (log2_exact(B) < 0) return c.fail(WBTE_ERR_SIZE, "batch size must be a power of two");
    const size_t LT = LINE_SZ * LINES_PER_POINT * B;
    uint8_t* dkl = c.out(key_lines, LT);
    uint8_t* dgl = c.out(generator_lines, LT);
    uint8_t* dml = c.out(mix_lines, LT);
    uint8_t* dsk_out = scaled_keys ? c.out(scaled_keys, G2_AFF * B) : nullptr;
    uint8_t* dg_out = generators ? c.out(generators, G2_AFF * B) : nullptr;
    uint8_t* dmx_out = mixes ? c.out(mixes, G2_AFF * B) : nullptr;
    const uint8_t* dkeys = c.in(fraction_keys, G2_AFF * B);
    const uint8_t* dsum = c.in(key_sum, G2_AFF);
    const uint8_t* sc = c.in(scalars, 6 * FR_SZ * B);
    PfeConvTables tab(B);
    const int32_t* drot = c.in_vec(tab.rot);
    const int64_t* doff2 = c.in_vec(tab.offs2);
    std::vector<int64_t> offs3(B + 1);
    for (uint64_t i = 0; i <= B; i++) offs3[i] = (int64_t)(3 * i);
    const int64_t* doff3 = c.in_vec(offs3);
    uint8_t* sk = c.alloc(G2_AFF * B);
    uint8_t* wk = c.alloc(G2_AFF * B);
    uint8_t* gens = c.alloc(G2_AFF * B);
    uint8_t* t1 = c.alloc(G2_AFF * B);
    uint8_t* t2 = c.alloc(G2_AFF * B);
    uint8_t* triples = c.alloc(3 * G2_AFF * B);
    uint8_t* mx = c.alloc(G2_AFF * B);
    const uint8_t* tw = B > 1 ? twiddles(c, (int64_t)B, false) : nullptr;
    const uint8_t* twi = B > 1 ? twiddles(c, (int64_t)B, true) : nullptr;
    if (!c.ok()) return c.finish();
    const uint8_t *inv2b = sc, *E = sc + FR_SZ * B, *cvec = sc + 2 * FR_SZ * B, *s2 = sc + 3 * FR_SZ * B,
                  *neg_s2 = sc + 4 * FR_SZ * B, *neg_mix = sc + 5 * FR_SZ * B;
    // scaled keys DK/(2B), their weighted convolution, generators [s2] G2 (pfe/src/decryption.rs:151-214)
    launch_mul_batch(GROUP_G2, sk, dkeys, 1, inv2b, (int64_t)B, c.s);
    cudaMemcpyAsync(wk, sk, G2_AFF * B, cudaMemcpyDeviceToDevice, c.s);
    pfe_conv_group(c, GROUP_G2, wk, E, cvec, drot, doff2, B, tw, twi);
    launch_mul_generator(GROUP_G2, gens, s2, (int64_t)B, c.s);
    // final mix = weighted - s2 * key_sum - (s1_bar * opening coefficient) * scaled key (:216-230)
    launch_mul_batch(GROUP_G2, t1, dsum, 0, neg_s2, (int64_t)B, c.s);
    launch_mul_batch(GROUP_G2, t2, sk, 1, neg_mix, (int64_t)B, c.s);
    cudaMemcpy2DAsync(triples, 3 * G2_AFF, wk, G2_AFF, G2_AFF, B, cudaMemcpyDeviceToDevice, c.s);
    cudaMemcpy2DAsync(triples + G2_AFF, 3 * G2_AFF, t1, G2_AFF, G2_AFF, B, cudaMemcpyDeviceToDevice, c.s);
    cudaMemcpy2DAsync(triples + 2 * G2_AFF, 3 * G2_AFF, t2, G2_AFF, G2_AFF, B, cudaMemcpyDeviceToDevice, c.s);
    launch_segment_sum(GROUP_G2, mx, triples, doff3, (int64_t)B, c.s);
    launch_prepare_lines(dkl, sk, (int64_t)B, c.s);
    launch_prepare_lines(dgl, gens, (int64_t)B, c.s);
    launch_prepare_lines(dml, mx, (int64_t)B, c.s);
    if (dsk_out) cudaMemcpyAsync(dsk_out, sk, G2_AFF * B, cudaMemcpyDeviceToDevice, c.s);
    if (dg_out) cudaMemcpyAsync(dg_out, gens, G2_AFF * B, cudaMemcpyDeviceToDevice, c.s);
    if (dmx_out) cudaMemcpyAsync(dmx_out, mx, G2_AFF * B, cudaMemcpyDeviceToDevice, c.s);
    return c.finish();
}

int32_t wbte_pfe_precompute(wbte_ctx* ctx, void* weighted_first, void* weighted_pairings, const void* first,
                            const void* key_lines, const void* scalars, uint64_t B) {
    return wbte_pfe_precompute_many(ctx, weighted_first, weighted_pairings, first, key_lines, scalars, B, 1);
}

int32_t wbte_pfe_precompute_many(wbte_ctx* ctx, void* weighted_first, void* weighted_pairings, const void* first,
                                 const void* key_lines, const void* scalars, uint64_t B, uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!weighted_first || !weighted_pairings || !first || !key_lines || !scalars || B == 0 || K == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    if (log2_exact(B) < 0) return c.fail(WBTE_ERR_SIZE, "batch size must be a power of two");
    const uint64_t n = B * K;
    uint8_t* dwf = c.out(weighted_first, G1_AFF * n);
    uint8_t* dwp = c.out(weighted_pairings, GT_SZ * n);
    const uint8_t* dfirst = c.in(first, G1_AFF * n);
    const uint8_t* dkl = c.in(key_lines, LINE_SZ * LINES_PER_POINT * B);
    const uint8_t* sc = c.in(scalars, 2 * FR_SZ * B);
    PfeConvTables tab(B, K);
    const int32_t* drot = c.in_vec(tab.rot);
    const int32_t* dslot = c.in_vec(tab.slot);
    const int64_t* doff2 = c.in_vec(tab.offs2);
    uint8_t* x = c.alloc(G1_AFF * n);
    uint8_t* f = c.alloc(GT_SZ * n);
    uint8_t* E = c.alloc(FR_SZ * n);
    uint8_t* cvec = c.alloc(FR_SZ * n);
    const uint8_t* tw = B > 1 ? twiddles(c, (int64_t)B, false) : nullptr;
    const uint8_t* twi = B > 1 ? twiddles(c, (int64_t)B, true) : nullptr;
    if (!c.ok()) return c.finish();
    // the B scalars of each kind, repeated for every batch
    launch_gather(E, sc, dslot, (int64_t)n, FR_SZ, c.s);
    launch_gather(cvec, sc + FR_SZ * B, dslot, (int64_t)n, FR_SZ, c.s);
    // weighted convolution of the first components and of e(first_i, DK_i/(2B)) (pfe/src/decryption.rs:259-298)
    cudaMemcpyAsync(x, dfirst, G1_AFF * n, cudaMemcpyDeviceToDevice, c.s);
    pfe_conv_group(c, GROUP_G1, x, E, cvec, drot, doff2, B, tw, twi, K);
    launch_miller_lines(f, dkl, dfirst, (int64_t)n, c.s, (int64_t)B);
    launch_final_exp(f, f, (int64_t)n, FE_FULL, c.s);
    pfe_conv_gt(c, f, E, cvec, drot, B, tw, twi, K);
    cudaMemcpyAsync(dwf, x, G1_AFF * n, cudaMemcpyDeviceToDevice, c.s);
    cudaMemcpyAsync(dwp, f, GT_SZ * n, cudaMemcpyDeviceToDevice, c.s);
    return c.finish();
}

int32_t wbte_pfe_open(wbte_ctx* ctx, void* messages, const void* first, const void* second, const void* third,
                      const void* weighted_first, const void* weighted_pairings, const void* pre_decryption_key,
                      const void* neg_scaled_s1, const void* key_lines, const void* generator_lines,
                      const void* mix_lines, uint64_t B) {
    return wbte_pfe_open_many(ctx, messages, first, second, third, weighted_first, weighted_pairings,
                              pre_decryption_key, neg_scaled_s1, key_lines, generator_lines, mix_lines, B, 1);
}

int32_t wbte_pfe_open_many(wbte_ctx* ctx, void* messages, const void* first, const void* second, const void* third,
                           const void* weighted_first, const void* weighted_pairings, const void* pre_decryption_key,
                           const void* neg_scaled_s1, const void* key_lines, const void* generator_lines,
                           const void* mix_lines, uint64_t B, uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!messages || !first || !second || !third || !weighted_first || !weighted_pairings || !pre_decryption_key ||
        !neg_scaled_s1 || !key_lines || !generator_lines || !mix_lines || B == 0 || K == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    const size_t LT = LINE_SZ * LINES_PER_POINT * B;
    const uint64_t n = B * K;
    uint8_t* dm = c.out(messages, GT_SZ * n);
    const uint8_t* d1 = c.in(first, G1_AFF * n);
    const uint8_t* d2 = c.in(second, G1_AFF * n);
    const uint8_t* d3 = c.in(third, GT_SZ * n);
    const uint8_t* dwf = c.in(weighted_first, G1_AFF * n);
    const uint8_t* dwp = c.in(weighted_pairings, GT_SZ * n);
    const uint8_t* dpdk = c.in(pre_decryption_key, G1_AFF * K);
    const uint8_t* ds1 = c.in(neg_scaled_s1, FR_SZ * B);
    const uint8_t* dkl = c.in(key_lines, LT);
    const uint8_t* dgl = c.in(generator_lines, LT);
    const uint8_t* dml = c.in(mix_lines, LT);
    PfeConvTables tab(B, K);
    const int64_t* doff2 = c.in_vec(tab.offs2);
    const int32_t* dslot = c.in_vec(tab.slot);
    const int32_t* dbatch = c.in_vec(tab.batch);
    uint8_t* npdk = c.alloc(G1_AFF * n);
    uint8_t* s1 = c.alloc(FR_SZ * n);
    uint8_t* pairs = c.alloc(2 * G1_AFF * n);
    uint8_t* d = c.alloc(G1_AFF * n);
    uint8_t* b1 = c.alloc(G1_AFF * n);
    uint8_t* f0 = c.alloc(GT_SZ * n);
    uint8_t* f1 = c.alloc(GT_SZ * n);
    uint8_t* f2 = c.alloc(GT_SZ * n);
    if (!c.ok()) return c.finish();
    // b1_i = weighted_first_i - 2B s1_i (second_i - pdk) (pfe/src/decryption.rs:434-447), pdk of the slot's batch
    launch_gather(npdk, dpdk, dbatch, (int64_t)n, G1_AFF, c.s);
    launch_negate(GROUP_G1, npdk, npdk, (int64_t)n, c.s);
    launch_gather(s1, ds1, dslot, (int64_t)n, FR_SZ, c.s);
    cudaMemcpy2DAsync(pairs, 2 * G1_AFF, d2, G1_AFF, G1_AFF, n, cudaMemcpyDeviceToDevice, c.s);
    cudaMemcpy2DAsync(pairs + G1_AFF, 2 * G1_AFF, npdk, G1_AFF, G1_AFF, n, cudaMemcpyDeviceToDevice, c.s);
    launch_segment_sum(GROUP_G1, d, pairs, doff2, (int64_t)n, c.s);
    launch_mul_batch(GROUP_G1, d, d, 1, s1, (int64_t)n, c.s);
    cudaMemcpy2DAsync(pairs, 2 * G1_AFF, dwf, G1_AFF, G1_AFF, n, cudaMemcpyDeviceToDevice, c.s);
    cudaMemcpy2DAsync(pairs + G1_AFF, 2 * G1_AFF, d, G1_AFF, G1_AFF, n, cudaMemcpyDeviceToDevice, c.s);
    launch_segment_sum(GROUP_G1, b1, pairs, doff2, (int64_t)n, c.s);
    // mask_i = e(second_i, [s2]) e(b1_i, DK_i/(2B)) e(first_i, mix_i) / weighted_pairings_i (:449-465)
    launch_miller_lines(f0, dgl, d2, (int64_t)n, c.s, (int64_t)B);
    launch_miller_lines(f1, dkl, b1, (int64_t)n, c.s, (int64_t)B);
    launch_miller_lines(f2, dml, d1, (int64_t)n, c.s, (int64_t)B);
    launch_fp12_mul(f0, f0, 1, f1, 1, false, (int64_t)n, c.s);
    launch_fp12_mul(f0, f0, 1, f2, 1, false, (int64_t)n, c.s);
    launch_final_exp(f0, f0, (int64_t)n, FE_FULL, c.s);
    launch_fp12_mul(f0, f0, 1, dwp, 1, true, (int64_t)n, c.s);
    launch_fp12_mul(dm, d3, 1, f0, 1, true, (int64_t)n, c.s);
    return c.finish();
}

// ------------------------------------------- weighted_btx, K batches per call
// The batched form: K batches of the same size B and the same accepted
// committee go through each phase in one launch sequence, so every kernel
// sees K times the work of one batch.  Arrays are batch-major (batch q first).
int32_t wbte_wbtx_partial_decrypt_many(wbte_ctx* ctx, void* sigma, const void* first, uint64_t B, const void* q,
                                       uint64_t T, uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (T == 0 || K == 0) return c.finish();
    if (!sigma || !first || !q || B == 0) return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    uint8_t* dsig = c.out(sigma, G1_AFF * T * K);
    const uint8_t* dfirst = c.in(first, G1_AFF * B * K);
    const uint8_t* dq = c.in(q, FR_SZ * T);
    uint8_t* scalars = c.alloc(FR_SZ * T * B);
    std::vector<int64_t> base(T * K);
    std::vector<int32_t> vsel(T * K);
    for (uint64_t b = 0; b < K; b++)
        for (uint64_t j = 0; j < T; j++) {
            base[b * T + j] = (int64_t)(b * B);
            vsel[b * T + j] = (int32_t)j;
        }
    const int64_t* db = c.in_vec(base);
    const int32_t* dv = c.in_vec(vsel);
    if (!c.ok()) return c.finish();
    // sigma[b T + j] = sum_i q_j^(i+1) first[b B + i] (weighted_btx/src/decryption.rs:205-233)
    for (uint64_t j = 0; j < T; j++) launch_fr_powers(scalars + FR_SZ * B * j, dq + FR_SZ * j, (int64_t)B, 1, c.s);
    launch_msm_family(GROUP_G1, dsig, dfirst, db, nullptr, scalars, dv, (int32_t)T, (int64_t)(T * K), (int64_t)B, c.s);
    return c.finish();
}

int32_t wbte_wbtx_vk_tables(wbte_ctx* ctx, void* tables, const wbte_wbtx_key* key, const int64_t* party_indices,
                            uint64_t T, uint64_t B) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (check_key(c, key)) return c.finish();
    if (T == 0 || B == 0) return c.finish();
    if (!tables || !party_indices) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    if (B > key->max_batch_size) return c.fail(WBTE_ERR_SIZE, "batch size out of range");
    const uint64_t N = key->party_count;
    std::vector<int64_t> idx(T * B);
    for (uint64_t t = 0; t < T; t++) {
        if (party_indices[t] < 0 || (uint64_t)party_indices[t] >= N) return c.fail(WBTE_ERR_INVALID_ARG, "invalid party index");
        for (uint64_t i = 0; i < B; i++) idx[t * B + i] = (int64_t)(i * N) + party_indices[t];
    }
    uint8_t* d = c.out(tables, FIXED_TABLE_BYTES * T * B);
    const uint8_t* dvk = c.in(key->verification_keys, G2_AFF * key->max_batch_size * N);
    const int64_t* didx = c.in_vec(idx);
    if (c.ok()) launch_fixed_tables_g2(d, dvk, didx, (int64_t)(T * B), c.s);
    return c.finish();
}

int32_t wbte_wbtx_verify_shares_many(wbte_ctx* ctx, int32_t* ok, const wbte_wbtx_key* key, const void* first, uint64_t B,
                                     const void* sigma, const int64_t* party_indices, const void* challenges,
                                     uint64_t T, uint64_t K, const void* vk_tables) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!ok) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    for (uint64_t b = 0; b < K; b++) ok[b] = 0;
    if (check_key(c, key)) return c.finish();
    if (K == 0) return c.finish();
    if (T == 0) {
        for (uint64_t b = 0; b < K; b++) ok[b] = 1;
        return c.finish();
    }
    if (!first || !sigma || !party_indices || !challenges) return c.fail(WBTE_ERR_INVALID_ARG, "null argument");
    if (B == 0 || B > key->max_batch_size) return c.fail(WBTE_ERR_SIZE, "batch size out of range");
    const uint64_t N = key->party_count, P1 = B + 1;
    std::vector<int32_t> pidx(T);
    for (uint64_t j = 0; j < T; j++) {
        if (party_indices[j] < 0 || (uint64_t)party_indices[j] >= N) return c.fail(WBTE_ERR_INVALID_ARG, "invalid party index");
        pidx[j] = (int32_t)party_indices[j];
    }
    // first carries the identity at invalid slots, whose pairings are 1, so
    // every slot enters the product (weighted_btx/src/decryption.rs:358-422)
    const uint8_t* dfirst = c.in(first, G1_AFF * B * K);
    const uint8_t* dsig = c.in(sigma, G1_AFF * T * K);
    const uint8_t* dch = c.in(challenges, FR_SZ * T * K);
    const uint8_t* dvk = c.in(key->verification_keys, G2_AFF * key->max_batch_size * N);
    uint8_t* agg = c.alloc(G1_AFF * K);
    uint8_t* aggvk = c.alloc(G2_AFF * B * K);
    uint8_t* P = c.alloc(G1_AFF * P1 * K);
    uint8_t* Q = c.alloc(G2_AFF * P1 * K);
    uint8_t* f = c.alloc(GT_SZ * P1 * K);
    uint8_t* prod = c.alloc(GT_SZ * K);
    uint8_t* flags = c.alloc(K);
    std::vector<int64_t> sbase(K), vbase(B * K);
    std::vector<int32_t> svsel(K), vvsel(B * K), gidx(K, 0);
    for (uint64_t b = 0; b < K; b++) {
        sbase[b] = (int64_t)(b * T);
        svsel[b] = (int32_t)b;
        for (uint64_t i = 0; i < B; i++) {
            vbase[b * B + i] = (int64_t)(i * N);
            vvsel[b * B + i] = (int32_t)b;
        }
    }
    const int64_t* dsbase = c.in_vec(sbase);
    const int32_t* dsvsel = c.in_vec(svsel);
    const int64_t* dvbase = c.in_vec(vbase);
    const int32_t* dvvsel = c.in_vec(vvsel);
    const int32_t* dpidx = c.in_vec(pidx);
    const int32_t* dgidx = c.in_vec(gidx);
    uint8_t* g2 = g2_generator_dev(c);
    if (!c.ok()) return c.finish();
    launch_msm_family(GROUP_G1, agg, dsig, dsbase, nullptr, dch, dsvsel, (int32_t)K, (int64_t)K, (int64_t)T, c.s);
    launch_negate(GROUP_G1, agg, agg, (int64_t)K, c.s);
    if (vk_tables) {
        // the committee's fixed-base tables: table t B + i holds party t's key at slot i
        std::vector<int64_t> tbase(B * K);
        std::vector<int32_t> tidx(T);
        for (uint64_t b = 0; b < K; b++)
            for (uint64_t i = 0; i < B; i++) tbase[b * B + i] = (int64_t)i;
        for (uint64_t t = 0; t < T; t++) tidx[t] = (int32_t)(t * B);
        const uint8_t* dtab = c.in(vk_tables, FIXED_TABLE_BYTES * T * B);
        const int64_t* dtbase = c.in_vec(tbase);
        const int32_t* dtidx = c.in_vec(tidx);
        if (!c.ok()) return c.finish();
        launch_fixed_msm_g2(aggvk, dtab, dtbase, dtidx, dch, dvvsel, (int64_t)(B * K), (int64_t)T, c.s);
    } else {
        launch_msm_family(GROUP_G2, aggvk, dvk, dvbase, dpidx, dch, dvvsel, (int32_t)K, (int64_t)(B * K), (int64_t)T, c.s);
    }
    cudaMemcpy2DAsync(P, G1_AFF * P1, dfirst, G1_AFF * B, G1_AFF * B, K, cudaMemcpyDeviceToDevice, c.s);
    cudaMemcpy2DAsync(P + G1_AFF * B, G1_AFF * P1, agg, G1_AFF, G1_AFF, K, cudaMemcpyDeviceToDevice, c.s);
    cudaMemcpy2DAsync(Q, G2_AFF * P1, aggvk, G2_AFF * B, G2_AFF * B, K, cudaMemcpyDeviceToDevice, c.s);
    uint8_t* gcol = c.alloc(G2_AFF * K);
    if (!c.ok()) return c.finish();
    launch_gather(gcol, g2, dgidx, (int64_t)K, G2_AFF, c.s);
    cudaMemcpy2DAsync(Q + G2_AFF * B, G2_AFF * P1, gcol, G2_AFF, G2_AFF, K, cudaMemcpyDeviceToDevice, c.s);
    const int64_t runs = launch_miller_chunks(f, P, Q, (int64_t)P1, (int64_t)K, miller_chunk((int64_t)(P1 * K)), c.s);
    fp12_segments_product(c, prod, f, runs, (int64_t)K);
    launch_final_exp(prod, prod, (int64_t)K, FE_FULL, c.s);
    launch_fp12_is_one(flags, prod, (int64_t)K, c.s);
    std::vector<uint8_t> h(K);
    if (c.to_host(h.data(), flags, K))
        for (uint64_t b = 0; b < K; b++) ok[b] = h[b] ? 1 : 0;
    return c.finish();
}

int32_t wbte_wbtx_precompute_many(wbte_ctx* ctx, void* beta, const void* kernel_lines, const void* first,
                                  const uint8_t* valid, uint64_t B, uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!beta || !kernel_lines || !first || !valid || B == 0 || K == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    const uint64_t m = next_pow2(2 * B);
    uint8_t* dbeta = c.out(beta, GT_SZ * B * K);
    const uint8_t* dl = c.in(kernel_lines, LINE_SZ * LINES_PER_POINT * m);
    const uint8_t* dfirst = c.in(first, G1_AFF * B * K);
    const uint8_t* dvalid = c.in(valid, B * K);
    uint8_t* x = c.zeros(G1_AFF * m * K);
    uint8_t* work = c.alloc(G1_XYZZ * m * K);
    uint8_t* f = c.alloc(GT_SZ * m * K);
    const uint8_t* tw = twiddles(c, (int64_t)m, false);
    const uint8_t* twi = twiddles(c, (int64_t)m, true);
    if (!c.ok()) return c.finish();
    // per batch: G1 transform of the zero-padded first components, prepared
    // Miller loops against the shared kernel lines, easy part, truncated
    // cyclotomic inverse transform, hard part (weighted_btx/src/decryption.rs:555-603)
    cudaMemcpy2DAsync(x, G1_AFF * m, dfirst, G1_AFF * B, G1_AFF * B, K, cudaMemcpyDeviceToDevice, c.s);
    launch_group_ntt(GROUP_G1, x, work, tw, (int64_t)m, c.s, (int64_t)K);
    launch_miller_lines(f, dl, x, (int64_t)(m * K), c.s, (int64_t)m);
    launch_final_exp(f, f, (int64_t)(m * K), FE_EASY, c.s);
    launch_cyclotomic_prefix_ifft(f, twi, (int64_t)m, (int64_t)B, c.s, (int64_t)K);
    cudaMemcpy2DAsync(dbeta, GT_SZ * B, f, GT_SZ * m, GT_SZ * B, K, cudaMemcpyDeviceToDevice, c.s);
    launch_final_exp(dbeta, dbeta, (int64_t)(B * K), FE_HARD, c.s);
    launch_fp12_mask(dbeta, dvalid, (int64_t)(B * K), c.s);
    return c.finish();
}

// alpha[b B + i] = prod_t Miller(sigma[b T + t], opening_keys[i T + t]) before
// the final exponentiation (weighted_btx/src/decryption.rs:607-695): one
// multi-Miller loop per slot over the prepared opening keys when their line
// tables are given, else T unprepared loops and their product
static bool opening_miller(Call& c, uint8_t* alpha, const uint8_t* dk, const void* opening_lines, const uint8_t* ds,
                           uint64_t T, uint64_t B, uint64_t K) {
    const uint64_t BT = B * T;
    if (opening_lines) {
        const uint8_t* dl = c.in(opening_lines, LINE_SZ * LINES_PER_POINT * BT);
        if (!c.ok()) return false;
        launch_miller_lines_multi(alpha, dl, ds, (int64_t)(B * K), (int64_t)B, (int)T, c.s);
        return true;
    }
    uint8_t* P = c.alloc(G1_AFF * BT * K);
    uint8_t* f = c.alloc(GT_SZ * BT * K);
    std::vector<int32_t> pidx(BT * K);
    for (uint64_t b = 0; b < K; b++)
        for (uint64_t x = 0; x < BT; x++) pidx[b * BT + x] = (int32_t)(b * T + x % T);
    std::vector<int64_t> offs(B * K + 1);
    for (uint64_t i = 0; i <= B * K; i++) offs[i] = (int64_t)(i * T);
    const int32_t* dpidx = c.in_vec(pidx);
    const int64_t* doffs = c.in_vec(offs);
    if (!c.ok()) return false;
    launch_gather(P, ds, dpidx, (int64_t)(BT * K), G1_AFF, c.s);
    launch_miller(f, P, dk, (int64_t)(BT * K), c.s, 0, (int64_t)BT);
    launch_fp12_segment_product(alpha, f, doffs, (int64_t)(B * K), c.s);
    return true;
}

int32_t wbte_wbtx_open_many(wbte_ctx* ctx, void* messages, const void* opening_keys, const void* opening_lines,
                            const void* sigma, uint64_t T, const void* second, const void* beta, const uint8_t* valid,
                            uint64_t B, uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!messages || !opening_keys || !sigma || !second || !beta || !valid || B == 0 || T == 0 || K == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    uint8_t* dm = c.out(messages, GT_SZ * B * K);
    const uint8_t* dk = c.in(opening_keys, G2_AFF * B * T);
    const uint8_t* ds = c.in(sigma, G1_AFF * T * K);
    const uint8_t* d2 = c.in(second, GT_SZ * B * K);
    const uint8_t* db = c.in(beta, GT_SZ * B * K);
    const uint8_t* dv = c.in(valid, B * K);
    uint8_t* alpha = c.alloc(GT_SZ * B * K);
    if (!c.ok() || !opening_miller(c, alpha, dk, opening_lines, ds, T, B, K)) return c.finish();
    launch_final_exp(alpha, alpha, (int64_t)(B * K), FE_FULL, c.s);
    launch_unmask(dm, d2, alpha, db, dv, (int64_t)(B * K), c.s);
    return c.finish();
}

int32_t wbte_wbtx_decrypt_many(wbte_ctx* ctx, void* messages, const void* kernel_lines, const void* opening_keys,
                               const void* opening_lines, const void* first, const void* second, const uint8_t* valid,
                               const void* sigma, uint64_t T, uint64_t B, uint64_t K) {
    if (!ctx) return WBTE_ERR_INVALID_ARG;
    Call c(ctx);
    if (!messages || !kernel_lines || !opening_keys || !first || !second || !valid || !sigma || B == 0 || T == 0 ||
        K == 0)
        return c.fail(WBTE_ERR_INVALID_ARG, "null argument or empty batch");
    const uint64_t m = next_pow2(2 * B), n = B * K;
    uint8_t* dm = c.out(messages, GT_SZ * n);
    const uint8_t* dl = c.in(kernel_lines, LINE_SZ * LINES_PER_POINT * m);
    const uint8_t* dk = c.in(opening_keys, G2_AFF * B * T);
    const uint8_t* dfirst = c.in(first, G1_AFF * n);
    const uint8_t* d2 = c.in(second, GT_SZ * n);
    const uint8_t* dv = c.in(valid, n);
    const uint8_t* ds = c.in(sigma, G1_AFF * T * K);
    uint8_t* x = c.zeros(G1_AFF * m * K);
    uint8_t* work = c.alloc(G1_XYZZ * m * K);
    uint8_t* f = c.alloc(GT_SZ * m * K);
    uint8_t* y = c.alloc(GT_SZ * n);
    uint8_t* alpha = c.alloc(GT_SZ * n);
    const uint8_t* tw = twiddles(c, (int64_t)m, false);
    const uint8_t* twi = twiddles(c, (int64_t)m, true);
    if (!c.ok()) return c.finish();
    // the cross terms up to the truncated cyclotomic transform, as precompute
    cudaMemcpy2DAsync(x, G1_AFF * m, dfirst, G1_AFF * B, G1_AFF * B, K, cudaMemcpyDeviceToDevice, c.s);
    launch_group_ntt(GROUP_G1, x, work, tw, (int64_t)m, c.s, (int64_t)K);
    launch_miller_lines(f, dl, x, (int64_t)(m * K), c.s, (int64_t)m);
    launch_final_exp(f, f, (int64_t)(m * K), FE_EASY, c.s);
    launch_cyclotomic_prefix_ifft(f, twi, (int64_t)m, (int64_t)B, c.s, (int64_t)K);
    // the opening's pairings up to their easy part
    if (!opening_miller(c, alpha, dk, opening_lines, ds, T, B, K)) return c.finish();
    launch_final_exp(alpha, alpha, (int64_t)n, FE_EASY, c.s);
    // beta / alpha = hard(t) / hard(easy(a)) = hard(t conj(easy(a))): the hard
    // part is a fixed power, a homomorphism of the cyclotomic subgroup, where
    // conjugation is the inverse; one hard part per slot instead of two
    cudaMemcpy2DAsync(y, GT_SZ * B, f, GT_SZ * m, GT_SZ * B, K, cudaMemcpyDeviceToDevice, c.s);
    launch_fp12_mul(y, y, 1, alpha, 1, true, (int64_t)n, c.s);
    launch_final_exp(y, y, (int64_t)n, FE_HARD, c.s);
    // messages = second beta / alpha at valid slots, one elsewhere
    launch_fp12_mul(dm, d2, 1, y, 1, false, (int64_t)n, c.s);
    launch_fp12_mask(dm, dv, (int64_t)n, c.s);
    return c.finish();
}

}  // extern "C"
