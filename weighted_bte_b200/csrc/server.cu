// The served form in the C ABI: resident key handles (wbte_crs_upload_*) and
// a request loop (wbte_server_create, wbte_submit, wbte_poll) that decrypts
// waiting requests of one setup, batch size and committee together through
// the batched entry points (wbte_wbtx_decrypt_many, wbte_wpfe_decrypt_many).
//
// A Rust or C caller validates ciphertexts and accepts shares with the
// other ABI calls (the crates' host logic), then submits the decryption of
// the accepted batch -- precompute and open, weighted_btx/src/decryption.rs:555-695
// and weighted_pfe/src/decryption.rs:540-644 -- and polls for the messages.
//
// Worker threads each own a library context on the server's device (and so
// a CUDA stream); prepared committees (the reference's reusable
// DecryptionPrecomputation, weighted_btx/src/decryption.rs:424-426) are kept in
// HBM per (setup, batch size, accepted parties) and shared by the workers.
// Admission: a request enters a group only while the estimated device
// memory of the running groups stays within the budget.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "wbte.h"

namespace {

constexpr size_t G1B = 96, G2B = 192, GTB = 576, FRB = 32, LINES = 68 * 288;

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    bool alloc(size_t bytes) {
        n = bytes ? bytes : 16;
        if (cudaMalloc(&p, n) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            return false;
        }
        return true;
    }
    // copy from host or device memory (unified addressing)
    bool load(const void* src, size_t bytes) {
        if (!alloc(bytes)) return false;
        if (!src || bytes == 0) return true;
        return cudaMemcpy(p, src, bytes, cudaMemcpyDefault) == cudaSuccess;
    }
};

}  // namespace

struct wbte_crs {
    int32_t scheme = 0;
    int32_t device = 0;
    uint64_t batch_size = 0;  // weighted_btx: the maximum batch size; weighted_pfe: the class size
    std::vector<int64_t> offsets;
    DevBuf domain, vk, m1, m2, global, mask_scalars;
    wbte_wbtx_key wk{};
    wbte_wpfe_key pk{};
};

namespace {

struct Request {
    uint64_t ticket = 0;
    const wbte_crs* crs = nullptr;
    uint64_t B = 0, T = 0;
    std::vector<uint8_t> first, second, valid, sigma;
    std::vector<int64_t> parties;
    void* messages = nullptr;
    size_t need = 0;
    bool done = false;
    int32_t status = WBTE_OK;
};

using Key = std::tuple<const wbte_crs*, uint64_t, std::vector<int64_t>>;

struct Committee {
    bool ready = false;
    int32_t status = WBTE_OK;
    DevBuf a, b, c, d;  // weighted_btx: kernel lines, opening keys, opening lines; weighted_pfe: by_party,
                        // total lines, mask lines, by_party lines
};

size_t request_bytes(const wbte_crs* crs, uint64_t B, uint64_t T) {
    if (crs->scheme == WBTE_SCHEME_WBTX) {
        uint64_t m = 1;
        while (m < 2 * B) m <<= 1;
        return B * (G1B + GTB + 1) + m * (3 * G1B + GTB) + B * GTB * 3 + T * G1B + (1u << 20);
    }
    return B * (6400 + 480 * T) + (1u << 20);
}

size_t committee_bytes(const wbte_crs* crs, uint64_t B, uint64_t T) {
    if (crs->scheme == WBTE_SCHEME_WBTX) {
        uint64_t m = 1;
        while (m < 2 * B) m <<= 1;
        return m * LINES + B * T * (G2B + LINES) + m * G2B * 4;
    }
    return B * T * (G2B + LINES + 64 * G2B) + 2 * B * LINES;
}

}  // namespace

struct wbte_server {
    int32_t device = 0;
    uint32_t max_group = 1;
    uint64_t budget = 0, in_use = 0, next_ticket = 1;
    bool closing = false;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Request*> queue;
    std::map<uint64_t, std::unique_ptr<Request>> tickets;
    std::map<Key, std::shared_ptr<Committee>> committees;
    std::vector<std::thread> workers;

    void work();
    std::shared_ptr<Committee> committee(wbte_ctx* ctx, const Request& r);
    void run_group(wbte_ctx* ctx, std::vector<Request*>& group);
};

std::shared_ptr<Committee> wbte_server::committee(wbte_ctx* ctx, const Request& r) {
    Key key{r.crs, r.B, r.parties};
    std::shared_ptr<Committee> cm;
    bool owner = false;
    {
        std::unique_lock<std::mutex> lk(mu);
        auto it = committees.find(key);
        if (it == committees.end()) {
            cm = std::make_shared<Committee>();
            committees[key] = cm;
            owner = true;
        } else {
            cm = it->second;
            cv.wait(lk, [&] { return cm->ready; });
        }
    }
    if (!owner) return cm;
    // prepared on this worker's stream and completed before other workers
    // (on their own streams) may read it
    int32_t st = WBTE_OK;
    const uint64_t B = r.B, T = r.T;
    if (r.crs->scheme == WBTE_SCHEME_WBTX) {
        uint64_t m = 1;
        while (m < 2 * B) m <<= 1;
        if (!cm->a.alloc(LINES * m) || !cm->b.alloc(G2B * B * T) || !cm->c.alloc(LINES * B * T)) {
            st = WBTE_ERR_OOM;
        } else {
            st = wbte_wbtx_prepare(ctx, &r.crs->wk, r.parties.data(), T, B, cm->a.p, cm->b.p, nullptr);
            if (st == WBTE_OK) st = wbte_g2_prepare_lines(ctx, cm->c.p, cm->b.p, B * T);
        }
    } else {
        if (!cm->a.alloc(G2B * B * T) || !cm->b.alloc(LINES * B) || !cm->c.alloc(LINES * B) ||
            !cm->d.alloc(LINES * B * T)) {
            st = WBTE_ERR_OOM;
        } else {
            st = wbte_wpfe_prepare(ctx, &r.crs->pk, r.parties.data(), T, r.crs->mask_scalars.p, cm->a.p, cm->b.p,
                                   cm->c.p, nullptr, nullptr);
            if (st == WBTE_OK) st = wbte_g2_prepare_lines(ctx, cm->d.p, cm->a.p, B * T);
        }
    }
    if (st == WBTE_OK) st = wbte_ctx_synchronize(ctx);
    {
        std::lock_guard<std::mutex> lk(mu);
        cm->status = st;
        cm->ready = true;
        if (st != WBTE_OK) committees.erase(key);
    }
    cv.notify_all();
    return cm;
}

void wbte_server::run_group(wbte_ctx* ctx, std::vector<Request*>& group) {
    Request& h = *group[0];
    const uint64_t B = h.B, T = h.T, K = group.size();
    std::shared_ptr<Committee> cm = committee(ctx, h);
    int32_t st = cm->status;
    std::vector<uint8_t> first, second, valid, sigma, out;
    if (st == WBTE_OK) {
        first.reserve(G1B * B * K);
        second.reserve(GTB * B * K);
        sigma.reserve(G1B * T * K);
        for (Request* r : group) {
            first.insert(first.end(), r->first.begin(), r->first.end());
            second.insert(second.end(), r->second.begin(), r->second.end());
            sigma.insert(sigma.end(), r->sigma.begin(), r->sigma.end());
            valid.insert(valid.end(), r->valid.begin(), r->valid.end());
        }
        out.resize(GTB * B * K);
        if (h.crs->scheme == WBTE_SCHEME_WBTX)
            st = wbte_wbtx_decrypt_many(ctx, out.data(), cm->a.p, cm->b.p, cm->c.p, first.data(), second.data(),
                                        valid.data(), sigma.data(), T, B, K);
        else
            st = wbte_wpfe_decrypt_many(ctx, out.data(), sigma.data(), T, cm->a.p, cm->d.p, cm->b.p, cm->c.p,
                                        first.data(), second.data(), h.crs->mask_scalars.p, B, K);
    }
    for (uint64_t q = 0; q < K; q++) {
        Request* r = group[q];
        if (st == WBTE_OK) memcpy(r->messages, out.data() + GTB * B * q, GTB * B);
        r->status = st;
    }
}

void wbte_server::work() {
    wbte_ctx* ctx = nullptr;
    int32_t cst = wbte_ctx_create(device, 0, &ctx);
    while (true) {
        std::vector<Request*> group;
        {
            std::unique_lock<std::mutex> lk(mu);
            // the head request fits the budget (or nothing else runs), or the
            // server is closing with nothing left to do
            cv.wait(lk, [&] {
                return (!queue.empty() && (in_use == 0 || in_use + queue.front()->need <= budget)) ||
                       (closing && queue.empty());
            });
            if (queue.empty()) break;
            // the head and the waiting requests of the same setup, batch size
            // and committee, in arrival order, within the budget
            Request* head = queue.front();
            queue.pop_front();
            group.push_back(head);
            in_use += head->need;
            for (auto it = queue.begin(); it != queue.end() && group.size() < max_group;) {
                Request* r = *it;
                if (r->crs == head->crs && r->B == head->B && r->parties == head->parties &&
                    in_use + r->need <= budget) {
                    group.push_back(r);
                    in_use += r->need;
                    it = queue.erase(it);
                } else {
                    ++it;
                }
            }
        }
        if (cst != WBTE_OK) {
            for (Request* r : group) r->status = cst;
        } else {
            run_group(ctx, group);
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            for (Request* r : group) {
                in_use -= r->need;
                r->done = true;
            }
        }
        cv.notify_all();
    }
    if (ctx) wbte_ctx_destroy(ctx);
}

extern "C" {

int32_t wbte_crs_upload_wbtx(wbte_ctx* ctx, const wbte_wbtx_key* key, wbte_crs** out) {
    if (!ctx || !key || !out || !key->party_offsets || key->party_count == 0 || key->max_batch_size == 0)
        return WBTE_ERR_INVALID_ARG;
    *out = nullptr;
    if ((uint64_t)key->party_offsets[key->party_count] != key->total_weight) return WBTE_ERR_INVALID_ARG;
    int dev = 0;
    cudaGetDevice(&dev);
    auto c = std::make_unique<wbte_crs>();
    c->scheme = WBTE_SCHEME_WBTX;
    c->device = dev;
    c->batch_size = key->max_batch_size;
    const uint64_t L = key->max_batch_size, N = key->party_count, W = key->total_weight;
    c->offsets.assign(key->party_offsets, key->party_offsets + N + 1);
    if (!c->domain.load(key->domain_points, FRB * W) || !c->vk.load(key->verification_keys, G2B * L * N) ||
        !c->m1.load(key->negative_material, G2B * L * W) ||
        !c->m2.load(key->positive_material, G2B * (L > 1 ? L - 1 : 0) * W))
        return WBTE_ERR_OOM;
    c->wk = *key;
    c->wk.domain_points = c->domain.p;
    c->wk.verification_keys = c->vk.p;
    c->wk.negative_material = c->m1.p;
    c->wk.positive_material = c->m2.p;
    c->wk.party_offsets = c->offsets.data();
    *out = c.release();
    return WBTE_OK;
}

int32_t wbte_crs_upload_wpfe(wbte_ctx* ctx, const wbte_wpfe_key* key, const void* mask_scalars, wbte_crs** out) {
    if (!ctx || !key || !mask_scalars || !out || !key->party_offsets || key->party_count == 0 ||
        key->batch_size == 0)
        return WBTE_ERR_INVALID_ARG;
    *out = nullptr;
    if ((uint64_t)key->party_offsets[key->party_count] != key->total_weight) return WBTE_ERR_INVALID_ARG;
    if (key->batch_size & (key->batch_size - 1)) return WBTE_ERR_SIZE;
    int dev = 0;
    cudaGetDevice(&dev);
    auto c = std::make_unique<wbte_crs>();
    c->scheme = WBTE_SCHEME_WPFE;
    c->device = dev;
    c->batch_size = key->batch_size;
    const uint64_t B = key->batch_size, N = key->party_count, W = key->total_weight;
    c->offsets.assign(key->party_offsets, key->party_offsets + N + 1);
    if (!c->domain.load(key->domain_points, FRB * W) || !c->vk.load(key->verification_keys, G2B * B * N) ||
        !c->m1.load(key->d1, G2B * B * W) || !c->m2.load(key->d2, G2B * B * W) ||
        !c->global.load(key->global_key, G2B) || !c->mask_scalars.load(mask_scalars, 2 * FRB * B))
        return WBTE_ERR_OOM;
    c->pk = *key;
    c->pk.domain_points = c->domain.p;
    c->pk.verification_keys = c->vk.p;
    c->pk.d1 = c->m1.p;
    c->pk.d2 = c->m2.p;
    c->pk.global_key = c->global.p;
    c->pk.party_offsets = c->offsets.data();
    *out = c.release();
    return WBTE_OK;
}

int32_t wbte_crs_destroy(wbte_crs* crs) {
    if (!crs) return WBTE_ERR_INVALID_ARG;
    cudaSetDevice(crs->device);
    delete crs;
    return WBTE_OK;
}

int32_t wbte_server_create(int32_t device, uint32_t slots, uint32_t max_group, uint64_t hbm_budget_bytes,
                           wbte_server** out) {
    if (!out || slots == 0 || max_group == 0) return WBTE_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return WBTE_ERR_CUDA;
    }
    auto s = std::make_unique<wbte_server>();
    s->device = device;
    s->max_group = max_group;
    if (hbm_budget_bytes == 0) {
        size_t fr = 0, total = 0;
        cudaSetDevice(device);
        if (cudaMemGetInfo(&fr, &total) != cudaSuccess) return WBTE_ERR_CUDA;
        hbm_budget_bytes = fr / 2;
    }
    s->budget = hbm_budget_bytes;
    wbte_server* raw = s.release();
    for (uint32_t i = 0; i < slots; i++) raw->workers.emplace_back([raw] { raw->work(); });
    *out = raw;
    return WBTE_OK;
}

int32_t wbte_submit(wbte_server* srv, const wbte_request* req, uint64_t* ticket) {
    if (!srv || !req || !ticket || !req->crs || !req->first || !req->second || !req->sigma || !req->party_indices ||
        !req->messages || req->batch_size == 0 || req->party_count == 0)
        return WBTE_ERR_INVALID_ARG;
    const wbte_crs* crs = req->crs;
    const uint64_t B = req->batch_size, T = req->party_count;
    if (crs->scheme == WBTE_SCHEME_WBTX && B > crs->batch_size) return WBTE_ERR_SIZE;
    if (crs->scheme == WBTE_SCHEME_WPFE && B != crs->batch_size) return WBTE_ERR_SIZE;
    const uint64_t N = crs->scheme == WBTE_SCHEME_WBTX ? crs->wk.party_count : crs->pk.party_count;
    for (uint64_t k = 0; k < T; k++) {
        if (req->party_indices[k] < 0 || (uint64_t)req->party_indices[k] >= N) return WBTE_ERR_INVALID_ARG;
        if (k && req->party_indices[k - 1] >= req->party_indices[k]) return WBTE_ERR_INVALID_ARG;
    }
    auto r = std::make_unique<Request>();
    r->crs = crs;
    r->B = B;
    r->T = T;
    r->messages = req->messages;
    r->parties.assign(req->party_indices, req->party_indices + T);
    r->need = request_bytes(crs, B, T) + committee_bytes(crs, B, T);
    if (r->need > srv->budget) return WBTE_ERR_OOM;
    r->first.resize(G1B * B);
    r->second.resize(GTB * B);
    r->sigma.resize(G1B * T);
    if (cudaMemcpy(r->first.data(), req->first, G1B * B, cudaMemcpyDefault) != cudaSuccess ||
        cudaMemcpy(r->second.data(), req->second, GTB * B, cudaMemcpyDefault) != cudaSuccess ||
        cudaMemcpy(r->sigma.data(), req->sigma, G1B * T, cudaMemcpyDefault) != cudaSuccess) {
        cudaGetLastError();
        return WBTE_ERR_CUDA;
    }
    if (crs->scheme == WBTE_SCHEME_WBTX) {
        r->valid.assign(B, 1);
        if (req->valid && cudaMemcpy(r->valid.data(), req->valid, B, cudaMemcpyDefault) != cudaSuccess) {
            cudaGetLastError();
            return WBTE_ERR_CUDA;
        }
    }
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->closing) return WBTE_ERR_INVALID_ARG;
    r->ticket = srv->next_ticket++;
    *ticket = r->ticket;
    srv->queue.push_back(r.get());
    srv->tickets[r->ticket] = std::move(r);
    srv->cv.notify_all();
    return WBTE_OK;
}

int32_t wbte_poll(wbte_server* srv, uint64_t ticket, uint64_t timeout_ns, int32_t* status) {
    if (!srv || !status) return WBTE_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->tickets.find(ticket);
    if (it == srv->tickets.end()) return WBTE_ERR_INVALID_ARG;
    Request* r = it->second.get();
    if (!srv->cv.wait_for(lk, std::chrono::nanoseconds(timeout_ns), [&] { return r->done; }))
        return WBTE_ERR_TIMEOUT;
    *status = r->status;
    srv->tickets.erase(ticket);
    return WBTE_OK;
}

int32_t wbte_server_destroy(wbte_server* srv) {
    if (!srv) return WBTE_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->closing = true;
    }
    srv->cv.notify_all();
    for (auto& t : srv->workers) t.join();
    cudaSetDevice(srv->device);
    delete srv;
    return WBTE_OK;
}

}  // extern "C"
