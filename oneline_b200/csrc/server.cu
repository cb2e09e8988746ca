// A serving loop for parse and search requests of mixed sizes (no reference
// counterpart: the reference exposes one blocking call per document,
// crates/oneline-gpu/src/parser.rs). Requests are queued as they arrive and
// taken by worker threads, each with its own context and CUDA stream, so
// requests that arrive while others run are admitted as soon as a worker frees
// up and their kernels overlap on the device. Parsed documents (text, line
// arrays, tree links) stay resident in a store bounded by an HBM budget: a new
// document evicts the least recently used idle ones, and is refused
// (OL_ERR_ADMISSION) when the documents in use leave no room. Search requests
// name a resident document and never upload text again.
//
// Every result carries a digest of its outputs computed on the device (offsets,
// kinds and the four tree arrays of a parse; counts and hits of a search), so a
// result computed in a busy server can be compared with the same request run
// alone.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "runtime.h"

using namespace ol;

namespace {

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Request {
    uint64_t id = 0;
    uint32_t kind = 0;  // 0 parse, 1 search
    const uint8_t *text = nullptr;
    uint64_t len = 0;
    uint64_t doc_id = 0;
    std::vector<std::string> patterns;
    uint64_t submit_ns = 0;
};

struct Entry {
    ol_doc *doc = nullptr;
    ol_tree *tree = nullptr;
    uint64_t bytes = 0;
    uint32_t refs = 0;
    uint64_t last_use = 0;
};

}  // namespace

struct ol_server {
    int device = 0;
    uint32_t n_workers = 0;
    uint64_t budget = 0;
    uint64_t max_hits = 0;
    std::vector<ol_ctx *> ctxs;
    std::vector<std::thread> threads;
    std::mutex qmu;
    std::condition_variable qcv;
    std::deque<Request *> queue;
    bool stopping = false;
    std::mutex rmu;
    std::condition_variable rcv;
    std::unordered_map<uint64_t, ol_request_result> results;
    std::atomic<uint64_t> next_id{1}, next_doc{1};
    std::mutex smu;
    std::unordered_map<uint64_t, Entry> store;
    uint64_t used = 0, tick = 0;
    std::atomic<uint64_t> evictions{0}, refusals{0};
};

namespace {

uint64_t resident_bytes(const ol_doc *d) {
    const uint64_t text = d->text_len ? (uint64_t)d->text_buf.bytes : 0;
    return text + (uint64_t)d->line_cap * 6 + (uint64_t)d->line_count * 16;  // offsets, kinds, depth8; tree
}

// Takes idle documents out of the store, least recently used first, until
// `need` more bytes fit; the caller frees them after releasing smu (freeing
// takes the owning context's lock, which a worker may hold while it waits for
// smu). Called with smu held; returns false when the documents in use leave no
// room.
bool make_room(ol_server *s, uint64_t need, std::vector<Entry> &evicted) {
    uint64_t busy = 0;  // documents in use cannot go: refuse before evicting anything
    for (auto &kv : s->store)
        if (kv.second.refs) busy += kv.second.bytes;
    if (busy + need > s->budget) return false;
    while (s->used + need > s->budget) {
        uint64_t victim = 0, best = UINT64_MAX;
        for (auto &kv : s->store)
            if (kv.second.refs == 0 && kv.second.last_use < best) {
                best = kv.second.last_use;
                victim = kv.first;
            }
        if (!victim) return false;
        evicted.push_back(s->store[victim]);
        s->store.erase(victim);
        s->used -= evicted.back().bytes;
        s->evictions++;
    }
    return true;
}

void free_entries(std::vector<Entry> &v) {
    for (auto &e : v) {
        ol_tree_free(e.tree);
        ol_doc_free(e.doc);
    }
    v.clear();
}

void run_parse(ol_server *s, ol_ctx *ctx, unsigned long long *d_digest, Request *r, ol_request_result &res) {
    ol_doc *d = nullptr;
    ol_tree *t = nullptr;
    ol_status st = ol_doc_upload(ctx, r->text, r->len, &d);
    if (st == OL_OK) st = ol_tree_build(ctx, d, 0, &t);  // any depth
    if (st == OL_OK) {
        const uint32_t L = d->line_count;
        cudaStream_t cs = ctx->stream;
        unsigned long long h = 0;
        cudaError_t e = cudaMemsetAsync(d_digest, 0, 8, cs);
        if (e == cudaSuccess && L) e = launch_digest_u32(d->offsets, L, 1, d_digest, cs);
        if (e == cudaSuccess && L) e = launch_digest_u8(d->kinds, L, 2, d_digest, cs);
        const void *arr[4] = {t->parent_buf.ptr, t->end_buf.ptr, t->fc_buf.ptr, t->ns_buf.ptr};
        for (uint32_t k = 0; k < 4 && e == cudaSuccess && L; k++)
            e = launch_digest_u32((const uint32_t *)arr[k], L, 3 + k, d_digest, cs);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d_digest, 8, cudaMemcpyDeviceToHost, cs);
        if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
        if (e != cudaSuccess) st = ctx_cuda(ctx, e, "digest");
        res.digest = h ^ ((uint64_t)L * 0x9E3779B97F4A7C15ull);
        res.line_count = L;
    }
    std::vector<Entry> evicted;
    if (st == OL_OK) {
        const uint64_t bytes = resident_bytes(d);
        std::lock_guard<std::mutex> g(s->smu);
        if (!make_room(s, bytes, evicted)) {
            st = OL_ERR_ADMISSION;
            s->refusals++;
        } else {
            Entry e;
            e.doc = d;
            e.tree = t;
            e.bytes = bytes;
            e.last_use = s->tick++;
            res.doc_id = s->next_doc++;
            s->store[res.doc_id] = e;
            s->used += bytes;
            d = nullptr;
            t = nullptr;
        }
    }
    free_entries(evicted);
    if (t) ol_tree_free(t);
    if (d) ol_doc_free(d);
    res.status = st;
}

void run_search(ol_server *s, ol_ctx *ctx, unsigned long long *d_digest, ol_hit *d_hits, Request *r,
                ol_request_result &res) {
    Entry e;
    {
        std::lock_guard<std::mutex> g(s->smu);
        auto it = s->store.find(r->doc_id);
        if (it == s->store.end()) {
            res.status = OL_ERR_NOT_FOUND;
            return;
        }
        it->second.refs++;
        it->second.last_use = s->tick++;
        e = it->second;
    }
    std::vector<const uint8_t *> p;
    std::vector<uint32_t> lens;
    for (auto &x : r->patterns) {
        p.push_back((const uint8_t *)x.data());
        lens.push_back((uint32_t)x.size());
    }
    ol_status st;
    {
        std::lock_guard<std::recursive_mutex> cg(ctx->mu);  // released before smu is taken again
        ol_patset *set = nullptr;
        st = ol_patset_compile(ctx, e.doc, p.data(), lens.data(), (uint32_t)p.size(), &set);
        std::vector<uint32_t> counts(p.size());
        uint64_t total = 0;
        HitDest dest;
        dest.dev = d_hits;
        if (st == OL_OK) st = many_run(ctx, e.doc, set, s->max_hits, 0, counts.data(), &total, dest, nullptr, nullptr, 0);
        if (st == OL_OK) {
            const uint64_t k = std::min<uint64_t>(total, s->max_hits);
            unsigned long long h = 0;
            cudaStream_t cs = ctx->stream;
            cudaError_t ce = cudaMemsetAsync(d_digest, 0, 8, cs);
            if (ce == cudaSuccess && k) ce = launch_digest_u32((const uint32_t *)d_hits, 2 * k, 7, d_digest, cs);
            if (ce == cudaSuccess) ce = cudaMemcpyAsync(&h, d_digest, 8, cudaMemcpyDeviceToHost, cs);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(cs);
            if (ce != cudaSuccess) st = ctx_cuda(ctx, ce, "digest");
            for (size_t i = 0; i < counts.size(); i++) h = h * 0x100000001B3ull ^ counts[i];  // counts on the host
            res.digest = h ^ total;
            res.total_hits = total;
        }
        if (set) ol_patset_free(set);
    }
    {
        std::lock_guard<std::mutex> g(s->smu);
        auto it = s->store.find(r->doc_id);
        if (it != s->store.end()) it->second.refs--;
    }
    res.doc_id = r->doc_id;
    res.status = st;
}

void worker(ol_server *s, uint32_t w) {
    ol_ctx *ctx = s->ctxs[w];
    cudaSetDevice(s->device);
    unsigned long long *d_digest = nullptr;
    ol_hit *d_hits = nullptr;
    cudaMalloc(&d_digest, 8);
    if (s->max_hits) cudaMalloc(&d_hits, s->max_hits * sizeof(ol_hit));
    for (;;) {
        Request *r = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->qmu);
            s->qcv.wait(lk, [&] { return s->stopping || !s->queue.empty(); });
            if (s->queue.empty()) break;
            r = s->queue.front();
            s->queue.pop_front();
        }
        ol_request_result res{};
        res.id = r->id;
        res.kind = r->kind;
        res.submit_ns = r->submit_ns;
        res.start_ns = now_ns();
        res.worker = w;
        if (r->kind == 0)
            run_parse(s, ctx, d_digest, r, res);
        else
            run_search(s, ctx, d_digest, d_hits, r, res);
        res.end_ns = now_ns();
        delete r;
        {
            std::lock_guard<std::mutex> g(s->rmu);
            s->results[res.id] = res;
        }
        s->rcv.notify_all();
    }
    cudaFree(d_digest);
    if (d_hits) cudaFree(d_hits);
}

ol_status submit(ol_server *s, Request *r, uint64_t *id) {
    r->id = s->next_id++;
    r->submit_ns = now_ns();
    *id = r->id;
    {
        std::lock_guard<std::mutex> g(s->qmu);
        if (s->stopping) {
            delete r;
            return OL_ERR_INVALID_ARG;
        }
        s->queue.push_back(r);
    }
    s->qcv.notify_one();
    return OL_OK;
}

}  // namespace

extern "C" ol_status ol_server_create(int32_t device, uint32_t workers, uint64_t store_budget, uint64_t max_hits,
                                      ol_server **out) {
    if (!out || workers == 0 || workers > 64) return OL_ERR_INVALID_ARG;
    *out = nullptr;
    auto s = new ol_server();
    s->device = device;
    s->n_workers = workers;
    s->budget = store_budget;
    s->max_hits = max_hits;
    for (uint32_t w = 0; w < workers; w++) {
        ol_ctx *c = nullptr;
        ol_status st = ol_ctx_create(device, &c);
        if (st != OL_OK) {
            for (ol_ctx *x : s->ctxs) ol_ctx_destroy(x);
            delete s;
            return st;
        }
        s->ctxs.push_back(c);
    }
    // Grow the device's memory pool once, up front: the resident store and the
    // workers' scratch are then carved from memory the pool already holds (its
    // release threshold keeps freed memory), instead of growing it while
    // requests wait.
    {
        void *p = nullptr;
        const size_t warm = store_budget + (size_t)workers * (512ull << 20);
        cudaStream_t st = s->ctxs[0]->stream;
        cudaSetDevice(device);
        if (cudaMallocAsync(&p, warm, st) == cudaSuccess) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
        cudaGetLastError();
    }
    for (uint32_t w = 0; w < workers; w++) s->threads.emplace_back(worker, s, w);
    *out = s;
    return OL_OK;
}

extern "C" void ol_server_destroy(ol_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->qmu);
        s->stopping = true;
    }
    s->qcv.notify_all();
    for (auto &t : s->threads) t.join();
    for (auto &kv : s->store) {
        ol_tree_free(kv.second.tree);
        ol_doc_free(kv.second.doc);
    }
    s->store.clear();
    for (ol_ctx *c : s->ctxs) ol_ctx_destroy(c);
    delete s;
}

extern "C" ol_status ol_server_submit_parse(ol_server *s, const uint8_t *text, uint64_t len, uint64_t *request_id) {
    if (!s || !request_id || (len && !text)) return OL_ERR_INVALID_ARG;
    auto r = new Request();
    r->kind = 0;
    r->text = text;
    r->len = len;
    return submit(s, r, request_id);
}

extern "C" ol_status ol_server_submit_search(ol_server *s, uint64_t doc_id, const uint8_t *const *patterns,
                                             const uint32_t *lens, uint32_t n, uint64_t *request_id) {
    if (!s || !request_id || !n || !patterns || !lens) return OL_ERR_INVALID_ARG;
    auto r = new Request();
    r->kind = 1;
    r->doc_id = doc_id;
    for (uint32_t i = 0; i < n; i++) r->patterns.emplace_back((const char *)patterns[i], lens[i]);
    return submit(s, r, request_id);
}

extern "C" ol_status ol_server_wait(ol_server *s, uint64_t request_id, ol_request_result *out) {
    if (!s || !out) return OL_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->rmu);
    s->rcv.wait(lk, [&] { return s->results.count(request_id) != 0; });
    *out = s->results[request_id];
    s->results.erase(request_id);
    return OL_OK;
}

extern "C" ol_status ol_server_stats(ol_server *s, uint64_t *resident_docs, uint64_t *resident_bytes_out,
                                     uint64_t *evictions, uint64_t *refusals) {
    if (!s) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(s->smu);
    if (resident_docs) *resident_docs = s->store.size();
    if (resident_bytes_out) *resident_bytes_out = s->used;
    if (evictions) *evictions = s->evictions;
    if (refusals) *refusals = s->refusals;
    return OL_OK;
}
