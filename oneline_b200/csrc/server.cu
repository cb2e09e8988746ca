// A serving loop for parse and search requests of mixed sizes (no reference
// counterpart: the reference exposes one blocking call per document,
// crates/oneline-gpu/src/parser.rs). Requests are queued as they arrive and
// taken by worker threads, each with its own context and CUDA stream.
//
// Continuous batching: a worker that frees up takes its share of the requests
// queued at that moment (the queue divided among the idle workers, up to a
// step's limits) and serves them together; under light load a step is one
// request and the workers serve requests side by side, under load the steps
// grow:
//   * admission first: each parse request reserves its estimated resident
//     bytes against the store budget, counting the reservations of requests
//     still in flight on other workers; least recently used idle documents
//     are evicted to make room, and a request that cannot fit is refused
//     (OL_ERR_ADMISSION) before any upload;
//   * the admitted parse requests are uploaded, parsed and linked as one batch
//     (one pinned-ring upload, one parse, one tree build for all of them),
//     then split into resident documents with one copy launch;
//   * search requests on the same resident document are merged into one
//     pattern set and one dictionary pass, and each request gets its own slice
//     of the (pattern, offset)-ordered hits;
//   * a step serves its searches before its parses (a search never waits for
//     a parse of its own step: it names a document that already exists), and
//     each request's result is published as soon as it is ready.
// Workers run steps concurrently, so requests that arrive while others are on
// the GPU start on the next free worker and their kernels overlap on the
// device. Results (offsets, kinds and the four tree arrays of a parse; counts
// and hits of a search) are downloaded into host memory, and into the caller's
// buffers when given, before the request completes, so the reported latency
// includes the download. Every result carries a digest of its outputs,
// computed on the host from the downloaded arrays, to compare a request served
// in a busy mix with the same request alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "runtime.h"

using namespace ol;

namespace {

constexpr uint32_t kStepMaxRequests = 256;            // requests one step takes at most
constexpr uint64_t kStepMaxParseBytes = 64ull << 20;  // parse text one step takes at most
constexpr uint64_t kStagingBytes = 64ull << 20;        // pinned download staging per worker (grown on demand)
constexpr uint64_t kStagingMaxBytes = 2ull << 30;

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// The digest of one array: the sum (mod 2^64) over i of
// splitmix64(seed << 56 ^ i << 24 ^ a[i] * 0x9E3779B97F4A7C15), a sum of
// per-element hashes, so two arrays that differ in one element or in order
// differ in digest with overwhelming odds.
uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}

uint64_t elem_digest(uint32_t seed, uint64_t i, uint64_t v) {
    return mix64(((uint64_t)seed << 56) ^ (i << 24) ^ (v * 0x9E3779B97F4A7C15ull));
}

template <class T>
uint64_t array_digest(const T *a, uint64_t n, uint32_t seed) {
    uint64_t acc = 0;
    for (uint64_t i = 0; i < n; i++) acc += elem_digest(seed, i, a[i]);
    return acc;
}

// A search result's digest: its first k hits as (pattern within the request,
// offset) pairs of u32 (seed 7), then the per-pattern counts folded in, then
// the total.
uint64_t search_digest(const ol_hit *hits, uint64_t k, uint32_t pattern_base, const uint32_t *counts, uint32_t n,
                       uint64_t total) {
    uint64_t h = 0;
    for (uint64_t j = 0; j < k; j++) {
        h += elem_digest(7, 2 * j, hits[j].pattern - pattern_base);
        h += elem_digest(7, 2 * j + 1, hits[j].offset);
    }
    for (uint32_t i = 0; i < n; i++) h = h * 0x100000001B3ull ^ counts[i];
    return h ^ total;
}

struct Request {
    uint64_t id = 0;
    uint32_t kind = 0;  // 0 parse, 1 search
    const uint8_t *text = nullptr;
    uint64_t len = 0;
    uint64_t doc_id = 0;
    std::vector<std::string> patterns;
    uint64_t submit_ns = 0;
    bool has_pdest = false, has_sdest = false;
    ol_parse_dest pdest{};
    ol_search_dest sdest{};
    uint64_t reserved = 0;  // bytes reserved in the store at admission
};

struct Entry {
    ol_doc *doc = nullptr;
    ol_tree *tree = nullptr;
    uint64_t bytes = 0;
    uint32_t refs = 0;
    uint64_t last_use = 0;
};

// Pinned host staging of one worker, grown on demand (never while copies into
// it are in flight: every step reserves what it needs before enqueuing them).
struct Staging {
    uint8_t *ptr = nullptr;
    uint64_t bytes = 0;
    bool reserve(uint64_t need) {
        if (need <= bytes) return true;
        if (need > kStagingMaxBytes) return false;
        const uint64_t want = std::min(kStagingMaxBytes, std::max<uint64_t>(need, bytes * 2));
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
        if (cudaMallocHost((void **)&ptr, want) != cudaSuccess) {
            cudaGetLastError();
            ptr = nullptr;
            return false;
        }
        bytes = want;
        return true;
    }
};

}  // namespace

struct ol_server {
    int device = 0;
    uint32_t n_workers = 0;
    uint64_t budget = 0;
    uint64_t max_hits = 0;
    uint32_t flags = 0;
    std::vector<ol_ctx *> ctxs;
    std::vector<Staging> staging;
    std::vector<std::thread> threads;
    std::mutex qmu;
    std::condition_variable qcv;
    std::deque<Request *> queue;
    bool stopping = false;
    bool paused = false;  // workers take no request while set (ol_server_pause)
    uint32_t idle = 0;    // workers waiting for requests
    std::mutex rmu;
    std::condition_variable rcv;
    std::unordered_map<uint64_t, ol_request_result> results;
    std::atomic<uint64_t> next_id{1}, next_doc{1};
    std::mutex smu;
    std::unordered_map<uint64_t, Entry> store;
    std::set<std::pair<uint64_t, uint64_t>> lru;  // (last_use, document id) of every resident document
    uint64_t used = 0, reserved = 0, tick = 0;
    uint64_t busy = 0;  // bytes of the resident documents in use (refs > 0)
    std::atomic<uint64_t> evictions{0}, refusals{0}, steps{0}, served{0}, largest_step{0};
};

namespace {

uint64_t resident_bytes(const ol_doc *d) {
    const uint64_t text = d->text_len ? (uint64_t)d->text_buf.bytes : 0;
    return text + (uint64_t)d->line_cap * 6 + (uint64_t)d->line_count * 16;  // offsets, kinds, depth8; tree
}

// What a document of `len` bytes will hold in the store: its padded text, line
// arrays for the estimated line count (with head room) and four tree arrays.
uint64_t estimate_resident(const uint8_t *text, uint64_t len) {
    if (len == 0) return 0;
    const uint64_t lines = round_lines(estimate_lines(text, len));
    return (uint64_t)parse_tiles(len) * kParseTile + kTextPad + lines * 22;
}

// Takes idle documents out of the store, least recently used first, until
// `need` more bytes fit beside the documents in use and the reservations of
// requests in flight; the caller frees them after releasing smu (freeing takes
// the owning context's lock, which a worker may hold while it waits for smu).
// Called with smu held; returns false, evicting nothing, when the documents in
// use and the reservations leave no room.
bool make_room(ol_server *s, uint64_t need, std::vector<Entry> &evicted) {
    if (s->reserved + s->busy + need > s->budget) return false;
    // the least recently used first; documents in use are skipped (few)
    auto it = s->lru.begin();
    while (s->used + s->reserved + need > s->budget) {
        auto victim = s->store.end();
        while (it != s->lru.end()) {  // the index holds exactly the resident documents
            victim = s->store.find(it->second);
            if (victim == s->store.end()) {
                it = s->lru.erase(it);
                continue;
            }
            if (victim->second.refs == 0) break;
            ++it;
        }
        if (it == s->lru.end()) return false;
        evicted.push_back(victim->second);
        s->store.erase(victim);
        it = s->lru.erase(it);
        s->used -= evicted.back().bytes;
        s->evictions++;
    }
    return true;
}

// Marks a resident document used now (the most recently used).
void touch(ol_server *s, uint64_t id, Entry &e) {
    s->lru.erase({e.last_use, id});
    e.last_use = s->tick++;
    s->lru.insert({e.last_use, id});
}

void free_entries(std::vector<Entry> &v) {
    for (auto &e : v) {
        ol_tree_free(e.tree);
        ol_doc_free(e.doc);
    }
    v.clear();
}

// A parsed document's six arrays in host memory.
struct HostLines {
    const uint32_t *offsets = nullptr;
    const uint8_t *kinds = nullptr;
    const uint32_t *links[4] = {nullptr, nullptr, nullptr, nullptr};
};

// The result of a parse request from its arrays: the digest, and the arrays
// into the caller's buffers when they have room for every line.
void finish_parse(const Request *r, uint64_t L, const HostLines &h, ol_request_result &res) {
    uint64_t dg = array_digest(h.offsets, L, 1) + array_digest(h.kinds, L, 2);
    for (int k = 0; k < 4; k++) dg += array_digest(h.links[k], L, 3 + k);
    res.digest = dg ^ (L * 0x9E3779B97F4A7C15ull);
    res.line_count = L;
    if (!r->has_pdest || r->pdest.cap < L || L == 0) return;
    const ol_parse_dest &d = r->pdest;
    if (d.offsets) memcpy(d.offsets, h.offsets, L * 4);
    if (d.kinds) memcpy(d.kinds, h.kinds, L);
    uint32_t *outs[4] = {d.parent, d.subtree_end, d.first_child, d.next_sibling};
    for (int k = 0; k < 4; k++)
        if (outs[k]) memcpy(outs[k], h.links[k], L * 4);
}

// Puts a parsed document into the store (its reservation becomes its real
// size), or refuses it when the real size does not fit after all.
void commit_doc(ol_server *s, Request *r, ol_doc *&d, ol_tree *&t, ol_request_result &res) {
    std::vector<Entry> evicted;
    {
        std::lock_guard<std::mutex> g(s->smu);
        s->reserved -= r->reserved;
        r->reserved = 0;
        const uint64_t bytes = resident_bytes(d);
        if (!make_room(s, bytes, evicted)) {
            res.status = OL_ERR_ADMISSION;
            s->refusals++;
        } else {
            Entry e;
            e.doc = d;
            e.tree = t;
            e.bytes = bytes;
            e.last_use = s->tick++;
            res.doc_id = s->next_doc++;
            s->store[res.doc_id] = e;
            s->lru.insert({e.last_use, res.doc_id});
            s->used += bytes;
            d = nullptr;
            t = nullptr;
        }
    }
    free_entries(evicted);
}

void release_reservation(ol_server *s, Request *r) {
    std::lock_guard<std::mutex> g(s->smu);
    s->reserved -= r->reserved;
    r->reserved = 0;
}

uint64_t staged_bytes(const ol_doc *d) { return ((uint64_t)d->line_count * 21 + 63) & ~63ull; }

// Enqueues the download of one resident document's six arrays into staging at
// `at` (bytes), which the caller has reserved.
void stage_doc(ol_ctx *ctx, Staging &stg, uint64_t &at, const ol_doc *d, const ol_tree *t, HostLines &h) {
    const uint64_t L = d->line_count;
    cudaStream_t st = ctx->stream;
    uint32_t *offs = (uint32_t *)(stg.ptr + at);
    uint32_t *links = offs + L;
    uint8_t *kinds = (uint8_t *)(links + 4 * L);
    const void *src[4] = {t->parent_buf.ptr, t->end_buf.ptr, t->fc_buf.ptr, t->ns_buf.ptr};
    if (L) {
        GpuPass pass(ctx, "download");
        cudaMemcpyAsync(offs, d->offsets, L * 4, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(kinds, d->kinds, L, cudaMemcpyDeviceToHost, st);
        for (int k = 0; k < 4; k++) cudaMemcpyAsync(links + k * L, src[k], L * 4, cudaMemcpyDeviceToHost, st);
    }
    h.offsets = offs;
    h.kinds = kinds;
    for (int k = 0; k < 4; k++) h.links[k] = links + k * L;
    at += staged_bytes(d);
}

// The admitted parse requests of one step: one resident document each, equal
// to ol_doc_upload + ol_tree_build of that document alone.
void run_parses(ol_server *s, ol_ctx *ctx, Staging &stg, std::vector<Request *> &reqs,
                std::vector<ol_request_result *> &res) {
    const size_t n = reqs.size();
    std::vector<ol_doc *> docs(n, nullptr);
    std::vector<ol_tree *> trees(n, nullptr);
    std::vector<ol_status> st(n, OL_OK);
    if (n == 1 || (s->flags & OL_SERVER_NO_COALESCE)) {
        for (size_t i = 0; i < n; i++) {
            st[i] = ol_doc_upload(ctx, reqs[i]->text, reqs[i]->len, &docs[i]);
            if (st[i] == OL_OK) st[i] = ol_tree_build(ctx, docs[i], 0, &trees[i]);  // any depth
        }
    } else {
        std::vector<const uint8_t *> parts(n);
        std::vector<uint64_t> lens(n);
        for (size_t i = 0; i < n; i++) {
            parts[i] = reqs[i]->text;
            lens[i] = reqs[i]->len;
        }
        ol_batch *b = nullptr;
        ol_status bs = batch_from_parts(ctx, parts.data(), lens.data(), (uint32_t)n, &b);
        if (bs == OL_OK) bs = ol_batch_build_trees(ctx, b);
        if (bs == OL_OK) bs = batch_split(ctx, b, docs, trees);
        if (b) ol_batch_free(b);
        if (bs != OL_OK) {
            docs.assign(n, nullptr);
            trees.assign(n, nullptr);
            for (size_t i = 0; i < n; i++) st[i] = bs;
        }
    }
    // every document's downloads into staging reserved once, then one wait
    std::vector<HostLines> host(n);
    uint64_t at = 0, need = 64;
    for (size_t i = 0; i < n; i++)
        if (st[i] == OL_OK) need += staged_bytes(docs[i]);
    if (!stg.reserve(need))
        for (size_t i = 0; i < n; i++)
            if (st[i] == OL_OK) st[i] = OL_ERR_OOM;
    {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        cudaSetDevice(ctx->device);
        for (size_t i = 0; i < n; i++)
            if (st[i] == OL_OK) stage_doc(ctx, stg, at, docs[i], trees[i], host[i]);
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            ol_status cs = ctx_cuda(ctx, e, "server download");
            for (size_t i = 0; i < n; i++)
                if (st[i] == OL_OK) st[i] = cs;
        }
    }
    prof_mark(ctx, "server: parse step");
    for (size_t i = 0; i < n; i++) {
        Request *r = reqs[i];
        res[i]->status = st[i];
        if (st[i] == OL_OK) {
            finish_parse(r, docs[i]->line_count, host[i], *res[i]);
            commit_doc(s, r, docs[i], trees[i], *res[i]);
        } else {
            release_reservation(s, r);
        }
        if (trees[i]) ol_tree_free(trees[i]);
        if (docs[i]) ol_doc_free(docs[i]);
        res[i]->end_ns = now_ns();
    }
}

// A search request inside a merged pass: its patterns are [first, first + n)
// of the merged set.
struct SearchPart {
    Request *r;
    ol_request_result *res;
    uint32_t first = 0, n = 0;
};

uint64_t hit_cap_of(const ol_server *s, const Request *r) { return r->has_sdest ? r->sdest.max_hits : s->max_hits; }

// One dictionary pass over a resident document for the merged patterns of
// `parts`, with room for `hit_cap` hits in staging. When every hit a request
// keeps fits, each request gets its slice of the (pattern, offset)-ordered
// hits; otherwise *overflow is set and no result is written.
ol_status search_pass(ol_server *s, ol_ctx *ctx, Staging &stg, const Entry &e, std::vector<SearchPart> &parts,
                      uint64_t hit_cap, bool &overflow) {
    std::vector<const uint8_t *> p;
    std::vector<uint32_t> lens;
    for (auto &x : parts) {
        x.first = (uint32_t)p.size();
        x.n = (uint32_t)x.r->patterns.size();
        for (auto &q : x.r->patterns) {
            p.push_back((const uint8_t *)q.data());
            lens.push_back((uint32_t)q.size());
        }
    }
    std::lock_guard<std::recursive_mutex> cg(ctx->mu);
    cudaSetDevice(ctx->device);
    ol_patset *set = nullptr;
    ol_status st = ol_patset_compile(ctx, e.doc, p.data(), lens.data(), (uint32_t)p.size(), &set);
    std::vector<uint32_t> counts(p.size());
    uint64_t total = 0;
    if (st == OL_OK && !stg.reserve(hit_cap * sizeof(ol_hit) + 64)) st = OL_ERR_OOM;
    if (st == OL_OK) {
        HitDest dest;
        dest.host = (ol_hit *)stg.ptr;
        st = many_run(ctx, e.doc, set, hit_cap, 0, counts.data(), &total, dest, nullptr, nullptr, 0);
    }
    if (set) ol_patset_free(set);
    overflow = false;
    if (st != OL_OK) return st;
    // every request needs the hits up to the end of the part of its slice it keeps
    uint64_t need = 0, at = 0;
    for (auto &x : parts) {
        uint64_t tot = 0;
        for (uint32_t i = 0; i < x.n; i++) tot += counts[x.first + i];
        need = std::max(need, at + std::min(tot, hit_cap_of(s, x.r)));
        at += tot;
    }
    if (need > hit_cap) {
        overflow = true;
        return OL_OK;
    }
    const ol_hit *hits = (const ol_hit *)stg.ptr;
    uint64_t base = 0;  // the request's first hit
    for (auto &x : parts) {
        Request *r = x.r;
        ol_request_result &res = *x.res;
        uint64_t tot = 0;
        for (uint32_t i = 0; i < x.n; i++) tot += counts[x.first + i];
        const uint64_t k = std::min(tot, hit_cap_of(s, r));
        const ol_hit *mine = hits + base;
        res.digest = search_digest(mine, k, x.first, counts.data() + x.first, x.n, tot);
        res.total_hits = tot;
        if (r->has_sdest) {
            if (r->sdest.counts) memcpy(r->sdest.counts, counts.data() + x.first, (size_t)x.n * 4);
            if (r->sdest.hits)
                for (uint64_t j = 0; j < k; j++) r->sdest.hits[j] = ol_hit{mine[j].pattern - x.first, mine[j].offset};
        }
        res.status = OL_OK;
        base += tot;
    }
    return OL_OK;
}

bool patterns_ok(const Request *r) {
    if (r->patterns.empty() || r->patterns.size() > OL_MAX_DICT_PATTERNS) return false;
    for (auto &q : r->patterns)
        if (q.size() < OL_MIN_SET_PATTERN_LEN || q.size() > OL_MAX_SET_PATTERN_LEN) return false;
    return true;
}

// The search requests of one step on one resident document: one merged pass,
// or, when the merged hits outgrow the room, one pass per request.
void run_search_group(ol_server *s, ol_ctx *ctx, Staging &stg, uint64_t doc_id, std::vector<SearchPart> &parts) {
    Entry e;
    bool found = false;
    {
        std::lock_guard<std::mutex> g(s->smu);
        auto it = s->store.find(doc_id);
        if (it != s->store.end()) {
            if (it->second.refs++ == 0) s->busy += it->second.bytes;
            touch(s, doc_id, it->second);
            e = it->second;
            found = true;
        }
    }
    if (!found) {
        for (auto &x : parts) x.res->status = OL_ERR_NOT_FOUND;
    } else {
        // The merged pass uses the staging the worker already holds and never
        // grows it: pinned allocations are slow and freeing pinned memory waits
        // for the whole device, which would stall every worker.
        uint64_t cap = 0;
        for (auto &x : parts) cap += hit_cap_of(s, x.r);
        cap = std::min<uint64_t>(cap, (stg.bytes - 64) / sizeof(ol_hit));
        bool overflow = false;
        ol_status st = parts.size() > 1 ? search_pass(s, ctx, stg, e, parts, cap, overflow) : OL_OK;
        if (st == OL_OK && (overflow || parts.size() == 1)) {
            for (auto &x : parts) {
                std::vector<SearchPart> one{x};
                bool of1 = false;
                ol_status s1 = search_pass(s, ctx, stg, e, one, hit_cap_of(s, x.r), of1);
                if (s1 == OL_OK && of1) s1 = OL_ERR_OOM;  // a request alone always fits its own cap
                x.res->status = s1;
            }
        } else if (st != OL_OK) {
            for (auto &x : parts) x.res->status = st;
        }
        std::lock_guard<std::mutex> g(s->smu);
        auto it = s->store.find(doc_id);
        if (it != s->store.end() && --it->second.refs == 0) s->busy -= it->second.bytes;
    }
    prof_mark(ctx, "server: search step");
    for (auto &x : parts) {
        x.res->doc_id = doc_id;
        x.res->end_ns = now_ns();
    }
}

void publish(ol_server *s, const std::vector<ol_request_result *> &done) {
    if (done.empty()) return;
    {
        std::lock_guard<std::mutex> g(s->rmu);
        for (auto *x : done) s->results[x->id] = *x;
    }
    s->rcv.notify_all();
}

// One step: the requests taken from the queue together.
void run_step(ol_server *s, uint32_t w, std::vector<Request *> &step) {
    ol_ctx *ctx = s->ctxs[w];
    Staging &stg = s->staging[w];
    std::vector<ol_request_result> res(step.size());
    const uint64_t start = now_ns();
    for (size_t i = 0; i < step.size(); i++) {
        res[i] = ol_request_result{};
        res[i].id = step[i]->id;
        res[i].kind = step[i]->kind;
        res[i].submit_ns = step[i]->submit_ns;
        res[i].start_ns = start;
        res[i].worker = w;
        res[i].status = OL_ERR_CUDA;
    }
    // Admission of the parse requests, before any work.
    std::vector<Request *> parses;
    std::vector<ol_request_result *> parse_res, refused;
    std::vector<Entry> evicted;
    {
        std::lock_guard<std::mutex> g(s->smu);
        for (size_t i = 0; i < step.size(); i++) {
            Request *r = step[i];
            if (r->kind != 0) continue;
            const uint64_t need = estimate_resident(r->text, r->len);
            if (!make_room(s, need, evicted)) {
                res[i].status = OL_ERR_ADMISSION;
                res[i].end_ns = now_ns();
                s->refusals++;
                refused.push_back(&res[i]);
                continue;
            }
            r->reserved = need;
            s->reserved += need;
            parses.push_back(r);
            parse_res.push_back(&res[i]);
        }
    }
    free_entries(evicted);
    publish(s, refused);
    // Search requests first (short, and never waiting on a parse of this
    // step), merged per document; each group's results go out when done.
    std::map<uint64_t, std::vector<SearchPart>> groups;
    std::vector<ol_request_result *> bad;
    for (size_t i = 0; i < step.size(); i++) {
        Request *r = step[i];
        if (r->kind != 1) continue;
        if (!patterns_ok(r)) {
            res[i].status = OL_ERR_BAD_PATTERN;
            res[i].doc_id = r->doc_id;
            res[i].end_ns = now_ns();
            bad.push_back(&res[i]);
            continue;
        }
        groups[r->doc_id].push_back(SearchPart{r, &res[i]});
    }
    publish(s, bad);
    for (auto &kv : groups) {
        run_search_group(s, ctx, stg, kv.first, kv.second);
        std::vector<ol_request_result *> done;
        for (auto &x : kv.second) done.push_back(x.res);
        publish(s, done);
    }
    if (!parses.empty()) {
        run_parses(s, ctx, stg, parses, parse_res);
        publish(s, parse_res);
    }
    for (Request *r : step) delete r;
    s->steps++;
    s->served += step.size();
    uint64_t big = s->largest_step.load();
    while (step.size() > big && !s->largest_step.compare_exchange_weak(big, step.size())) {
    }
}

void worker(ol_server *s, uint32_t w) {
    cudaSetDevice(s->device);
    const uint32_t limit = (s->flags & OL_SERVER_NO_COALESCE) ? 1u : kStepMaxRequests;
    for (;;) {
        std::vector<Request *> step;
        {
            std::unique_lock<std::mutex> lk(s->qmu);
            s->idle++;
            s->qcv.wait(lk, [&] { return s->stopping || (!s->paused && !s->queue.empty()); });
            s->idle--;
            if (s->queue.empty()) break;
            // this worker's share of the queue: the rest is left to the idle ones
            const uint64_t share = (s->queue.size() + s->idle) / (s->idle + 1);
            const uint64_t take = std::min<uint64_t>(limit, std::max<uint64_t>(share, 1));
            uint64_t parse_bytes = 0;
            while (!s->queue.empty() && step.size() < take) {
                Request *r = s->queue.front();
                if (!step.empty() && r->kind == 0 && parse_bytes + r->len > kStepMaxParseBytes) break;
                if (r->kind == 0) parse_bytes += r->len;
                step.push_back(r);
                s->queue.pop_front();
            }
        }
        run_step(s, w, step);
    }
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

extern "C" ol_status ol_server_create_ex(int32_t device, uint32_t workers, uint64_t store_budget, uint64_t max_hits,
                                         uint32_t flags, ol_server **out) {
    if (!out || workers == 0 || workers > 64 || (flags & ~(uint32_t)OL_SERVER_NO_COALESCE)) return OL_ERR_INVALID_ARG;
    *out = nullptr;
    auto s = new ol_server();
    s->device = device;
    s->n_workers = workers;
    s->budget = store_budget;
    s->max_hits = max_hits;
    s->flags = flags;
    s->staging.resize(workers);
    for (uint32_t w = 0; w < workers; w++) {
        ol_ctx *c = nullptr;
        ol_status st = ol_ctx_create(device, &c);
        if (st == OL_OK && !s->staging[w].reserve(kStagingBytes)) {
            ol_ctx_destroy(c);
            st = OL_ERR_OOM;  // the pinned staging could not be allocated: refuse to start
        }
        if (st != OL_OK) {
            for (ol_ctx *x : s->ctxs) ol_ctx_destroy(x);
            for (auto &g : s->staging)
                if (g.ptr) cudaFreeHost(g.ptr);
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

extern "C" ol_status ol_server_create(int32_t device, uint32_t workers, uint64_t store_budget, uint64_t max_hits,
                                      ol_server **out) {
    return ol_server_create_ex(device, workers, store_budget, max_hits, 0, out);
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
    s->lru.clear();
    for (ol_ctx *c : s->ctxs) ol_ctx_destroy(c);
    for (auto &g : s->staging)
        if (g.ptr) cudaFreeHost(g.ptr);
    delete s;
}

extern "C" ol_status ol_server_submit_parse_to(ol_server *s, const uint8_t *text, uint64_t len,
                                               const ol_parse_dest *dest, uint64_t *request_id) {
    if (!s || !request_id || (len && !text)) return OL_ERR_INVALID_ARG;
    if (len > OL_MAX_GPU_INPUT_LEN) return OL_ERR_INPUT_TOO_LARGE;
    auto r = new Request();
    r->kind = 0;
    r->text = text;
    r->len = len;
    if (dest) {
        r->has_pdest = true;
        r->pdest = *dest;
    }
    return submit(s, r, request_id);
}

extern "C" ol_status ol_server_submit_parse(ol_server *s, const uint8_t *text, uint64_t len, uint64_t *request_id) {
    return ol_server_submit_parse_to(s, text, len, nullptr, request_id);
}

extern "C" ol_status ol_server_submit_search_to(ol_server *s, uint64_t doc_id, const uint8_t *const *patterns,
                                                const uint32_t *lens, uint32_t n, const ol_search_dest *dest,
                                                uint64_t *request_id) {
    if (!s || !request_id || !n || !patterns || !lens) return OL_ERR_INVALID_ARG;
    auto r = new Request();
    r->kind = 1;
    r->doc_id = doc_id;
    for (uint32_t i = 0; i < n; i++) r->patterns.emplace_back((const char *)patterns[i], lens[i]);
    if (dest) {
        r->has_sdest = true;
        r->sdest = *dest;
    }
    return submit(s, r, request_id);
}

extern "C" ol_status ol_server_submit_search(ol_server *s, uint64_t doc_id, const uint8_t *const *patterns,
                                             const uint32_t *lens, uint32_t n, uint64_t *request_id) {
    return ol_server_submit_search_to(s, doc_id, patterns, lens, n, nullptr, request_id);
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

extern "C" ol_status ol_server_pause(ol_server *s, uint32_t paused) {
    if (!s) return OL_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> g(s->qmu);
        s->paused = paused != 0;
    }
    s->qcv.notify_all();
    return OL_OK;
}

extern "C" ol_status ol_server_steps(ol_server *s, uint64_t *steps, uint64_t *requests, uint64_t *largest_step) {
    if (!s) return OL_ERR_INVALID_ARG;
    if (steps) *steps = s->steps;
    if (requests) *requests = s->served;
    if (largest_step) *largest_step = s->largest_step;
    return OL_OK;
}
