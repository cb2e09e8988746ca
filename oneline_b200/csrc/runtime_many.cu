// C ABI for dictionary search: GpuParser::compile_patterns / search_many and
// GpuPatternSet::{len, is_empty} (crates/oneline-gpu/src/many.rs:139-176,
// 391-646). Hits are every (pattern, offset), duplicates once per id, ordered
// by (pattern, offset) as ManyPatterns orders them
// (crates/oneline-simd/src/search.rs:259-282).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "runtime.h"

using namespace ol;

// The trie path of a run of one byte, as compiled: node and unique pattern
// (or NONE) at each depth 4..K.
struct DictRunPath {
    uint32_t byte = 0, K = 0;
    uint32_t node[ol::kDictMaxLen + 1] = {};
    uint32_t u[ol::kDictMaxLen + 1] = {};
};

struct ol_patset {
    ol_ctx *ctx = nullptr;
    uint32_t n_ids = 0, n_u = 0, n_nodes = 0;
    DevBuf blob;
    DictSet dev{};
    const uint32_t *u_of_id = nullptr, *dup_start = nullptr, *dup_ids = nullptr;
    std::vector<DictRunPath> runs;  // the longest byte runs (at most kDictMaxChains)
};

namespace {

struct TrieNode {
    std::vector<std::pair<uint8_t, uint32_t>> kids;
    uint32_t out = NONE;
};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

uint32_t bits_for(uint32_t v) {  // bits needed to hold values 0..v
    uint32_t b = 0;
    while (b < 32 && (v >> b)) b++;
    return b;
}

// Scratch of one dictionary search, carved from ctx->dict_small.
struct ManyScratch {
    uint32_t *sample_counts, *light_count, *light_base, *heavy_u, *heavy_totals, *heavy_counts, *heavy_bases;
    uint32_t *light_n, *error, *id_counts, *sort_hist, *sort_totals;
    uint8_t *heavy_of_u;
    unsigned long long *id_base, *total, *stats;
    DictChain *chains;
};

}  // namespace

extern "C" ol_status ol_patset_compile(ol_ctx *ctx, const ol_doc *doc, const uint8_t *const *patterns,
                                       const uint32_t *lens, uint32_t n, ol_patset **out) {
    (void)doc;  // the reference samples the document to size its filter; this filter is fixed
    if (!ctx || !out || (n && (!patterns || !lens))) return OL_ERR_INVALID_ARG;
    *out = nullptr;
    if (n == 0 || n > OL_MAX_DICT_PATTERNS)
        return ctx_fail(ctx, OL_ERR_BAD_PATTERN,
                        "pattern count " + std::to_string(n) + " is outside 1.." + std::to_string(OL_MAX_DICT_PATTERNS));
    for (uint32_t i = 0; i < n; i++)
        if (!patterns[i] || lens[i] < OL_MIN_SET_PATTERN_LEN || lens[i] > OL_MAX_SET_PATTERN_LEN)
            return ctx_fail(ctx, OL_ERR_BAD_PATTERN,
                            "pattern " + std::to_string(i) + " has " + std::to_string(lens[i]) + " bytes; set patterns need " +
                                std::to_string(OL_MIN_SET_PATTERN_LEN) + ".." + std::to_string(OL_MAX_SET_PATTERN_LEN));

    // Unique patterns, in order of first appearance.
    std::unordered_map<std::string, uint32_t> uniq;
    std::vector<uint32_t> u_of_id(n);
    std::vector<const std::string *> u_str;
    uniq.reserve(n * 2);
    for (uint32_t i = 0; i < n; i++) {
        auto r = uniq.emplace(std::string((const char *)patterns[i], lens[i]), (uint32_t)uniq.size());
        if (r.second) u_str.push_back(&r.first->first);
        u_of_id[i] = r.first->second;
    }
    const uint32_t U = (uint32_t)u_str.size();

    // Trie over the unique patterns; the node after the first four bytes of each.
    std::vector<TrieNode> trie(1);
    std::unordered_map<uint32_t, uint32_t> key_node;
    for (uint32_t u = 0; u < U; u++) {
        const std::string &p = *u_str[u];
        uint32_t v = 0;
        for (size_t j = 0; j < p.size(); j++) {
            uint8_t b = (uint8_t)p[j];
            uint32_t next = NONE;
            for (auto &k : trie[v].kids)
                if (k.first == b) next = k.second;
            if (next == NONE) {
                next = (uint32_t)trie.size();
                trie[v].kids.emplace_back(b, next);
                trie.emplace_back();
            }
            v = next;
            if (j == kDictMinLen - 1) {
                uint32_t key;
                memcpy(&key, p.data(), 4);
                key_node[key] = v;
            }
        }
        trie[v].out = u;
    }
    const uint32_t n_nodes = (uint32_t)trie.size();
    if (n_nodes >= (1u << 24)) return ctx_fail(ctx, OL_ERR_BAD_PATTERN, "pattern set too large for the trie");
    std::vector<uint4> nodes(n_nodes);
    std::vector<uint32_t> extra, dense;
    for (uint32_t v = 0; v < n_nodes; v++) {
        auto &k = trie[v].kids;
        std::sort(k.begin(), k.end());
        uint4 r{trie[v].out, (uint32_t)k.size(), 0, 0};
        auto pack = [](const std::pair<uint8_t, uint32_t> &e) { return (e.second << 8) | e.first; };
        if (k.size() > kDictDenseMin) {
            // many children: a 256-entry table, one load per step
            r.y |= kDictDenseFlag;
            r.w = (uint32_t)(dense.size() / 256);
            dense.resize(dense.size() + 256, NONE);
            for (auto &e : k) dense[(size_t)r.w * 256 + e.first] = e.second;
        } else {
            if (!k.empty()) r.z = pack(k[0]);
            if (k.size() == 2) r.w = pack(k[1]);
            if (k.size() > 2) {
                r.w = (uint32_t)extra.size();
                for (size_t i = 1; i < k.size(); i++) extra.push_back(pack(k[i]));
            }
        }
        nodes[v] = r;
    }
    if (extra.empty()) extra.push_back(0);
    if (dense.empty()) dense.push_back(NONE);

    // Byte runs: the trie path c^4, c^5, ... of each byte c that starts a
    // pattern with c^4; the longest ones (at least kDictChainMin deep) let
    // walks inside long runs of c skip down the path (dict_walk).
    std::vector<DictRunPath> runs;
    for (uint32_t c = 0; c < 256; c++) {
        auto it = key_node.find(c * 0x01010101u);
        if (it == key_node.end()) continue;
        DictRunPath r;
        r.byte = c;
        uint32_t v = it->second, d = kDictMinLen;
        r.node[d] = v;
        r.u[d] = trie[v].out;
        while (d < kDictMaxLen) {
            uint32_t next = NONE;
            for (auto &k : trie[v].kids)
                if (k.first == c) next = k.second;
            if (next == NONE) break;
            v = next;
            d++;
            r.node[d] = v;
            r.u[d] = trie[v].out;
        }
        r.K = d;
        if (r.K >= kDictChainMin) runs.push_back(r);
    }
    std::sort(runs.begin(), runs.end(), [](const DictRunPath &x, const DictRunPath &y) { return x.K > y.K; });
    if (runs.size() > kDictMaxChains) runs.resize(kDictMaxChains);

    // Filter and hash table over the distinct first-four-byte keys.
    std::vector<uint32_t> filter(1u << (kDictFilterBits - 5), 0);
    uint32_t table_bits = 10;
    while ((1u << table_bits) < 2 * key_node.size()) table_bits++;
    std::vector<uint2> table(1u << table_bits, make_uint2(0, NONE));
    uint32_t max_probe = 0;
    for (auto &kv : key_node) {
        uint32_t key = kv.first;
        uint32_t h1 = dict_filter_h1(key), h2 = dict_filter_h2(key);
        filter[h1 >> 5] |= 1u << (h1 & 31);
        filter[h2 >> 5] |= 1u << (h2 & 31);
        uint32_t slot = dict_table_h(key, table_bits), dist = 0;
        while (table[slot].y != NONE) {
            slot = (slot + 1) & ((1u << table_bits) - 1);
            dist++;
        }
        table[slot] = make_uint2(key, kv.second);
        max_probe = std::max(max_probe, dist);
    }

    // Ids grouped by unique pattern.
    std::vector<uint32_t> dup_start(U + 1, 0), dup_ids(n);
    for (uint32_t i = 0; i < n; i++) dup_start[u_of_id[i] + 1]++;
    for (uint32_t u = 0; u < U; u++) dup_start[u + 1] += dup_start[u];
    {
        std::vector<uint32_t> fill(dup_start.begin(), dup_start.end() - 1);
        for (uint32_t i = 0; i < n; i++) dup_ids[fill[u_of_id[i]]++] = i;
    }

    // One device blob.
    size_t off_filter = 0, sz_filter = filter.size() * 4;
    size_t off_table = align256(off_filter + sz_filter), sz_table = table.size() * 8;
    size_t off_nodes = align256(off_table + sz_table), sz_nodes = nodes.size() * 16;
    size_t off_extra = align256(off_nodes + sz_nodes), sz_extra = extra.size() * 4;
    size_t off_dense = align256(off_extra + sz_extra), sz_dense = dense.size() * 4;
    size_t off_uid = align256(off_dense + sz_dense), sz_uid = (size_t)n * 4;
    size_t off_ds = align256(off_uid + sz_uid), sz_ds = dup_start.size() * 4;
    size_t off_di = align256(off_ds + sz_ds), sz_di = dup_ids.size() * 4;
    size_t total = align256(off_di + sz_di);
    std::vector<uint8_t> host(total, 0);
    memcpy(host.data() + off_filter, filter.data(), sz_filter);
    memcpy(host.data() + off_table, table.data(), sz_table);
    memcpy(host.data() + off_nodes, nodes.data(), sz_nodes);
    memcpy(host.data() + off_extra, extra.data(), sz_extra);
    memcpy(host.data() + off_dense, dense.data(), sz_dense);
    memcpy(host.data() + off_uid, u_of_id.data(), sz_uid);
    memcpy(host.data() + off_ds, dup_start.data(), sz_ds);
    memcpy(host.data() + off_di, dup_ids.data(), sz_di);

    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    ol_patset *s = new ol_patset();
    s->ctx = ctx;
    s->n_ids = n;
    s->n_u = U;
    s->n_nodes = n_nodes;
    cudaError_t e = s->blob.reserve(total, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->blob.ptr, host.data(), total, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        s->blob.release(ctx->stream);
        delete s;
        return ctx_cuda(ctx, e, "compile_patterns");
    }
    uint8_t *b = (uint8_t *)s->blob.ptr;
    s->dev.filter = (const uint32_t *)(b + off_filter);
    s->dev.table = (const uint2 *)(b + off_table);
    s->dev.table_bits = table_bits;
    s->dev.max_probe = max_probe;
    s->dev.nodes = (const uint4 *)(b + off_nodes);
    s->dev.extra = (const uint32_t *)(b + off_extra);
    s->dev.dense = (const uint32_t *)(b + off_dense);
    s->dev.n_u = U;
    s->u_of_id = (const uint32_t *)(b + off_uid);
    s->dup_start = (const uint32_t *)(b + off_ds);
    s->dup_ids = (const uint32_t *)(b + off_di);
    s->runs = std::move(runs);
    *out = s;
    return OL_OK;
}

extern "C" void ol_patset_free(ol_patset *s) {
    if (!s) return;
    if (s->ctx) {
        std::lock_guard<std::recursive_mutex> g(s->ctx->mu);
        cudaSetDevice(s->ctx->device);
        s->blob.release(s->ctx->stream);
    }
    delete s;
}

extern "C" uint32_t ol_patset_len(const ol_patset *s) { return s ? s->n_ids : 0; }
extern "C" uint32_t ol_patset_unique(const ol_patset *s) { return s ? s->n_u : 0; }


// The whole search; hits go to d_hits (capacity max_hits) when given, else to
// host_hits through ctx->dict_hits. counts (n_ids) and *total are host outputs.
// seg_start/seg_end (device, n_seg): batches, whose hits stay inside a document.
ol_status ol::many_run(ol_ctx *ctx, const ol_doc *d, const ol_patset *set, uint64_t max_hits, uint32_t heavy_min_hits,
                       uint32_t *counts, uint64_t *total, const HitDest &dest,
                       const unsigned long long *seg_start, const unsigned long long *seg_end, uint32_t n_seg) {
    cudaStream_t st = ctx->stream;
    const uint32_t n = set->n_ids, U = set->n_u;
    const uint64_t N = d->text_len;
    *total = 0;
    memset(counts, 0, (size_t)n * 4);
    if (N < kDictMinLen) return OL_OK;
    const uint32_t n_tiles = (uint32_t)((N + kDictTile - 1) / kDictTile);
    const uint32_t n_words = n_tiles * kDictWordsPerTile;
    const uint32_t hblocks = dict_heavy_blocks(n_words), hld = scan_ld(hblocks);

    // Small scratch (sort histograms sized for the worst light count: grown below if needed).
    auto carve = [](size_t &at, size_t bytes) {
        size_t o = at;
        at = align256(at + bytes);
        return o;
    };
    size_t at = 0;
    size_t o_sample = carve(at, (size_t)U * 4), o_lcount = carve(at, (size_t)U * 4), o_lbase = carve(at, (size_t)U * 4);
    size_t o_heavy_of = carve(at, U), o_heavy_u = carve(at, kDictMaxHeavy * 4), o_htot = carve(at, kDictMaxHeavy * 4);
    size_t o_hcounts = carve(at, (size_t)kDictMaxHeavy * hld * 4), o_hbases = carve(at, (size_t)kDictMaxHeavy * hld * 4);
    size_t o_ln = carve(at, 16), o_idc = carve(at, (size_t)n * 4), o_idb = carve(at, (size_t)n * 8), o_tot = carve(at, 16);
    size_t o_stot = carve(at, 256 * 4), o_stats = carve(at, 16);
    size_t o_chains = carve(at, kDictMaxChains * sizeof(DictChain));
    const size_t fixed = at;
    cudaError_t e = ctx->dict_small.reserve(fixed, st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "search_many");
    auto scratch_at = [&](uint8_t *b) {
        ManyScratch m;
        m.sample_counts = (uint32_t *)(b + o_sample);
        m.light_count = (uint32_t *)(b + o_lcount);
        m.light_base = (uint32_t *)(b + o_lbase);
        m.heavy_of_u = b + o_heavy_of;
        m.heavy_u = (uint32_t *)(b + o_heavy_u);
        m.heavy_totals = (uint32_t *)(b + o_htot);
        m.heavy_counts = (uint32_t *)(b + o_hcounts);
        m.heavy_bases = (uint32_t *)(b + o_hbases);
        m.light_n = (uint32_t *)(b + o_ln);
        m.error = m.light_n + 1;
        m.id_counts = (uint32_t *)(b + o_idc);
        m.id_base = (unsigned long long *)(b + o_idb);
        m.total = (unsigned long long *)(b + o_tot);
        m.sort_totals = (uint32_t *)(b + o_stot);
        m.stats = (unsigned long long *)(b + o_stats);
        m.chains = (DictChain *)(b + o_chains);
        m.sort_hist = (uint32_t *)(b + fixed);
        return m;
    };
    ManyScratch m = scratch_at((uint8_t *)ctx->dict_small.ptr);

    // 1. Counts on a sample of tiles (every tile when the text is small) pick
    //    the heavy patterns: those expected to have at least `threshold` hits.
    const uint32_t stride = std::max<uint32_t>(1, n_tiles / 256);
    const uint32_t n_work = (n_tiles + stride - 1) / stride;
    DictMatchArgs ma{};
    ma.set = set->dev;
    ma.text = d->text;
    ma.text_len = N;
    ma.n_tiles = n_tiles;
    ma.tile_stride = stride;
    ma.count_only = 1;
    ma.counts = m.sample_counts;
    ma.error = m.error;
    ma.seg_start = seg_start;
    ma.seg_end = seg_end;
    ma.n_seg = n_seg;
    // an armed injected timeout is taken by this search's first match pass
    ma.force_timeout = (ctx->inject & OL_INJECT_DICT_WAIT_TIMEOUT) ? 1u : 0u;
    ctx->inject &= ~OL_INJECT_DICT_WAIT_TIMEOUT;
    e = cudaMemsetAsync(m.sample_counts, 0, (size_t)U * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(m.light_n, 0, 16, st);
    if (e == cudaSuccess) {
        GpuPass pass(ctx, "dictionary: sample counts");
        e = launch_dict_match(ma, ctx->sm_count, st, ctx->tune.dict_slice, ctx->tune.dict_blocks_per_sm);
    }
    std::vector<uint32_t> sample(U);
    uint32_t flags[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(sample.data(), m.sample_counts, (size_t)U * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(flags, m.light_n, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    prof_mark(ctx, "dictionary: wait for the sample");
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "search_many sample");
    if (flags[1] & OL_DEVERR_TIMEOUT) return ctx_fail(ctx, OL_ERR_TIMEOUT, "search_many: a bounded wait ran out");
    const double scale = (double)n_tiles / (double)n_work;
    const double threshold = heavy_min_hits ? (double)heavy_min_hits : std::max(4096.0, (double)N / (double)std::max<uint32_t>(ctx->tune.dict_heavy_divisor, 1));
    std::vector<std::pair<double, uint32_t>> cand;
    double light_est = 0;
    for (uint32_t u = 0; u < U; u++) {
        double ex = sample[u] * scale;
        if (sample[u] && ex >= threshold)
            cand.emplace_back(-ex, u);
        else
            light_est += ex;
    }
    std::sort(cand.begin(), cand.end());
    if (cand.size() > kDictMaxHeavy) {
        for (size_t i = kDictMaxHeavy; i < cand.size(); i++) light_est += -cand[i].first;
        cand.resize(kDictMaxHeavy);
    }
    const uint32_t H = (uint32_t)cand.size();
    std::vector<uint8_t> heavy_of(U, 0xFF);
    std::vector<uint32_t> heavy_u(kDictMaxHeavy, 0);
    for (uint32_t h = 0; h < H; h++) {
        heavy_u[h] = cand[h].second;
        heavy_of[cand[h].second] = (uint8_t)h;
    }
    // The byte-run chains of this search: heavy bits accumulated down each run,
    // and its light patterns.
    std::vector<DictChain> chains(set->runs.size());
    uint32_t chain_bytes = 0;
    for (size_t j = 0; j < set->runs.size(); j++) {
        const DictRunPath &r = set->runs[j];
        DictChain &c = chains[j];
        memset(&c, 0, sizeof c);
        c.byte = r.byte;
        c.K = r.K;
        chain_bytes |= r.byte << (8 * j);
        uint32_t acc = 0;
        for (uint32_t dd = kDictMinLen; dd <= r.K; dd++) {
            c.node[dd] = r.node[dd];
            const uint32_t u = r.u[dd];
            if (u != NONE) {
                if (heavy_of[u] != 0xFF)
                    acc |= 1u << heavy_of[u];
                else
                    c.light[c.n_light++] = (dd << 24) | u;
            }
            c.cum[dd] = acc;
        }
    }
    e = cudaMemcpyAsync(m.heavy_of_u, heavy_of.data(), U, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && !chains.empty())
        e = cudaMemcpyAsync(m.chains, chains.data(), chains.size() * sizeof(DictChain), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m.heavy_u, heavy_u.data(), kDictMaxHeavy * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && H) e = ctx->dict_bitmap.reserve((size_t)H * n_words * 4, st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "search_many");

    // 2. The match pass; grown and re-run if the light keys overflow.
    uint64_t cap = std::min<uint64_t>(0xFFFFFFF0ull, (uint64_t)(light_est * 1.25) + 65536);
    uint32_t light_n = 0;
    for (int attempt = 0; attempt < 3; attempt++) {
        e = ctx->dict_keys.reserve((size_t)cap * 16, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(m.light_count, 0, (size_t)U * 4, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(m.light_n, 0, 16, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(m.stats, 0, 16, st);
        ma.stats = m.stats;
        ma.force_timeout = 0;
        ma.tile_stride = 1;
        ma.count_only = 0;
        ma.counts = m.light_count;
        ma.heavy_of_u = m.heavy_of_u;
        ma.n_heavy = H;
        ma.bitmap = H ? (uint32_t *)ctx->dict_bitmap.ptr : nullptr;
        ma.light_keys = (unsigned long long *)ctx->dict_keys.ptr;
        ma.light_cap = (uint32_t)cap;
        ma.light_n = m.light_n;
        ma.chains = m.chains;
        ma.n_chains = (uint32_t)chains.size();
        ma.chain_bytes = chain_bytes;
        if (e == cudaSuccess) {
            GpuPass pass(ctx, "dictionary: match");
            e = launch_dict_match(ma, ctx->sm_count, st, ctx->tune.dict_slice, ctx->tune.dict_blocks_per_sm);
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(flags, m.light_n, 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        prof_mark(ctx, "dictionary: wait for the match pass");
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "search_many match");
        if (flags[1] & OL_DEVERR_TIMEOUT) return ctx_fail(ctx, OL_ERR_TIMEOUT, "search_many: a bounded wait ran out");
        light_n = flags[0];
        if (light_n <= cap) break;
        cap = (uint64_t)light_n + 1024;
        if (attempt == 2) return ctx_fail(ctx, OL_ERR_CUDA, "search_many: light hit count kept growing");
    }

    // 3. Heavy ranks, light order, per-id slots.
    GpuPass order_pass(ctx, "dictionary: rank and sort");
    if (H) {
        e = launch_dict_heavy_count((const uint32_t *)ctx->dict_bitmap.ptr, n_words, H, m.heavy_counts, hld, st);
        if (e == cudaSuccess) e = launch_scan_columns(m.heavy_counts, m.heavy_bases, m.heavy_totals, hblocks, H, hld, st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "search_many heavy");
    }
    unsigned long long *keys = (unsigned long long *)ctx->dict_keys.ptr;
    if (light_n > 1) {
        const size_t hist_bytes = (size_t)2 * 256 * scan_ld(dict_sort_chunks(light_n)) * 4;
        if (ctx->dict_small.bytes < fixed + hist_bytes) {
            // keep the scratch written so far: grow into a fresh buffer and copy it over
            DevBuf grown;
            e = grown.reserve(fixed + hist_bytes, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(grown.ptr, ctx->dict_small.ptr, fixed, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) {
                grown.release(st);
                return ctx_cuda(ctx, e, "search_many sort");
            }
            ctx->dict_small.release(st);
            ctx->dict_small = grown;
            m = scratch_at((uint8_t *)ctx->dict_small.ptr);
        }
        e = launch_dict_sort(keys, keys + cap, light_n, 32 + bits_for(U - 1), m.sort_hist, m.sort_totals, st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "search_many sort");
    }
    DictEmitArgs ea{};
    ea.n_ids = n;
    ea.n_u = U;
    ea.n_heavy = H;
    ea.n_words = n_words;
    ea.u_of_id = set->u_of_id;
    ea.dup_start = set->dup_start;
    ea.dup_ids = set->dup_ids;
    ea.heavy_of_u = m.heavy_of_u;
    ea.heavy_u = m.heavy_u;
    ea.heavy_totals = m.heavy_totals;
    ea.heavy_bases = m.heavy_bases;
    ea.ld = hld;
    ea.bitmap = H ? (const uint32_t *)ctx->dict_bitmap.ptr : nullptr;
    ea.light_count = m.light_count;
    ea.light_base = m.light_base;
    ea.light_keys = keys;
    ea.light_n = light_n;
    ea.id_counts = m.id_counts;
    ea.id_base = m.id_base;
    ea.total = m.total;
    e = launch_dict_ids(ea, st);
    order_pass.done();
    unsigned long long tot = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&tot, m.total, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(counts, m.id_counts, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    unsigned long long walk[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(walk, m.stats, 16, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    prof_mark(ctx, "dictionary: wait for the slots");
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "search_many ids");
    *total = tot;
    ctx->dict_stats[0] = N;
    ctx->dict_stats[1] = walk[0];
    ctx->dict_stats[2] = walk[1];
    ctx->dict_stats[3] = H;
    ctx->dict_stats[4] = light_n;
    ctx->dict_stats[5] = tot;

    // 4. Hits.
    const uint64_t k = std::min<uint64_t>(tot, max_hits);
    if (k == 0) return OL_OK;
    ea.max_hits = k;
    const size_t off_at = (k * 4 + 255) & ~(size_t)255;  // pair form in scratch: patterns, then offsets
    if (dest.off && !dest.pair_on_host) {
        ea.hit_pat = dest.pat;
        ea.hit_off = reinterpret_cast<unsigned long long *>(dest.off);
    } else if (dest.dev) {
        ea.hits = reinterpret_cast<uint2 *>(dest.dev);
    } else {
        const size_t need = dest.off ? off_at + k * 8 : k * 8;
        if ((e = ctx->dict_hits.reserve(need, st)) != cudaSuccess) return ctx_cuda(ctx, e, "search_many hits");
        if (dest.off) {
            ea.hit_pat = (uint32_t *)ctx->dict_hits.ptr;
            ea.hit_off = (unsigned long long *)((uint8_t *)ctx->dict_hits.ptr + off_at);
        } else {
            ea.hits = (uint2 *)ctx->dict_hits.ptr;
        }
    }
    {
        GpuPass pass(ctx, "dictionary: emit");
        e = launch_dict_emit(ea, st);
    }
    if (e == cudaSuccess && (dest.host || dest.pair_on_host)) {
        GpuPass pass(ctx, "download");
        if (dest.pair_on_host) {
            e = cudaMemcpyAsync(dest.pat, ea.hit_pat, k * 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(dest.off, ea.hit_off, k * 8, cudaMemcpyDeviceToHost, st);
        } else {
            e = cudaMemcpyAsync(dest.host, ea.hits, k * 8, cudaMemcpyDeviceToHost, st);
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    prof_mark(ctx, "dictionary: emit hits");
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "search_many emit");
    return OL_OK;
}

extern "C" ol_status ol_search_many(ol_ctx *ctx, const ol_doc *d, const ol_patset *set, uint64_t max_hits,
                                    uint32_t *counts, uint64_t *total_hits, ol_hit *hits) {
    if (!ctx || !d || !set || !counts || !total_hits || (max_hits && !hits)) return OL_ERR_INVALID_ARG;
    if (set->ctx != ctx) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "pattern set belongs to another context");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    HitDest dest;
    dest.host = hits;
    return many_run(ctx, d, set, max_hits, 0, counts, total_hits, dest, nullptr, nullptr, 0);
}

extern "C" ol_status ol_search_many_device(ol_ctx *ctx, const ol_doc *d, const ol_patset *set, uint64_t max_hits,
                                           uint32_t heavy_min_hits, uint32_t *counts, uint64_t *total_hits,
                                           ol_hit *d_hits) {
    if (!ctx || !d || !set || !counts || !total_hits || (max_hits && !d_hits)) return OL_ERR_INVALID_ARG;
    if (set->ctx != ctx) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "pattern set belongs to another context");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    HitDest dest;
    dest.dev = d_hits;
    return many_run(ctx, d, set, max_hits, heavy_min_hits, counts, total_hits, dest, nullptr, nullptr, 0);
}

extern "C" ol_status ol_search_many_u64(ol_ctx *ctx, const ol_doc *d, const ol_patset *set, uint64_t max_hits,
                                        uint32_t *counts, uint64_t *total_hits, uint32_t *patterns, uint64_t *offsets) {
    if (!ctx || !d || !set || !counts || !total_hits || (max_hits && (!patterns || !offsets))) return OL_ERR_INVALID_ARG;
    if (set->ctx != ctx) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "pattern set belongs to another context");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    HitDest dest;
    dest.pat = patterns;
    dest.off = offsets;
    dest.pair_on_host = true;
    return many_run(ctx, d, set, max_hits, 0, counts, total_hits, dest, nullptr, nullptr, 0);
}

extern "C" ol_status ol_search_many_device_u64(ol_ctx *ctx, const ol_doc *d, const ol_patset *set, uint64_t max_hits,
                                               uint32_t heavy_min_hits, uint32_t *counts, uint64_t *total_hits,
                                               uint32_t *d_patterns, uint64_t *d_offsets) {
    if (!ctx || !d || !set || !counts || !total_hits || (max_hits && (!d_patterns || !d_offsets)))
        return OL_ERR_INVALID_ARG;
    if (((uintptr_t)d_offsets & 7) || ((uintptr_t)d_patterns & 3))
        return ctx_fail(ctx, OL_ERR_INVALID_ARG, "d_offsets must be 8-byte and d_patterns 4-byte aligned");
    if (set->ctx != ctx) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "pattern set belongs to another context");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    HitDest dest;
    dest.pat = d_patterns;
    dest.off = d_offsets;
    return many_run(ctx, d, set, max_hits, heavy_min_hits, counts, total_hits, dest, nullptr, nullptr, 0);
}

extern "C" ol_status ol_dict_stats(ol_ctx *ctx, uint64_t *out) {
    if (!ctx || !out) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    for (int i = 0; i < 6; i++) out[i] = ctx->dict_stats[i];
    return OL_OK;
}
