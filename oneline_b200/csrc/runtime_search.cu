// C ABI for substring search (GpuParser::search_document / search_raw,
// crates/oneline-gpu/src/search.rs:32-140), plus the batched form that
// searches up to eight patterns per pass over the text.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "runtime.h"

using namespace ol;

static uint32_t halo_for(uint32_t m) { return ((m > 0 ? m - 1 : 0) + 15u) & ~15u; }

namespace {

// Enqueues searches of n patterns over doc, at most 8 per launch (longer than
// the staged limit: one per launch). Results stay on the device: d_totals[i]
// and d_outs[i]. Pattern bytes are copied to device memory first.
cudaError_t enqueue_multi(ol_ctx *ctx, const ol_doc *d, const uint8_t *const *pats, const uint32_t *lens, uint32_t n,
                          const uint32_t *max_out, uint32_t *d_totals, uint32_t *const *d_outs) {
    cudaStream_t st = ctx->stream;
    uint32_t n_tiles = (uint32_t)((d->text_len + kSearchTile - 1) / kSearchTile);
    size_t total_bytes = 0;
    for (uint32_t i = 0; i < n; i++) total_bytes += (lens[i] + 15) & ~15u;
    cudaError_t e = ctx->pattern_dev.reserve(std::max<size_t>(total_bytes, 16), st);
    if (e == cudaSuccess) e = ctx->scratch_a.reserve((size_t)scan_ld(n_tiles) * kSearchMaxPatterns * 4 * 2, st);
    if (e != cudaSuccess) return e;
    // Patterns travel through pinned host staging so the copy is truly async
    // and the caller's buffers may be reused once this call returns.
    if (ctx->pat_host_bytes < total_bytes) {
        if (ctx->pat_host) {
            cudaStreamSynchronize(st);
            cudaFreeHost(ctx->pat_host);
        }
        ctx->pat_host = nullptr;
        ctx->pat_host_bytes = 0;
        if ((e = cudaMallocHost((void **)&ctx->pat_host, std::max<size_t>(total_bytes, 4096))) != cudaSuccess) return e;
        ctx->pat_host_bytes = std::max<size_t>(total_bytes, 4096);
    } else {
        // the previous pattern upload must have left the staging buffer
        if ((e = cudaEventSynchronize(ctx->pat_done)) != cudaSuccess) return e;
    }
    std::vector<size_t> at(n);
    size_t w = 0;
    for (uint32_t i = 0; i < n; i++) {
        at[i] = w;
        memcpy(ctx->pat_host + w, pats[i], lens[i]);
        w += (lens[i] + 15) & ~15u;
    }
    uint8_t *dpat = (uint8_t *)ctx->pattern_dev.ptr;
    if ((e = cudaMemcpyAsync(dpat, ctx->pat_host, std::max<size_t>(w, 1), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(ctx->pat_done, st)) != cudaSuccess) return e;
    std::vector<const uint8_t *> dp(n);
    for (uint32_t i = 0; i < n; i++) dp[i] = dpat + at[i];
    return ol::launch_multi(ctx, d, pats, dp.data(), lens, n, max_out, d_totals, d_outs);
}

}  // namespace

// Launches the searches of n patterns already in device memory (dpats[i]; the
// same bytes on the host: hpats[i]) over doc, at most 8 per launch (longer
// than the staged limit: one per launch). Only stream operations: a CUDA
// graph can capture it once the context's scratch is large enough.
cudaError_t ol::launch_multi(ol_ctx *ctx, const ol_doc *d, const uint8_t *const *hpats, const uint8_t *const *dpats,
                             const uint32_t *lens, uint32_t n, const uint32_t *max_out, uint32_t *d_totals,
                             uint32_t *const *d_outs) {
    GpuPass pass(ctx, "search");
    cudaStream_t st = ctx->stream;
    uint32_t n_tiles = (uint32_t)((d->text_len + kSearchTile - 1) / kSearchTile);
    const size_t col_words = (size_t)scan_ld(n_tiles) * kSearchMaxPatterns;  // counts, then bases
    cudaError_t e = ctx->scratch_a.reserve(col_words * 4 * 2, st);
    // staging: kSearchStageCap tile offsets per tile, then the overflow flags
    // then the flagged tiles' count and list
    const size_t stage_bytes = (size_t)n_tiles * kSearchStageCap * 2;
    const size_t list_at = (stage_bytes + n_tiles + 15) & ~size_t(15);
    if (e == cudaSuccess && ctx->tune.search_staged)
        e = ctx->search_stage.reserve(list_at + 16 + (size_t)n_tiles * 4, st);
    if (e != cudaSuccess) return e;
    uint32_t i = 0;
    while (i < n) {
        SearchArgs a{};
        a.text = d->text;
        a.text_len = d->text_len;
        a.n_tiles = n_tiles;
        a.ld = scan_ld(n_tiles);
        a.counts = (uint32_t *)ctx->scratch_a.ptr;
        a.bases = (uint32_t *)ctx->scratch_a.ptr + col_words;
        a.stage = ctx->tune.search_staged ? (uint16_t *)ctx->search_stage.ptr : nullptr;
        a.overflow = (uint8_t *)ctx->search_stage.ptr + stage_bytes;
        a.overflow_n = (uint32_t *)((uint8_t *)ctx->search_stage.ptr + list_at);
        a.overflow_list = a.overflow_n + 4;
        a.stage_cap = kSearchStageCap;
        uint32_t halo = 0;
        bool alone = halo_for(lens[i]) > kSearchMaxStagedPattern;
        uint32_t first = i;
        while (i < n && a.np < kSearchMaxPatterns) {
            bool long_pat = halo_for(lens[i]) > kSearchMaxStagedPattern;
            if (a.np > 0 && (alone || long_pat)) break;
            search_add_pattern(a, hpats[i], dpats[i], lens[i], d_outs[i], max_out[i]);
            halo = std::max(halo, halo_for(lens[i]));
            i++;
            if (alone) break;
        }
        a.halo = halo;
        a.totals = d_totals + first;
        if ((e = launch_search(a, st)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

namespace {

// Blocking multi-pattern search into host buffers.
ol_status search_multi_host(ol_ctx *ctx, const ol_doc *d, const uint8_t *const *pats, const uint32_t *lens, uint32_t n,
                            const uint32_t *max_matches, uint32_t *totals, uint32_t *const *outs) {
    for (uint32_t i = 0; i < n; i++) totals[i] = 0;
    if (d->text_len == 0 || n == 0) return OL_OK;
    cudaStream_t st = ctx->stream;
    // Patterns longer than the text cannot match: skip them.
    std::vector<uint32_t> idx;
    size_t out_words = 0;
    for (uint32_t i = 0; i < n; i++)
        if (lens[i] <= d->text_len) {
            idx.push_back(i);
            out_words += std::max<uint32_t>(max_matches[i], 1);
        }
    if (idx.empty()) return OL_OK;
    cudaError_t e = ctx->search_out.reserve(out_words * 4 + 64 * 4, st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "search");
    uint32_t *dev = (uint32_t *)ctx->search_out.ptr;
    uint32_t *d_totals = dev;  // 64 slots
    std::vector<const uint8_t *> p2;
    std::vector<uint32_t> l2, m2;
    std::vector<uint32_t *> o2;
    size_t w = 64;
    for (uint32_t i : idx) {
        p2.push_back(pats[i]);
        l2.push_back(lens[i]);
        m2.push_back(max_matches[i]);
        o2.push_back(dev + w);
        w += std::max<uint32_t>(max_matches[i], 1);
    }
    for (size_t c = 0; c < idx.size(); c += 64) {
        uint32_t cn = (uint32_t)std::min<size_t>(64, idx.size() - c);
        e = enqueue_multi(ctx, d, p2.data() + c, l2.data() + c, cn, m2.data() + c, d_totals, o2.data() + c);
        uint32_t tot_h[64];
        if (e == cudaSuccess) e = cudaMemcpyAsync(tot_h, d_totals, cn * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        prof_mark(ctx, "search: wait for totals");
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "search");
        {
            GpuPass pass(ctx, "download");
            for (uint32_t j = 0; j < cn; j++) {
                uint32_t i = idx[c + j];
                totals[i] = tot_h[j];
                uint32_t k = std::min(tot_h[j], max_matches[i]);
                if (k > 0 && (e = cudaMemcpyAsync(outs[i], o2[c + j], (size_t)k * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
                    return ctx_cuda(ctx, e, "search download");
            }
        }
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return ctx_cuda(ctx, e, "search download");
        prof_mark(ctx, "search: download matches");
    }
    return OL_OK;
}

}  // namespace

extern "C" ol_status ol_search(ol_ctx *ctx, const ol_doc *d, const uint8_t *pattern, uint32_t pat_len, uint32_t max_matches,
                               uint32_t *total, uint32_t *out) {
    if (!ctx || !d || !total || (max_matches && !out)) return OL_ERR_INVALID_ARG;
    if (pat_len == 0 || !pattern) return ctx_fail(ctx, OL_ERR_BAD_PATTERN, "pattern must not be empty");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return search_multi_host(ctx, d, &pattern, &pat_len, 1, &max_matches, total, &out);
}

extern "C" ol_status ol_search_multi(ol_ctx *ctx, const ol_doc *d, const uint8_t *const *patterns, const uint32_t *lens,
                                     uint32_t n, const uint32_t *max_matches, uint32_t *totals, uint32_t *const *outs) {
    if (!ctx || !d || (n && (!patterns || !lens || !max_matches || !totals || !outs))) return OL_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < n; i++) {
        if (lens[i] == 0 || !patterns[i]) return ctx_fail(ctx, OL_ERR_BAD_PATTERN, "pattern " + std::to_string(i) + " is empty");
        if (max_matches[i] && !outs[i]) return OL_ERR_INVALID_ARG;
    }
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return search_multi_host(ctx, d, patterns, lens, n, max_matches, totals, outs);
}

extern "C" ol_status ol_search_raw(ol_ctx *ctx, const uint8_t *text, uint64_t len, const uint8_t *pattern, uint32_t pat_len,
                                   uint32_t max_matches, uint32_t *total, uint32_t *out) {
    if (!ctx || !total || (max_matches && !out) || (len && !text)) return OL_ERR_INVALID_ARG;
    if (len > OL_MAX_GPU_INPUT_LEN) return ctx_fail(ctx, OL_ERR_INPUT_TOO_LARGE, "input too large");
    if (pat_len == 0 || !pattern) return ctx_fail(ctx, OL_ERR_BAD_PATTERN, "pattern must not be empty");
    *total = 0;
    if (len == 0) return OL_OK;
    ol_doc *d = nullptr;
    // Upload without a line scan: the search needs only the text.
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    ol_status s = new_text_doc(ctx, text, len, &d);
    if (s == OL_OK) s = search_multi_host(ctx, d, &pattern, &pat_len, 1, &max_matches, total, &out);
    ol_doc_free(d);
    return s;
}

extern "C" ol_status ol_search_async(ol_ctx *ctx, const ol_doc *d, const uint8_t *pattern, uint32_t pat_len,
                                     uint32_t max_matches, uint32_t *d_total, uint32_t *d_out) {
    return ol_search_multi_async(ctx, d, &pattern, &pat_len, 1, &max_matches, d_total, &d_out);
}

extern "C" ol_status ol_search_multi_async(ol_ctx *ctx, const ol_doc *d, const uint8_t *const *patterns, const uint32_t *lens,
                                           uint32_t n, const uint32_t *max_matches, uint32_t *d_totals, uint32_t *const *d_outs) {
    if (!ctx || !d || (n && (!patterns || !lens || !max_matches || !d_totals || !d_outs))) return OL_ERR_INVALID_ARG;
    for (uint32_t i = 0; i < n; i++) {
        if (lens[i] == 0 || !patterns[i]) return ctx_fail(ctx, OL_ERR_BAD_PATTERN, "pattern " + std::to_string(i) + " is empty");
        if (max_matches[i] && !d_outs[i]) return OL_ERR_INVALID_ARG;
    }
    if (n == 0) return OL_OK;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    // Patterns that cannot fit in the text report 0 and are not launched.
    std::vector<const uint8_t *> p2;
    std::vector<uint32_t> l2, m2, map;
    std::vector<uint32_t *> o2;
    for (uint32_t i = 0; i < n; i++) {
        if (lens[i] > d->text_len) {
            cudaError_t e = cudaMemsetAsync(d_totals + i, 0, 4, st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "search");
            continue;
        }
        p2.push_back(patterns[i]);
        l2.push_back(lens[i]);
        m2.push_back(max_matches[i]);
        o2.push_back(d_outs[i]);
        map.push_back(i);
    }
    // Launches write totals of consecutive patterns: run maximal runs of kept
    // patterns whose indices are consecutive.
    size_t a = 0;
    while (a < map.size()) {
        size_t b = a + 1;
        while (b < map.size() && map[b] == map[b - 1] + 1) b++;
        cudaError_t e = enqueue_multi(ctx, d, p2.data() + a, l2.data() + a, (uint32_t)(b - a), m2.data() + a,
                                      d_totals + map[a], o2.data() + a);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "search");
        a = b;
    }
    return OL_OK;
}
