// C ABI for tree links (GpuParser::build_tree / build_tree_reusing /
// download_links, crates/oneline-gpu/src/tree.rs:53-290).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "runtime.h"

using namespace ol;

ol_status ol::tree_alloc(ol_ctx *ctx, ol_tree *t, uint32_t L) {
    cudaStream_t st = ctx->stream;
    uint32_t cap = round_lines(std::max<uint32_t>(L, 1));
    if (t->capacity >= cap && t->parent_buf.ptr) return OL_OK;
    t->parent_buf.release(st);
    t->end_buf.release(st);
    t->fc_buf.release(st);
    t->ns_buf.release(st);
    cudaError_t e = t->parent_buf.reserve((size_t)cap * 4, st);
    if (e == cudaSuccess) e = t->end_buf.reserve((size_t)cap * 4, st);
    if (e == cudaSuccess) e = t->fc_buf.reserve((size_t)cap * 4, st);
    if (e == cudaSuccess) e = t->ns_buf.reserve((size_t)cap * 4, st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "allocate tree");
    t->capacity = cap;
    return OL_OK;
}

namespace {

// Enqueues the fast (depth < 32) tree kernels.
cudaError_t enqueue_tree_fast(ol_ctx *ctx, const ol_doc *d, ol_tree *t) {
    cudaStream_t st = ctx->stream;
    uint32_t L = d->line_count;
    uint32_t n_tiles = (L + kTreeTile - 1) / kTreeTile;
    size_t words = (size_t)n_tiles * kTreeLevels;
    cudaError_t e = ctx->scratch_a.reserve(words * 4 * 4, st);
    if (e != cudaSuccess) return e;
    TreeArgs a{};
    a.kinds = d->kinds;
    a.depth8 = d->depth8;
    a.L = L;
    a.n_tiles = n_tiles;
    a.levels = std::min<uint32_t>(d->max_depth + 1, kTreeLevels);
    uint32_t *w = (uint32_t *)ctx->scratch_a.ptr;
    a.tile_last = w;
    a.tile_first = w + words;
    a.in_last = w + 2 * words;
    a.in_first = w + 3 * words;
    a.stats = d->stats;
    a.parent = (uint32_t *)t->parent_buf.ptr;
    a.subtree_end = (uint32_t *)t->end_buf.ptr;
    a.first_child = (uint32_t *)t->fc_buf.ptr;
    a.next_sibling = (uint32_t *)t->ns_buf.ptr;
    return launch_tree_fast(a, st);
}

// Any-depth path: exact depths, 32-ary min tree, per-line searches.
cudaError_t enqueue_tree_deep(ol_ctx *ctx, const ol_doc *d, ol_tree *t) {
    cudaStream_t st = ctx->stream;
    uint32_t L = d->line_count;
    TreeDeepArgs a{};
    a.L = L;
    size_t total = 0;
    uint32_t len = L, n_levels = 0;
    uint32_t lens[8];
    while (true) {
        lens[n_levels++] = len;
        total += (size_t)len * 4;
        if (len <= 1 || n_levels == 8) break;
        len = (len + 31) / 32;
    }
    cudaError_t e = ctx->scratch_c.reserve(total, st);
    if (e != cudaSuccess) return e;
    size_t at = 0;
    for (uint32_t l = 0; l < n_levels; l++) {
        a.levels[l] = (uint32_t *)((uint8_t *)ctx->scratch_c.ptr + at);
        a.level_len[l] = lens[l];
        at += (size_t)lens[l] * 4;
    }
    a.n_levels = n_levels;
    a.keys = a.levels[0];
    e = launch_classify_lines(d->text, d->text_len, d->offsets, L, nullptr, a.levels[0], st);
    if (e != cudaSuccess) return e;
    a.parent = (uint32_t *)t->parent_buf.ptr;
    a.subtree_end = (uint32_t *)t->end_buf.ptr;
    a.first_child = (uint32_t *)t->fc_buf.ptr;
    a.next_sibling = (uint32_t *)t->ns_buf.ptr;
    return launch_tree_deep(a, st);
}

ol_status build(ol_ctx *ctx, const ol_doc *d, ol_tree *t, uint32_t flags, bool wait) {
    uint32_t L = d->line_count;
    t->line_count = L;
    if (L == 0) return OL_OK;
    bool deep = d->max_depth >= kTreeLevels;
    if (deep && (flags & OL_TREE_STRICT_DEPTH))
        return ctx_fail(ctx, OL_ERR_TOO_DEEP,
                        "a content line is nested " + std::to_string(d->max_depth) +
                            " levels deep; the tree kernels track at most 32 levels (0..31)");
    ol_status s = tree_alloc(ctx, t, L);
    if (s != OL_OK) return s;
    t->deep = deep;
    cudaError_t e;
    {
        GpuPass pass(ctx, "tree");
        e = deep ? enqueue_tree_deep(ctx, d, t) : enqueue_tree_fast(ctx, d, t);
    }
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "tree");
    if (!wait) return OL_OK;
    uint32_t err = 0;
    e = cudaMemcpyAsync(&ctx->host_counters->error, &d->stats->error, 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    prof_mark(ctx, "tree: wait for links");
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "tree");
    err = ctx->host_counters->error;
    if (err & OL_DEVERR_DEEP) return ctx_fail(ctx, OL_ERR_CUDA, "tree: depth above the fast path reached the kernels");
    return OL_OK;
}

}  // namespace

// The tree kernels for doc into t (sized for doc's lines), enqueued only: a
// CUDA graph can capture it once t and the context's scratch are large enough.
cudaError_t ol::enqueue_tree(ol_ctx *ctx, const ol_doc *d, ol_tree *t) {
    const uint32_t L = d->line_count;
    t->line_count = L;
    if (L == 0) return cudaSuccess;
    if (tree_alloc(ctx, t, L) != OL_OK) return cudaErrorMemoryAllocation;
    t->deep = d->max_depth >= kTreeLevels;
    return t->deep ? enqueue_tree_deep(ctx, d, t) : enqueue_tree_fast(ctx, d, t);
}

extern "C" ol_status ol_tree_build_reusing(ol_ctx *ctx, const ol_doc *d, ol_tree *previous, uint32_t flags, ol_tree **out) {
    if (!ctx || !d || !out) {
        if (previous) ol_tree_free(previous);
        return OL_ERR_INVALID_ARG;
    }
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    *out = nullptr;
    ol_tree *t = previous ? previous : new ol_tree();
    t->ctx = ctx;
    ol_status s = build(ctx, d, t, flags, true);
    if (s != OL_OK) {
        ol_tree_free(t);
        return s;
    }
    *out = t;
    return OL_OK;
}

extern "C" ol_status ol_tree_build(ol_ctx *ctx, const ol_doc *d, uint32_t flags, ol_tree **out) {
    return ol_tree_build_reusing(ctx, d, nullptr, flags, out);
}

extern "C" ol_status ol_tree_rebuild_async(ol_ctx *ctx, const ol_doc *d, ol_tree *t) {
    if (!ctx || !d || !t) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return build(ctx, d, t, 0, false);
}

extern "C" void ol_tree_free(ol_tree *t) {
    if (!t) return;
    ol_ctx *ctx = t->ctx;
    if (ctx) {
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        cudaSetDevice(ctx->device);
        t->parent_buf.release(ctx->stream);
        t->end_buf.release(ctx->stream);
        t->fc_buf.release(ctx->stream);
        t->ns_buf.release(ctx->stream);
    }
    delete t;
}

extern "C" uint64_t ol_tree_line_count(const ol_tree *t) { return t ? t->line_count : 0; }

extern "C" ol_status ol_tree_read(ol_ctx *ctx, const ol_tree *t, uint32_t *parent, uint32_t *subtree_end,
                                  uint32_t *first_child, uint32_t *next_sibling, uint64_t cap) {
    if (!ctx || !t) return OL_ERR_INVALID_ARG;
    if (cap < t->line_count) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "output capacity is smaller than the line count");
    if (t->line_count == 0) return OL_OK;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    size_t bytes = (size_t)t->line_count * 4;
    cudaError_t e = cudaSuccess;
    struct {
        uint32_t *dst;
        const void *src;
    } parts[4] = {{parent, t->parent_buf.ptr}, {subtree_end, t->end_buf.ptr}, {first_child, t->fc_buf.ptr}, {next_sibling, t->ns_buf.ptr}};
    for (auto &p : parts)
        if (p.dst && e == cudaSuccess) e = cudaMemcpyAsync(p.dst, p.src, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return ctx_cuda(ctx, e, "download tree");
}
