// C ABI for the node query filter: GpuParser::query_document, query_subtree,
// query_raw and query (crates/oneline-gpu/src/document.rs:94-127, 165-190,
// tree.rs:292-313, query.rs:228-329). Results are QueryResult
// (query.rs:10-19): the true total and the first min(total, max_matches)
// matching line indices, ascending.
#include <cuda_runtime.h>

#include <string>

#include "runtime.h"

using namespace ol;

namespace {

// Runs the filter over lines [lo, hi) of a resident document (or over `nodes`
// when given) and downloads the result.
ol_status run_query(ol_ctx *ctx, const ol_doc *d, const FlatNode *nodes, uint32_t lines, uint32_t lo, uint32_t hi,
                    uint32_t kind, uint32_t depth, uint32_t max_matches, uint32_t *total, uint32_t *out) {
    cudaStream_t st = ctx->stream;
    *total = 0;
    if (hi <= lo) return OL_OK;
    const uint32_t blocks = query_blocks(hi - lo), ld = scan_ld(blocks);
    const size_t small = ((size_t)2 * ld + 4) * 4;
    cudaError_t e = ctx->search_out.reserve(small + (size_t)std::max<uint32_t>(max_matches, 1) * 4, st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "query");
    uint32_t *w = (uint32_t *)ctx->search_out.ptr;
    QueryArgs a{};
    if (!nodes) {
        a.kinds = d->kinds;
        a.depth8 = d->depth8;
        a.text = d->text;
        a.offsets = d->offsets;
        a.text_len = d->text_len;
    }
    a.nodes = nodes;
    a.lines = lines;
    a.lo = lo;
    a.hi = hi;
    a.target_kind = kind;
    a.target_depth = depth;
    a.counts = w;
    a.bases = w + ld;
    a.total = w + 2 * ld;
    a.out = w + 2 * ld + 4;
    a.max_out = max_matches;
    {
        GpuPass pass(ctx, "query");
        e = launch_query(a, st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(total, a.total, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    prof_mark(ctx, "query: wait for the count");
    const uint32_t k = std::min(*total, max_matches);
    if (e == cudaSuccess && k) {
        GpuPass pass(ctx, "download");
        e = cudaMemcpyAsync(out, a.out, (size_t)k * 4, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    prof_mark(ctx, "query: download matches");
    return ctx_cuda(ctx, e, "query");
}

}  // namespace

extern "C" ol_status ol_query_document(ol_ctx *ctx, const ol_doc *d, uint32_t kind, uint32_t depth, uint32_t max_matches,
                                       uint32_t *total, uint32_t *out) {
    if (!ctx || !d || !total || (max_matches && !out)) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return run_query(ctx, d, nullptr, d->line_count, 0, d->line_count, kind, depth, max_matches, total, out);
}

extern "C" ol_status ol_query_subtree(ol_ctx *ctx, const ol_doc *d, const ol_tree *t, uint64_t root, uint32_t kind,
                                      uint32_t depth, uint32_t max_matches, uint32_t *total, uint32_t *out) {
    if (!ctx || !d || !t || !total || (max_matches && !out)) return OL_ERR_INVALID_ARG;
    if (root >= t->line_count || t->line_count != d->line_count)
        return ctx_fail(ctx, OL_ERR_INVALID_ARG,
                        "line " + std::to_string(root) + " is out of range (document has " +
                            std::to_string(d->line_count) + " lines, tree has " + std::to_string(t->line_count) + ")");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    uint32_t end = 0;
    cudaError_t e = cudaMemcpyAsync(&end, (const uint32_t *)t->end_buf.ptr + root, 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "query_subtree");
    return run_query(ctx, d, nullptr, d->line_count, (uint32_t)root, end, kind, depth, max_matches, total, out);
}

extern "C" ol_status ol_query_raw(ol_ctx *ctx, const uint8_t *text, uint64_t len, uint32_t kind, uint32_t depth,
                                  uint32_t max_matches, uint32_t *total, uint32_t *out) {
    if (!ctx || !total || (max_matches && !out) || (len && !text)) return OL_ERR_INVALID_ARG;
    *total = 0;
    if (len > OL_MAX_GPU_INPUT_LEN) return ctx_fail(ctx, OL_ERR_INPUT_TOO_LARGE, "input too large");
    if (len == 0) return OL_OK;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    ol_doc *d = nullptr;
    ol_status s = ol_doc_upload(ctx, text, len, &d);
    if (s == OL_OK) s = ol_query_document(ctx, d, kind, depth, max_matches, total, out);
    ol_doc_free(d);
    return s;
}

extern "C" ol_status ol_query(ol_ctx *ctx, const uint8_t *text, uint64_t len, const uint32_t *offsets, uint64_t n_lines,
                              uint32_t kind, uint32_t depth, uint32_t max_matches, uint32_t *total, uint32_t *out) {
    if (!ctx || !total || (max_matches && !out) || (n_lines && (!offsets || !text))) return OL_ERR_INVALID_ARG;
    *total = 0;
    if (len > OL_MAX_GPU_INPUT_LEN) return ctx_fail(ctx, OL_ERR_INPUT_TOO_LARGE, "input too large");
    if (n_lines == 0) return OL_OK;
    if (len == 0) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "line offsets given for an empty text");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    ol_doc *d = nullptr;
    ol_status s = new_text_doc(ctx, text, len, &d);
    if (s != OL_OK) return s;
    cudaError_t e = ctx->scratch_b.reserve((size_t)n_lines * 4, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->scratch_b.ptr, offsets, (size_t)n_lines * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = ctx->scratch_c.reserve((size_t)n_lines * sizeof(FlatNode), st);
    if (e == cudaSuccess)
        e = launch_classify_lines(d->text, len, (const uint32_t *)ctx->scratch_b.ptr, (uint32_t)n_lines,
                                  (FlatNode *)ctx->scratch_c.ptr, nullptr, st);
    s = ctx_cuda(ctx, e, "query");
    if (s == OL_OK)
        s = run_query(ctx, d, (const FlatNode *)ctx->scratch_c.ptr, (uint32_t)n_lines, 0, (uint32_t)n_lines, kind, depth,
                      max_matches, total, out);
    ol_doc_free(d);
    return s;
}
