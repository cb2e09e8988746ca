// C ABI for substring search (GpuParser::search_document / search_raw,
// crates/oneline-gpu/src/search.rs:32-140).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "runtime.h"

using namespace ol;

namespace {

// Enqueues one search over doc; results stay on the device.
cudaError_t enqueue_search(ol_ctx *ctx, const ol_doc *d, const uint8_t *pattern, uint32_t m, uint32_t max_out,
                           uint32_t *d_total, uint32_t *d_out, uint32_t *d_ticket, uint32_t *d_error) {
    cudaStream_t st = ctx->stream;
    uint32_t n_tiles = (uint32_t)((d->text_len + kSearchTile - 1) / kSearchTile);
    cudaError_t e = ctx->scratch_a.reserve((size_t)n_tiles * 8, st);
    if (e == cudaSuccess) e = ctx->pattern_dev.reserve(std::max<size_t>(m, 16), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->scratch_a.ptr, 0, (size_t)n_tiles * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_ticket, 0, 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_total, 0, 4, st);
    // The pattern travels by value through a pageable copy: stream ordered, and
    // the call returns only after the source has been read.
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->pattern_dev.ptr, pattern, m, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    SearchArgs a{};
    a.text = d->text;
    a.text_len = d->text_len;
    a.pattern = (const uint8_t *)ctx->pattern_dev.ptr;
    a.pat_len = m;
    a.n_tiles = n_tiles;
    a.tile_status = (uint64_t *)ctx->scratch_a.ptr;
    a.ticket = d_ticket;
    a.total = d_total;
    a.error = d_error;
    a.out = d_out;
    a.max_out = max_out;
    return launch_search(a, st);
}

ol_status search_doc(ol_ctx *ctx, const ol_doc *d, const uint8_t *pattern, uint32_t m, uint32_t max_matches,
                     uint32_t *total, uint32_t *out) {
    *total = 0;
    if (d->text_len == 0 || d->text_len < m) return OL_OK;
    cudaStream_t st = ctx->stream;
    cudaError_t e = ctx->search_out.reserve((size_t)std::max<uint32_t>(max_matches, 1) * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(&ctx->counters->error, 0, 4, st);
    if (e == cudaSuccess)
        e = enqueue_search(ctx, d, pattern, m, max_matches, &ctx->counters->total, (uint32_t *)ctx->search_out.ptr,
                           &ctx->counters->ticket, &ctx->counters->error);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->host_counters, ctx->counters, sizeof(CtxCounters), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "search");
    if (ctx->host_counters->error & OL_DEVERR_TIMEOUT) return ctx_fail(ctx, OL_ERR_TIMEOUT, "search: a look-back wait timed out");
    *total = ctx->host_counters->total;
    uint32_t n = std::min(*total, max_matches);
    if (n > 0) {
        e = cudaMemcpyAsync(out, ctx->search_out.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "search download");
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
    return search_doc(ctx, d, pattern, pat_len, max_matches, total, out);
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
    if (s == OL_OK) s = search_doc(ctx, d, pattern, pat_len, max_matches, total, out);
    ol_doc_free(d);
    return s;
}

extern "C" ol_status ol_search_async(ol_ctx *ctx, const ol_doc *d, const uint8_t *pattern, uint32_t pat_len,
                                     uint32_t max_matches, uint32_t *d_total, uint32_t *d_out) {
    if (!ctx || !d || !d_total || (max_matches && !d_out)) return OL_ERR_INVALID_ARG;
    if (pat_len == 0 || !pattern) return ctx_fail(ctx, OL_ERR_BAD_PATTERN, "pattern must not be empty");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    if (d->text_len < pat_len) return ctx_cuda(ctx, cudaMemsetAsync(d_total, 0, 4, ctx->stream), "search");
    return ctx_cuda(ctx,
                    enqueue_search(ctx, d, pattern, pat_len, max_matches, d_total, d_out, &ctx->counters->ticket,
                                   &ctx->counters->error),
                    "search");
}
