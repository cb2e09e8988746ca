// The parse-then-search pipeline of a resident document as one CUDA graph:
// re-parse (newline count, column scan, tile parse, fix-up), tree links and a
// multi-pattern search, captured once and replayed with a single launch. The
// graph has two branches: the parse and the tree on one private context's
// stream, the search (which reads only the text) on a second one, so the
// search's blocks fill the SMs that the parse's small passes leave idle. No
// reference counterpart (the reference records wgpu command buffers per call,
// crates/oneline-gpu/src/parser.rs).
//
// The graph bakes in device addresses: the document's buffers, the tree's, the
// output buffers, the pattern copies and the scratch memory of a private
// context that only the pipeline uses, so nothing else can move them. The
// document, tree and outputs must outlive the pipeline and keep their sizes
// (replays re-parse the same resident text).
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "runtime.h"

using namespace ol;

struct ol_pipeline {
    ol_ctx *pctx = nullptr;  // private: its scratch is baked into the graph
    ol_ctx *sctx = nullptr;  // private, the search branch's: its own stream and scratch
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    DevBuf patterns;
    uint32_t kernels = 0;    // kernel launches one replay performs
};

namespace {

// The search reads only the text, which the parse does not write: it runs on
// the second context's stream beside the parse and the tree.
cudaError_t enqueue_step(ol_pipeline *p, ol_doc *d, ol_tree *t, const uint8_t *const *hp,
                         const std::vector<const uint8_t *> &dp, const std::vector<uint32_t> &lens,
                         const uint32_t *max_matches, uint32_t *d_totals, uint32_t *const *d_outs) {
    ol_ctx *pctx = p->pctx, *sctx = p->sctx;
    cudaError_t e = cudaEventRecord(p->fork, pctx->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sctx->stream, p->fork, 0);
    if (e == cudaSuccess) e = enqueue_parse(pctx, d);
    if (e == cudaSuccess) e = enqueue_tree(pctx, d, t);
    if (e == cudaSuccess && !dp.empty())
        e = launch_multi(sctx, d, hp, dp.data(), lens.data(), (uint32_t)dp.size(), max_matches, d_totals, d_outs);
    if (e == cudaSuccess) e = cudaEventRecord(p->join, sctx->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(pctx->stream, p->join, 0);
    return e;
}

}  // namespace

extern "C" void ol_pipeline_free(ol_pipeline *p) {
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->pctx) {
        cudaSetDevice(p->pctx->device);
        cudaStreamSynchronize(p->pctx->stream);
        if (p->sctx) cudaStreamSynchronize(p->sctx->stream);
        p->patterns.release(p->pctx->stream);
        if (p->fork) cudaEventDestroy(p->fork);
        if (p->join) cudaEventDestroy(p->join);
        if (p->sctx) ol_ctx_destroy(p->sctx);
        ol_ctx_destroy(p->pctx);
    }
    delete p;
}

extern "C" ol_status ol_pipeline_capture(ol_ctx *ctx, ol_doc *d, ol_tree *t, const uint8_t *const *patterns,
                                         const uint32_t *lens, uint32_t n, const uint32_t *max_matches,
                                         uint32_t *d_totals, uint32_t *const *d_outs, ol_pipeline **out) {
    if (!ctx || !d || !t || !out || (n && (!patterns || !lens || !max_matches || !d_totals || !d_outs)))
        return OL_ERR_INVALID_ARG;
    *out = nullptr;
    if (t->line_count != d->line_count || d->text_len == 0)
        return ctx_fail(ctx, OL_ERR_INVALID_ARG, "the pipeline needs a non-empty document and its built tree");
    for (uint32_t i = 0; i < n; i++) {
        if (!patterns[i] || lens[i] == 0) return ctx_fail(ctx, OL_ERR_BAD_PATTERN, "pattern " + std::to_string(i) + " is empty");
        if (lens[i] > d->text_len)
            return ctx_fail(ctx, OL_ERR_BAD_PATTERN, "pattern " + std::to_string(i) + " is longer than the document");
        if (max_matches[i] && !d_outs[i]) return OL_ERR_INVALID_ARG;
    }
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    // the document and tree were made on ctx's stream
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "pipeline");
    auto p = new ol_pipeline();
    ol_status s = ol_ctx_create(ctx->device, &p->pctx);
    if (s != OL_OK) {
        delete p;
        return ctx_fail(ctx, s, "pipeline: could not create its context");
    }
    ol_ctx *pc = p->pctx;
    pc->tune = ctx->tune;
    s = ol_ctx_create(ctx->device, &p->sctx);
    if (s == OL_OK && (cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming) != cudaSuccess ||
                       cudaEventCreateWithFlags(&p->join, cudaEventDisableTiming) != cudaSuccess))
        s = OL_ERR_CUDA;
    if (s != OL_OK) {
        ol_pipeline_free(p);
        return ctx_fail(ctx, s, "pipeline: could not create its search context");
    }
    p->sctx->tune = ctx->tune;
    // pattern copies, 16-byte aligned
    std::vector<size_t> at(n);
    size_t w = 0;
    for (uint32_t i = 0; i < n; i++) {
        at[i] = w;
        w += (lens[i] + 15) & ~size_t(15);
    }
    std::vector<uint8_t> host(std::max<size_t>(w, 16), 0);
    for (uint32_t i = 0; i < n; i++) memcpy(host.data() + at[i], patterns[i], lens[i]);
    e = p->patterns.reserve(host.size(), pc->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(p->patterns.ptr, host.data(), host.size(), cudaMemcpyHostToDevice, pc->stream);
    std::vector<const uint8_t *> dp(n);
    std::vector<uint32_t> ln(lens, lens + n);
    for (uint32_t i = 0; i < n; i++) dp[i] = (const uint8_t *)p->patterns.ptr + at[i];
    // One plain run sizes every scratch buffer; the capture must then allocate nothing.
    const uint64_t l0 = ol_launch_count();
    if (e == cudaSuccess) e = cudaStreamSynchronize(pc->stream);  // the pattern copies
    if (e == cudaSuccess) e = enqueue_step(p, d, t, patterns, dp, ln, max_matches, d_totals, d_outs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(pc->stream);
    p->kernels = (uint32_t)(ol_launch_count() - l0);
    void *before[8] = {pc->scratch_a.ptr, pc->scratch_b.ptr,   p->sctx->scratch_a.ptr, t->parent_buf.ptr, t->end_buf.ptr,
                       p->patterns.ptr,   pc->parse_slot.ptr, p->sctx->search_stage.ptr};
    if (e == cudaSuccess) e = cudaStreamBeginCapture(pc->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t ce = enqueue_step(p, d, t, patterns, dp, ln, max_matches, d_totals, d_outs);
        e = cudaStreamEndCapture(pc->stream, &p->graph);
        if (ce != cudaSuccess) e = ce;
    }
    void *after[8] = {pc->scratch_a.ptr, pc->scratch_b.ptr,   p->sctx->scratch_a.ptr, t->parent_buf.ptr, t->end_buf.ptr,
                      p->patterns.ptr,   pc->parse_slot.ptr, p->sctx->search_stage.ptr};
    if (e == cudaSuccess && memcmp(before, after, sizeof before) != 0) e = cudaErrorStreamCaptureInvalidated;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, p->graph, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ol_pipeline_free(p);
        return ctx_cuda(ctx, e, "pipeline capture");
    }
    *out = p;
    return OL_OK;
}

extern "C" ol_status ol_pipeline_launch(ol_pipeline *p) {
    if (!p) return OL_ERR_INVALID_ARG;
    cudaSetDevice(p->pctx->device);
    cudaError_t e = cudaGraphLaunch(p->exec, p->pctx->stream);
    return e == cudaSuccess ? OL_OK : OL_ERR_CUDA;
}

extern "C" void *ol_pipeline_stream(const ol_pipeline *p) { return p ? (void *)p->pctx->stream : nullptr; }

extern "C" uint32_t ol_pipeline_kernels(const ol_pipeline *p) { return p ? p->kernels : 0; }

extern "C" ol_status ol_pipeline_sync(ol_pipeline *p) {
    if (!p) return OL_ERR_INVALID_ARG;
    cudaSetDevice(p->pctx->device);
    return cudaStreamSynchronize(p->pctx->stream) == cudaSuccess ? OL_OK : OL_ERR_CUDA;
}
