// Host runtime behind the C ABI (include/oneline_cuda.h): contexts, resident
// documents, trees and searches. Replaces the wgpu host side of
// crates/oneline-gpu (parser.rs, document.rs, scan.rs, parse.rs, tree.rs,
// search.rs, staging.rs): device memory comes from the stream-ordered
// allocator, uploads go through a pinned staging ring (or straight from
// pinned caller memory), and every public call leaves the context usable on
// error.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/oneline_cuda.h"
#include "ol_common.cuh"
#include "ol_kernels.h"
#include "runtime.h"

using namespace ol;

// ------------------------------------------------------------ utilities ----

namespace ol {

static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

ol_status ctx_fail(ol_ctx *ctx, ol_status code, const std::string &msg) {
    if (ctx) ctx->last_error = msg;
    return code;
}

ol_status ctx_cuda(ol_ctx *ctx, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return OL_OK;
    cudaGetLastError();  // clear a non-sticky error
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return ctx_fail(ctx, OL_ERR_OOM, msg);
    return ctx_fail(ctx, OL_ERR_CUDA, msg);
}

cudaError_t DevBuf::reserve(size_t need, cudaStream_t st) {
    if (need <= bytes) return cudaSuccess;
    release(st);
    void *p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, need, st);
    if (e != cudaSuccess) return e;
    ptr = p;
    bytes = need;
    return cudaSuccess;
}

void DevBuf::release(cudaStream_t st) {
    if (ptr) cudaFreeAsync(ptr, st);
    ptr = nullptr;
    bytes = 0;
}

uint32_t parse_tiles(uint64_t len) { return (uint32_t)((len + kParseTile - 1) / kParseTile); }
uint64_t text_alloc_bytes(uint64_t len) { return (uint64_t)parse_tiles(len) * kParseTile + kTextPad; }
uint32_t round_lines(uint64_t n) { return (uint32_t)std::min<uint64_t>(((n + kTreeTile - 1) / kTreeTile) * kTreeTile, 0xFFFFF000ull); }

// Line-count estimate from four 64 KiB windows (the idea of
// crates/oneline-simd/src/lib.rs:265-277), with head room.
uint64_t estimate_lines(const uint8_t *host, uint64_t len) {
    const uint64_t W = 64 << 10;
    if (len <= 4 * W) {
        uint64_t n = 1;
        for (uint64_t i = 0; i < len; i++) n += host[i] == '\n';
        return n;
    }
    uint64_t nl = 0, span = len - W;
    for (int w = 0; w < 4; w++) {
        const uint8_t *p = host + span / 3 * w;
        for (uint64_t i = 0; i < W; i++) nl += p[i] == '\n';
    }
    double per_byte = (double)(nl + 4) / (double)(4 * W);
    uint64_t est = (uint64_t)(per_byte * (double)len * 1.25) + 4096;
    return std::min<uint64_t>(est, len + 1);
}

}  // namespace ol

// ---------------------------------------------------------------- context --

extern "C" ol_status ol_ctx_create(int32_t device, ol_ctx **out) {
    if (!out) return OL_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return OL_ERR_CUDA;
    if (device < 0 || device >= n) return OL_ERR_INVALID_ARG;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return OL_ERR_CUDA;
    ol_ctx *c = new ol_ctx();
    c->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
        snprintf(c->name, sizeof c->name, "%s", prop.name);
        c->sm_count = prop.multiProcessorCount;
    }
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        delete c;
        return OL_ERR_CUDA;
    }
    if ((e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->copy_ready, cudaEventDisableTiming)) != cudaSuccess) {
        ol_ctx_destroy(c);
        return OL_ERR_CUDA;
    }
    // Keep freed pool memory around: documents come and go.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    e = cudaMallocAsync((void **)&c->counters, sizeof(CtxCounters), c->stream);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->pat_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->host_counters, sizeof(CtxCounters));
    for (int i = 0; i < kRingSlots && e == cudaSuccess; i++) {
        e = cudaMallocHost((void **)&c->ring[i], kRingBytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ring_done[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        ol_ctx_destroy(c);
        return OL_ERR_CUDA;
    }
    // kernel variants recorded for this device by ol_autotune, when the
    // environment names a tuning file (absent file or device: the defaults)
    if (const char *tf = getenv("OL_TUNING_FILE")) load_tuning(c, tf);
    *out = c;
    return OL_OK;
}

extern "C" void ol_ctx_destroy(ol_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->scratch_a.release(ctx->stream);
    ctx->scratch_b.release(ctx->stream);
    ctx->scratch_c.release(ctx->stream);
    ctx->parse_slot.release(ctx->stream);
    ctx->search_out.release(ctx->stream);
    ctx->search_stage.release(ctx->stream);
    ctx->pattern_dev.release(ctx->stream);
    ctx->dict_small.release(ctx->stream);
    ctx->dict_bitmap.release(ctx->stream);
    ctx->dict_keys.release(ctx->stream);
    ctx->dict_hits.release(ctx->stream);
    if (ctx->counters) cudaFreeAsync(ctx->counters, ctx->stream);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->host_counters) cudaFreeHost(ctx->host_counters);
    if (ctx->pat_host) cudaFreeHost(ctx->pat_host);
    if (ctx->pat_done) cudaEventDestroy(ctx->pat_done);
    for (int i = 0; i < kRingSlots; i++) {
        if (ctx->ring[i]) cudaFreeHost(ctx->ring[i]);
        if (ctx->ring_done[i]) cudaEventDestroy(ctx->ring_done[i]);
    }
    prof_discard(ctx);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    for (cudaEvent_t ev : ctx->chunk_done) cudaEventDestroy(ev);
    if (ctx->copy_ready) cudaEventDestroy(ctx->copy_ready);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

extern "C" const char *ol_last_error(const ol_ctx *ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

extern "C" ol_status ol_ctx_device_name(ol_ctx *ctx, char *buf, size_t cap) {
    if (!ctx || !buf || cap == 0) return OL_ERR_INVALID_ARG;
    snprintf(buf, cap, "%s", ctx->name);
    return OL_OK;
}

extern "C" ol_status ol_ctx_sync(ol_ctx *ctx) {
    if (!ctx) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return ctx_cuda(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
}

extern "C" void *ol_ctx_stream(ol_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

extern "C" ol_status ol_ctx_inject(ol_ctx *ctx, uint32_t faults) {
    if (!ctx) return OL_ERR_INVALID_ARG;
    if (faults & ~(uint32_t)OL_INJECT_DICT_WAIT_TIMEOUT) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "unknown fault flag");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    ctx->inject = faults;
    return OL_OK;
}

// --------------------------------------------------------------- upload ----

namespace ol {

// Copies len host bytes to dev. Pinned sources go in one DMA; pageable ones
// through the ring: the copy of chunk i+1 into a pinned slot overlaps the DMA
// of chunk i (crates/oneline-gpu/src/staging.rs:59-117).
cudaError_t h2d(ol_ctx *ctx, uint8_t *dev, const uint8_t *host, uint64_t len) {
    GpuPass pass(ctx, "upload: copy to device");
    cudaPointerAttributes attr;
    cudaError_t e = cudaPointerGetAttributes(&attr, host);
    if (e == cudaSuccess && (attr.type == cudaMemoryTypeHost || attr.type == cudaMemoryTypeManaged))
        return cudaMemcpyAsync(dev, host, len, cudaMemcpyHostToDevice, ctx->stream);
    cudaGetLastError();
    for (uint64_t off = 0, i = 0; off < len; off += kRingBytes, i++) {
        int slot = (int)(i % kRingSlots);
        uint64_t n = std::min<uint64_t>(kRingBytes, len - off);
        if ((e = cudaEventSynchronize(ctx->ring_done[slot])) != cudaSuccess) return e;
        memcpy(ctx->ring[slot], host + off, n);
        if ((e = cudaMemcpyAsync(dev + off, ctx->ring[slot], n, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(ctx->ring_done[slot], ctx->stream)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// The staged parse's arguments for doc, with the context's scratch reserved
// and the document's counters reset (enqueued on the context stream).
static cudaError_t parse_args(ol_ctx *ctx, ol_doc *d, ParseArgs &a) {
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    uint32_t n_tiles = parse_tiles(d->text_len);
    if ((e = ctx->scratch_a.reserve((size_t)scan_ld(n_tiles) * 8, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(d->stats, 0, sizeof(DocStats), st)) != cudaSuccess) return e;
    a = ParseArgs{};
    a.text = d->text;
    a.text_len = d->text_len;
    a.n_tiles = n_tiles;
    a.tile_count = (uint32_t *)ctx->scratch_a.ptr;
    a.tile_base = (uint32_t *)ctx->scratch_a.ptr + scan_ld(n_tiles);  // 16-byte aligned
    a.stats = d->stats;
    a.offsets = d->offsets;
    a.kinds = d->kinds;
    a.depth8 = d->depth8;
    a.line_cap = d->line_cap;
    a.fixup = d->fixup;
    a.fixup_cap = n_tiles;
    // staged form: slots, then the per-tile flags, then the redo count and list
    const size_t slot_bytes = (size_t)n_tiles * kParseSlotCap * 4;
    const size_t list_at = (slot_bytes + n_tiles + 15) & ~size_t(15);
    if ((e = ctx->parse_slot.reserve(list_at + 16 + (size_t)n_tiles * 4, st)) != cudaSuccess) return e;
    uint8_t *ps = (uint8_t *)ctx->parse_slot.ptr;
    a.slot = (uint32_t *)ps;
    a.slot_over = ps + slot_bytes;
    a.redo_n = (uint32_t *)(ps + list_at);
    a.redo_list = a.redo_n + 4;
    a.slot_cap = kParseSlotCap;
    return cudaSuccess;
}

// Enqueues the parse of doc's resident text into its buffers.
cudaError_t enqueue_parse(ol_ctx *ctx, ol_doc *d) {
    GpuPass pass(ctx, "parse");
    ParseArgs a;
    cudaError_t e = parse_args(ctx, d, a);
    return e == cudaSuccess ? launch_parse(a, ctx->stream) : e;
}

// The upload chunk after which the stage pass runs on the tiles that have
// arrived (a 16 MiB ring slot for pageable text).
constexpr uint64_t kOverlapChunk = 32ull << 20;
constexpr size_t kMaxChunksInFlight = 64;

cudaError_t upload_parse_overlapped(ol_ctx *ctx, ol_doc *d, const uint8_t *host, uint64_t len) {
    cudaStream_t st = ctx->stream, cs = ctx->copy_stream;
    cudaError_t e;
    while (ctx->chunk_done.size() < kMaxChunksInFlight) {
        cudaEvent_t ev;
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return e;
        ctx->chunk_done.push_back(ev);
    }
    GpuPass parse_pass(ctx, "parse (overlapped with the upload)");
    ParseArgs a;
    if ((e = parse_args(ctx, d, a)) != cudaSuccess) return e;
    if ((e = launch_parse_begin(a, st)) != cudaSuccess) return e;
    // the copies start after the document's buffers exist on the main stream
    if ((e = cudaEventRecord(ctx->copy_ready, st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(cs, ctx->copy_ready, 0)) != cudaSuccess) return e;
    cudaPointerAttributes attr;
    const bool pinned = cudaPointerGetAttributes(&attr, host) == cudaSuccess &&
                        (attr.type == cudaMemoryTypeHost || attr.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    const uint64_t chunk = pinned ? std::max<uint64_t>(kOverlapChunk, (len + kMaxChunksInFlight - 1) / kMaxChunksInFlight)
                                  : kRingBytes;
    GpuPass copy_pass(ctx, "upload: copy to device", cs);
    uint32_t t0 = 0;
    for (uint64_t off = 0, i = 0; off < len; off += chunk, i++) {
        const uint64_t n = std::min<uint64_t>(chunk, len - off);
        cudaEvent_t landed;
        if (pinned) {
            landed = ctx->chunk_done[i % kMaxChunksInFlight];
            if ((e = cudaMemcpyAsync(d->text + off, host + off, n, cudaMemcpyHostToDevice, cs)) != cudaSuccess) return e;
        } else {
            const int slot = (int)(i % kRingSlots);  // the ring: the copy of chunk i+1 into a pinned slot
            landed = ctx->ring_done[slot];            // overlaps the DMA of chunk i (staging.rs:59-117)
            if ((e = cudaEventSynchronize(landed)) != cudaSuccess) return e;
            memcpy(ctx->ring[slot], host + off, n);
            if ((e = cudaMemcpyAsync(d->text + off, ctx->ring[slot], n, cudaMemcpyHostToDevice, cs)) != cudaSuccess)
                return e;
        }
        if ((e = cudaEventRecord(landed, cs)) != cudaSuccess) return e;
        // tiles whose bytes and halo have landed: (t + 1) * tile + halo <= off + n
        const uint64_t have = off + n;
        const uint32_t t1 = have == len ? a.n_tiles
                                        : (uint32_t)(have >= kParseHalo ? (have - kParseHalo) / kParseTile : 0);
        if (t1 > t0) {
            if ((e = cudaStreamWaitEvent(st, landed, 0)) != cudaSuccess) return e;
            if ((e = launch_parse_tiles(a, t0, t1, st)) != cudaSuccess) return e;
            t0 = t1;
        }
    }
    copy_pass.done();
    return launch_parse_end(a, st);
}

ol_status alloc_lines(ol_ctx *ctx, ol_doc *d, uint64_t cap_lines) {
    cudaStream_t st = ctx->stream;
    uint32_t cap = round_lines(std::max<uint64_t>(cap_lines, 1));
    d->offsets_buf.release(st);
    d->kinds_buf.release(st);
    d->depth8_buf.release(st);
    cudaError_t e = d->offsets_buf.reserve((size_t)cap * 4, st);
    if (e == cudaSuccess) e = d->kinds_buf.reserve(cap, st);
    if (e == cudaSuccess) e = d->depth8_buf.reserve(cap, st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "allocate line arrays");
    d->offsets = (uint32_t *)d->offsets_buf.ptr;
    d->kinds = (uint8_t *)d->kinds_buf.ptr;
    d->depth8 = (uint8_t *)d->depth8_buf.ptr;
    d->line_cap = cap;
    return OL_OK;
}

// Runs the parse (with one exact-size retry when the estimate was too low),
// waits, and records the line count. With nodes_out, the 16-byte nodes are
// materialised into ctx->scratch_c as well.
ol_status parse_doc(ol_ctx *ctx, ol_doc *d, uint64_t est_lines, FlatNode **nodes_out, const uint8_t *host_text) {
    cudaStream_t st = ctx->stream;
    for (int attempt = 0; attempt < 2; attempt++) {
        ol_status s = alloc_lines(ctx, d, est_lines);
        if (s != OL_OK) return s;
        // the first attempt uploads the text as it parses; a retry finds it resident
        cudaError_t e = attempt == 0 && host_text ? upload_parse_overlapped(ctx, d, host_text, d->text_len)
                                                  : enqueue_parse(ctx, d);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&d->host_stats, d->stats, sizeof(DocStats), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return ctx_cuda(ctx, e, "parse");
        const DocStats &hs = d->host_stats;
        if (hs.error & OL_DEVERR_FIXUP) return ctx_fail(ctx, OL_ERR_CUDA, "parse: fix-up list overflow");
        if (hs.error & OL_DEVERR_CAPACITY) {
            est_lines = hs.line_count;  // exact now
            continue;
        }
        d->line_count = hs.line_count;
        d->max_depth = hs.max_content_depth;
        if (nodes_out) {
            e = ctx->scratch_c.reserve((size_t)d->line_cap * sizeof(FlatNode), st);
            if (e == cudaSuccess)
                e = launch_classify_lines(d->text, d->text_len, d->offsets, d->line_count, (FlatNode *)ctx->scratch_c.ptr,
                                          nullptr, st);
            if (e != cudaSuccess) return ctx_cuda(ctx, e, "materialise nodes");
            *nodes_out = (FlatNode *)ctx->scratch_c.ptr;
        }
        return OL_OK;
    }
    return ctx_fail(ctx, OL_ERR_CUDA, "parse: line capacity retry failed");
}

ol_status new_doc(ol_ctx *ctx, uint64_t len, ol_doc **out) {
    if (len > OL_MAX_GPU_INPUT_LEN)
        return ctx_fail(ctx, OL_ERR_INPUT_TOO_LARGE,
                        "input is " + std::to_string(len) + " bytes; the GPU path addresses at most " +
                            std::to_string(OL_MAX_GPU_INPUT_LEN) + " bytes (32-bit offsets)");
    ol_doc *d = new ol_doc();
    d->ctx = ctx;
    d->text_len = len;
    if (len == 0) {
        *out = d;
        return OL_OK;
    }
    cudaStream_t st = ctx->stream;
    uint64_t alloc = text_alloc_bytes(len);
    uint32_t n_tiles = parse_tiles(len);
    cudaError_t e = d->text_buf.reserve(alloc, st);
    if (e == cudaSuccess) e = d->misc_buf.reserve(sizeof(DocStats) + (size_t)n_tiles * sizeof(uint2), st);
    if (e == cudaSuccess) e = cudaMemsetAsync((uint8_t *)d->text_buf.ptr + len, 0, alloc - len, st);
    if (e != cudaSuccess) {
        ol_doc_free(d);
        return ctx_cuda(ctx, e, "allocate document");
    }
    d->text = (uint8_t *)d->text_buf.ptr;
    d->stats = (DocStats *)d->misc_buf.ptr;
    d->fixup = (uint2 *)((uint8_t *)d->misc_buf.ptr + sizeof(DocStats));
    *out = d;
    return OL_OK;
}

}  // namespace ol

static ol_status upload_common(ol_ctx *ctx, const uint8_t *text, uint64_t len, bool device_src, ol_doc **out) {
    if (!ctx || !out || (len && !text)) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    *out = nullptr;
    ol_doc *d = nullptr;
    ol_status s = new_doc(ctx, len, &d);
    if (s != OL_OK) return s;
    if (len == 0) {
        *out = d;
        return OL_OK;
    }
    cudaError_t e;
    uint64_t est;
    if (device_src) {
        e = cudaMemcpyAsync(d->text, text, len, cudaMemcpyDeviceToDevice, ctx->stream);
        est = len / 24 + 4096;  // no host copy to sample; a low guess costs one retry
    } else {
        est = estimate_lines(text, len);
        e = cudaSuccess;
    }
    if (e != cudaSuccess) {
        ol_doc_free(d);
        return ctx_cuda(ctx, e, "upload");
    }
    s = parse_doc(ctx, d, est, nullptr, device_src ? nullptr : text);
    prof_mark(ctx, "upload: wait for parse");
    if (s != OL_OK) {
        ol_doc_free(d);
        return s;
    }
    *out = d;
    return OL_OK;
}

extern "C" ol_status ol_doc_upload(ol_ctx *ctx, const uint8_t *text, uint64_t len, ol_doc **out) {
    return upload_common(ctx, text, len, false, out);
}

extern "C" ol_status ol_doc_upload_device(ol_ctx *ctx, const uint8_t *dev_text, uint64_t len, ol_doc **out) {
    return upload_common(ctx, dev_text, len, true, out);
}

extern "C" void ol_doc_free(ol_doc *d) {
    if (!d) return;
    ol_ctx *ctx = d->ctx;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    d->text_buf.release(ctx->stream);
    d->misc_buf.release(ctx->stream);
    d->offsets_buf.release(ctx->stream);
    d->kinds_buf.release(ctx->stream);
    d->depth8_buf.release(ctx->stream);
    delete d;
}

extern "C" uint64_t ol_doc_line_count(const ol_doc *d) { return d ? d->line_count : 0; }
extern "C" uint64_t ol_doc_text_len(const ol_doc *d) { return d ? d->text_len : 0; }
extern "C" uint64_t ol_doc_max_depth(const ol_doc *d) { return d ? d->max_depth : 0; }

extern "C" ol_status ol_doc_reparse_async(ol_ctx *ctx, ol_doc *d) {
    if (!ctx || !d) return OL_ERR_INVALID_ARG;
    if (d->text_len == 0) return OL_OK;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return ctx_cuda(ctx, enqueue_parse(ctx, d), "reparse");
}

static ol_status read_array(ol_ctx *ctx, const ol_doc *d, void *out, const void *src, size_t elem, uint64_t cap) {
    if (!ctx || !d || (d->line_count && !out)) return OL_ERR_INVALID_ARG;
    if (cap < d->line_count) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "output capacity is smaller than the line count");
    if (d->line_count == 0) return OL_OK;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaError_t e;
    {
        GpuPass pass(ctx, "download");
        e = cudaMemcpyAsync(out, src, (size_t)d->line_count * elem, cudaMemcpyDeviceToHost, ctx->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    prof_mark(ctx, "download");
    return ctx_cuda(ctx, e, "download");
}

extern "C" ol_status ol_doc_read_offsets(ol_ctx *ctx, const ol_doc *d, uint32_t *out, uint64_t cap) {
    return read_array(ctx, d, out, d ? d->offsets : nullptr, 4, cap);
}

extern "C" ol_status ol_doc_read_kinds(ol_ctx *ctx, const ol_doc *d, uint8_t *out, uint64_t cap) {
    return read_array(ctx, d, out, d ? d->kinds : nullptr, 1, cap);
}

extern "C" ol_status ol_doc_read_nodes(ol_ctx *ctx, const ol_doc *d, ol_flat_node *out, uint64_t cap) {
    if (!ctx || !d || (d->line_count && !out)) return OL_ERR_INVALID_ARG;
    if (cap < d->line_count) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "output capacity is smaller than the line count");
    if (d->line_count == 0) return OL_OK;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    cudaError_t e = ctx->scratch_c.reserve((size_t)d->line_count * sizeof(FlatNode), st);
    if (e == cudaSuccess)
        e = launch_classify_lines(d->text, d->text_len, d->offsets, d->line_count, (FlatNode *)ctx->scratch_c.ptr, nullptr, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, ctx->scratch_c.ptr, (size_t)d->line_count * sizeof(FlatNode), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return ctx_cuda(ctx, e, "materialise nodes");
}

extern "C" ol_status ol_doc_device_views(const ol_doc *d, const uint8_t **text, const uint32_t **offsets,
                                         const uint8_t **kinds, const uint8_t **depth8) {
    if (!d) return OL_ERR_INVALID_ARG;
    if (text) *text = d->text;
    if (offsets) *offsets = d->offsets;
    if (kinds) *kinds = d->kinds;
    if (depth8) *depth8 = d->depth8;
    return OL_OK;
}

// ------------------------------------------------------------- one-shot ----

extern "C" ol_status ol_parse_raw(ol_ctx *ctx, const uint8_t *text, uint64_t len, uint32_t *offsets,
                                  ol_flat_node *nodes, uint64_t cap, uint64_t *line_count) {
    if (!ctx || !line_count) return OL_ERR_INVALID_ARG;
    ol_doc *d = nullptr;
    ol_status s;
    {
        if (len > OL_MAX_GPU_INPUT_LEN) return ctx_fail(ctx, OL_ERR_INPUT_TOO_LARGE, "input too large");
        std::lock_guard<std::recursive_mutex> g(ctx->mu);
        cudaSetDevice(ctx->device);
        s = new_doc(ctx, len, &d);
        if (s != OL_OK) return s;
        if (len > 0) {
            cudaError_t e = cudaSuccess;
            FlatNode *dn = nullptr;
            s = parse_doc(ctx, d, estimate_lines(text, len), nodes ? &dn : nullptr, text);  // upload overlapped
            *line_count = d->line_count;
            if (s == OL_OK && d->line_count <= cap && d->line_count > 0) {
                cudaStream_t st = ctx->stream;
                if (offsets) e = cudaMemcpyAsync(offsets, d->offsets, (size_t)d->line_count * 4, cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess && nodes)
                    e = cudaMemcpyAsync(nodes, dn, (size_t)d->line_count * sizeof(FlatNode), cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) s = ctx_cuda(ctx, e, "download");
            }
        } else {
            *line_count = 0;
        }
    }
    ol_doc_free(d);
    return s;
}

extern "C" ol_status ol_scan_line_offsets(ol_ctx *ctx, const uint8_t *text, uint64_t len, uint32_t *offsets, uint64_t cap,
                                          uint64_t *line_count) {
    return ol_parse_raw(ctx, text, len, offsets, nullptr, cap, line_count);
}

extern "C" ol_status ol_parse_with_offsets(ol_ctx *ctx, const uint8_t *text, uint64_t len, const uint32_t *offsets,
                                           uint64_t n_lines, ol_flat_node *nodes) {
    if (!ctx || (n_lines && (!offsets || !nodes))) return OL_ERR_INVALID_ARG;
    if (len > OL_MAX_GPU_INPUT_LEN) return ctx_fail(ctx, OL_ERR_INPUT_TOO_LARGE, "input too large");
    if (n_lines == 0) return OL_OK;
    if (len == 0) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "line offsets given for an empty text");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    ol_doc *d = nullptr;
    ol_status s = new_doc(ctx, len, &d);
    if (s != OL_OK) return s;
    cudaError_t e = h2d(ctx, d->text, text, len);
    if (e == cudaSuccess) e = ctx->scratch_b.reserve((size_t)n_lines * 4, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->scratch_b.ptr, offsets, (size_t)n_lines * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = ctx->scratch_c.reserve((size_t)n_lines * sizeof(FlatNode), st);
    if (e == cudaSuccess)
        e = launch_classify_lines(d->text, len, (const uint32_t *)ctx->scratch_b.ptr, (uint32_t)n_lines,
                                  (FlatNode *)ctx->scratch_c.ptr, nullptr, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(nodes, ctx->scratch_c.ptr, (size_t)n_lines * sizeof(FlatNode), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    s = ctx_cuda(ctx, e, "parse with offsets");
    // free without re-locking
    d->text_buf.release(st);
    d->misc_buf.release(st);
    delete d;
    return s;
}

// A document holding only the uploaded text (no line scan): for one-shot search.
ol_status ol::new_text_doc(ol_ctx *ctx, const uint8_t *text, uint64_t len, ol_doc **out) {
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    ol_doc *d = nullptr;
    ol_status s = new_doc(ctx, len, &d);
    if (s != OL_OK) return s;
    if (len) {
        cudaError_t e = h2d(ctx, d->text, text, len);
        if (e != cudaSuccess) {
            ol_doc_free(d);
            return ctx_cuda(ctx, e, "upload");
        }
    }
    *out = d;
    return OL_OK;
}

extern "C" uint64_t ol_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }
