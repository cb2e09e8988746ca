// C ABI for batches of documents (no reference counterpart: the reference
// parses, links and searches one document per call, parser.rs:424-445,
// tree.rs:34-67, many.rs:391-399). A batch lays its documents end to end in
// one resident text, with a '\n' after every non-empty document that lacks
// one, so that every document's lines, kinds and depths are exactly its own;
// one parse, one tree build and one dictionary pass then cover all documents,
// and batch kernels keep tree links and hits inside their document.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "runtime.h"

using namespace ol;

struct ol_batch {
    ol_ctx *ctx = nullptr;
    ol_doc *doc = nullptr;        // the concatenated text, parsed
    ol_tree *tree = nullptr;      // per-document links once built
    uint32_t n = 0;
    std::vector<uint64_t> start;  // document i: bytes [start[i], start[i] + len[i]) of the text
    std::vector<uint64_t> len;
    std::vector<uint32_t> line_start;  // n + 1 entries
    DevBuf table;                 // device: seg_start[n], seg_end[n] (u64), line_start[n + 1] (u32)
    const unsigned long long *seg_start = nullptr, *seg_end = nullptr;
    uint32_t *d_line_start = nullptr;
};

namespace {

// Lays n documents end to end, each non-empty one that does not end in '\n'
// followed by one: their starts and lengths go to b; returns the text length.
uint64_t batch_layout(ol_batch *b, const uint8_t *const *parts, const uint64_t *lens, uint32_t n) {
    b->n = n;
    b->start.resize(n);
    b->len.resize(n);
    uint64_t T = 0;
    for (uint32_t i = 0; i < n; i++) {
        const uint64_t l = lens[i];
        b->start[i] = T;
        b->len[i] = l;
        T += l + ((l && parts[i][l - 1] != '\n') ? 1 : 0);
    }
    return T;
}

bool needs_separator(const ol_batch *b, uint32_t i) {
    const uint64_t next = i + 1 < b->n ? b->start[i + 1] : b->doc->text_len;
    return next > b->start[i] + b->len[i];
}

// Fills the batch text through the pinned ring (any host memory): documents
// and separators packed on the host, 16 MiB per copy.
cudaError_t batch_fill_ring(ol_ctx *ctx, ol_batch *b, const uint8_t *const *parts) {
    cudaStream_t st = ctx->stream;
    uint64_t at = 0, ring_i = 0, fill = 0;
    uint8_t *slot = nullptr;
    auto flush = [&]() -> cudaError_t {
        if (!fill) return cudaSuccess;
        int k = (int)(ring_i % kRingSlots);
        cudaError_t r = cudaMemcpyAsync(b->doc->text + at, slot, fill, cudaMemcpyHostToDevice, st);
        if (r == cudaSuccess) r = cudaEventRecord(ctx->ring_done[k], st);
        at += fill;
        fill = 0;
        ring_i++;
        slot = nullptr;
        return r;
    };
    auto put = [&](const uint8_t *src, uint64_t nbytes) -> cudaError_t {
        while (nbytes) {
            if (!slot) {
                int k = (int)(ring_i % kRingSlots);
                cudaError_t r = cudaEventSynchronize(ctx->ring_done[k]);
                if (r != cudaSuccess) return r;
                slot = ctx->ring[k];
            }
            const uint64_t c = std::min<uint64_t>(nbytes, kRingBytes - fill);
            memcpy(slot + fill, src, c);
            fill += c;
            src += c;
            nbytes -= c;
            if (fill == kRingBytes) {
                cudaError_t r = flush();
                if (r != cudaSuccess) return r;
            }
        }
        return cudaSuccess;
    };
    static const uint8_t nl = '\n';
    cudaError_t e = cudaSuccess;
    for (uint32_t i = 0; e == cudaSuccess && i < b->n; i++) {
        if (b->len[i]) e = put(parts[i], b->len[i]);
        if (e == cudaSuccess && needs_separator(b, i)) e = put(&nl, 1);
    }
    if (e == cudaSuccess) e = flush();
    return e;
}

// Fills the batch text from page-locked host memory: the documents' bytes
// [in_off[0], in_off[n]) of data cross PCIe in one copy as they lie, then
// batch_pack_kernel moves every document to its place and writes its
// separator, so the host copies nothing.
cudaError_t batch_fill_pinned(ol_ctx *ctx, ol_batch *b, const uint8_t *data, const uint64_t *in_off) {
    cudaStream_t st = ctx->stream;
    const uint32_t n = b->n;
    const uint64_t in_bytes = in_off[n] - in_off[0];
    std::vector<BatchPackDoc> docs(n);
    std::vector<uint32_t> item_start(n + 1);
    uint64_t items = 0;
    for (uint32_t i = 0; i < n; i++) {
        docs[i] = BatchPackDoc{in_off[i] - in_off[0], b->start[i], b->len[i], needs_separator(b, i) ? 1u : 0u, 0u};
        item_start[i] = (uint32_t)items;
        items += batch_pack_items(b->len[i]);
    }
    item_start[n] = (uint32_t)items;
    if (items > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    const size_t table = ((size_t)n * sizeof(BatchPackDoc) + (size_t)(n + 1) * 4 + 255) & ~(size_t)255;
    DevBuf tmp;
    cudaError_t e = tmp.reserve(table + std::max<uint64_t>(in_bytes, 16), st);
    uint8_t *base = (uint8_t *)tmp.ptr;
    if (e == cudaSuccess) e = cudaMemcpyAsync(base, docs.data(), (size_t)n * sizeof(BatchPackDoc), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(base + (size_t)n * sizeof(BatchPackDoc), item_start.data(), (size_t)(n + 1) * 4,
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && in_bytes) {
        GpuPass pass(ctx, "batch upload: copy to device");
        e = cudaMemcpyAsync(base + table, data + in_off[0], in_bytes, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) {
        GpuPass pass(ctx, "batch upload: lay out documents");
        e = launch_batch_pack((const BatchPackDoc *)base, (const uint32_t *)(base + (size_t)n * sizeof(BatchPackDoc)), n,
                              (uint32_t)items, base + table, b->doc->text, st);
    }
    tmp.release(st);  // stream-ordered: freed after the pack
    // the pageable tables must stay until their copies are done
    cudaError_t s2 = cudaStreamSynchronize(st);
    return e != cudaSuccess ? e : s2;
}

bool is_page_locked(const void *p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

// Uploads the laid-out documents (from parts, or when `pinned` is set from
// page-locked data at in_off), parses the text and builds the document tables.
ol_status batch_build(ol_ctx *ctx, const uint8_t *const *parts, const uint64_t *lens, uint32_t n, const uint8_t *pinned,
                      const uint64_t *in_off, ol_batch **out) {
    *out = nullptr;
    auto b = new ol_batch();
    b->ctx = ctx;
    const uint64_t T = batch_layout(b, parts, lens, n);
    if (T > OL_MAX_GPU_INPUT_LEN) {
        delete b;
        return ctx_fail(ctx, OL_ERR_INPUT_TOO_LARGE, "batch text of " + std::to_string(T) + " bytes exceeds the 32-bit limit");
    }
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    ol_status s = new_doc(ctx, T, &b->doc);
    cudaError_t e = cudaSuccess;
    if (s == OL_OK) {
        if (pinned) {
            e = batch_fill_pinned(ctx, b, pinned, in_off);
        } else {
            GpuPass pass(ctx, "batch upload: pack on the host and copy");
            e = batch_fill_ring(ctx, b, parts);
        }
    }
    if (s == OL_OK && e != cudaSuccess) s = ctx_cuda(ctx, e, "batch upload");
    prof_mark(ctx, "batch upload: documents in device memory");
    if (s == OL_OK && T) s = parse_doc(ctx, b->doc, T / 24 + 4096, nullptr);
    prof_mark(ctx, "batch upload: parse");
    // Document ranges and first lines on the device.
    const size_t tbytes = (size_t)n * 16 + (size_t)(n + 1) * 4;
    if (s == OL_OK) {
        std::vector<uint8_t> host(tbytes);
        std::vector<uint64_t> ends(n);
        for (uint32_t i = 0; i < n; i++) ends[i] = b->start[i] + b->len[i];
        memcpy(host.data(), b->start.data(), (size_t)n * 8);
        memcpy(host.data() + (size_t)n * 8, ends.data(), (size_t)n * 8);
        e = b->table.reserve(tbytes, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(b->table.ptr, host.data(), (size_t)n * 16, cudaMemcpyHostToDevice, st);
        b->seg_start = (const unsigned long long *)b->table.ptr;
        b->seg_end = b->seg_start + n;
        b->d_line_start = (uint32_t *)((uint8_t *)b->table.ptr + (size_t)n * 16);
        if (e == cudaSuccess)
            e = launch_batch_line_starts(b->doc->offsets, b->doc->line_count, b->seg_start, n, b->d_line_start, st);
        b->line_start.resize(n + 1);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->line_start.data(), b->d_line_start, (size_t)(n + 1) * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) s = ctx_cuda(ctx, e, "batch tables");
        prof_mark(ctx, "batch upload: document tables");
    }
    if (s != OL_OK) {
        ol_batch_free(b);
        return s;
    }
    *out = b;
    return OL_OK;
}

}  // namespace

// The batch of documents parts[i][0 .. lens[i]) (host memory), uploaded and
// parsed (see ol_batch_upload).
ol_status ol::batch_from_parts(ol_ctx *ctx, const uint8_t *const *parts, const uint64_t *lens, uint32_t n,
                               ol_batch **out) {
    return batch_build(ctx, parts, lens, n, nullptr, nullptr, out);
}

extern "C" ol_status ol_batch_upload(ol_ctx *ctx, const uint8_t *data, const uint64_t *doc_offsets, uint32_t n,
                                     ol_batch **out) {
    if (!ctx || !out || !doc_offsets || n == 0) return OL_ERR_INVALID_ARG;
    *out = nullptr;
    for (uint32_t i = 0; i < n; i++)
        if (doc_offsets[i + 1] < doc_offsets[i]) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "document offsets must not decrease");
    if (doc_offsets[n] > doc_offsets[0] && !data) return OL_ERR_INVALID_ARG;
    std::vector<const uint8_t *> parts(n);
    std::vector<uint64_t> lens(n);
    for (uint32_t i = 0; i < n; i++) {
        parts[i] = data ? data + doc_offsets[i] : nullptr;
        lens[i] = doc_offsets[i + 1] - doc_offsets[i];
    }
    // page-locked input crosses PCIe as it lies and is laid out on the device
    const bool pinned = doc_offsets[n] > doc_offsets[0] && is_page_locked(data + doc_offsets[0]) &&
                        is_page_locked(data + doc_offsets[n] - 1);
    return batch_build(ctx, parts.data(), lens.data(), n, pinned ? data : nullptr, doc_offsets, out);
}

extern "C" void ol_batch_free(ol_batch *b) {
    if (!b) return;
    if (b->tree) ol_tree_free(b->tree);
    if (b->doc) ol_doc_free(b->doc);
    if (b->ctx) {
        std::lock_guard<std::recursive_mutex> g(b->ctx->mu);
        cudaSetDevice(b->ctx->device);
        b->table.release(b->ctx->stream);
    }
    delete b;
}

extern "C" uint32_t ol_batch_docs(const ol_batch *b) { return b ? b->n : 0; }

extern "C" uint64_t ol_batch_text_len(const ol_batch *b) { return b && b->doc ? b->doc->text_len : 0; }

extern "C" ol_status ol_batch_doc_info(const ol_batch *b, uint32_t i, uint64_t *text_start, uint64_t *text_len,
                                       uint64_t *first_line, uint64_t *line_count) {
    if (!b || i >= b->n) return OL_ERR_INVALID_ARG;
    if (text_start) *text_start = b->start[i];
    if (text_len) *text_len = b->len[i];
    const uint32_t ls = b->line_start[i], le = b->len[i] ? b->line_start[i + 1] : ls;
    if (first_line) *first_line = ls;
    if (line_count) *line_count = le - ls;
    return OL_OK;
}

extern "C" ol_status ol_batch_build_trees(ol_ctx *ctx, ol_batch *b) {
    if (!ctx || !b || b->ctx != ctx) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    ol_tree *t = nullptr;
    ol_status s = ol_tree_build_reusing(ctx, b->doc, b->tree, 0, &t);  // any depth: each document is checked alone
    b->tree = nullptr;
    if (s != OL_OK) return s;
    b->tree = t;
    const uint32_t L = b->doc->line_count;
    uint32_t *p = (uint32_t *)t->parent_buf.ptr, *e = (uint32_t *)t->end_buf.ptr, *fc = (uint32_t *)t->fc_buf.ptr,
             *ns = (uint32_t *)t->ns_buf.ptr;
    cudaError_t ce;
    {
        GpuPass pass(ctx, "batch: links kept inside documents");
        ce = launch_batch_tree_fixup(b->d_line_start, b->n, L, b->doc->kinds, p, e, fc, p, e, fc, ns, ctx->stream);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
    prof_mark(ctx, "batch: wait for the links");
    return ctx_cuda(ctx, ce, "batch trees");
}

// Lines of document i: offsets relative to the document, kinds, and tree links
// as line indices within the document (NONE stays NONE). Any output may be
// NULL; cap must be at least the document's line count.
extern "C" ol_status ol_batch_read_doc(ol_ctx *ctx, const ol_batch *b, uint32_t i, uint32_t *offsets, uint8_t *kinds,
                                       uint32_t *parent, uint32_t *subtree_end, uint32_t *first_child,
                                       uint32_t *next_sibling, uint64_t cap) {
    if (!ctx || !b || i >= b->n) return OL_ERR_INVALID_ARG;
    uint64_t ls, lc;
    ol_batch_doc_info(b, i, nullptr, nullptr, &ls, &lc);
    if (cap < lc) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "output capacity is smaller than the document's line count");
    if (lc == 0) return OL_OK;
    if ((parent || subtree_end || first_child || next_sibling) && !b->tree)
        return ctx_fail(ctx, OL_ERR_INVALID_ARG, "the batch's trees are not built");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaSuccess;
    struct Part {
        void *dst;
        const void *src;
        size_t elem;
        bool rebase;    // subtract the document's first line / byte
    } parts[6] = {
        {offsets, b->doc->offsets, 4, true},
        {kinds, b->doc->kinds, 1, false},
        {parent, b->tree ? b->tree->parent_buf.ptr : nullptr, 4, true},
        {subtree_end, b->tree ? b->tree->end_buf.ptr : nullptr, 4, true},
        {first_child, b->tree ? b->tree->fc_buf.ptr : nullptr, 4, true},
        {next_sibling, b->tree ? b->tree->ns_buf.ptr : nullptr, 4, true},
    };
    for (auto &p : parts)
        if (p.dst && e == cudaSuccess)
            e = cudaMemcpyAsync(p.dst, (const uint8_t *)p.src + ls * p.elem, lc * p.elem, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "batch read");
    if (offsets)
        for (uint64_t j = 0; j < lc; j++) offsets[j] -= (uint32_t)b->start[i];
    for (int k = 2; k < 6; k++) {
        uint32_t *a = (uint32_t *)parts[k].dst;
        if (!a) continue;
        for (uint64_t j = 0; j < lc; j++)
            if (a[j] != NONE) a[j] -= (uint32_t)ls;
    }
    return OL_OK;
}

// Dictionary search over every document of the batch at once. Hits are
// {pattern, offset in the batch text} in (pattern, offset) order, which is
// (pattern, document, offset) order; no hit crosses a document boundary.
// counts and *total_hits are host outputs, d_hits device memory.
extern "C" ol_status ol_batch_search_many(ol_ctx *ctx, const ol_batch *b, const ol_patset *set, uint64_t max_hits,
                                          uint32_t heavy_min_hits, uint32_t *counts, uint64_t *total_hits,
                                          ol_hit *d_hits) {
    if (!ctx || !b || !set || !counts || !total_hits || (max_hits && !d_hits)) return OL_ERR_INVALID_ARG;
    if (b->ctx != ctx) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "batch belongs to another context");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    HitDest dest;
    dest.dev = d_hits;
    return many_run(ctx, b->doc, set, max_hits, heavy_min_hits, counts, total_hits, dest, b->seg_start,
                    b->seg_end, b->n);
}

// Splits a parsed batch whose trees are built into its documents: each gets
// its own resident document and tree, equal to what ol_doc_upload and
// ol_tree_build of that document alone give, with one copy launch for all of
// them. docs[i] / trees[i] are new handles on ctx (an empty document gets a
// document without lines and a tree of 0 lines).
ol_status ol::batch_split(ol_ctx *ctx, ol_batch *b, std::vector<ol_doc *> &docs, std::vector<ol_tree *> &trees) {
    if (!b->tree) return ctx_fail(ctx, OL_ERR_INVALID_ARG, "batch_split: the batch's trees are not built");
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const uint32_t n = b->n;
    docs.assign(n, nullptr);
    trees.assign(n, nullptr);
    std::vector<BatchSplitDoc> table;
    std::vector<uint32_t> item_start, which;
    uint32_t items = 0;
    ol_status s = OL_OK;
    cudaError_t e = cudaSuccess;
    for (uint32_t i = 0; i < n && s == OL_OK; i++) {
        uint64_t ls, lc;
        ol_batch_doc_info(b, i, nullptr, nullptr, &ls, &lc);
        s = new_doc(ctx, b->len[i], &docs[i]);
        if (s != OL_OK) break;
        trees[i] = new ol_tree();
        trees[i]->ctx = ctx;
        if (b->len[i] == 0) continue;
        ol_doc *d = docs[i];
        s = alloc_lines(ctx, d, lc);
        if (s == OL_OK) s = tree_alloc(ctx, trees[i], (uint32_t)lc);
        if (s != OL_OK) break;
        if ((e = cudaMemsetAsync(d->stats, 0, sizeof(DocStats), st)) != cudaSuccess) break;
        d->line_count = (uint32_t)lc;
        trees[i]->line_count = (uint32_t)lc;
        BatchSplitDoc x;
        x.text_start = b->start[i];
        x.text_len = b->len[i];
        x.first_line = (uint32_t)ls;
        x.lines = (uint32_t)lc;
        x.text = d->text;
        x.offsets = d->offsets;
        x.kinds = d->kinds;
        x.depth8 = d->depth8;
        x.parent = (uint32_t *)trees[i]->parent_buf.ptr;
        x.subtree_end = (uint32_t *)trees[i]->end_buf.ptr;
        x.first_child = (uint32_t *)trees[i]->fc_buf.ptr;
        x.next_sibling = (uint32_t *)trees[i]->ns_buf.ptr;
        table.push_back(x);
        item_start.push_back(items);
        which.push_back(i);
        items += batch_split_items(x.text_len, x.lines);
    }
    const uint32_t m = (uint32_t)table.size();
    std::vector<uint32_t> depth(m, 0);
    if (s == OL_OK && e == cudaSuccess && m) {
        const size_t t_bytes = (size_t)m * sizeof(BatchSplitDoc), i_at = (t_bytes + 15) & ~size_t(15);
        const size_t d_at = (i_at + (size_t)m * 4 + 15) & ~size_t(15);
        e = ctx->scratch_b.reserve(d_at + (size_t)m * 4, st);
        uint8_t *base = (uint8_t *)ctx->scratch_b.ptr;
        if (e == cudaSuccess) e = cudaMemcpyAsync(base, table.data(), t_bytes, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(base + i_at, item_start.data(), (size_t)m * 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(base + d_at, 0, (size_t)m * 4, st);
        BatchSplitSrc src;
        src.text = b->doc->text;
        src.offsets = b->doc->offsets;
        src.kinds = b->doc->kinds;
        src.depth8 = b->doc->depth8;
        src.parent = (const uint32_t *)b->tree->parent_buf.ptr;
        src.subtree_end = (const uint32_t *)b->tree->end_buf.ptr;
        src.first_child = (const uint32_t *)b->tree->fc_buf.ptr;
        src.next_sibling = (const uint32_t *)b->tree->ns_buf.ptr;
        if (e == cudaSuccess) {
            GpuPass pass(ctx, "batch: split into documents");
            e = launch_batch_split((const BatchSplitDoc *)base, (const uint32_t *)(base + i_at), m, items, src,
                                   (uint32_t *)(base + d_at), st);
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(depth.data(), base + d_at, (size_t)m * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (s == OL_OK && e != cudaSuccess) s = ctx_cuda(ctx, e, "batch split");
    if (s != OL_OK) {
        for (auto &t : trees) ol_tree_free(t);
        for (auto &d : docs) ol_doc_free(d);
        docs.clear();
        trees.clear();
        return s;
    }
    for (uint32_t k = 0; k < m; k++) {
        const uint32_t i = which[k];
        docs[i]->max_depth = depth[k];
        trees[i]->deep = depth[k] >= kTreeLevels;
    }
    return OL_OK;
}
