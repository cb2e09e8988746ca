// Batches of documents: many documents parsed, linked and searched as one
// resident text. Documents are laid end to end, with a '\n' appended to every
// non-empty document that does not end in one, so every document starts on a
// line of its own and keeps exactly its own lines, kinds and depths. These
// kernels keep the tree links and the search hits from crossing a document
// boundary. The reference has no batch form: it parses one document per call
// (crates/oneline-gpu/src/parser.rs:424-445); the per-document semantics are
// those of core links.rs:52-82 and simd search.rs:259-282.
#include <cuda_runtime.h>

#include <algorithm>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

// line_start[i] = the first line at or after document i's first byte (its
// first line when it has any); line_start[n] = L.
__global__ void batch_line_starts_kernel(const uint32_t *__restrict__ offsets, uint32_t L,
                                         const unsigned long long *__restrict__ seg_start, uint32_t n,
                                         uint32_t *__restrict__ line_start) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) {
        line_start[n] = L;
        return;
    }
    const unsigned long long s = seg_start[i];
    uint32_t lo = 0, hi = L;  // first line with offset >= s
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((unsigned long long)__ldg(offsets + mid) < s)
            lo = mid + 1;
        else
            hi = mid;
    }
    line_start[i] = lo;
}

// The document of line j: the last i with line_start[i] <= j among documents
// that have lines (empty documents share their successor's start).
__device__ __forceinline__ uint32_t doc_of_line(const uint32_t *line_start, uint32_t n, uint32_t j) {
    uint32_t lo = 0, hi = n;  // last i in [0, n) with line_start[i] <= j
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(line_start + mid) <= j)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Tree links of the whole text restricted to each line's document: a parent
// before the document becomes NONE, a subtree end past it becomes the
// document's end, a first child past it NONE, and next_sibling is recomputed
// from the restricted links (parents equal after restriction).
//
// It may run in place (outputs = inputs): a thread reads another line's parent
// only inside its own document, where the raw and the restricted parent
// restrict to the same value.
__global__ void batch_tree_fixup_kernel(const uint32_t *__restrict__ line_start, uint32_t n, uint32_t L,
                                        const uint8_t *__restrict__ kinds, const uint32_t *parent_in,
                                        const uint32_t *end_in, const uint32_t *fc_in, uint32_t *parent,
                                        uint32_t *subtree_end, uint32_t *first_child, uint32_t *next_sibling) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= L) return;
    const uint32_t d = doc_of_line(line_start, n, j);
    const uint32_t ls = __ldg(line_start + d), le = __ldg(line_start + d + 1);  // d is the last start <= j
    auto clamp_parent = [&](uint32_t p) { return (p != NONE && p >= ls) ? p : NONE; };
    const uint32_t p = clamp_parent(parent_in[j]);
    const uint32_t e = min(end_in[j], le);
    const uint32_t f = fc_in[j];
    uint32_t ns = NONE;
    // blank lines have no siblings; otherwise the end is a sibling when it lies
    // in the document and the restricted parents agree
    if (__ldg(kinds + j) != KIND_BLANK && e < le && clamp_parent(parent_in[e]) == p) ns = e;
    parent[j] = p;
    subtree_end[j] = e;
    first_child[j] = (f != NONE && f < le) ? f : NONE;
    next_sibling[j] = ns;
}

// Documents of a parsed, linked batch copied into their own resident buffers,
// all in one launch. Work item k of document i covers its text bytes
// [k * 4096, +4096) and its lines [k * 1024, +1024); offsets lose the
// document's first byte, tree links its first line (NONE stays NONE), and
// max_depth[i] receives the document's deepest non-blank line (from depth8,
// so 255 stands for 255 or more).
constexpr uint32_t kSplitBytes = 4096, kSplitLines = 1024;

__global__ void batch_split_kernel(const BatchSplitDoc *__restrict__ docs, const uint32_t *__restrict__ item_start,
                                   uint32_t n, BatchSplitSrc src, uint32_t *__restrict__ max_depth) {
    const uint32_t item = blockIdx.x;
    uint32_t lo = 0, hi = n;  // the last document i with item_start[i] <= item
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(item_start + mid) <= item)
            lo = mid;
        else
            hi = mid;
    }
    const BatchSplitDoc d = docs[lo];
    const uint32_t k = item - __ldg(item_start + lo);
    const uint64_t b0 = (uint64_t)k * kSplitBytes;
    for (uint64_t j = b0 + threadIdx.x; j < d.text_len && j < b0 + kSplitBytes; j += blockDim.x)
        d.text[j] = src.text[d.text_start + j];
    const uint32_t l0 = k * kSplitLines;
    uint32_t deepest = 0;
    for (uint32_t j = l0 + threadIdx.x; j < d.lines && j < l0 + kSplitLines; j += blockDim.x) {
        const uint32_t g = d.first_line + j;
        const uint8_t kind = src.kinds[g], depth = src.depth8[g];
        d.offsets[j] = src.offsets[g] - (uint32_t)d.text_start;
        d.kinds[j] = kind;
        d.depth8[j] = depth;
        if (kind != KIND_BLANK) deepest = max(deepest, (uint32_t)depth);
        auto rebase = [&](uint32_t v) { return v == NONE ? NONE : v - d.first_line; };
        d.parent[j] = rebase(src.parent[g]);
        d.subtree_end[j] = rebase(src.subtree_end[g]);
        d.first_child[j] = rebase(src.first_child[g]);
        d.next_sibling[j] = rebase(src.next_sibling[g]);
    }
    for (int o = 16; o > 0; o >>= 1) deepest = max(deepest, __shfl_xor_sync(0xFFFFFFFFu, deepest, o));
    if ((threadIdx.x & 31) == 0 && deepest) atomicMax(max_depth + lo, deepest);
}

// Item `blockIdx.x` of the documents' items (item_start: the prefix sum of
// batch_pack_items): the document's bytes [64 KiB k, 64 KiB (k + 1)), and its
// separator in its last item.
__global__ void batch_pack_kernel(const BatchPackDoc *__restrict__ docs, const uint32_t *__restrict__ item_start,
                                  uint32_t n, const uint8_t *__restrict__ in, uint8_t *__restrict__ text) {
    const uint32_t item = blockIdx.x;
    uint32_t lo = 0, hi = n;  // the last document i with item_start[i] <= item
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(item_start + mid) <= item)
            lo = mid;
        else
            hi = mid;
    }
    const BatchPackDoc d = docs[lo];
    const uint64_t b0 = (uint64_t)(item - __ldg(item_start + lo)) * kBatchPackBytes;
    const uint64_t b1 = min(d.len, b0 + kBatchPackBytes);
    const uint8_t *src = in + d.src;
    uint8_t *dst = text + d.dst;
    for (uint64_t j = b0 + threadIdx.x; j < b1; j += blockDim.x) dst[j] = src[j];
    if (d.sep && threadIdx.x == 0 && b0 + kBatchPackBytes >= d.len) dst[d.len] = '\n';
}

uint32_t batch_pack_items(uint64_t len) { return (uint32_t)std::max<uint64_t>((len + kBatchPackBytes - 1) / kBatchPackBytes, 1); }

cudaError_t launch_batch_pack(const BatchPackDoc *docs, const uint32_t *item_start, uint32_t n, uint32_t items,
                              const uint8_t *in, uint8_t *text, cudaStream_t st) {
    if (n == 0 || items == 0) return cudaSuccess;
    batch_pack_kernel<<<items, 256, 0, st>>>(docs, item_start, n, in, text); OL_LAUNCHED();
    return cudaGetLastError();
}

uint32_t batch_split_items(uint64_t text_len, uint32_t lines) {
    const uint64_t a = (text_len + kSplitBytes - 1) / kSplitBytes, b = (lines + kSplitLines - 1) / kSplitLines;
    return (uint32_t)std::max<uint64_t>(std::max(a, b), 1);
}

cudaError_t launch_batch_split(const BatchSplitDoc *docs, const uint32_t *item_start, uint32_t n, uint32_t items,
                               const BatchSplitSrc &src, uint32_t *max_depth, cudaStream_t st) {
    if (n == 0 || items == 0) return cudaSuccess;
    batch_split_kernel<<<items, 256, 0, st>>>(docs, item_start, n, src, max_depth); OL_LAUNCHED();
    return cudaGetLastError();
}

cudaError_t launch_batch_line_starts(const uint32_t *offsets, uint32_t L, const unsigned long long *seg_start, uint32_t n,
                                     uint32_t *line_start, cudaStream_t st) {
    batch_line_starts_kernel<<<(n + 1 + 255) / 256, 256, 0, st>>>(offsets, L, seg_start, n, line_start); OL_LAUNCHED();
    return cudaGetLastError();
}

cudaError_t launch_batch_tree_fixup(const uint32_t *line_start, uint32_t n, uint32_t L, const uint8_t *kinds,
                                    const uint32_t *parent_in,
                                    const uint32_t *end_in, const uint32_t *fc_in, uint32_t *parent, uint32_t *subtree_end,
                                    uint32_t *first_child, uint32_t *next_sibling, cudaStream_t st) {
    if (L == 0 || n == 0) return cudaSuccess;
    batch_tree_fixup_kernel<<<(L + 255) / 256, 256, 0, st>>>(line_start, n, L, kinds, parent_in, end_in, fc_in, parent,
                                                             subtree_end, first_child, next_sibling); OL_LAUNCHED();
    return cudaGetLastError();
}

}  // namespace ol
