// Host-side state behind the C ABI handles.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/oneline_cuda.h"
#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

constexpr int kRingSlots = 4;
constexpr uint64_t kRingBytes = 16ull << 20;  // 4 x 16 MiB pinned staging ring
constexpr uint64_t kTextPad = kSearchMaxStagedPattern + kParseHalo + 64;

// A device allocation from the stream-ordered pool, grown on demand.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t need, cudaStream_t st);
    void release(cudaStream_t st);
};

struct Prof;

// Small per-context device words (a status word read back by the tree build).
struct CtxCounters {
    uint32_t error;
    uint32_t pad[15];
};

}  // namespace ol

struct ol_ctx {
    int device = 0;
    int sm_count = 0;
    char name[256] = {0};
    cudaStream_t stream = nullptr;
    std::recursive_mutex mu;
    std::string last_error;
    ol::DevBuf scratch_a;  // tile status words
    ol::DevBuf scratch_b;  // second status array / uploaded offsets
    ol::DevBuf scratch_c;  // nodes and other per-call outputs
    ol::DevBuf search_out;
    ol::DevBuf search_stage;  // staged search hits, 16 KiB per text tile
    ol::DevBuf parse_slot;    // staged parse lines, 4 KiB per text tile
    ol_tuning tune{512, 0, 512, 1};  // kernel variants in use (ol_autotune / ol_tuning_set)
    uint64_t dict_stats[6] = {0, 0, 0, 0, 0, 0};  // the last dictionary search (ol_dict_stats)
    uint32_t inject = 0;  // OL_INJECT_* faults armed for the next operation they name (ol_ctx_inject)
    ol::Prof *prof = nullptr;  // open profile (ol_profile_begin), or null
    cudaStream_t copy_stream = nullptr;  // uploads that overlap the parse
    cudaEvent_t copy_ready = nullptr;    // the main stream's work before an upload
    std::vector<cudaEvent_t> chunk_done; // one per upload chunk in flight
    ol::DevBuf pattern_dev;
    ol::DevBuf dict_small;   // dictionary search: per-pattern counts, ranks, slots
    ol::DevBuf dict_bitmap;  // heavy-pattern bitmaps
    ol::DevBuf dict_keys;    // light-hit keys and the sort's second buffer
    ol::DevBuf dict_hits;    // hits of the blocking search before the download
    ol::CtxCounters *counters = nullptr;
    ol::CtxCounters *host_counters = nullptr;  // pinned
    uint8_t *pat_host = nullptr;  // pinned staging for pattern bytes
    size_t pat_host_bytes = 0;
    cudaEvent_t pat_done = nullptr;
    uint8_t *ring[ol::kRingSlots] = {nullptr};
    cudaEvent_t ring_done[ol::kRingSlots] = {nullptr};
};

struct ol_doc {
    ol_ctx *ctx = nullptr;
    uint64_t text_len = 0;
    uint32_t line_count = 0;
    uint32_t max_depth = 0;
    uint32_t line_cap = 0;
    ol::DevBuf text_buf, misc_buf, offsets_buf, kinds_buf, depth8_buf;
    uint8_t *text = nullptr;
    uint32_t *offsets = nullptr;
    uint8_t *kinds = nullptr;
    uint8_t *depth8 = nullptr;
    ol::DocStats *stats = nullptr;
    uint2 *fixup = nullptr;
    ol::DocStats host_stats{};
};

struct ol_tree {
    ol_ctx *ctx = nullptr;
    uint32_t line_count = 0;
    uint32_t capacity = 0;
    bool deep = false;
    ol::DevBuf parent_buf, end_buf, fc_buf, ns_buf;
};

namespace ol {
// Profiling (profile.cu): a GPU pass is timed by CUDA events recorded on the
// context's stream at construction and destruction, when a profile is open;
// prof_mark ends a host step.
struct GpuPass {
    ol_ctx *ctx;
    cudaStream_t stream;
    int index = -1;
    GpuPass(ol_ctx *c, const char *label) : GpuPass(c, label, nullptr) {}
    GpuPass(ol_ctx *c, const char *label, cudaStream_t on);  // on: a stream of ctx (null: its main stream)
    ~GpuPass() { done(); }
    void done();  // ends the pass here instead of at destruction
    GpuPass(const GpuPass &) = delete;
    GpuPass &operator=(const GpuPass &) = delete;
};
void prof_mark(ol_ctx *ctx, const char *label);
void prof_discard(ol_ctx *ctx);

ol_status ctx_fail(ol_ctx *ctx, ol_status code, const std::string &msg);
ol_status ctx_cuda(ol_ctx *ctx, cudaError_t e, const char *what);
uint32_t parse_tiles(uint64_t len);
uint32_t round_lines(uint64_t n);
ol_status new_text_doc(ol_ctx *ctx, const uint8_t *text, uint64_t len, ol_doc **out);
ol_status new_doc(ol_ctx *ctx, uint64_t len, ol_doc **out);
// Parses doc's text and waits (one retry with the exact line count when the
// estimate was low). With host_text, the text is uploaded first, overlapped
// with the parse.
ol_status parse_doc(ol_ctx *ctx, ol_doc *d, uint64_t est_lines, FlatNode **nodes_out,
                    const uint8_t *host_text = nullptr);
cudaError_t enqueue_parse(ol_ctx *ctx, ol_doc *d);
// Copies host bytes to device memory on the context stream (pinned: one DMA;
// pageable: through the pinned staging ring).
cudaError_t h2d(ol_ctx *ctx, uint8_t *dev, const uint8_t *host, uint64_t len);
// Uploads host text into doc (allocated, line arrays reserved) and parses it,
// the copy of each chunk overlapping the stage pass of the chunks before it.
cudaError_t upload_parse_overlapped(ol_ctx *ctx, ol_doc *d, const uint8_t *host, uint64_t len);
cudaError_t enqueue_tree(ol_ctx *ctx, const ol_doc *d, ol_tree *t);
cudaError_t launch_multi(ol_ctx *ctx, const ol_doc *d, const uint8_t *const *hpats, const uint8_t *const *dpats,
                         const uint32_t *lens, uint32_t n, const uint32_t *max_out, uint32_t *d_totals,
                         uint32_t *const *d_outs);
// Sets ctx->tune from the line for ctx's device in the tuning file at path.
ol_status load_tuning(ol_ctx *ctx, const char *path);
// Where a dictionary search puts its hits: ManyHits on the host or the device,
// or the (pattern u32, offset u64) pair of arrays on the host or the device.
struct HitDest {
    ol_hit *host = nullptr;
    ol_hit *dev = nullptr;
    uint32_t *pat = nullptr;
    uint64_t *off = nullptr;
    bool pair_on_host = false;
};
ol_status batch_from_parts(ol_ctx *ctx, const uint8_t *const *parts, const uint64_t *lens, uint32_t n, ol_batch **out);
ol_status batch_split(ol_ctx *ctx, ol_batch *b, std::vector<ol_doc *> &docs, std::vector<ol_tree *> &trees);
uint64_t estimate_lines(const uint8_t *host, uint64_t len);
ol_status alloc_lines(ol_ctx *ctx, ol_doc *d, uint64_t cap_lines);
ol_status tree_alloc(ol_ctx *ctx, ol_tree *t, uint32_t L);
ol_status many_run(ol_ctx *ctx, const ol_doc *d, const ol_patset *set, uint64_t max_hits, uint32_t heavy_min_hits,
                   uint32_t *counts, uint64_t *total, const HitDest &dest,
                   const unsigned long long *seg_start, const unsigned long long *seg_end, uint32_t n_seg);
}  // namespace ol
