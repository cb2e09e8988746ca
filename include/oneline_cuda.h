/* oneline_cuda.h — C ABI of the B200 (sm_100a) parse-and-search engine.
 *
 * Drop-in boundary for the oneline GPU path (tomet-lang/oneline, crate
 * oneline-gpu). Every entry point takes plain pointers and sizes; no C++ or
 * torch types cross it. Each declaration names the reference interface it
 * replaces (file:line within the reference project).
 *
 * Conventions
 *   - Every call returns an ol_status; OL_OK is 0. ol_last_error(ctx) gives a
 *     message for the last failure on that context. A failed call never leaves
 *     the context unusable (crates/oneline-gpu/src/tests.rs:353-373, 571-591).
 *   - Output arrays are caller-allocated with an explicit capacity; true totals
 *     are always returned even when the output was truncated.
 *   - Handles (ol_ctx, ol_doc, ol_tree, ol_patset) are owned by the caller and
 *     freed with the matching *_free / *_destroy call. Calls on one context are
 *     serialized internally; handles may be used from any thread.
 *   - Input text is copied to device memory; the host pointer is not retained.
 */
#ifndef ONELINE_CUDA_H
#define ONELINE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t ol_status;
enum {
    OL_OK = 0,
    OL_ERR_INVALID_ARG = 1,     /* null handle, bad flag, capacity too small where required */
    OL_ERR_INPUT_TOO_LARGE = 2, /* text longer than OL_MAX_GPU_INPUT_LEN (util.rs:8-17) */
    OL_ERR_BAD_PATTERN = 3,     /* empty pattern, bad set size or length (search.rs:41-46, many.rs:159-173) */
    OL_ERR_TOO_DEEP = 4,        /* strict tree build: a content line has depth >= 32 (tree.rs:218-223) */
    OL_ERR_OOM = 5,             /* device allocation failed */
    OL_ERR_ADMISSION = 6,       /* a budgeted store refused the document */
    OL_ERR_TIMEOUT = 7,         /* a bounded device wait ran out */
    OL_ERR_CUDA = 8,            /* any other CUDA runtime error */
    OL_ERR_NOT_FOUND = 9        /* unknown document id in a store */
};

/* NodeKind codes (crates/oneline-core/src/lib.rs:39-51). */
enum {
    OL_KIND_BLANK = 0, OL_KIND_TEXT = 1, OL_KIND_HEADING = 2, OL_KIND_ELEMENT = 3,
    OL_KIND_LIST = 4, OL_KIND_CONNECT = 5, OL_KIND_ORDERED_LIST = 6, OL_KIND_COMMENT = 7
};

#define OL_NONE 0xFFFFFFFFu                  /* crates/oneline-core/src/links.rs:6 */
#define OL_MAX_GPU_INPUT_LEN 0xFFFFFFFCull   /* u32::MAX - 3, crates/oneline-gpu/src/util.rs:8 */
#define OL_MAX_PATTERN_LEN 64u               /* crates/oneline-gpu/src/lib.rs:66 (drop-in search limit) */
#define OL_MAX_PATTERNS 2048u                /* crates/oneline-gpu/src/many.rs:14 (drop-in set limit) */
#define OL_MIN_SET_PATTERN_LEN 4u            /* crates/oneline-gpu/src/many.rs:17 */
#define OL_MAX_SET_PATTERN_LEN 64u           /* crates/oneline-gpu/src/many.rs:18 */
#define OL_MAX_TREE_DEPTH 32u                /* crates/oneline-gpu/src/tree.rs:12 */

/* FlatNode, 16 bytes (crates/oneline-core/src/lib.rs:86-96). */
typedef struct ol_flat_node {
    uint32_t depth;
    uint32_t kind;
    uint32_t span_start;
    uint32_t span_len;
} ol_flat_node;

/* ManyHit (crates/oneline-gpu/src/many.rs:77-82). */
typedef struct ol_hit {
    uint32_t pattern;
    uint32_t offset;
} ol_hit;

typedef struct ol_ctx ol_ctx;
typedef struct ol_doc ol_doc;
typedef struct ol_tree ol_tree;
typedef struct ol_patset ol_patset;

/* ---- context: GpuParser::new / adapter_name (crates/oneline-gpu/src/parser.rs:94-142, 470-479) */
ol_status ol_ctx_create(int32_t device, ol_ctx **out);
void ol_ctx_destroy(ol_ctx *ctx);
const char *ol_last_error(const ol_ctx *ctx);
ol_status ol_ctx_device_name(ol_ctx *ctx, char *buf, size_t cap);
/* Blocks until every operation enqueued on the context's stream is done. */
ol_status ol_ctx_sync(ol_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order work. */
void *ol_ctx_stream(ol_ctx *ctx);
/* Test hook, like the reference's test-only candidate_capacity_cap
 * (crates/oneline-gpu/src/parser.rs:20-23, many.rs:450-458): arms host-side
 * faults for the next operation on ctx that they name, so that error paths run
 * without faulting the GPU. OL_INJECT_DICT_WAIT_TIMEOUT: the next dictionary
 * search's blocks take their bounded-wait timeout branch once their filter
 * copy has landed; the call returns OL_ERR_TIMEOUT and the context stays
 * usable. 0 disarms. */
#define OL_INJECT_DICT_WAIT_TIMEOUT 1u
ol_status ol_ctx_inject(ol_ctx *ctx, uint32_t faults);
/* Kernels this library has launched in this process, over all contexts (every
 * launch counts itself). For benchmarks; no reference counterpart. */
uint64_t ol_launch_count(void);

/* ---- profiling: StageTimer / Profile (crates/oneline-gpu/src/timing.rs:16-124)
 *      behind GpuParser::profile_upload, profile_query_document
 *      (document.rs:136-157), profile_search_document, profile_search_raw
 *      (search.rs:143-173), profile_search_many (many.rs:401-410),
 *      profile_build_tree, profile_build_tree_reusing (tree.rs:69-82) and
 *      profile_query_raw (query.rs:275). Between ol_profile_begin and
 *      ol_profile_end every GPU pass the context enqueues (upload copy, parse,
 *      tree, search, dictionary stages, query, download) is timed by CUDA
 *      events on its stream, and every blocking step marks the host time spent
 *      since the previous mark. ol_profile_end waits for the stream and fills
 *      *out: wall_ns is the host time from begin to the last mark,
 *      gpu_total_ns the sum of the passes (Profile::gpu_total). At most
 *      OL_PROFILE_MAX_STEPS of each are kept. */
#define OL_PROFILE_MAX_STEPS 32
#define OL_PROFILE_LABEL_LEN 40
typedef struct ol_profile_step {
    char label[OL_PROFILE_LABEL_LEN];
    uint64_t ns;
} ol_profile_step;
typedef struct ol_profile {
    uint64_t wall_ns;
    uint64_t gpu_total_ns;
    uint32_t n_host_steps;
    uint32_t n_gpu_passes;
    ol_profile_step host_steps[OL_PROFILE_MAX_STEPS];
    ol_profile_step gpu_passes[OL_PROFILE_MAX_STEPS];
} ol_profile;
ol_status ol_profile_begin(ol_ctx *ctx);
ol_status ol_profile_end(ol_ctx *ctx, ol_profile *out);

/* ---- resident documents: GpuParser::upload, GpuDocument::{line_count,text_len}
 *      (crates/oneline-gpu/src/document.rs:16-90, 111-127) */
ol_status ol_doc_upload(ol_ctx *ctx, const uint8_t *text, uint64_t len, ol_doc **out);
/* Same, for text already in this device's memory (copied device-to-device). */
ol_status ol_doc_upload_device(ol_ctx *ctx, const uint8_t *dev_text, uint64_t len, ol_doc **out);
void ol_doc_free(ol_doc *doc);
uint64_t ol_doc_line_count(const ol_doc *doc);
uint64_t ol_doc_text_len(const ol_doc *doc);
/* Deepest non-blank line (0 for an empty document). */
uint64_t ol_doc_max_depth(const ol_doc *doc);
/* Re-runs the scan + classify kernels over the resident text into the
 * document's own buffers, enqueued on the context stream without waiting. */
ol_status ol_doc_reparse_async(ol_ctx *ctx, ol_doc *doc);
/* Downloads: line_offsets (scan.rs:138-146), kinds (u8 NodeKind per line) and
 * 16-byte nodes (parse.rs:69-80). cap = entries the output can hold; it must be
 * at least the line count. */
ol_status ol_doc_read_offsets(ol_ctx *ctx, const ol_doc *doc, uint32_t *out, uint64_t cap);
ol_status ol_doc_read_kinds(ol_ctx *ctx, const ol_doc *doc, uint8_t *out, uint64_t cap);
ol_status ol_doc_read_nodes(ol_ctx *ctx, const ol_doc *doc, ol_flat_node *out, uint64_t cap);
/* Device pointers of a resident document (valid until ol_doc_free). */
ol_status ol_doc_device_views(const ol_doc *doc, const uint8_t **text, const uint32_t **offsets, const uint8_t **kinds,
                              const uint8_t **depth8);

/* ---- the .olb binary format: FlatTree::save_to_file / open_mmap as planned in
 *      .agents/tasks/phase4-zero-copy-binary-serialization.md:13-36 (64-byte
 *      header "ONELINE\0", version 1, text_len, line_count, section offsets,
 *      CRC-32; then the text, FlatNode[line_count] and u32 line offsets, each
 *      section on a 64-byte boundary). ol_doc_save_olb writes a resident
 *      document's text, nodes and offsets. ol_doc_load_olb maps a file and
 *      makes it a resident document without parsing: the text, offsets and
 *      nodes are copied to the device (by DMA from the mapped pages where they
 *      can be registered) and the kinds and depths come from the nodes. A file
 *      whose header, sections or offsets do not hold together is refused with
 *      OL_ERR_INVALID_ARG; with OL_OLB_VERIFY its checksum is checked too. */
#define OL_OLB_VERIFY 1u
ol_status ol_doc_save_olb(ol_ctx *ctx, const ol_doc *doc, const char *path);
ol_status ol_doc_load_olb(ol_ctx *ctx, const char *path, uint32_t flags, ol_doc **out);

/* ---- one-shot parse: GpuParser::parse_raw, scan_line_offsets, parse(input, offsets)
 *      (crates/oneline-gpu/src/parse.rs:86-125, scan.rs:127-136). *line_count
 *      always receives the true count; outputs are written when cap allows. */
ol_status ol_parse_raw(ol_ctx *ctx, const uint8_t *text, uint64_t len, uint32_t *offsets, ol_flat_node *nodes,
                       uint64_t cap, uint64_t *line_count);
ol_status ol_scan_line_offsets(ol_ctx *ctx, const uint8_t *text, uint64_t len, uint32_t *offsets, uint64_t cap,
                               uint64_t *line_count);
ol_status ol_parse_with_offsets(ol_ctx *ctx, const uint8_t *text, uint64_t len, const uint32_t *offsets,
                                uint64_t n_lines, ol_flat_node *nodes);

/* ---- tree: GpuParser::build_tree / build_tree_reusing / download_links,
 *      GpuTree::line_count (crates/oneline-gpu/src/tree.rs:34-67, 278-290) */
#define OL_TREE_STRICT_DEPTH 1u  /* fail with OL_ERR_TOO_DEEP like the reference when depth >= 32 */
ol_status ol_tree_build(ol_ctx *ctx, const ol_doc *doc, uint32_t flags, ol_tree **out);
/* Reuses `previous`'s buffers when large enough; `previous` is consumed (freed
 * or adopted) whatever the outcome. */
ol_status ol_tree_build_reusing(ol_ctx *ctx, const ol_doc *doc, ol_tree *previous, uint32_t flags, ol_tree **out);
/* Re-runs the tree kernels for `doc` into `tree` (same line count), no wait. */
ol_status ol_tree_rebuild_async(ol_ctx *ctx, const ol_doc *doc, ol_tree *tree);
void ol_tree_free(ol_tree *tree);
uint64_t ol_tree_line_count(const ol_tree *tree);
/* Any output may be NULL. cap must be >= the line count. */
ol_status ol_tree_read(ol_ctx *ctx, const ol_tree *tree, uint32_t *parent, uint32_t *subtree_end, uint32_t *first_child,
                       uint32_t *next_sibling, uint64_t cap);

/* ---- substring search: GpuParser::search_document / search_raw
 *      (crates/oneline-gpu/src/search.rs:84-140). Any pattern length >= 1 is
 *      accepted here (the reference's 64-byte cap is applied by the drop-in
 *      wrappers). out receives the first min(total, max_matches) offsets in
 *      ascending order. */
ol_status ol_search(ol_ctx *ctx, const ol_doc *doc, const uint8_t *pattern, uint32_t pat_len, uint32_t max_matches,
                    uint32_t *total, uint32_t *out);
ol_status ol_search_raw(ol_ctx *ctx, const uint8_t *text, uint64_t len, const uint8_t *pattern, uint32_t pat_len,
                        uint32_t max_matches, uint32_t *total, uint32_t *out);
/* Enqueues the search without waiting: *d_total and d_out are device pointers. */
ol_status ol_search_async(ol_ctx *ctx, const ol_doc *doc, const uint8_t *pattern, uint32_t pat_len,
                          uint32_t max_matches, uint32_t *d_total, uint32_t *d_out);
/* n patterns in one call (up to eight share each pass over the text); per
 * pattern i: totals[i] and the first min(totals[i], max_matches[i]) offsets in
 * outs[i], ascending. Extension of search_document for callers with several
 * patterns (no single reference counterpart; semantics per pattern as above). */
ol_status ol_search_multi(ol_ctx *ctx, const ol_doc *doc, const uint8_t *const *patterns, const uint32_t *lens,
                          uint32_t n, const uint32_t *max_matches, uint32_t *totals, uint32_t *const *outs);
/* Same, enqueued without waiting; d_totals (n entries) and d_outs[i] are device pointers. */
ol_status ol_search_multi_async(ol_ctx *ctx, const ol_doc *doc, const uint8_t *const *patterns, const uint32_t *lens,
                                uint32_t n, const uint32_t *max_matches, uint32_t *d_totals, uint32_t *const *d_outs);

/* ---- node queries: GpuParser::query_document / query_subtree / query_raw /
 *      query (crates/oneline-gpu/src/document.rs:94-127, tree.rs:292-313,
 *      query.rs:228-329). kind: a NodeKind code, 0 for any (the reference maps
 *      None to 0, so Blank cannot be asked for either); depth: OL_ANY_DEPTH for
 *      any. *total receives the number of matching lines, out the first
 *      min(total, max_matches) of them in ascending order (the reference returns
 *      an arbitrary subset when truncated). query_subtree considers lines
 *      [root, subtree_end[root]). */
#define OL_ANY_DEPTH 0xFFFFFFFFu
ol_status ol_query_document(ol_ctx *ctx, const ol_doc *doc, uint32_t kind, uint32_t depth, uint32_t max_matches,
                            uint32_t *total, uint32_t *out);
ol_status ol_query_subtree(ol_ctx *ctx, const ol_doc *doc, const ol_tree *tree, uint64_t root, uint32_t kind,
                           uint32_t depth, uint32_t max_matches, uint32_t *total, uint32_t *out);
ol_status ol_query_raw(ol_ctx *ctx, const uint8_t *text, uint64_t len, uint32_t kind, uint32_t depth,
                       uint32_t max_matches, uint32_t *total, uint32_t *out);
ol_status ol_query(ol_ctx *ctx, const uint8_t *text, uint64_t len, const uint32_t *offsets, uint64_t n_lines,
                   uint32_t kind, uint32_t depth, uint32_t max_matches, uint32_t *total, uint32_t *out);

/* ---- the parse-then-search pipeline as one CUDA graph. No reference
 *      counterpart. Captures, once, a re-parse of the resident document, its
 *      tree links (into `tree`, already built for it) and a search of n
 *      patterns (as ol_search_multi_async: d_totals, d_outs on the device);
 *      ol_pipeline_launch then replays all of it with one graph launch on the
 *      pipeline's own stream; inside the graph the search runs on a second
 *      branch beside the parse and the tree. The pipeline keeps the scratch
 *      memory of two private contexts; the document, tree and output buffers
 *      must outlive it. */
typedef struct ol_pipeline ol_pipeline;
ol_status ol_pipeline_capture(ol_ctx *ctx, ol_doc *doc, ol_tree *tree, const uint8_t *const *patterns,
                              const uint32_t *lens, uint32_t n, const uint32_t *max_matches, uint32_t *d_totals,
                              uint32_t *const *d_outs, ol_pipeline **out);
ol_status ol_pipeline_launch(ol_pipeline *pipeline);
ol_status ol_pipeline_sync(ol_pipeline *pipeline);
/* The stream replays run on (a cudaStream_t), and the kernels one replay launches. */
void *ol_pipeline_stream(const ol_pipeline *pipeline);
uint32_t ol_pipeline_kernels(const ol_pipeline *pipeline);
void ol_pipeline_free(ol_pipeline *pipeline);

/* ---- tuning. No reference counterpart (the reference fixes its workgroup
 *      sizes per shader). Kernel variants a context uses, chosen by measuring
 *      them on a document with ol_autotune and recorded per device (name and SM
 *      count) in a text file that ol_tuning_load reads back. The variants change
 *      speed, never results. */
typedef struct ol_tuning {
    uint32_t dict_slice;          /* dictionary: text positions per warp work item (256, 512, 1024) */
    uint32_t dict_blocks_per_sm;  /* dictionary: resident blocks per SM of the persistent pass (0: all that fit) */
    uint32_t dict_heavy_divisor;  /* dictionary: patterns expected to occur text_len / divisor times or more
                                     are collected as bitmaps */
    uint32_t search_staged;       /* substring search: 1 stages each tile's hits in one pass, 0 counts then
                                     recomputes in the writing pass */
} ol_tuning;
ol_status ol_tuning_get(ol_ctx *ctx, ol_tuning *out);
ol_status ol_tuning_set(ol_ctx *ctx, const ol_tuning *tuning);
/* Times the variants on doc: the dictionary variants with `set` (may be NULL),
 * the search variants with the n patterns (n may be 0). Sets the fastest on
 * ctx, writes them to *out, and records them in the file at `path` (may be
 * NULL) under this device. */
ol_status ol_autotune(ol_ctx *ctx, const ol_doc *doc, const ol_patset *set, const uint8_t *const *patterns,
                      const uint32_t *lens, uint32_t n, const char *path, ol_tuning *out);
/* Sets the variants recorded for this device in `path`; OL_ERR_NOT_FOUND when
 * the file has none. */
ol_status ol_tuning_load(ol_ctx *ctx, const char *path);

/* ---- dictionary search: GpuParser::compile_patterns / search_many,
 *      GpuPatternSet::{len, is_empty} (crates/oneline-gpu/src/many.rs:139-176,
 *      391-399). A set holds 1..OL_MAX_DICT_PATTERNS patterns of
 *      OL_MIN_SET_PATTERN_LEN..OL_MAX_SET_PATTERN_LEN bytes (the reference caps
 *      the count at OL_MAX_PATTERNS; the drop-in wrappers apply that cap).
 *      Results follow ManyResult (many.rs:84-94): counts[i] per pattern, the
 *      total, and the first min(total, max_hits) hits in (pattern, offset)
 *      order, the order of ManyPatterns::find_all (oneline-simd
 *      search.rs:259-282). Identical patterns are reported once per id. `doc`
 *      may be NULL: the compiled set does not depend on the document. */
#define OL_MAX_DICT_PATTERNS 65536u
ol_status ol_patset_compile(ol_ctx *ctx, const ol_doc *doc, const uint8_t *const *patterns, const uint32_t *lens,
                            uint32_t n, ol_patset **out);
void ol_patset_free(ol_patset *set);
uint32_t ol_patset_len(const ol_patset *set);
/* Distinct patterns in the set. */
uint32_t ol_patset_unique(const ol_patset *set);
ol_status ol_search_many(ol_ctx *ctx, const ol_doc *doc, const ol_patset *set, uint64_t max_hits, uint32_t *counts,
                         uint64_t *total_hits, ol_hit *hits);
/* Same, with the hits left in device memory (d_hits holds max_hits entries);
 * counts and *total_hits are host outputs. heavy_min_hits: patterns expected
 * to occur at least this often are collected as bitmaps rather than sorted
 * keys (0: automatic). It changes the speed, never the result. */
ol_status ol_search_many_device(ol_ctx *ctx, const ol_doc *doc, const ol_patset *set, uint64_t max_hits,
                                uint32_t heavy_min_hits, uint32_t *counts, uint64_t *total_hits, ol_hit *d_hits);
/* The same results in the hit form the north-star workload states, (pattern
 * id u32, byte offset u64): hit i is (patterns[i], offsets[i]), two arrays of
 * max_hits entries, in (pattern, offset) order. It extends ManyHit's u32
 * offset (crates/oneline-gpu/src/many.rs:77-82) to 64 bits; the values are
 * the same. ol_search_many_u64 writes host arrays; ol_search_many_device_u64
 * device arrays (d_offsets 8-byte aligned). */
ol_status ol_search_many_u64(ol_ctx *ctx, const ol_doc *doc, const ol_patset *set, uint64_t max_hits, uint32_t *counts,
                             uint64_t *total_hits, uint32_t *patterns, uint64_t *offsets);
ol_status ol_search_many_device_u64(ol_ctx *ctx, const ol_doc *doc, const ol_patset *set, uint64_t max_hits,
                                    uint32_t heavy_min_hits, uint32_t *counts, uint64_t *total_hits,
                                    uint32_t *d_patterns, uint64_t *d_offsets);
/* Work of the last dictionary search on ctx, for tuning and reports: out[0]
 * text bytes, [1] positions walked in the trie (filter and table hits), [2] trie
 * nodes visited, [3] patterns collected as bitmaps, [4] hits collected as sorted
 * keys, [5] total hits. */
ol_status ol_dict_stats(ol_ctx *ctx, uint64_t out[6]);

/* ---- batches of documents. No counterpart in the reference, which handles
 *      one document per call (GpuParser::upload / build_tree / search_many,
 *      parser.rs:424-445, tree.rs:34-67, many.rs:391-399); per document the
 *      results equal those calls'. The n documents are bytes
 *      [doc_offsets[i], doc_offsets[i+1]) of data; they are laid end to end in
 *      one resident text (a '\n' follows every non-empty document that lacks
 *      one), parsed in one pass, linked in one pass, and searched in one pass.
 *      Tree builds accept any depth. */
typedef struct ol_batch ol_batch;
ol_status ol_batch_upload(ol_ctx *ctx, const uint8_t *data, const uint64_t *doc_offsets, uint32_t n, ol_batch **out);
void ol_batch_free(ol_batch *batch);
uint32_t ol_batch_docs(const ol_batch *batch);
/* Bytes of the batch text (documents and separators). */
uint64_t ol_batch_text_len(const ol_batch *batch);
/* Where document i lies: its bytes in the batch text and its lines. */
ol_status ol_batch_doc_info(const ol_batch *batch, uint32_t i, uint64_t *text_start, uint64_t *text_len,
                            uint64_t *first_line, uint64_t *line_count);
/* parent / subtree_end / first_child / next_sibling of every document. */
ol_status ol_batch_build_trees(ol_ctx *ctx, ol_batch *batch);
/* Document i's offsets (from its own first byte), kinds and links (line
 * indices within the document). Any output may be NULL. */
ol_status ol_batch_read_doc(ol_ctx *ctx, const ol_batch *batch, uint32_t i, uint32_t *offsets, uint8_t *kinds,
                            uint32_t *parent, uint32_t *subtree_end, uint32_t *first_child, uint32_t *next_sibling,
                            uint64_t cap);
/* Dictionary search of every document: hits {pattern, offset in the batch
 * text} in (pattern, offset) order, i.e. (pattern, document, offset); no hit
 * crosses a document. counts and *total_hits on the host, d_hits on the device
 * (room for max_hits). */
ol_status ol_batch_search_many(ol_ctx *ctx, const ol_batch *batch, const ol_patset *set, uint64_t max_hits,
                               uint32_t heavy_min_hits, uint32_t *counts, uint64_t *total_hits, ol_hit *d_hits);

/* ---- serving. No counterpart in the reference (one blocking call per
 *      document). A server owns `workers` threads, each with its own context
 *      and stream. Continuous batching: a worker that frees up takes every
 *      request queued at that moment and serves them as one step: parse
 *      requests are admitted against the store budget before any upload
 *      (counting the reservations of requests in flight; refused with
 *      OL_ERR_ADMISSION when they cannot fit), then uploaded, parsed and
 *      linked as one batch; search requests on the same document share one
 *      dictionary pass. Steps of different workers overlap on the device.
 *      Parsed documents (text, line arrays, tree links) stay resident in a
 *      store of at most store_budget bytes: the least recently used idle
 *      documents are evicted to make room. A search names a resident document
 *      (OL_ERR_NOT_FOUND once evicted) and searches it for
 *      1..OL_MAX_DICT_PATTERNS set patterns of OL_MIN_SET_PATTERN_LEN..
 *      OL_MAX_SET_PATTERN_LEN bytes, keeping up to max_hits hits. A request
 *      completes once its results are in host memory (the caller's buffers
 *      when given); each result carries a digest of its outputs, to compare a
 *      request served in a busy mix with the same request alone. */
typedef struct ol_server ol_server;
typedef struct ol_request_result {
    uint64_t id;
    uint32_t kind;        /* 0 parse, 1 search */
    ol_status status;
    uint32_t worker;
    uint32_t pad;
    uint64_t doc_id;      /* parse: the new resident document; search: the document searched */
    uint64_t line_count;  /* parse */
    uint64_t total_hits;  /* search */
    uint64_t digest;      /* parse: offsets, kinds, parent, subtree_end, first_child, next_sibling; search: counts, hits */
    uint64_t submit_ns, start_ns, end_ns;  /* steady clock */
} ol_request_result;
ol_status ol_server_create(int32_t device, uint32_t workers, uint64_t store_budget, uint64_t max_hits, ol_server **out);
/* Same, with flags. OL_SERVER_NO_COALESCE: one request per step (the plain
 * per-request form, for comparison). */
#define OL_SERVER_NO_COALESCE 1u
ol_status ol_server_create_ex(int32_t device, uint32_t workers, uint64_t store_budget, uint64_t max_hits,
                              uint32_t flags, ol_server **out);
/* Where a request's results go (host memory that must stay valid until the
 * request completes). Parse: every array holds `cap` entries and is written
 * when the document's line count fits (any pointer may be NULL). Search:
 * counts[i] for the request's pattern i, and its first min(total, max_hits)
 * hits, pattern = index in the request's list (either pointer may be NULL;
 * max_hits also caps what the digest covers). */
typedef struct ol_parse_dest {
    uint64_t cap;
    uint32_t *offsets;
    uint8_t *kinds;
    uint32_t *parent, *subtree_end, *first_child, *next_sibling;
} ol_parse_dest;
typedef struct ol_search_dest {
    uint64_t max_hits;
    uint32_t *counts;
    ol_hit *hits;
} ol_search_dest;
/* Finishes the queued requests, then frees every resident document. */
void ol_server_destroy(ol_server *server);
/* The text must stay valid until the request completes. */
ol_status ol_server_submit_parse(ol_server *server, const uint8_t *text, uint64_t len, uint64_t *request_id);
ol_status ol_server_submit_search(ol_server *server, uint64_t doc_id, const uint8_t *const *patterns,
                                  const uint32_t *lens, uint32_t n, uint64_t *request_id);
/* The same with the results copied to `dest` (may be NULL). */
ol_status ol_server_submit_parse_to(ol_server *server, const uint8_t *text, uint64_t len, const ol_parse_dest *dest,
                                    uint64_t *request_id);
ol_status ol_server_submit_search_to(ol_server *server, uint64_t doc_id, const uint8_t *const *patterns,
                                     const uint32_t *lens, uint32_t n, const ol_search_dest *dest,
                                     uint64_t *request_id);
/* Blocks until the request is done and returns its result (once). */
ol_status ol_server_wait(ol_server *server, uint64_t request_id, ol_request_result *out);
ol_status ol_server_stats(ol_server *server, uint64_t *resident_docs, uint64_t *resident_bytes, uint64_t *evictions,
                          uint64_t *refusals);
/* While paused, workers finish their current step and take no new request;
 * requests still queue (for draining, and to hand a set of requests to one
 * step). Destroying a paused server serves what is queued first. */
ol_status ol_server_pause(ol_server *server, uint32_t paused);
/* Steps served, requests served, and the most requests one step took. */
ol_status ol_server_steps(ol_server *server, uint64_t *steps, uint64_t *requests, uint64_t *largest_step);

/* ---- substring search that allocates nothing. No counterpart in the
 *      reference: an addition for callers that cannot call cudaMalloc, such as a
 *      serving process whose own allocator reserved the GPU's memory up front, or
 *      a latency-critical loop that must not stall the device on cudaMalloc /
 *      cudaFree. It takes no context: everything is the caller's except one fixed
 *      scratch array of 1 MiB + 256 B inside this library, which every GPU that
 *      loads the library holds until the process exits.
 *
 *   d_text      device text, 16-byte aligned, at most OL_NOALLOC_MAX_TEXT_LEN
 *               bytes; longer texts are refused with OL_ERR_INPUT_TOO_LARGE.
 *   text_cap    bytes readable at d_text, at least OL_NOALLOC_TEXT_CAP(text_len)
 *               (whole 16 KiB tiles plus 64 bytes; what lies past text_len is
 *               read but never matched, so it may hold anything).
 *   pattern     host memory, 1..OL_MAX_PATTERN_LEN bytes, read before return
 *               (its bytes travel in a kernel's arguments): the buffer may be
 *               overwritten as soon as the call returns, pinned or not.
 *   d_total     device u32: the number of occurrences.
 *   d_out       device u32[max_matches]: the first min(total, max_matches)
 *               offsets, ascending (may be NULL when max_matches is 0).
 *   stream      a cudaStream_t (NULL: the legacy default stream); the call only
 *               enqueues, results are ready when the stream reaches them.
 *   err/err_cap optional buffer for a message when the status is not OL_OK.
 *
 * Call it with the device that owns the buffers current. The first call on a
 * device looks up the scratch array's device address (cudaGetSymbolAddress),
 * and so does the first call after the device's context was created anew
 * (cudaDeviceReset); make that first call before any stream capture. Every call on a device uses
 * the same scratch array: calls that overlap on the GPU (on streams with no
 * ordering between them) race and may return wrong results. */
#define OL_NOALLOC_MAX_TEXT_LEN (256ull << 20)
#define OL_NOALLOC_TEXT_CAP(len) ((((uint64_t)(len) + 16383ull) / 16384ull) * 16384ull + 64ull)
ol_status ol_search_noalloc(const uint8_t *d_text, uint64_t text_len, uint64_t text_cap, const uint8_t *pattern,
                            uint32_t pat_len, uint32_t max_matches, uint32_t *d_total, uint32_t *d_out, void *stream,
                            char *err, uint32_t err_cap);

#ifdef __cplusplus
}
#endif
#endif /* ONELINE_CUDA_H */
