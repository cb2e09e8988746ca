// Kernel argument blocks and launch entry points shared between the kernels
// (*.cu) and the host runtime (runtime.cu). Device pointers only.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace ol {

// Kernels launched by this library in this process (every launch site counts
// itself), read through ol_launch_count().
void count_launch();
#define OL_LAUNCHED() ::ol::count_launch()

struct FlatNode;
struct DocStats;

constexpr uint32_t kParseTile = 16384;  // text bytes per parse tile
constexpr uint32_t kParseHalo = 256;    // bytes staged past a tile
constexpr uint32_t kTreeTile = 4096;    // lines per tree tile (256 threads x 16)
constexpr uint32_t kTreeLevels = 32;    // depth levels of the fast tree path

struct ParseArgs {
    const uint8_t *text;  // padded: n_tiles * kParseTile + kParseHalo readable bytes
    uint64_t text_len;
    uint32_t n_tiles;
    uint32_t *tile_count;   // n_tiles newline counts (pass 1)
    uint32_t *tile_base;    // n_tiles exclusive prefix sums (pass 2)
    DocStats *stats;        // fixup_count/error zeroed before the launch
    uint32_t *offsets;      // line_cap entries
    uint8_t *kinds;
    uint8_t *depth8;        // min(depth, 255)
    uint32_t line_cap;
    uint2 *fixup;           // (line index, start) of lines longer than the halo
    uint32_t fixup_cap;
    // Staged form (nullptr: count pass + recomputing pass): per tile a slot of
    // slot_cap line words, a flag per tile whose lines did not fit, and the
    // count and list of those tiles.
    uint32_t *slot;
    uint8_t *slot_over;
    uint32_t *redo_n;
    uint32_t *redo_list;
    uint32_t slot_cap;
    uint32_t first_tile;  // staged pass 1: block b takes tile first_tile + b (launches over tile ranges)
};
constexpr uint32_t kParseSlotCap = 1024;  // staged lines per tile

cudaError_t launch_parse(const ParseArgs &a, cudaStream_t st);
// The staged form in three parts, for a parse that starts while the text is
// still arriving: begin (reset the redo list), the stage pass over tiles
// [t0, t1) (any ranges that together cover every tile once, each launched once
// its tiles and their 256-byte halo are in device memory), then end (the scan,
// the copy pass, the redo and fix-up passes).
cudaError_t launch_parse_begin(const ParseArgs &a, cudaStream_t st);
cudaError_t launch_parse_tiles(const ParseArgs &a, uint32_t t0, uint32_t t1, cudaStream_t st);
cudaError_t launch_parse_end(const ParseArgs &a, cudaStream_t st);

// Exclusive scan of each of `cols` columns of a column-major u32 matrix:
// column c is `rows` entries at in + c * ld (in, out 16-byte aligned, ld a
// multiple of 4); out has the same layout; totals[c] (optional) receives
// column c's sum.
cudaError_t launch_scan_columns(const uint32_t *in, uint32_t *out, uint32_t *totals, uint32_t rows, uint32_t cols,
                                uint32_t ld, cudaStream_t st);
// Column stride for per-tile count columns: rows rounded up to a multiple of 4.
inline uint32_t scan_ld(uint32_t rows) { return (rows + 3u) & ~3u; }
cudaError_t launch_classify_lines(const uint8_t *text, uint64_t N, const uint32_t *offsets, uint32_t L, FlatNode *nodes,
                                  uint32_t *depth32, cudaStream_t st);

struct TreeArgs {
    const uint8_t *kinds;
    const uint8_t *depth8;
    uint32_t L;
    uint32_t n_tiles;        // ceil(L / kTreeTile)
    uint32_t levels;         // max content depth + 1 (<= kTreeLevels)
    uint32_t *tile_last;     // n_tiles * kTreeLevels: last content line + 1 of each depth in the tile (0: none)
    uint32_t *tile_first;    // n_tiles * kTreeLevels: first content line of each depth in the tile (NONE: none)
    uint32_t *in_last;       // exclusive prefix max of tile_last over the tiles
    uint32_t *in_first;      // exclusive suffix min of tile_first over the tiles
    DocStats *stats;
    uint32_t *parent;
    uint32_t *subtree_end;   // optional
    uint32_t *first_child;
    uint32_t *next_sibling;
};

cudaError_t launch_tree_fast(const TreeArgs &a, cudaStream_t st);

// Any-depth path (content lines deeper than kTreeLevels-1).
struct TreeDeepArgs {
    const uint32_t *keys;    // depth of content lines, NONE for blank lines
    uint32_t L;
    uint32_t *levels[8];     // levels[0] = keys, levels[k] = min over 32 of levels[k-1]
    uint32_t level_len[8];
    uint32_t n_levels;
    uint32_t *parent;
    uint32_t *subtree_end;
    uint32_t *first_child;
    uint32_t *next_sibling;
};

cudaError_t launch_tree_deep(const TreeDeepArgs &a, cudaStream_t st);

constexpr uint32_t kSearchTile = 16384;
constexpr uint32_t kSearchMaxStagedPattern = 4096;
constexpr uint32_t kSearchMaxPatterns = 8;  // patterns per launch

// Per-pattern constants of a search launch, computed on the host from the
// pattern bytes (search_add_pattern) and read by every block as kernel
// parameters.
struct SearchPatMeta {
    uint32_t pre[4];  // bytes 0..3, each replicated into a word (0 past the end)
    uint32_t anc[4];  // anchor words (len >= 8): bytes [r, r + 4) little-endian, r = 1..4
    uint32_t len;
    uint32_t f4;      // byte 0 replicated
};

struct SearchArgs {
    const uint8_t *text;     // padded: n_tiles * kSearchTile + kSearchMaxStagedPattern + 16 readable bytes
    uint64_t text_len;
    uint32_t n_tiles;
    uint32_t np;                                // patterns in this launch (1..8)
    uint32_t halo;                              // round_up(longest - 1, 16); > 4096 only when np == 1
    const uint8_t *pat[kSearchMaxPatterns];     // device copies
    uint32_t pat_len[kSearchMaxPatterns];
    uint32_t *out[kSearchMaxPatterns];          // ascending offsets, first max_out[p] of them
    uint32_t max_out[kSearchMaxPatterns];
    uint32_t ld;             // column stride of counts and bases: scan_ld(n_tiles)
    uint32_t *counts;        // [np][ld] matches per tile (pass 1), 16-byte aligned
    uint32_t *bases;         // [np][ld] exclusive scans (pass 2), 16-byte aligned
    uint32_t *totals;        // kSearchMaxPatterns totals (pass 2)
    // Staged form (nullptr: count pass + recomputing write pass): per tile a
    // slot of stage_cap 16-bit tile offsets, and a flag per tile whose hits did
    // not fit (recomputed by the write pass).
    uint16_t *stage;
    uint8_t *overflow;
    uint32_t stage_cap;
    uint32_t *overflow_n;     // staged form: count, then list, of the flagged tiles (n_tiles entries)
    uint32_t *overflow_list;
    SearchPatMeta meta[kSearchMaxPatterns];
    uint32_t anchor_hash[kSearchMaxPatterns * 4];  // anchor-map bits of the patterns of >= 8 bytes
    uint32_t n_anchor;
    uint32_t len_class[3];  // bit p: pattern p has <= 4 bytes; 5..7 bytes; 8 or more (search_add_pattern)
};
constexpr uint32_t kSearchStageCap = 8192;  // staged hits per tile (all patterns of a launch)

// Appends a pattern to a launch (slot a.np): its device copy, and the
// constants the kernels take from its host bytes.
void search_add_pattern(SearchArgs &a, const uint8_t *host, const uint8_t *dev, uint32_t len, uint32_t *out,
                        uint32_t max_out);
cudaError_t launch_search(const SearchArgs &a, cudaStream_t st);

// ---------------------------------------------------------------- query --

struct QueryArgs {
    const uint8_t *kinds;    // resident document (kinds, depth8, text, offsets) ...
    const uint8_t *depth8;
    const uint8_t *text;
    const uint32_t *offsets;
    uint64_t text_len;
    const FlatNode *nodes;   // ... or materialised nodes (then the four above are unused)
    uint32_t lines;          // lines in the document
    uint32_t lo, hi;         // range [lo, hi) of lines considered
    uint32_t target_kind;    // 0: any
    uint32_t target_depth;   // NONE: any
    uint32_t *counts;        // per block of 4096 lines, 16-byte aligned
    uint32_t *bases;         // same size, 16-byte aligned
    uint32_t *total;         // device
    uint32_t *out;           // ascending line indices, first max_out of them
    uint32_t max_out;
};
uint32_t query_blocks(uint32_t lines);
cudaError_t launch_query(const QueryArgs &a, cudaStream_t st);

// ------------------------------------------------------------ dictionary --

constexpr uint32_t kDictTile = 16384;         // text bytes per tile (the parse tile: same padding)
constexpr uint32_t kDictHalo = 80;            // staged past the tile: > longest pattern, 16-byte multiple
constexpr uint32_t kDictMinLen = 4;           // the filter keys on a pattern's first 4 bytes
constexpr uint32_t kDictMaxLen = 64;
constexpr uint32_t kDictMaxHeavy = 32;        // patterns whose hits go to bitmaps in one search
constexpr uint32_t kDictFilterBits = 17;      // 2^17-bit two-hash filter (16 KiB of shared memory)
constexpr uint32_t kDictWordsPerTile = kDictTile / 32;
constexpr uint32_t kDictSortChunk = 512;      // keys per warp in the light-hit radix sort

// Filter and table hashes of a pattern's first four bytes (little-endian u32);
// the host compiler uses the same functions.
__host__ __device__ inline uint32_t dict_filter_h1(uint32_t w) { return (w * 0x85EBCA77u) >> (32 - kDictFilterBits); }
__host__ __device__ inline uint32_t dict_filter_h2(uint32_t w) { return (w * 0xC2B2AE3Du) >> (32 - kDictFilterBits); }
__host__ __device__ inline uint32_t dict_table_h(uint32_t w, uint32_t bits) { return (w * 0x9E3779B1u) >> (32 - bits); }

// Device view of a compiled pattern set. Patterns are deduplicated ("unique
// patterns" u); a trie over them gives, for a text position whose first four
// bytes match some pattern's, every unique pattern starting there.
struct DictSet {
    const uint32_t *filter;  // 2^kDictFilterBits bits
    const uint2 *table;      // open addressing: {first 4 bytes, trie node at depth 4}; empty: .y == NONE
    uint32_t table_bits;
    uint32_t max_probe;      // longest probe distance of any key
    const uint4 *nodes;      // {unique pattern ending here or NONE, edge count (| kDictDenseFlag),
                             //  edge 0, edge 1 | extra start | dense table}
    const uint32_t *extra;   // edges 1.. of nodes with 3..kDictDenseMin children; edge = (child << 8) | byte,
                             // sorted by byte
    const uint32_t *dense;   // 256 children (NONE: no edge) per node with more than kDictDenseMin children
    uint32_t n_u;
};
constexpr uint32_t kDictDenseMin = 8;
constexpr uint32_t kDictDenseFlag = 0x80000000u;

// A byte run in the trie: the path c^4, c^5, ..., c^K (K <= kDictMaxLen) of
// one byte c, built per search. A walk that starts inside a run of c jumps to
// the deepest chain node its run reaches: the heavy patterns on the way are
// one mask, the light ones a short list.
constexpr uint32_t kDictMaxChains = 4;
constexpr uint32_t kDictChainMin = 8;  // shorter chains are walked node by node
struct DictChain {
    uint32_t byte, K, n_light, pad;
    uint32_t node[kDictMaxLen + 1];   // trie node of c^d, d = 4..K
    uint32_t cum[kDictMaxLen + 1];    // heavy bits of the patterns c^4 .. c^d
    uint32_t light[kDictMaxLen + 1];  // (d << 24) | u of the light patterns on the chain, d ascending
};

struct DictMatchArgs {
    DictSet set;
    const uint8_t *text;     // padded like every resident text
    uint64_t text_len;
    uint32_t n_tiles;
    uint32_t tile_stride;    // tiles 0, s, 2s, ... (count mode samples)
    uint32_t count_only;     // 1: counts[u] += every hit; 0: heavy bitmaps + light keys
    uint32_t *counts;        // per unique pattern (count mode: all hits; else light hits)
    const uint8_t *heavy_of_u;  // heavy index or 0xFF
    uint32_t n_heavy;
    uint32_t *bitmap;        // [n_heavy][n_tiles * kDictWordsPerTile]
    unsigned long long *light_keys;  // (u << 32) | offset, unordered
    uint32_t light_cap;
    uint32_t *light_n;
    uint32_t *error;
    // Batches: hits must lie inside one document, [seg_start[i], seg_end[i])
    // (sorted, disjoint); nullptr: the whole text is one document.
    const unsigned long long *seg_start;
    const unsigned long long *seg_end;
    uint32_t n_seg;
    unsigned long long *stats;  // optional: += candidates walked, trie nodes visited
    // Byte-run chains (not in count mode): n_chains of them, their bytes
    // packed in chain_bytes (byte j = chain j's byte).
    const DictChain *chains;
    uint32_t n_chains;
    uint32_t chain_bytes;
    // Test hook (ol_ctx_inject): each block takes its wait-timeout branch
    // after its filter copy has landed, as if the bounded wait had run out.
    uint32_t force_timeout;
};

cudaError_t launch_dict_match(const DictMatchArgs &a, int sm_count, cudaStream_t st, uint32_t slice = 512,
                              uint32_t blocks_per_sm = 0);
// Per (4096-word block, heavy pattern) popcounts, [n_heavy][ld] column-major.
cudaError_t launch_dict_heavy_count(const uint32_t *bitmap, uint32_t n_words, uint32_t n_heavy, uint32_t *counts,
                                    uint32_t ld, cudaStream_t st);
uint32_t dict_heavy_blocks(uint32_t n_words);
// Stable LSD radix sort of n 64-bit keys on bits [0, key_bits), 8 per pass;
// the result ends in keys (tmp is the other buffer); hist needs
// 2 * 256 * scan_ld(chunks) words and digit totals 256 words.
cudaError_t launch_dict_sort(unsigned long long *keys, unsigned long long *tmp, uint32_t n, uint32_t key_bits,
                             uint32_t *hist, uint32_t *totals, cudaStream_t st);
uint32_t dict_sort_chunks(uint32_t n);

struct DictEmitArgs {
    uint32_t n_ids, n_u, n_heavy, n_words;
    const uint32_t *u_of_id;
    const uint32_t *dup_start;   // [n_u + 1]
    const uint32_t *dup_ids;     // ids grouped by unique pattern, ascending
    const uint8_t *heavy_of_u;
    const uint32_t *heavy_u;     // [n_heavy]
    const uint32_t *heavy_totals;
    const uint32_t *heavy_bases; // [n_heavy][ld]
    uint32_t ld;
    const uint32_t *bitmap;
    const uint32_t *light_count; // [n_u]
    uint32_t *light_base;        // [n_u] (written by the id pass)
    const unsigned long long *light_keys;  // sorted
    uint32_t light_n;
    uint32_t *id_counts;         // [n_ids]
    unsigned long long *id_base; // [n_ids]
    unsigned long long *total;
    uint2 *hits;                 // {pattern, offset}
    unsigned long long max_hits;
    // The (pattern u32, offset u64) form: when hit_off is set, hits go to
    // these two arrays instead of `hits`.
    uint32_t *hit_pat;
    unsigned long long *hit_off;
};
cudaError_t launch_dict_ids(const DictEmitArgs &a, cudaStream_t st);

// Digests (digest.cu): *out += sum of per-element hashes of a[0..n).
cudaError_t launch_digest_u32(const uint32_t *a, uint64_t n, uint32_t seed, unsigned long long *out, cudaStream_t st);
cudaError_t launch_digest_u8(const uint8_t *a, uint64_t n, uint32_t seed, unsigned long long *out, cudaStream_t st);

// Batches (batch.cu).
cudaError_t launch_batch_line_starts(const uint32_t *offsets, uint32_t L, const unsigned long long *seg_start, uint32_t n,
                                     uint32_t *line_start, cudaStream_t st);
cudaError_t launch_batch_tree_fixup(const uint32_t *line_start, uint32_t n, uint32_t L, const uint8_t *kinds,
                                    const uint32_t *parent_in, const uint32_t *end_in, const uint32_t *fc_in,
                                    uint32_t *parent, uint32_t *subtree_end, uint32_t *first_child,
                                    uint32_t *next_sibling, cudaStream_t st);
cudaError_t launch_dict_emit(const DictEmitArgs &a, cudaStream_t st);

// One document of a batch copied from the caller's bytes (uploaded as they
// lie) to its place in the batch text: len bytes from in + src to text + dst,
// then a '\n' at text + dst + len when sep is set (batch_pack).
struct BatchPackDoc {
    uint64_t src, dst, len;
    uint32_t sep, pad;
};
// Work items of a document (batch_pack_kernel: kBatchPackBytes each, at least one).
constexpr uint32_t kBatchPackBytes = 65536;
uint32_t batch_pack_items(uint64_t len);
cudaError_t launch_batch_pack(const BatchPackDoc *docs, const uint32_t *item_start, uint32_t n, uint32_t items,
                              const uint8_t *in, uint8_t *text, cudaStream_t st);

// One document of a batch and the buffers it is copied into (batch_split).
struct BatchSplitDoc {
    uint64_t text_start, text_len;  // bytes of the batch text
    uint32_t first_line, lines;     // lines of the batch
    uint8_t *text;
    uint32_t *offsets;
    uint8_t *kinds, *depth8;
    uint32_t *parent, *subtree_end, *first_child, *next_sibling;
};
struct BatchSplitSrc {
    const uint8_t *text;
    const uint32_t *offsets;
    const uint8_t *kinds, *depth8;
    const uint32_t *parent, *subtree_end, *first_child, *next_sibling;
};
// Work items of a document (batch_split_kernel: 4096 bytes and 1024 lines each).
uint32_t batch_split_items(uint64_t text_len, uint32_t lines);
// item_start[i]: the first work item of document i (a prefix sum of
// batch_split_items); items: their total.
cudaError_t launch_batch_split(const BatchSplitDoc *docs, const uint32_t *item_start, uint32_t n, uint32_t items,
                               const BatchSplitSrc &src, uint32_t *max_depth, cudaStream_t st);

}  // namespace ol
