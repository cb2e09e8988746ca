// Kernel argument blocks and launch entry points shared between the kernels
// (*.cu) and the host runtime (runtime.cu). Device pointers only.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace ol {

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
};

cudaError_t launch_parse(const ParseArgs &a, cudaStream_t st);

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
};

cudaError_t launch_search(const SearchArgs &a, cudaStream_t st);

}  // namespace ol
