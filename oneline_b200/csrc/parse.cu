// Kernel (a)+(b): newline scan fused with per-line classification.
//
// Staged form (the default), no block ever waits on another:
//   1. parse_stage_kernel: per 16 KiB tile, the newline count (16-byte
//      coalesced vector loads, exact byte SWAR, popc, warp scans), the
//      newline positions in order, and the classification of every line
//      starting in the tile from shared memory, staged as one word per line
//      in the tile's slot;
//   2. scan_columns_kernel: exclusive scan of the tile counts = every tile's
//      first line index;
//   3. parse_copy_kernel: one warp per tile writes the staged lines at their
//      line indices; parse_redo_kernel parses the tiles with more lines than
//      a slot holds again, in place.
// The text is read once. The recomputing form (newline_count_kernel, the
// scan, parse_tiles_kernel) reads it twice and needs no slots. A single pass
// with a decoupled look-back was measured slower here: the look-back chain
// fell behind the tile rate. A line that runs past the tile plus a 256-byte
// halo is queued for a small fix-up kernel, which reads it from global memory
// once the offsets array is complete.
//
// Replaces crates/oneline-gpu/src/scan.wgsl:20-237 (three passes + a host read
// of the line count) and shader.wgsl:34-134 (one thread per line, byte loads
// from global memory). Semantics: crates/oneline-simd/src/lib.rs:49-66 (line
// starts) and crates/oneline-simd/src/line.rs:8-81 (classification).
#include <cuda_runtime.h>

#include <algorithm>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

constexpr uint32_t PT_THREADS = 256;
constexpr uint32_t PT_STEPS = 4;                          // 16-byte pieces per thread
constexpr uint32_t PT_TILE = PT_THREADS * 16 * PT_STEPS;  // 16384
constexpr uint32_t PT_HALO = 256;
constexpr uint32_t PT_LIST = 1024;                        // newline positions listed per round

static_assert(PT_TILE == kParseTile && PT_HALO == kParseHalo, "tile geometry");

struct ParseSmem {
    alignas(16) uint8_t text[PT_TILE + PT_HALO + 16];  // +16: word reads may run 3 bytes past
    uint16_t nl[PT_LIST + 1];        // newline positions of the current round, ascending
    uint32_t warp_tot[PT_STEPS][8];  // newline count per (step, warp)
    uint32_t warp_base[PT_STEPS][8];
    uint32_t halo_first;             // first newline in the halo (local), or NONE
    uint32_t tile_nl;                // newlines in the tile
};

// Staged form: a tile's lines as one word each, (start, kind, depth8) or a
// marker, in its slot of PT_LIST words.
constexpr uint32_t kSlotNone = 0xFFFFFFFFu;  // a final '\n' that starts no line
constexpr uint32_t kSlotFixup = 1u << 26;    // the line runs past the halo: the fix-up kernel classifies it
__device__ __forceinline__ uint32_t slot_word(uint32_t s, uint32_t kind, uint32_t depth) {
    return s | (kind << 15) | (min(depth, 255u) << 18);  // s <= 16384: 15 bits
}

// 4 bytes of shared memory from any byte offset.
__device__ __forceinline__ uint32_t lds4(const uint8_t *base, uint32_t off) {
    const uint32_t *w = reinterpret_cast<const uint32_t *>(base) + (off >> 2);
    return __funnelshift_r(w[0], w[1], (off & 3) * 8);
}

// High bit of every byte of w equal to '|'.
__device__ __forceinline__ uint32_t pipe_bits(uint32_t w) { return zero_bytes(w ^ 0x7C7C7C7Cu); }

// parse_line (crates/oneline-simd/src/line.rs:8-44) for a line held in shared
// memory at tile-local [s, e), e = its '\n' or the text end; the bytes from e
// to e+3 are readable. The prefix is read as alternating runs: a run of '|'
// four bytes per step (byte SWAR), then a run of blanks; it continues only
// while another '|' follows the blanks.
__device__ __forceinline__ uint32_t classify_smem(const uint8_t *t, uint32_t s, uint32_t e, uint32_t &depth_out) {
    uint32_t eff = e;
    while (eff > s && t[eff - 1] == '\r') eff--;
    uint32_t c = s, depth = 0;
    if (s < eff && t[s] == '|') {
        for (;;) {
            // run of '|' (stops at a non-'|' byte, at the latest at eff)
            for (;;) {
                uint32_t other = ~pipe_bits(lds4(t, c)) & 0x80808080u;
                if (other) {
                    uint32_t nb = (__ffs(other) - 8) >> 3;
                    depth += nb;
                    c += nb;
                    break;
                }
                depth += 4;
                c += 4;
            }
            // run of blanks; the prefix goes on only if a '|' follows it
            uint32_t b = c;
            while (b < eff && is_blank(t[b])) b++;
            if (b < eff && t[b] == '|') {
                c = b;
                continue;
            }
            c = b;
            break;
        }
    } else {
        while (c < eff && is_blank(t[c])) c++;
    }
    depth_out = depth;
    if (c >= eff) return KIND_BLANK;
    uint32_t w = lds4(t, c);
    return classify3((uint8_t)w, (uint8_t)(w >> 8), (uint8_t)(w >> 16), eff - c);
}

// Exact '\n' bits (high bit of each byte) of a 16-byte piece at tile-local lo;
// bytes at or past `valid` are cleared.
__device__ __forceinline__ void newline_bits(const uint4 &v, uint32_t lo, uint32_t valid, uint32_t z[4]) {
    const uint32_t NL4 = 0x0A0A0A0Au;
    z[0] = zero_bytes(v.x ^ NL4);
    z[1] = zero_bytes(v.y ^ NL4);
    z[2] = zero_bytes(v.z ^ NL4);
    z[3] = zero_bytes(v.w ^ NL4);
    if (lo + 16 > valid) {
#pragma unroll
        for (uint32_t i = 0; i < 4; i++) {
            uint32_t b0 = lo + 4 * i;  // bytes b0..b0+3; keep those < valid
            uint32_t keep = b0 >= valid ? 0u : (valid - b0 >= 4 ? 4u : valid - b0);
            z[i] &= keep == 4 ? 0xFFFFFFFFu : ((1u << (8 * keep)) - 1u);
        }
    }
}

// Pass 1: newlines per 16 KiB tile (positions < N).
__global__ void __launch_bounds__(PT_THREADS) newline_count_kernel(const uint8_t *__restrict__ text, uint64_t N,
                                                                    uint32_t *__restrict__ counts) {
    __shared__ uint32_t warp_sum[PT_THREADS / 32];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t t0 = (uint64_t)blockIdx.x * PT_TILE;
    const uint32_t valid = N - t0 >= PT_TILE ? PT_TILE : (uint32_t)(N - t0);
    uint4 v[PT_STEPS];
#pragma unroll
    for (uint32_t k = 0; k < PT_STEPS; k++) v[k] = ld_stream16(text + t0 + k * 4096 + tid * 16);
    uint32_t c = 0;
#pragma unroll
    for (uint32_t k = 0; k < PT_STEPS; k++) {
        uint32_t z[4];
        newline_bits(v[k], k * 4096 + tid * 16, valid, z);
        c += __popc(z[0]) + __popc(z[1]) + __popc(z[2]) + __popc(z[3]);
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if (lane == 0) warp_sum[warp] = c;
    __syncthreads();
    if (tid == 0) {
        uint32_t t = 0;
#pragma unroll
        for (uint32_t w = 0; w < PT_THREADS / 32; w++) t += warp_sum[w];
        counts[blockIdx.x] = t;
    }
}

// One tile: the block loads tile b, lists its newlines in position order
// (warp popc scans) and classifies every line that starts after one of them
// (plus line 0 for tile 0) from shared memory. Consecutive threads take
// consecutive lines. A line that runs past the tile plus a 256-byte halo is
// left to the fix-up kernel.
//   STAGE: the tile's newline count goes to tile_count and its lines, by
//     tile-local rank, to its slot (a tile with more lines than a slot holds
//     is listed for the recomputing form instead);
//   else: the tile's first line index comes from tile_base (the scan of the
//     counts), and offsets, kinds and depth8 are written in place.
template <bool STAGE>
__device__ __forceinline__ void parse_tile(const ParseArgs &a, ParseSmem &sm, uint32_t tile) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t t0 = (uint64_t)tile * PT_TILE;
    const uint64_t N = a.text_len;
    // bytes of this tile (and halo) that belong to the text
    const uint32_t valid = N - t0 >= PT_TILE + PT_HALO ? PT_TILE + PT_HALO : (uint32_t)(N - t0);

    // 1. Coalesced 16-byte loads: step k covers [t0 + k*4096, +4096), lane-major.
    uint4 v[PT_STEPS];
#pragma unroll
    for (uint32_t k = 0; k < PT_STEPS; k++) v[k] = ld_stream16(a.text + t0 + k * 4096 + tid * 16);
    uint4 vh = make_uint4(0, 0, 0, 0);
    if (tid < PT_HALO / 16) vh = ld_stream16(a.text + t0 + PT_TILE + tid * 16);
    if (tid == 0) {
        sm.halo_first = NONE;
        *reinterpret_cast<uint4 *>(&sm.text[PT_TILE + PT_HALO]) = make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (uint32_t k = 0; k < PT_STEPS; k++) *reinterpret_cast<uint4 *>(&sm.text[k * 4096 + tid * 16]) = v[k];
    if (tid < PT_HALO / 16) *reinterpret_cast<uint4 *>(&sm.text[PT_TILE + tid * 16]) = vh;

    // 2. Newline bits and their ranks within the warp: steps (0,1) and (2,3)
    //    packed in 16-bit fields.
    uint32_t nlm[PT_STEPS];  // bit b: byte b of the thread's piece in step k is a newline
    uint32_t cnt[PT_STEPS];
#pragma unroll
    for (uint32_t k = 0; k < PT_STEPS; k++) {
        uint32_t z[4];
        newline_bits(v[k], k * 4096 + tid * 16, valid, z);
        nlm[k] = gather16(z[0], z[1], z[2], z[3]);
        cnt[k] = __popc(nlm[k]);
    }
    uint32_t c01 = cnt[0] | (cnt[1] << 16), c23 = cnt[2] | (cnt[3] << 16);
    uint32_t i01 = c01, i23 = c23;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t1 = __shfl_up_sync(0xFFFFFFFFu, i01, o);
        uint32_t t2 = __shfl_up_sync(0xFFFFFFFFu, i23, o);
        if ((int)lane >= o) {
            i01 += t1;
            i23 += t2;
        }
    }
    const uint32_t r01 = i01 - c01, r23 = i23 - c23;
    if (lane == 31) {
        sm.warp_tot[0][warp] = i01 & 0xFFFF;
        sm.warp_tot[1][warp] = i01 >> 16;
        sm.warp_tot[2][warp] = i23 & 0xFFFF;
        sm.warp_tot[3][warp] = i23 >> 16;
    }
    __syncthreads();  // (a) halo_first initialised, warp totals visible
    if (tid < PT_HALO / 16) {
        const uint32_t lo = PT_TILE + tid * 16;
        uint32_t first = NONE;
        uint32_t zh[4];
        newline_bits(vh, lo, valid, zh);
#pragma unroll
        for (int i = 3; i >= 0; i--)
            if (zh[i]) first = lo + 4 * i + ((__ffs(zh[i]) - 8) >> 3);
        for (int o = 8; o > 0; o >>= 1) first = min(first, __shfl_xor_sync(0x0000FFFFu, first, o));
        if (tid == 0) sm.halo_first = first;
    }
    if (warp == 1) {
        // 32 (step, warp) totals in position order: index = k*8 + w.
        uint32_t c = sm.warp_tot[lane >> 3][lane & 7], inc = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += t;
        }
        sm.warp_base[lane >> 3][lane & 7] = inc - c;
        if (lane == 31) sm.tile_nl = inc;
    }
    __syncthreads();  // (b) bases and halo_first visible

    const uint32_t off = tile == 0 ? 1u : 0u;
    uint32_t nl_base, n_nl;
    if (STAGE) {
        n_nl = sm.tile_nl;
        nl_base = 0;
        const bool over = n_nl + off > a.slot_cap;
        if (tid == 0) {
            a.tile_count[tile] = n_nl;
            a.slot_over[tile] = over ? 1 : 0;
            if (over) a.redo_list[atomicAdd(a.redo_n, 1u)] = tile;
        }
        if (over) return;  // uniform
    } else {
        nl_base = a.tile_base[tile];  // newlines before this tile
        n_nl = a.tile_count[tile];
        if (tile == a.n_tiles - 1 && tid == 0)  // L = 1 + newlines before the last byte
            a.stats->line_count = 1u + nl_base + n_nl - (a.text[N - 1] == '\n');
    }
    const uint32_t n_lines = n_nl + off;
    const uint32_t halo_first = sm.halo_first;
    uint32_t *slot = STAGE ? a.slot + (size_t)tile * a.slot_cap : nullptr;
    uint32_t my_max = 0;

    // Lines are classified in rounds of PT_LIST (one round unless the tile
    // holds more than 1024 newlines): list the round's newline positions, then
    // classify and write the round's lines.
    for (uint32_t r0 = 0; r0 < n_lines; r0 += PT_LIST) {
        const int32_t w0 = (int32_t)r0 - (int32_t)off;  // rank of nl[0]
#pragma unroll
        for (uint32_t k = 0; k < PT_STEPS; k++) {
            uint32_t rr = (k & 1) ? ((k < 2 ? r01 : r23) >> 16) : ((k < 2 ? r01 : r23) & 0xFFFF);
            int32_t rk = (int32_t)(sm.warp_base[k][warp] + rr) - w0;
            if (rk > (int32_t)PT_LIST) continue;
            // one loop over the piece's 16-bit newline mask: the warp runs as
            // many rounds as its busiest lane has newlines in this piece
            uint32_t m = nlm[k];
            while (m) {
                const uint32_t b = __ffs(m) - 1;
                m &= m - 1;
                if (rk >= 0 && rk <= (int32_t)PT_LIST) sm.nl[rk] = (uint16_t)(k * 4096 + tid * 16 + b);
                rk++;
            }
        }
        __syncthreads();  // (c) list ready

        const uint32_t r_end = min(n_lines, r0 + PT_LIST);
        for (uint32_t j = r0 + tid; j < r_end; j += PT_THREADS) {
            int32_t q = (int32_t)j - (int32_t)off;  // newline that precedes the line (-1: none)
            uint32_t s = q < 0 ? 0u : sm.nl[q - w0] + 1u;  // tile-local
            if (s >= valid) {  // the final '\n' starts no line
                if (STAGE) slot[j] = kSlotNone;
                continue;
            }
            uint32_t idx = nl_base + j + 1 - off;
            if (!STAGE) {
                if (idx >= a.line_cap) {
                    atomicOr(&a.stats->error, OL_DEVERR_CAPACITY);
                    continue;
                }
                a.offsets[idx] = (uint32_t)t0 + s;
            }
            uint32_t e;
            if ((uint32_t)(q + 1) < n_nl) e = sm.nl[q + 1 - w0];
            else if (halo_first != NONE) e = halo_first;
            else if (valid < PT_TILE + PT_HALO) e = valid;  // the text ends in the staged bytes
            else {
                // runs past the halo: classified by the fix-up kernel
                if (STAGE) {
                    slot[j] = s | kSlotFixup;
                } else {
                    uint32_t fx = atomicAdd(&a.stats->fixup_count, 1u);
                    if (fx < a.fixup_cap) a.fixup[fx] = make_uint2(idx, (uint32_t)t0 + s);
                    else atomicOr(&a.stats->error, OL_DEVERR_FIXUP);
                }
                continue;
            }
            uint32_t depth;
            uint32_t kind = classify_smem(sm.text, s, e, depth);
            if (STAGE) {
                slot[j] = slot_word(s, kind, depth);
            } else {
                a.kinds[idx] = (uint8_t)kind;
                a.depth8[idx] = (uint8_t)min(depth, 255u);
            }
            if (kind != KIND_BLANK) my_max = max(my_max, depth);
        }
        __syncthreads();  // (d) the next round may overwrite the list
    }
    for (int o = 16; o > 0; o >>= 1) my_max = max(my_max, __shfl_xor_sync(0xFFFFFFFFu, my_max, o));
    if (lane == 0 && my_max) atomicMax(&a.stats->max_content_depth, my_max);
}

// Recomputing form, every tile (pass 3 after newline_count_kernel and the scan).
__global__ void __launch_bounds__(PT_THREADS, 6) parse_tiles_kernel(ParseArgs a) {
    __shared__ ParseSmem sm;
    parse_tile<false>(a, sm, blockIdx.x);
}

// Staged form, pass 1: every tile counts its newlines and stages its lines.
// Block b first asks L2 to prefetch the tile kPrefetchTilesAhead further on
// (when this launch covers it), which a block that starts soon will read.
__global__ void __launch_bounds__(PT_THREADS, 6) parse_stage_kernel(ParseArgs a) {
    __shared__ ParseSmem sm;
    if (threadIdx.x == 0 && blockIdx.x + kPrefetchTilesAhead < gridDim.x)  // inside this launch's tiles
        prefetch_l2(a.text + (uint64_t)(a.first_tile + blockIdx.x + kPrefetchTilesAhead) * kParseTile, kParseTile);
    parse_tile<true>(a, sm, a.first_tile + blockIdx.x);
}

// Staged form, pass 3: the tiles listed by pass 1 (more lines than a slot
// holds) in the recomputing form, now that their first line index is known.
__global__ void __launch_bounds__(PT_THREADS, 6) parse_redo_kernel(ParseArgs a) {
    __shared__ ParseSmem sm;
    const uint32_t n = *a.redo_n;
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        parse_tile<false>(a, sm, a.redo_list[i]);
        __syncthreads();  // shared memory is reused by the next tile
    }
}

// Staged form, pass 2: one warp per tile writes its staged lines at their
// line indices (the scan of the counts): offsets, kinds and depth8, or a
// fix-up entry for a line that runs past the halo.
constexpr uint32_t PC_TILES = 8;  // tiles per block
__global__ void __launch_bounds__(256) parse_copy_kernel(ParseArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t tile = blockIdx.x * PC_TILES + (threadIdx.x >> 5);
    if (tile >= a.n_tiles || a.slot_over[tile]) return;
    const uint32_t off = tile == 0 ? 1u : 0u;
    const uint32_t n_nl = a.tile_count[tile], nl_base = a.tile_base[tile];
    const uint32_t n_lines = n_nl + off;
    const uint32_t t0 = tile * PT_TILE;
    if (tile == a.n_tiles - 1 && lane == 0)  // L = 1 + newlines before the last byte
        a.stats->line_count = 1u + nl_base + n_nl - (a.text[a.text_len - 1] == '\n');
    const uint32_t *slot = a.slot + (size_t)tile * a.slot_cap;
    for (uint32_t j0 = 0; j0 < n_lines; j0 += 128) {
        uint32_t ws[4];  // four independent loads in flight per lane
#pragma unroll
        for (uint32_t r = 0; r < 4; r++) {
            const uint32_t j = j0 + r * 32 + lane;
            ws[r] = j < n_lines ? __ldg(slot + j) : kSlotNone;
        }
#pragma unroll
        for (uint32_t r = 0; r < 4; r++) {
            const uint32_t j = j0 + r * 32 + lane;
            const uint32_t w = ws[r];
            if (w == kSlotNone) continue;
            const uint32_t idx = nl_base + j + 1 - off;
            if (idx >= a.line_cap) {
                atomicOr(&a.stats->error, OL_DEVERR_CAPACITY);
                continue;
            }
            const uint32_t s = t0 + (w & 0x7FFFu);
            a.offsets[idx] = s;
            if (w & kSlotFixup) {
                const uint32_t fx = atomicAdd(&a.stats->fixup_count, 1u);
                if (fx < a.fixup_cap) a.fixup[fx] = make_uint2(idx, s);
                else atomicOr(&a.stats->error, OL_DEVERR_FIXUP);
                continue;
            }
            a.kinds[idx] = (uint8_t)((w >> 15) & 7u);
            a.depth8[idx] = (uint8_t)((w >> 18) & 0xFFu);
        }
    }
}

// Lines queued by the tile kernel: their end comes from the complete offsets
// array, their bytes from global memory. One warp per line (lane 0 works).
__global__ void parse_fixup_kernel(ParseArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t count = min(a.stats->fixup_count, a.fixup_cap);
    const uint32_t L = a.stats->line_count;
    if (L > a.line_cap) return;  // outputs overflowed: the host re-runs with room for L lines
    const uint64_t N = a.text_len;
    const uint32_t last_end = a.text[N - 1] == '\n' ? (uint32_t)(N - 1) : (uint32_t)N;
    for (uint32_t i = gw; i < count; i += nw) {
        if (lane != 0) continue;
        uint2 f = a.fixup[i];
        uint32_t idx = f.x, s = f.y;
        uint32_t e = idx + 1 < L ? a.offsets[idx + 1] - 1 : last_end;
        const uint8_t *t = a.text;
        FlatNode nd = classify_line(s, e, [t](uint32_t p) -> uint8_t { return __ldg(t + p); });
        if (idx >= a.line_cap) continue;
        a.kinds[idx] = (uint8_t)nd.kind;
        a.depth8[idx] = (uint8_t)min(nd.depth, 255u);
        if (nd.kind != KIND_BLANK) atomicMax(&a.stats->max_content_depth, nd.depth);
    }
}

// FlatNode of every line from the text and a complete offsets array (used for
// GpuParser::parse(input, offsets) and to materialise nodes of a resident
// document). One thread per line, bytes from global memory (read-only path).
__global__ void classify_lines_kernel(const uint8_t *__restrict__ text, uint64_t N, const uint32_t *__restrict__ offsets,
                                      uint32_t L, FlatNode *__restrict__ nodes, uint32_t *__restrict__ depth32) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L) return;
    uint32_t s = offsets[i];
    uint32_t last_end = text[N - 1] == '\n' ? (uint32_t)(N - 1) : (uint32_t)N;
    uint32_t e = i + 1 < L ? offsets[i + 1] - 1 : last_end;
    FlatNode nd = classify_line(s, e, [text](uint32_t p) -> uint8_t { return __ldg(text + p); });
    if (nodes) nodes[i] = nd;
    if (depth32) depth32[i] = nd.kind == KIND_BLANK ? NONE : nd.depth;
}

// ------------------------------------------------------------------ host ----

cudaError_t launch_parse(const ParseArgs &a, cudaStream_t st) {
    if (a.n_tiles == 0) return cudaSuccess;
    cudaError_t e;
    if (a.slot) {
        // staged: the text is read once; tiles with too many lines are redone
        if ((e = launch_parse_begin(a, st)) != cudaSuccess) return e;
        if ((e = launch_parse_tiles(a, 0, a.n_tiles, st)) != cudaSuccess) return e;
        return launch_parse_end(a, st);
    } else {
        newline_count_kernel<<<a.n_tiles, PT_THREADS, 0, st>>>(a.text, a.text_len, a.tile_count); OL_LAUNCHED();
        e = launch_scan_columns(a.tile_count, a.tile_base, nullptr, a.n_tiles, 1, scan_ld(a.n_tiles), st);
        if (e != cudaSuccess) return e;
        parse_tiles_kernel<<<a.n_tiles, PT_THREADS, 0, st>>>(a); OL_LAUNCHED();
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    uint32_t blocks = a.fixup_cap < 64 ? 8 : 64;
    parse_fixup_kernel<<<blocks, 256, 0, st>>>(a); OL_LAUNCHED();
    return cudaGetLastError();
}

cudaError_t launch_parse_begin(const ParseArgs &a, cudaStream_t st) {
    if (!a.slot || a.slot_cap > PT_LIST) return cudaErrorInvalidValue;  // a slot is listed in one round
    return cudaMemsetAsync(a.redo_n, 0, sizeof(uint32_t), st);
}

cudaError_t launch_parse_tiles(const ParseArgs &a, uint32_t t0, uint32_t t1, cudaStream_t st) {
    t1 = std::min(t1, a.n_tiles);
    if (t0 >= t1) return cudaSuccess;
    ParseArgs r = a;
    r.first_tile = t0;
    parse_stage_kernel<<<t1 - t0, PT_THREADS, 0, st>>>(r); OL_LAUNCHED();
    return cudaGetLastError();
}

cudaError_t launch_parse_end(const ParseArgs &a, cudaStream_t st) {
    if (a.n_tiles == 0) return cudaSuccess;
    cudaError_t e = launch_scan_columns(a.tile_count, a.tile_base, nullptr, a.n_tiles, 1, scan_ld(a.n_tiles), st);
    if (e != cudaSuccess) return e;
    parse_copy_kernel<<<(a.n_tiles + PC_TILES - 1) / PC_TILES, 256, 0, st>>>(a); OL_LAUNCHED();
    parse_redo_kernel<<<std::min(a.n_tiles, 512u), PT_THREADS, 0, st>>>(a); OL_LAUNCHED();
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const uint32_t blocks = a.fixup_cap < 64 ? 8 : 64;
    parse_fixup_kernel<<<blocks, 256, 0, st>>>(a); OL_LAUNCHED();
    return cudaGetLastError();
}

cudaError_t launch_classify_lines(const uint8_t *text, uint64_t N, const uint32_t *offsets, uint32_t L, FlatNode *nodes,
                                  uint32_t *depth32, cudaStream_t st) {
    if (L == 0) return cudaSuccess;
    classify_lines_kernel<<<(L + 255) / 256, 256, 0, st>>>(text, N, offsets, L, nodes, depth32); OL_LAUNCHED();
    return cudaGetLastError();
}

}  // namespace ol
