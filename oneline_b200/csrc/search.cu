// Kernel (d): substring search, every overlapping occurrence, ascending.
//
// Up to eight patterns are searched in one pass over the text; CTA b owns the
// 16 KiB tile b and stages it, plus a halo of (longest pattern - 1) bytes, in
// shared memory with 16-byte coalesced loads (in the stage pass, after asking
// L2 to prefetch the tile kPrefetchTilesAhead further on, which a block that
// starts soon will read). Every 16-byte piece is compared
// with each pattern of up to 4 bytes at all sixteen starts at once (byte SWAR
// on the piece shifted by 1, 2 and 3 bytes, built once for all patterns),
// which decides it. Longer patterns only mark candidate pieces: 5-7 byte ones
// by their first two bytes (the same SWAR), longer ones by a shared hash map
// of their anchor words (the 4-byte-aligned text word inside every
// occurrence). Candidate pieces are queued per warp and verified 32 at a
// time, one per lane: the first byte, the last, then every other byte, all
// sixteen starts at once. An occurrence must end inside the text (the buffer
// is zero padded: a pattern ending in NUL must not match the padding).
// Recomputing form, three launches, no block waits on another:
//   1. search_count_kernel: matches per (tile, pattern);
//   2. scan_columns_kernel: per pattern, the first output slot of every tile
//      and the total;
//   3. search_write_kernel: tiles with matches recompute them for the patterns
//      that have some and write every pattern's first max_out offsets in
//      ascending order, the whole block writing one contiguous range per
//      pattern: no host sort, and a truncated result is the lowest max_out
//      offsets.
// Patterns longer than kSearchMaxStagedPattern run alone (np = 1) and read
// their halo and verification bytes from global memory.
//
// Semantics: crates/oneline-simd/src/search.rs:88-114 (every overlapping
// occurrence, ascending). Replaces crates/oneline-gpu/src/search.wgsl:101-173
// (4-byte window filter, slot atomics, host sort).
#include <cuda_runtime.h>

#include <algorithm>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

constexpr uint32_t SR_THREADS = 256;
constexpr uint32_t SR_STEPS = 4;
constexpr uint32_t SR_PIECES = SR_THREADS * SR_STEPS;  // 16-byte pieces per tile
constexpr uint32_t SR_QCAP = 160;                       // per-warp candidate queue (< 32 left + 128 per pattern)
static_assert(SR_THREADS * 16 * SR_STEPS == kSearchTile, "search tile");

// Patterns of at least kAnchorMin bytes are filtered by their anchor words:
// every occurrence at start s covers the 4-byte-aligned text word at
// a = 4 * floor(s / 4) + 4 (1 <= a - s <= 4, and a + 4 <= s + 8 <= s + len),
// which equals the pattern's bytes [a - s, a - s + 4) -- one of four anchor
// words, r = a - s = 1..4. The starts of the 16-byte piece at lo map to the
// words at lo + 4, lo + 8, lo + 12 and lo + 16, four phases each. A 2^15-bit
// map of the anchors' hashes, shared by all patterns of the launch, tells
// which aligned text words may be one; those are compared exactly.
constexpr uint32_t kAnchorMin = 8;
constexpr uint32_t kAnchorBits = 15;

__host__ __device__ __forceinline__ uint32_t anchor_hash(uint32_t w) {
    return (w * 0x9E3779B1u) >> (32 - kAnchorBits);
}

struct alignas(16) PatMeta {
    uint4 pre;  // bytes 0..3 of the pattern, each replicated into a word (unused ones 0)
    uint4 anc;  // anchor words r = 1..4 (len >= kAnchorMin)
    const uint8_t *ptr;
    uint32_t len;
    uint32_t f4;  // first byte, replicated
};

struct SearchSmem {
    alignas(16) uint8_t text[kSearchTile + kSearchMaxStagedPattern + 16];  // stage pass: output staging after use
    uint32_t anchor_map[(1u << kAnchorBits) / 32];
    uint16_t queue[SR_THREADS / 32][SR_QCAP];  // (pattern << 10) | piece, per warp
    PatMeta pat[kSearchMaxPatterns];
    uint32_t count[kSearchMaxPatterns];
    uint32_t active;  // stage pass: patterns with matches in this tile (bit mask)
};

// 16 bytes of shared memory starting at any byte offset.
__device__ __forceinline__ uint4 lds16_unaligned(const uint8_t *smem, uint32_t off) {
    const uint32_t *w = reinterpret_cast<const uint32_t *>(smem) + (off >> 2);
    uint32_t sh = (off & 3) * 8;
    uint32_t a0 = w[0], a1 = w[1], a2 = w[2], a3 = w[3], a4 = w[4];
    return make_uint4(__funnelshift_r(a0, a1, sh), __funnelshift_r(a1, a2, sh), __funnelshift_r(a2, a3, sh),
                      __funnelshift_r(a3, a4, sh));
}

// High bit of each byte of x that is zero; may also flag a 0x01 byte right
// above a zero byte (a cheap first filter, confirmed by zero_bytes).
__device__ __forceinline__ uint32_t zero_bytes_loose(uint32_t x) { return (x - 0x01010101u) & ~x & 0x80808080u; }

// Bytes [off, off+16) of the tile-local text as four words: from shared
// memory when staged, else from global memory (bytes at or past N read as 0).
__device__ __forceinline__ uint4 window16(const uint8_t *smem, uint32_t off, bool staged, const uint8_t *g, uint64_t t0,
                                          uint64_t N) {
    if (staged) return lds16_unaligned(smem, off);
    uint8_t b[16];
#pragma unroll
    for (int r = 0; r < 16; r++) {
        uint64_t q = t0 + off + r;
        b[r] = q < N ? __ldg(g + q) : (uint8_t)0;
    }
    return *reinterpret_cast<uint4 *>(b);
}

// Clears the starts of the piece at tile-local lo that lie past N - m (they
// cannot match; the zero padding must not complete a pattern ending in NUL).
__device__ __forceinline__ void keep_valid_starts(uint64_t N, uint32_t m, uint64_t t0, uint32_t lo, uint32_t &c0,
                                                  uint32_t &c1, uint32_t &c2, uint32_t &c3) {
    const int64_t last_ok = (int64_t)N - (int64_t)m - (int64_t)t0;
    uint32_t keep[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int64_t room = last_ok - (int64_t)(lo + 4 * i) + 1;  // valid starts in word i
        keep[i] = room <= 0 ? 0u : (room >= 4 ? 0xFFFFFFFFu : ((1u << (8 * room)) - 1u));
    }
    c0 &= keep[0];
    c1 &= keep[1];
    c2 &= keep[2];
    c3 &= keep[3];
}

// Exact matches of a pattern at the sixteen starts of one piece (piece x
// covers tile bytes [16x, 16x+16)): first byte, then the last byte, then every
// other byte, all sixteen starts at once.
__device__ __forceinline__ uint32_t verify_piece(const SearchArgs &a, const SearchSmem &sm, const PatMeta &pm,
                                                 uint32_t piece, bool staged, bool tail_tile, uint64_t t0) {
    const uint32_t m = pm.len;
    const uint32_t lo = piece * 16;
    const uint4 v = *reinterpret_cast<const uint4 *>(&sm.text[lo]);
    uint32_t c0 = zero_bytes(v.x ^ pm.f4), c1 = zero_bytes(v.y ^ pm.f4);
    uint32_t c2 = zero_bytes(v.z ^ pm.f4), c3 = zero_bytes(v.w ^ pm.f4);
    if (tail_tile) keep_valid_starts(a.text_len, m, t0, lo, c0, c1, c2, c3);
    for (uint32_t jj = 1; jj < m && (c0 | c1 | c2 | c3); jj++) {
        const uint32_t j = jj == 1 ? m - 1 : jj - 1;  // last byte first, then 1, 2, ...
        const uint32_t P4 = __ldg(pm.ptr + j) * 0x01010101u;
        uint4 w = window16(sm.text, lo + j, staged, a.text, t0, a.text_len);
        c0 &= zero_bytes(w.x ^ P4);
        c1 &= zero_bytes(w.y ^ P4);
        c2 &= zero_bytes(w.z ^ P4);
        c3 &= zero_bytes(w.w ^ P4);
    }
    return gather16(c0, c1, c2, c3);
}

// Loads tile b (plus the halo) into shared memory, and (warp 0) the pattern
// table and the anchor map from the kernel parameters; the caller's
// __syncthreads publishes them.
__device__ __forceinline__ void load_tile(const SearchArgs &a, SearchSmem &sm, uint64_t t0) {
    const uint32_t tid = threadIdx.x;
    const bool staged = a.halo <= kSearchMaxStagedPattern;
    uint4 v[SR_STEPS];
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) v[k] = ld_stream16(a.text + t0 + k * 4096 + tid * 16);
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) *reinterpret_cast<uint4 *>(&sm.text[k * 4096 + tid * 16]) = v[k];
    const uint32_t halo = staged ? a.halo : 0u;
    for (uint32_t o = tid * 16; o < halo; o += SR_THREADS * 16)
        *reinterpret_cast<uint4 *>(&sm.text[kSearchTile + o]) = ld_stream16(a.text + t0 + kSearchTile + o);
    // 16 bytes past the halo: zeros when staged; unstaged, the bytes right
    // after the tile (the filter looks 3 bytes ahead; the text is padded)
    if (tid == 0)
        *reinterpret_cast<uint4 *>(&sm.text[kSearchTile + halo]) =
            staged ? make_uint4(0, 0, 0, 0) : ld_stream16(a.text + t0 + kSearchTile);
    if (tid < 32) {
        uint4 *am = reinterpret_cast<uint4 *>(sm.anchor_map);
        for (uint32_t o = tid; o < (1u << kAnchorBits) / 128; o += 32) am[o] = make_uint4(0, 0, 0, 0);
        __syncwarp();
        if (tid < a.n_anchor) {
            const uint32_t h = a.anchor_hash[tid];
            atomicOr(&sm.anchor_map[h >> 5], 1u << (h & 31));
        }
        if (tid < a.np) {
            const SearchPatMeta &m = a.meta[tid];
            PatMeta pm;
            pm.ptr = a.pat[tid];
            pm.len = m.len;
            pm.f4 = m.f4;
            pm.pre = make_uint4(m.pre[0], m.pre[1], m.pre[2], m.pre[3]);
            pm.anc = make_uint4(m.anc[0], m.anc[1], m.anc[2], m.anc[3]);
            sm.pat[tid] = pm;
            sm.count[tid] = 0;
        }
    }
}

// Runs the filter of every pattern in `mask` over the tile (staged in shared
// memory). Every lane takes its four pieces, one per step, and builds once for
// all patterns the windows of the piece shifted by 1, 2 and 3 bytes (the word
// after the piece comes from the next lane, or from shared memory for lane
// 31). A pattern of at most 4 bytes is compared whole at all sixteen starts at
// once (byte SWAR on the shifted windows) and its exact matches go to `sink`.
// A pattern of 5 to 7 bytes marks the pieces where its first two bytes occur
// (the same SWAR). Longer patterns share one test of the piece's four
// anchoring aligned words against the anchor map, whose cost does not grow
// with the number of patterns; a word found there is compared with each
// pattern's anchors. Marked pieces are queued per warp and verified 32 at a
// time, one per lane, so verification work follows the number of candidates.
// The pattern loops are not unrolled (the step loop is): with up to eight
// patterns a fully unrolled body outgrows the instruction cache. `sink(p, piece,
// matches)` receives every verified piece (matches may be 0) and every
// short-pattern piece with matches.
template <uint32_t NP, class Sink>
__device__ __forceinline__ void filter_tile(const SearchArgs &a, SearchSmem &sm, uint32_t mask, uint64_t t0, Sink sink) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool staged = a.halo <= kSearchMaxStagedPattern;
    const bool tail_tile = t0 + kSearchTile + a.halo + 16 > a.text_len;
    uint16_t *queue = sm.queue[warp];
    uint32_t qn = 0;  // queued entries (the same in every lane)
    auto drain = [&](uint32_t n) {
        for (uint32_t done = 0; done < n; done += 32) {
            if (done + lane < n) {
                uint32_t e = queue[done + lane];
                uint32_t p = e >> 10, piece = e & 1023u;
                sink(p, piece, verify_piece(a, sm, sm.pat[p], piece, staged, tail_tile, t0));
            }
        }
    };
    // patterns in `mask` by length: <= 4, 5-7, >= 8
    const uint32_t shorts = a.len_class[0] & mask, mids = a.len_class[1] & mask, anchored = a.len_class[2] & mask;
    uint32_t cand = 0;  // bit 4p + k: piece k has a candidate of pattern p (patterns over 4 bytes)
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) {
        const uint32_t piece = k * SR_THREADS + tid;
        const uint4 vk = *reinterpret_cast<const uint4 *>(&sm.text[piece * 16]);
        uint32_t w4 = __shfl_down_sync(0xFFFFFFFFu, vk.x, 1);
        if (lane == 31) w4 = *reinterpret_cast<const uint32_t *>(&sm.text[(piece + 1) * 16]);
        const uint32_t w[5] = {vk.x, vk.y, vk.z, vk.w, w4};
        uint32_t s1[4];
#pragma unroll
        for (int i = 0; i < 4; i++) s1[i] = __funnelshift_r(w[i], w[i + 1], 8);
        if (shorts) {  // uniform
            uint32_t s2[4], s3[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                s2[i] = __funnelshift_r(w[i], w[i + 1], 16);
                s3[i] = __funnelshift_r(w[i], w[i + 1], 24);
            }
#pragma unroll 1
            for (uint32_t bits = shorts; bits; bits &= bits - 1) {
                const uint32_t p = __ffs(bits) - 1;
                const uint4 pre = sm.pat[p].pre;
                const uint32_t m = sm.pat[p].len;
                uint32_t x[4];
#pragma unroll
                for (int i = 0; i < 4; i++) x[i] = w[i] ^ pre.x;
                if (m > 1)
#pragma unroll
                    for (int i = 0; i < 4; i++) x[i] |= s1[i] ^ pre.y;
                if (m > 2)
#pragma unroll
                    for (int i = 0; i < 4; i++) x[i] |= s2[i] ^ pre.z;
                if (m > 3)
#pragma unroll
                    for (int i = 0; i < 4; i++) x[i] |= s3[i] ^ pre.w;
                uint32_t c0 = zero_bytes(x[0]), c1 = zero_bytes(x[1]), c2 = zero_bytes(x[2]), c3 = zero_bytes(x[3]);
                if (tail_tile) keep_valid_starts(a.text_len, m, t0, piece * 16, c0, c1, c2, c3);
                if (c0 | c1 | c2 | c3) sink(p, piece, gather16(c0, c1, c2, c3));
            }
        }
#pragma unroll 1
        for (uint32_t bits = mids; bits; bits &= bits - 1) {  // the first two bytes (loose SWAR; exact as "any")
            const uint32_t p = __ffs(bits) - 1;
            const uint4 pre = sm.pat[p].pre;
            uint32_t acc = 0;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t x = (w[i] ^ pre.x) | (s1[i] ^ pre.y);
                acc |= (x - 0x01010101u) & ~x;
            }
            cand |= (uint32_t)((acc & 0x80808080u) != 0) << (4 * p + k);
        }
        if (anchored) {  // uniform
            // the four aligned words that anchor the piece's sixteen starts:
            // w[i] anchors the starts lo + 4i - 4 .. lo + 4i - 1 (i = 1..4)
            uint32_t hit = 0;
#pragma unroll
            for (int i = 1; i < 5; i++) {
                const uint32_t h = anchor_hash(w[i]);
                hit |= (sm.anchor_map[h >> 5] >> (h & 31)) & 1u;
            }
            if (hit) {  // rare: compare the anchors exactly
#pragma unroll 1
                for (uint32_t bits = anchored; bits; bits &= bits - 1) {
                    const uint32_t p = __ffs(bits) - 1;
                    const uint4 c = sm.pat[p].anc;
                    bool any = false;
#pragma unroll
                    for (int i = 1; i < 5; i++) any |= w[i] == c.x || w[i] == c.y || w[i] == c.z || w[i] == c.w;
                    cand |= (uint32_t)any << (4 * p + k);
                }
            }
        }
    }
    if (!__any_sync(0xFFFFFFFFu, cand != 0)) return;  // no candidate in the warp: nothing to verify
#pragma unroll 1
    for (uint32_t bits = mids | anchored; bits; bits &= bits - 1) {
        const uint32_t p = __ffs(bits) - 1;
        uint32_t cm = (cand >> (4 * p)) & 0xFu;
        if (!__any_sync(0xFFFFFFFFu, cm != 0)) continue;
        uint32_t n = __popc(cm), inc = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += t;
        }
        uint32_t pos = qn + inc - n;
        while (cm) {
            uint32_t k = __ffs(cm) - 1;
            cm &= cm - 1;
            queue[pos++] = (uint16_t)((p << 10) | (k * SR_THREADS + tid));
        }
        qn += __shfl_sync(0xFFFFFFFFu, inc, 31);
        __syncwarp();
        if (qn >= 32) {
            uint32_t full = qn & ~31u;
            drain(full);
            uint32_t rem = qn - full;
            uint16_t keep = lane < rem ? queue[full + lane] : (uint16_t)0;
            __syncwarp();
            if (lane < rem) queue[lane] = keep;
            qn = rem;
            __syncwarp();
        }
    }
    drain(qn);
}

// Pass 1: matches of every pattern in every tile (counts only). NP = a.np.
template <uint32_t NP>
__global__ void __launch_bounds__(SR_THREADS) search_count_kernel(SearchArgs a) {
    __shared__ SearchSmem sm;
    const uint32_t tid = threadIdx.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * kSearchTile;
    load_tile(a, sm, t0);
    __syncthreads();
    // Lanes verifying pieces of the same pattern add up their matches first:
    // one shared-memory atomic per (round, pattern) instead of one per piece.
    filter_tile<NP>(a, sm, 0xFFu, t0, [&](uint32_t p, uint32_t piece, uint32_t mk) {
        const uint32_t group = __match_any_sync(__activemask(), p);
        const uint32_t sum = __reduce_add_sync(group, __popc(mk));
        if ((threadIdx.x & 31) == __ffs(group) - 1 && sum) atomicAdd(&sm.count[p], sum);
    });
    __syncthreads();
    if (tid < a.np) a.counts[(size_t)tid * a.ld + blockIdx.x] = sm.count[tid];
}

// Pass 3: tiles with matches recompute the match masks of the patterns that
// have some; then, pattern by pattern, thread t takes pieces [4t, 4t+4) (in
// position order), a block scan of the per-thread match counts gives every
// thread its first output slot after the tile's base from pass 2, and each
// thread writes its matches there: the block's stores cover one contiguous
// range. Tiles without matches exit before loading text.
template <uint32_t NP>
__device__ __forceinline__ void write_tile(const SearchArgs &a, SearchSmem &sm, uint16_t (*match)[SR_PIECES],
                                           uint32_t *warp_sum, uint32_t tile) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t t0 = (uint64_t)tile * kSearchTile;
    // patterns with matches here whose output window is not yet full
    uint32_t want = 0;
    for (uint32_t p = 0; p < NP; p++) {
        size_t at = (size_t)p * a.ld + tile;
        if (a.counts[at] && a.bases[at] < a.max_out[p]) want |= 1u << p;
    }
    if (!want) return;
    load_tile(a, sm, t0);
    for (uint32_t o = tid; o < NP * SR_PIECES / 8; o += SR_THREADS)
        reinterpret_cast<uint4 *>(&match[0][0])[o] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    filter_tile<NP>(a, sm, want, t0, [&](uint32_t p, uint32_t piece, uint32_t mk) { match[p][piece] = (uint16_t)mk; });
    __syncthreads();
    for (uint32_t w = want; w; w &= w - 1) {
        const uint32_t p = __ffs(w) - 1;
        const uint2 m4 = *reinterpret_cast<const uint2 *>(&match[p][4 * tid]);  // my 4 pieces
        const uint32_t n = __popc(m4.x) + __popc(m4.y), inc0 = n;
        uint32_t inc = inc0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += t;
        }
        if (lane == 31) warp_sum[warp] = inc;
        __syncthreads();
        uint32_t before = 0;
        for (uint32_t x = 0; x < warp; x++) before += warp_sum[x];
        uint32_t r = a.bases[(size_t)p * a.ld + tile] + before + inc - n;
        const uint32_t max_out = a.max_out[p];
        uint32_t *out = a.out[p];
        const uint32_t mm[2] = {m4.x, m4.y};
#pragma unroll
        for (uint32_t h = 0; h < 2; h++) {
            uint32_t bits = mm[h];  // pieces 4t+2h (low 16 bits) and 4t+2h+1 (high 16 bits)
            while (bits && r < max_out) {
                uint32_t b = __ffs(bits) - 1;
                bits &= bits - 1;
                uint32_t piece = 4 * tid + 2 * h + (b >> 4);
                out[r++] = (uint32_t)(t0 + piece * 16 + (b & 15));
            }
        }
        __syncthreads();  // warp_sum is reused by the next pattern
    }
}

// Recomputing form: block b writes tile b. Staged form: a small grid takes
// the tiles the stage pass listed as overflowing their slots (usually none).
template <uint32_t NP>
__global__ void __launch_bounds__(SR_THREADS) search_write_kernel(SearchArgs a) {
    __shared__ SearchSmem sm;
    __shared__ uint16_t match[NP][SR_PIECES];
    __shared__ uint32_t warp_sum[SR_THREADS / 32];
    if (!a.stage) {
        write_tile<NP>(a, sm, match, warp_sum, blockIdx.x);
        return;
    }
    const uint32_t n = *a.overflow_n;
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) write_tile<NP>(a, sm, match, warp_sum, a.overflow_list[i]);
}

// ----------------------------------------------------------- staged path --
//
// With a staging buffer the filter and verification run once: pass 1
// (search_stage_kernel) keeps each tile's match masks in shared memory, counts
// every pattern's hits with one block scan for all patterns at once, and writes
// the tile's hits, in (pattern, position) order, as 16-bit tile offsets into the
// tile's staging slot. After the column scan, pass 2 (search_copy_kernel)
// copies them to their final slots. A tile with more hits than its staging slot
// holds is flagged and left to search_write_kernel, which recomputes it.

template <uint32_t NP>
__global__ void __launch_bounds__(SR_THREADS) search_stage_kernel(SearchArgs a) {
    constexpr uint32_t NQ = (NP + 1) / 2;  // packed count words, two patterns each
    __shared__ SearchSmem sm;
    __shared__ uint16_t match[NP][SR_PIECES];
    __shared__ uint32_t warp_sum[SR_THREADS / 32][NQ];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile = blockIdx.x;
    const uint64_t t0 = (uint64_t)tile * kSearchTile;
    if (tid == 0 && tile + kPrefetchTilesAhead < a.n_tiles)
        prefetch_l2(a.text + (uint64_t)(tile + kPrefetchTilesAhead) * kSearchTile, kSearchTile);
    load_tile(a, sm, t0);
    if (tid == 0) sm.active = 0;
    for (uint32_t o = tid; o < NP * SR_PIECES / 8; o += SR_THREADS)
        reinterpret_cast<uint4 *>(&match[0][0])[o] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    // the patterns with hits anywhere in the tile, as the filter finds them
    uint32_t found = 0;
    filter_tile<NP>(a, sm, (1u << NP) - 1u, t0, [&](uint32_t p, uint32_t piece, uint32_t mk) {
        match[p][piece] = (uint16_t)mk;
        found |= (mk != 0 ? 1u : 0u) << p;
    });
    found = __reduce_or_sync(0xFFFFFFFFu, found);
    if (lane == 0 && found) atomicOr(&sm.active, found);
    __syncthreads();
    const uint32_t active = sm.active;
    if (active == 0) {  // a tile without hits is done here
        if (tid < NP) a.counts[(size_t)tid * a.ld + tile] = 0;
        if (tid == 0) a.overflow[tile] = 0;
        return;
    }
    uint16_t *stage = reinterpret_cast<uint16_t *>(sm.text);  // the slot, assembled where the text was
    if ((active & (active - 1)) == 0) {  // hits of one pattern only: the usual tile
        const uint32_t p = __ffs(active) - 1;
        const uint2 m = *reinterpret_cast<const uint2 *>(&match[p][4 * tid]);
        const uint32_t mine = __popc(m.x) + __popc(m.y);
        uint32_t inc = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += t;
        }
        if (lane == 31) warp_sum[warp][0] = inc;
        __syncthreads();
        uint32_t before = 0, total = 0;
#pragma unroll
        for (uint32_t w = 0; w < SR_THREADS / 32; w++) {
            const uint32_t x = warp_sum[w][0];
            before += w < warp ? x : 0u;
            total += x;
        }
        if (tid < NP) a.counts[(size_t)tid * a.ld + tile] = tid == p ? total : 0u;
        const bool over = total > a.stage_cap;
        if (tid == 0) {
            a.overflow[tile] = over ? 1 : 0;
            if (over) a.overflow_list[atomicAdd(a.overflow_n, 1u)] = tile;
        }
        if (over) return;  // uniform: recomputed later
        uint32_t r = before + inc - mine;
        const uint32_t mm[2] = {m.x, m.y};
#pragma unroll
        for (uint32_t h = 0; h < 2; h++) {
            uint32_t bits = mm[h];
            while (bits) {
                const uint32_t b = __ffs(bits) - 1;
                bits &= bits - 1;
                stage[r++] = (uint16_t)((4 * tid + 2 * h + (b >> 4)) * 16 + (b & 15));
            }
        }
        __syncthreads();
        uint4 *dst = reinterpret_cast<uint4 *>(a.stage + (size_t)tile * a.stage_cap);
        const uint4 *src = reinterpret_cast<const uint4 *>(stage);
        for (uint32_t o = tid; o < (total + 7) / 8; o += SR_THREADS) dst[o] = src[o];
        return;
    }
    // my hits per pattern with hits (4 pieces: at most 64)
    uint2 m4[NP];
#pragma unroll
    for (uint32_t p = 0; p < NP; p++)
        m4[p] = ((active >> p) & 1u) ? *reinterpret_cast<const uint2 *>(&match[p][4 * tid]) : make_uint2(0, 0);
    // counts, two patterns per word; inclusive warp scans of the words that
    // hold a pattern with hits (tile totals stay below 2^16)
    uint32_t packed[NQ], inc[NQ];
#pragma unroll
    for (uint32_t q = 0; q < NQ; q++) packed[q] = 0;
#pragma unroll
    for (uint32_t p = 0; p < NP; p++)
        packed[p >> 1] |= (uint32_t)(__popc(m4[p].x) + __popc(m4[p].y)) << (16 * (p & 1));
#pragma unroll
    for (uint32_t q = 0; q < NQ; q++) {
        inc[q] = packed[q];
        if ((active >> (2 * q)) & 3u) {  // uniform
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc[q], o);
                if ((int)lane >= o) inc[q] += t;
            }
        }
        if (lane == 31) warp_sum[warp][q] = inc[q];
    }
    __syncthreads();
    uint32_t before[NQ], total[NQ];
#pragma unroll
    for (uint32_t q = 0; q < NQ; q++) {
        before[q] = total[q] = 0;
        if ((active >> (2 * q)) & 3u)
            for (uint32_t w = 0; w < SR_THREADS / 32; w++) {
                const uint32_t x = warp_sum[w][q];
                before[q] += w < warp ? x : 0u;
                total[q] += x;
            }
    }
    // tile totals per pattern, and where each pattern's hits start in the slot;
    // the slot is assembled in shared memory (the staged text is no longer
    // read) and stored with 16-byte writes
    static_assert(kSearchStageCap * 2 <= kSearchTile, "the slot fits where the tile text was");
    uint32_t start = 0;
#pragma unroll
    for (uint32_t p = 0; p < NP; p++) {
        const uint32_t sh = 16 * (p & 1);
        const uint32_t tot = (total[p >> 1] >> sh) & 0xFFFFu;
        const uint32_t mine = (packed[p >> 1] >> sh) & 0xFFFFu;
        uint32_t r = start + ((before[p >> 1] >> sh) & 0xFFFFu) + ((inc[p >> 1] >> sh) & 0xFFFFu) - mine;
        if (mine && start + tot <= a.stage_cap) {
            const uint32_t mm[2] = {m4[p].x, m4[p].y};
#pragma unroll
            for (uint32_t h = 0; h < 2; h++) {
                uint32_t bits = mm[h];
                while (bits) {
                    const uint32_t b = __ffs(bits) - 1;
                    bits &= bits - 1;
                    stage[r++] = (uint16_t)((4 * tid + 2 * h + (b >> 4)) * 16 + (b & 15));
                }
            }
        }
        if (tid == 0) a.counts[(size_t)p * a.ld + tile] = tot;
        start += tot;
    }
    if (tid == 0) {
        a.overflow[tile] = start > a.stage_cap ? 1 : 0;
        if (start > a.stage_cap) a.overflow_list[atomicAdd(a.overflow_n, 1u)] = tile;
    }
    if (start > a.stage_cap) return;  // uniform: recomputed later
    __syncthreads();
    uint4 *dst = reinterpret_cast<uint4 *>(a.stage + (size_t)tile * a.stage_cap);
    const uint4 *src = reinterpret_cast<const uint4 *>(stage);
    for (uint32_t o = tid; o < (start + 7) / 8; o += SR_THREADS) dst[o] = src[o];
}

// Pass 2 of the staged path: two warps per tile. Lane p reads pattern p's
// count and first output slot (all patterns at once: one memory round trip),
// a warp scan places each pattern's hits in the tile's slot, and the warps
// copy them to their final slots, alternate runs of 256 each.
constexpr uint32_t SC_WARPS = 2;                          // warps per tile
constexpr uint32_t SC_TILES = SR_THREADS / 32 / SC_WARPS;  // tiles per block
__global__ void __launch_bounds__(SR_THREADS) search_copy_kernel(SearchArgs a) {
    const uint32_t lane = threadIdx.x & 31, half = (threadIdx.x >> 5) % SC_WARPS;
    const uint32_t tile = blockIdx.x * SC_TILES + (threadIdx.x >> 5) / SC_WARPS;
    if (tile >= a.n_tiles || a.overflow[tile]) return;  // overflowing tiles: search_write_kernel
    uint32_t n = 0, base = 0, max_out = 0;
    if (lane < a.np) {
        const size_t at = (size_t)lane * a.ld + tile;
        n = a.counts[at];
        base = a.bases[at];
        max_out = a.max_out[lane];
    }
    uint32_t inc = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if ((int)lane >= o) inc += t;
    }
    if (__shfl_sync(0xFFFFFFFFu, inc, 31) == 0) return;
    const uint64_t t0 = (uint64_t)tile * kSearchTile;
    const uint16_t *slot = a.stage + (size_t)tile * a.stage_cap;
    for (uint32_t p = 0; p < a.np; p++) {
        const uint32_t np_ = __shfl_sync(0xFFFFFFFFu, n, p);
        if (np_ == 0) continue;
        const uint32_t b = __shfl_sync(0xFFFFFFFFu, base, p), mx = __shfl_sync(0xFFFFFFFFu, max_out, p);
        const uint32_t start = __shfl_sync(0xFFFFFFFFu, inc - n, p);
        const uint32_t lim = b >= mx ? 0u : min(np_, mx - b);  // the first max_out hits overall
        uint32_t *__restrict__ out = a.out[p] + b;
        const uint16_t *__restrict__ src = slot + start;
        // the tile's warps take alternate runs of 256 hits; eight independent
        // loads in flight per lane before the stores
        for (uint32_t i0 = half * 256; i0 < lim; i0 += 256 * SC_WARPS) {
            uint32_t v[8];
#pragma unroll
            for (uint32_t j = 0; j < 8; j++) {
                const uint32_t i = i0 + j * 32 + lane;
                v[j] = i < lim ? __ldg(src + i) : 0u;
            }
#pragma unroll
            for (uint32_t j = 0; j < 8; j++) {
                const uint32_t i = i0 + j * 32 + lane;
                if (i < lim) out[i] = (uint32_t)(t0 + v[j]);
            }
        }
    }
}

void search_add_pattern(SearchArgs &a, const uint8_t *host, const uint8_t *dev, uint32_t len, uint32_t *out,
                        uint32_t max_out) {
    const uint32_t p = a.np++;
    a.pat[p] = dev;
    a.pat_len[p] = len;
    a.out[p] = out;
    a.max_out[p] = max_out;
    SearchPatMeta &m = a.meta[p];
    m = SearchPatMeta{};
    m.len = len;
    a.len_class[len <= 4 ? 0 : len < kAnchorMin ? 1 : 2] |= 1u << p;
    m.f4 = (len ? host[0] : 0u) * 0x01010101u;
    for (uint32_t j = 0; j < 4 && j < len; j++) m.pre[j] = host[j] * 0x01010101u;
    if (len >= kAnchorMin)
        for (uint32_t r = 1; r <= 4; r++) {  // len >= 8: bytes r..r+3 exist
            m.anc[r - 1] = (uint32_t)host[r] | ((uint32_t)host[r + 1] << 8) | ((uint32_t)host[r + 2] << 16) |
                           ((uint32_t)host[r + 3] << 24);
            a.anchor_hash[a.n_anchor++] = anchor_hash(m.anc[r - 1]);
        }
}

constexpr uint32_t kSearchWriteGrid = 512;  // blocks of the staged form's write pass

template <uint32_t NP>
static cudaError_t launch_search_np(const SearchArgs &a, cudaStream_t st) {
    if (a.stage) {
        cudaError_t e0 = cudaMemsetAsync(a.overflow_n, 0, sizeof(uint32_t), st);
        if (e0 != cudaSuccess) return e0;
        search_stage_kernel<NP><<<a.n_tiles, SR_THREADS, 0, st>>>(a); OL_LAUNCHED();
        cudaError_t e = launch_scan_columns(a.counts, a.bases, a.totals, a.n_tiles, a.np, a.ld, st);
        if (e != cudaSuccess) return e;
        search_copy_kernel<<<(a.n_tiles + SC_TILES - 1) / SC_TILES, SR_THREADS, 0, st>>>(a); OL_LAUNCHED();
        search_write_kernel<NP><<<std::min(a.n_tiles, kSearchWriteGrid), SR_THREADS, 0, st>>>(a); OL_LAUNCHED();  // listed tiles
        return cudaGetLastError();
    }
    search_count_kernel<NP><<<a.n_tiles, SR_THREADS, 0, st>>>(a); OL_LAUNCHED();
    cudaError_t e = launch_scan_columns(a.counts, a.bases, a.totals, a.n_tiles, a.np, a.ld, st);
    if (e != cudaSuccess) return e;
    search_write_kernel<NP><<<a.n_tiles, SR_THREADS, 0, st>>>(a); OL_LAUNCHED();
    return cudaGetLastError();
}

// One instantiation per pattern count: the per-pattern loops unroll without
// guards and the shared match arrays hold only the launch's patterns.
cudaError_t launch_search(const SearchArgs &a, cudaStream_t st) {
    if (a.n_tiles == 0 || a.np == 0) return cudaSuccess;
    switch (a.np) {
        case 1: return launch_search_np<1>(a, st);
        case 2: return launch_search_np<2>(a, st);
        case 3: return launch_search_np<3>(a, st);
        case 4: return launch_search_np<4>(a, st);
        case 5: return launch_search_np<5>(a, st);
        case 6: return launch_search_np<6>(a, st);
        case 7: return launch_search_np<7>(a, st);
        case 8: return launch_search_np<8>(a, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ol
