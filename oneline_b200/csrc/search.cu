// Kernel (d): substring search, every overlapping occurrence, ascending.
//
// Up to eight patterns are searched in one pass over the text; CTA b owns the
// 16 KiB tile b and stages it, plus a halo of (longest pattern - 1) bytes, in
// shared memory with 16-byte coalesced loads. For each pattern a first-byte
// filter (byte SWAR over 16-byte pieces) queues candidate pieces per warp;
// queued pieces are verified 32 at a time, one per lane: the last byte, then
// every other byte, for all sixteen starts of the piece at once (byte SWAR on
// shifted windows). An occurrence must end inside the text (the buffer is zero
// padded: a pattern ending in NUL must not match the padding).
// Three launches, no block waits on another:
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

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

constexpr uint32_t SR_THREADS = 256;
constexpr uint32_t SR_STEPS = 4;
constexpr uint32_t SR_PIECES = SR_THREADS * SR_STEPS;  // 16-byte pieces per tile
constexpr uint32_t SR_QCAP = 160;                       // per-warp candidate queue (< 32 left + 128 per pattern)
static_assert(SR_THREADS * 16 * SR_STEPS == kSearchTile, "search tile");

struct PatMeta {
    const uint8_t *ptr;
    uint32_t len;
    uint32_t f4;  // first byte, replicated
};

struct SearchSmem {
    alignas(16) uint8_t text[kSearchTile + kSearchMaxStagedPattern + 16];  // write pass: output staging after use
    uint16_t queue[SR_THREADS / 32][SR_QCAP];  // (pattern << 10) | piece, per warp
    PatMeta pat[kSearchMaxPatterns];
    uint32_t count[kSearchMaxPatterns];
    uint32_t active;  // write pass: patterns with matches in this tile (bit mask)
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

// 16-bit mask (bit i = byte i) from the high bits of four SWAR words.
__device__ __forceinline__ uint32_t gather16(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3) {
    auto g = [](uint32_t c) { return (((c >> 7) * 0x00204081u) >> 21) & 0xFu; };
    return g(c0) | (g(c1) << 4) | (g(c2) << 8) | (g(c3) << 12);
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
    if (tail_tile) {  // starts past N - m cannot match
        const int64_t last_ok = (int64_t)a.text_len - (int64_t)m - (int64_t)t0;
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

// Loads tile b (plus the halo) into shared memory and the pattern table.
__device__ __forceinline__ void load_tile(const SearchArgs &a, SearchSmem &sm, uint64_t t0, uint4 v[SR_STEPS]) {
    const uint32_t tid = threadIdx.x;
    const bool staged = a.halo <= kSearchMaxStagedPattern;
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) v[k] = ld_stream16(a.text + t0 + k * 4096 + tid * 16);
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) *reinterpret_cast<uint4 *>(&sm.text[k * 4096 + tid * 16]) = v[k];
    const uint32_t halo = staged ? a.halo : 0u;
    for (uint32_t o = tid * 16; o < halo; o += SR_THREADS * 16)
        *reinterpret_cast<uint4 *>(&sm.text[kSearchTile + o]) = ld_stream16(a.text + t0 + kSearchTile + o);
    if (tid == 0) *reinterpret_cast<uint4 *>(&sm.text[kSearchTile + halo]) = make_uint4(0, 0, 0, 0);
    if (tid < a.np) {
        PatMeta pm;
        pm.ptr = a.pat[tid];
        pm.len = a.pat_len[tid];
        pm.f4 = __ldg(pm.ptr) * 0x01010101u;
        sm.pat[tid] = pm;
        sm.count[tid] = 0;
    }
}

// Runs the filter of every pattern in `mask` over the tile: every lane tests
// its four pieces with the loose first-byte SWAR (three operations per word);
// pieces with a candidate are queued per warp and verified 32 at a time, one
// per lane, so verification work follows the number of candidates. `sink(p,
// piece, matches)` receives every verified piece (matches may be 0).
template <class Sink>
__device__ __forceinline__ void filter_tile(const SearchArgs &a, SearchSmem &sm, const uint4 v[SR_STEPS], uint32_t mask,
                                            uint64_t t0, Sink sink) {
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
#pragma unroll 1
    for (uint32_t p = 0; p < a.np; p++) {
        if (!((mask >> p) & 1u)) continue;
        const uint32_t F4 = sm.pat[p].f4;
        uint32_t cm = 0;
#pragma unroll
        for (uint32_t k = 0; k < SR_STEPS; k++) {
            uint32_t c = zero_bytes_loose(v[k].x ^ F4) | zero_bytes_loose(v[k].y ^ F4) | zero_bytes_loose(v[k].z ^ F4) |
                         zero_bytes_loose(v[k].w ^ F4);
            cm |= (uint32_t)(c != 0) << k;
        }
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

// Pass 1: matches of every pattern in every tile (counts only).
__global__ void __launch_bounds__(SR_THREADS) search_count_kernel(SearchArgs a) {
    __shared__ SearchSmem sm;
    const uint32_t tid = threadIdx.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * kSearchTile;
    uint4 v[SR_STEPS];
    load_tile(a, sm, t0, v);
    __syncthreads();
    // Lanes verifying pieces of the same pattern add up their matches first:
    // one shared-memory atomic per (round, pattern) instead of one per piece.
    filter_tile(a, sm, v, 0xFFu, t0, [&](uint32_t p, uint32_t piece, uint32_t mk) {
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
__global__ void __launch_bounds__(SR_THREADS) search_write_kernel(SearchArgs a) {
    __shared__ SearchSmem sm;
    __shared__ uint16_t match[kSearchMaxPatterns][SR_PIECES];
    __shared__ uint32_t warp_sum[SR_THREADS / 32];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile = blockIdx.x;
    const uint64_t t0 = (uint64_t)tile * kSearchTile;
    if (a.stage && !a.overflow[tile]) return;  // written from the staged hits
    // patterns with matches here whose output window is not yet full
    uint32_t want = 0;
    for (uint32_t p = 0; p < a.np; p++) {
        size_t at = (size_t)p * a.ld + tile;
        if (a.counts[at] && a.bases[at] < a.max_out[p]) want |= 1u << p;
    }
    if (!want) return;
    uint4 v[SR_STEPS];
    load_tile(a, sm, t0, v);
    for (uint32_t o = tid; o < kSearchMaxPatterns * SR_PIECES / 8; o += SR_THREADS)
        reinterpret_cast<uint4 *>(&match[0][0])[o] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    filter_tile(a, sm, v, want, t0, [&](uint32_t p, uint32_t piece, uint32_t mk) { match[p][piece] = (uint16_t)mk; });
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

// ----------------------------------------------------------- staged path --
//
// With a staging buffer the filter and verification run once: pass 1
// (search_stage_kernel) keeps each tile's match masks in shared memory, counts
// every pattern's hits with one block scan for all patterns at once, and writes
// the tile's hits, in (pattern, position) order, as 16-bit tile offsets into the
// tile's staging slot. After the column scan, pass 2 (search_copy_kernel)
// copies them to their final slots. A tile with more hits than its staging slot
// holds is flagged and left to search_write_kernel, which recomputes it.

__global__ void __launch_bounds__(SR_THREADS) search_stage_kernel(SearchArgs a) {
    __shared__ SearchSmem sm;
    __shared__ uint16_t match[kSearchMaxPatterns][SR_PIECES];
    __shared__ uint32_t warp_sum[SR_THREADS / 32][4];
    __shared__ uint32_t tile_tot[kSearchMaxPatterns];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile = blockIdx.x;
    const uint64_t t0 = (uint64_t)tile * kSearchTile;
    uint4 v[SR_STEPS];
    load_tile(a, sm, t0, v);
    for (uint32_t o = tid; o < kSearchMaxPatterns * SR_PIECES / 8; o += SR_THREADS)
        reinterpret_cast<uint4 *>(&match[0][0])[o] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    filter_tile(a, sm, v, (1u << a.np) - 1u, t0,
                [&](uint32_t p, uint32_t piece, uint32_t mk) { match[p][piece] = (uint16_t)mk; });
    __syncthreads();
    // my hits per pattern (4 pieces: at most 64), two patterns per word
    uint2 m4[kSearchMaxPatterns];
    uint32_t packed[4] = {0, 0, 0, 0};
#pragma unroll
    for (uint32_t p = 0; p < kSearchMaxPatterns; p++) {
        m4[p] = p < a.np ? *reinterpret_cast<const uint2 *>(&match[p][4 * tid]) : make_uint2(0, 0);
        packed[p >> 1] |= (uint32_t)(__popc(m4[p].x) + __popc(m4[p].y)) << (16 * (p & 1));
    }
    // inclusive warp scans of the packed counts (tile totals stay below 2^16)
    uint32_t inc[4];
#pragma unroll
    for (uint32_t q = 0; q < 4; q++) {
        inc[q] = packed[q];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc[q], o);
            if ((int)lane >= o) inc[q] += t;
        }
        if (lane == 31) warp_sum[warp][q] = inc[q];
    }
    __syncthreads();
    uint32_t before[4] = {0, 0, 0, 0}, total[4] = {0, 0, 0, 0};
    for (uint32_t w = 0; w < SR_THREADS / 32; w++)
#pragma unroll
        for (uint32_t q = 0; q < 4; q++) {
            before[q] += w < warp ? warp_sum[w][q] : 0u;
            total[q] += warp_sum[w][q];
        }
    // tile totals per pattern, and where each pattern's hits start in the slot;
    // the slot is assembled in shared memory (the staged text is no longer
    // read) and stored with 16-byte writes
    static_assert(kSearchStageCap * 2 <= kSearchTile, "the slot fits where the tile text was");
    uint16_t *stage = reinterpret_cast<uint16_t *>(sm.text);
    uint32_t start = 0;
#pragma unroll
    for (uint32_t p = 0; p < kSearchMaxPatterns; p++) {
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
        if (tid == 0 && p < a.np) a.counts[(size_t)p * a.ld + tile] = tot;
        start += tot;
    }
    if (tid == 0) a.overflow[tile] = start > a.stage_cap ? 1 : 0;
    if (start == 0 || start > a.stage_cap) return;  // uniform: nothing to store, or recomputed later
    __syncthreads();
    uint4 *dst = reinterpret_cast<uint4 *>(a.stage + (size_t)tile * a.stage_cap);
    const uint4 *src = reinterpret_cast<const uint4 *>(stage);
    for (uint32_t o = tid; o < (start + 7) / 8; o += SR_THREADS) dst[o] = src[o];
}

__global__ void __launch_bounds__(SR_THREADS) search_copy_kernel(SearchArgs a) {
    const uint32_t tile = blockIdx.x;
    if (a.overflow[tile]) return;  // left to search_write_kernel
    const uint64_t t0 = (uint64_t)tile * kSearchTile;
    const uint16_t *slot = a.stage + (size_t)tile * a.stage_cap;
    uint32_t start = 0;
    for (uint32_t p = 0; p < a.np; p++) {
        const size_t at = (size_t)p * a.ld + tile;
        const uint32_t n = a.counts[at], base = a.bases[at], max_out = a.max_out[p];
        uint32_t *out = a.out[p];
        for (uint32_t i = threadIdx.x; i < n && base + i < max_out; i += SR_THREADS)
            out[base + i] = (uint32_t)(t0 + slot[start + i]);
        start += n;
    }
}

cudaError_t launch_search(const SearchArgs &a, cudaStream_t st) {
    if (a.n_tiles == 0 || a.np == 0) return cudaSuccess;
    if (a.stage) {
        search_stage_kernel<<<a.n_tiles, SR_THREADS, 0, st>>>(a); OL_LAUNCHED();
        cudaError_t e = launch_scan_columns(a.counts, a.bases, a.totals, a.n_tiles, a.np, a.ld, st);
        if (e != cudaSuccess) return e;
        search_copy_kernel<<<a.n_tiles, SR_THREADS, 0, st>>>(a); OL_LAUNCHED();
        search_write_kernel<<<a.n_tiles, SR_THREADS, 0, st>>>(a); OL_LAUNCHED();  // flagged tiles only
        return cudaGetLastError();
    }
    search_count_kernel<<<a.n_tiles, SR_THREADS, 0, st>>>(a); OL_LAUNCHED();
    cudaError_t e = launch_scan_columns(a.counts, a.bases, a.totals, a.n_tiles, a.np, a.ld, st);
    if (e != cudaSuccess) return e;
    search_write_kernel<<<a.n_tiles, SR_THREADS, 0, st>>>(a); OL_LAUNCHED();
    return cudaGetLastError();
}

}  // namespace ol
