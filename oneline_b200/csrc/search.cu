// Kernel (d): substring search, every overlapping occurrence, ascending.
//
// One launch searches up to eight patterns in one pass over the text. CTA b
// owns the 16 KiB tile b and stages it, plus a halo of (longest pattern - 1)
// bytes, in shared memory with 16-byte coalesced loads. For each pattern a
// first-byte filter (byte SWAR over 16-byte pieces) queues candidate pieces per
// warp; queued pieces are verified 32 at a time, one per lane: the last byte,
// then every other byte, for all sixteen starts of the piece at once (byte
// SWAR on shifted windows). An occurrence must end inside the text (the buffer
// is zero padded: a pattern ending in NUL must not match the padding). The
// match masks go to shared memory in position order; warp p then counts
// pattern p's matches, runs the decoupled look-back over the tile match counts
// of pattern p (the eight look-backs proceed in parallel) and writes the
// pattern's first max_out offsets in ascending order through a staging buffer,
// coalesced: no host sort, and a truncated result is the lowest max_out
// offsets.
//
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
static_assert(SR_THREADS * 16 * SR_STEPS == kSearchTile, "search tile");

constexpr uint32_t SR_QCAP = 160;  // per-warp candidate queue (< 32 left over + 128 per pattern)

struct SearchSmem {
    alignas(16) uint8_t text[kSearchTile + kSearchMaxStagedPattern + 16];  // phase B: output staging
    alignas(16) uint16_t match[kSearchMaxPatterns][SR_THREADS * SR_STEPS];  // per 16-byte piece, position order
    uint16_t queue[SR_THREADS / 32][SR_QCAP];  // (pattern << 10) | piece, per warp
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

// Exact matches of pattern p at the sixteen starts of one piece: first byte,
// then the last byte, then every other byte, all sixteen starts at once.
__device__ __forceinline__ uint32_t verify_piece(const SearchArgs &a, const SearchSmem &sm, uint32_t p, uint32_t piece,
                                                 bool staged, bool tail_tile, uint64_t t0) {
    const uint32_t m = a.pat_len[p];
    const uint8_t *pat = a.pat[p];
    const uint32_t F4 = __ldg(pat) * 0x01010101u;
    const uint32_t lo = piece * 16;  // position order: piece x covers tile bytes [16x, 16x+16)
    const uint4 v = *reinterpret_cast<const uint4 *>(&sm.text[lo]);
    uint32_t c0 = zero_bytes(v.x ^ F4), c1 = zero_bytes(v.y ^ F4), c2 = zero_bytes(v.z ^ F4), c3 = zero_bytes(v.w ^ F4);
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
        const uint32_t P4 = __ldg(pat + j) * 0x01010101u;
        uint4 w = window16(sm.text, lo + j, staged, a.text, t0, a.text_len);
        c0 &= zero_bytes(w.x ^ P4);
        c1 &= zero_bytes(w.y ^ P4);
        c2 &= zero_bytes(w.z ^ P4);
        c3 &= zero_bytes(w.w ^ P4);
    }
    return gather16(c0, c1, c2, c3);
}

__global__ void __launch_bounds__(SR_THREADS) search_kernel(SearchArgs a) {
    __shared__ SearchSmem sm;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile = blockIdx.x;
    const uint64_t t0 = (uint64_t)tile * kSearchTile;
    const uint64_t N = a.text_len;
    const bool staged = a.halo <= kSearchMaxStagedPattern;

    uint4 v[SR_STEPS];
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) v[k] = ld_stream16(a.text + t0 + k * 4096 + tid * 16);
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) *reinterpret_cast<uint4 *>(&sm.text[k * 4096 + tid * 16]) = v[k];
    const uint32_t halo = staged ? a.halo : 0u;
    for (uint32_t o = tid * 16; o < halo; o += SR_THREADS * 16)
        *reinterpret_cast<uint4 *>(&sm.text[kSearchTile + o]) = ld_stream16(a.text + t0 + kSearchTile + o);
    if (tid == 0) *reinterpret_cast<uint4 *>(&sm.text[kSearchTile + halo]) = make_uint4(0, 0, 0, 0);
    // clear the match masks of every pattern (64 bytes per thread)
    for (uint32_t o = tid; o < kSearchMaxPatterns * SR_THREADS * SR_STEPS / 8; o += SR_THREADS)
        reinterpret_cast<uint4 *>(&sm.match[0][0])[o] = make_uint4(0, 0, 0, 0);
    __syncthreads();

    // Phase A. Every lane runs the first-byte filter (loose byte SWAR, three
    // operations per word) on its four pieces for each pattern; pieces with a
    // candidate go to the warp's queue, and every 32 queued pieces are verified
    // together, one per lane, so that verification work follows the number of
    // candidates rather than the number of pieces.
    const bool tail_tile = t0 + kSearchTile + a.halo + 16 > N;
    uint16_t *queue = sm.queue[warp];
    uint32_t qn = 0;  // queued entries (the same in every lane)
#pragma unroll 1
    for (uint32_t p = 0; p < a.np; p++) {
        const uint32_t F4 = __ldg(a.pat[p]) * 0x01010101u;
        uint32_t cm = 0;
#pragma unroll
        for (uint32_t k = 0; k < SR_STEPS; k++) {
            uint32_t c = zero_bytes_loose(v[k].x ^ F4) | zero_bytes_loose(v[k].y ^ F4) | zero_bytes_loose(v[k].z ^ F4) |
                         zero_bytes_loose(v[k].w ^ F4);
            cm |= (c != 0) << k;
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
            uint32_t done = 0;
            for (; done + 32 <= qn; done += 32) {
                uint32_t e = queue[done + lane];
                uint32_t piece = e & 1023u;
                sm.match[e >> 10][piece] = (uint16_t)verify_piece(a, sm, e >> 10, piece, staged, tail_tile, t0);
            }
            uint32_t rem = qn - done;
            uint16_t keep = lane < rem ? queue[done + lane] : (uint16_t)0;
            __syncwarp();
            if (lane < rem) queue[lane] = keep;
            qn = rem;
            __syncwarp();
        }
    }
    if (lane < qn) {
        uint32_t e = queue[lane];
        uint32_t piece = e & 1023u;
        sm.match[e >> 10][piece] = (uint16_t)verify_piece(a, sm, e >> 10, piece, staged, tail_tile, t0);
    }
    __syncthreads();

    // Phase B: warp p counts, looks back and writes pattern p on its own.
    // Lane l owns pieces [32 l, 32 l + 32) of the tile, in position order.
    if (warp >= a.np) return;
    const uint32_t p = warp;
    const uint4 *row = reinterpret_cast<const uint4 *>(&sm.match[p][lane * 32]);
    uint32_t cnt = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        uint4 r = row[q];  // 8 pieces
        cnt += __popc(r.x) + __popc(r.y) + __popc(r.z) + __popc(r.w);
    }
    uint32_t inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if ((int)lane >= o) inc += t;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, inc, 31);
    uint64_t *st = a.tile_status + (uint64_t)tile * kSearchMaxPatterns + p;
    if (lane == 0) st_relaxed_u64(st, (uint64_t)total | (tile == 0 ? LB_PREFIX : LB_AGGREGATE));
    const uint32_t base =
        tile == 0 ? 0u : lb_sum_exclusive_wide(a.tile_status + p, tile, a.error, kSearchMaxPatterns);
    if (lane == 0) {
        if (tile != 0) st_relaxed_u64(st, (uint64_t)(base + total) | LB_PREFIX);
        if (tile == a.n_tiles - 1) a.totals[p] = base + total;
    }
    const uint32_t max_out = a.max_out[p];
    if (total == 0 || base >= max_out) return;
    // Ordered, coalesced output: chunk c is lane c's 32 pieces; its matches are
    // expanded into this warp's 2 KiB of staging, then copied out by all lanes.
    uint32_t *out = a.out[p];
    uint32_t *stg = reinterpret_cast<uint32_t *>(sm.text) + warp * 512;
    const uint32_t excl = inc - cnt;
    uint32_t nz = __ballot_sync(0xFFFFFFFFu, cnt != 0);
    while (nz) {
        const uint32_t c = __ffs(nz) - 1;
        nz &= nz - 1;
        const uint32_t c_base = base + __shfl_sync(0xFFFFFFFFu, excl, c);  // first output slot of the chunk
        const uint32_t c_total = __shfl_sync(0xFFFFFFFFu, cnt, c);
        if (c_base >= max_out) break;
        const uint32_t piece = c * 32 + lane;
        uint32_t mk = sm.match[p][piece], n = __popc(mk), pi = n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, pi, o);
            if ((int)lane >= o) pi += t;
        }
        uint32_t w = pi - n;
        while (mk) {
            uint32_t b = __ffs(mk) - 1;
            mk &= mk - 1;
            stg[w++] = (uint32_t)(t0 + piece * 16 + b);
        }
        __syncwarp();
        for (uint32_t i = lane; i < c_total && c_base + i < max_out; i += 32) out[c_base + i] = stg[i];
        __syncwarp();
    }
}

cudaError_t launch_search(const SearchArgs &a, cudaStream_t st) {
    if (a.n_tiles == 0 || a.np == 0) return cudaSuccess;
    search_kernel<<<a.n_tiles, SR_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace ol
