// Kernel (d): substring search, every overlapping occurrence, ascending.
//
// One launch searches up to eight patterns in one pass over the text. CTA b
// owns the 16 KiB tile b and stages it, plus a halo of (longest pattern - 1)
// bytes, in shared memory with 16-byte coalesced loads. For each pattern the
// candidates are the positions whose first byte equals the pattern's first
// byte and whose byte at +len-1 equals its last byte (byte SWAR on 16-byte
// pieces, then the last byte per candidate); each candidate is verified
// against the whole pattern and must end inside the text (the buffer is zero
// padded: a pattern ending in NUL must not match the padding). The match masks
// go to shared memory in position order; warp p then counts pattern p's
// matches, runs the decoupled look-back over the tile match counts of pattern
// p (the eight look-backs proceed in parallel) and writes the pattern's first
// max_out offsets in ascending order: no host sort, and a truncated result is
// the lowest max_out offsets.
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

struct SearchSmem {
    alignas(16) uint8_t text[kSearchTile + kSearchMaxStagedPattern + 16];
    alignas(16) uint16_t match[kSearchMaxPatterns][SR_THREADS * SR_STEPS];  // per 16-byte piece, position order
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

// Bytes [off, off+16) of the text as four words: from shared memory when
// staged, else from global memory (bytes at or past N read as zero).
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
    __syncthreads();

    // Phase A: for each pattern, the 16-bit match mask of each of my pieces.
    // Filter: first byte (SWAR over the piece) then the last byte (SWAR over the
    // piece shifted by len-1); verification: every other byte the same way, for
    // all sixteen starts at once, stopping when no candidate is left.
    // Only the last tiles hold starts whose occurrence would run past the text.
    const bool tail_tile = t0 + kSearchTile + a.halo + 16 > N;
#pragma unroll 1
    for (uint32_t p = 0; p < a.np; p++) {
        const uint32_t m = a.pat_len[p];
        const uint8_t *pat = a.pat[p];
        const uint32_t F4 = __ldg(pat) * 0x01010101u;
#pragma unroll
        for (uint32_t k = 0; k < SR_STEPS; k++) {
            const uint32_t lo = k * 4096 + tid * 16;
            // loose first-byte filter: 3 operations per word
            uint32_t c0 = zero_bytes_loose(v[k].x ^ F4), c1 = zero_bytes_loose(v[k].y ^ F4);
            uint32_t c2 = zero_bytes_loose(v[k].z ^ F4), c3 = zero_bytes_loose(v[k].w ^ F4);
            uint32_t mk = 0;
            if (c0 | c1 | c2 | c3) {
                // exact first byte (drops the loose test's false positives)
                c0 = zero_bytes(v[k].x ^ F4);
                c1 = zero_bytes(v[k].y ^ F4);
                c2 = zero_bytes(v[k].z ^ F4);
                c3 = zero_bytes(v[k].w ^ F4);
                if (tail_tile) {  // starts past N - m cannot match
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
                for (uint32_t jj = 1; jj < m && (c0 | c1 | c2 | c3); jj++) {
                    const uint32_t j = jj == 1 ? m - 1 : jj - 1;  // last byte first, then 1, 2, ...
                    const uint32_t P4 = __ldg(pat + j) * 0x01010101u;
                    uint4 w = window16(sm.text, lo + j, staged, a.text, t0, N);
                    c0 &= zero_bytes(w.x ^ P4);
                    c1 &= zero_bytes(w.y ^ P4);
                    c2 &= zero_bytes(w.z ^ P4);
                    c3 &= zero_bytes(w.w ^ P4);
                }
                mk = gather16(c0, c1, c2, c3);
            }
            sm.match[p][k * SR_THREADS + tid] = (uint16_t)mk;
        }
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
    const uint32_t base = tile == 0 ? 0u : lb_sum_exclusive(a.tile_status + p, tile, a.error, kSearchMaxPatterns);
    if (lane == 0) {
        if (tile != 0) st_relaxed_u64(st, (uint64_t)(base + total) | LB_PREFIX);
        if (tile == a.n_tiles - 1) a.totals[p] = base + total;
    }
    uint32_t r = base + inc - cnt;
    const uint32_t max_out = a.max_out[p];
    if (cnt == 0 || r >= max_out) return;
    uint32_t *out = a.out[p];
    const uint16_t *mine = &sm.match[p][lane * 32];
    for (uint32_t x = 0; x < 32 && r < max_out; x++) {
        uint32_t mk = mine[x];
        while (mk && r < max_out) {
            uint32_t b = __ffs(mk) - 1;
            mk &= mk - 1;
            out[r++] = (uint32_t)(t0 + (lane * 32 + x) * 16 + b);
        }
    }
}

cudaError_t launch_search(const SearchArgs &a, cudaStream_t st) {
    if (a.n_tiles == 0 || a.np == 0) return cudaSuccess;
    search_kernel<<<a.n_tiles, SR_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace ol
