// Kernel (d): substring search, every overlapping occurrence, ascending.
//
// Each CTA takes the next 16 KiB tile from a ticket counter and stages it plus
// a halo of pattern_len-1 bytes in shared memory with 16-byte coalesced loads.
// Candidates are positions whose first byte equals the pattern's first byte
// and whose byte at +len-1 equals its last byte (byte SWAR on 16-byte pieces);
// each candidate is verified against the whole pattern in shared memory and
// must end inside the text (the buffer is zero padded; a pattern ending in NUL
// must not match the padding). Matches are ranked in position order with warp
// popc scans, the tile's first output slot comes from a decoupled look-back
// over tile match counts, and the first max_out offsets are written in order:
// no host sort, and a truncated result is the lowest max_out offsets.
//
// Semantics: crates/oneline-simd/src/search.rs:88-114 (every overlapping
// occurrence, ascending). Replaces crates/oneline-gpu/src/search.wgsl:101-173
// (4-byte window filter, atomics, host sort).
#include <cuda_runtime.h>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

constexpr uint32_t SR_THREADS = 256;
constexpr uint32_t SR_STEPS = 4;
static_assert(SR_THREADS * 16 * SR_STEPS == kSearchTile, "search tile");

struct SearchSmem {
    alignas(16) uint8_t text[kSearchTile + kSearchMaxStagedPattern + 16];
    alignas(16) uint8_t pat[kSearchMaxStagedPattern];
    uint32_t warp_tot[SR_STEPS][8];
    uint32_t warp_base[SR_STEPS][8];
    uint32_t tile;
    uint32_t base;
};

// 16 bytes of shared memory starting at any byte offset.
__device__ __forceinline__ uint4 lds16_unaligned(const uint8_t *smem, uint32_t off) {
    const uint32_t *w = reinterpret_cast<const uint32_t *>(smem) + (off >> 2);
    uint32_t sh = (off & 3) * 8;
    uint32_t a0 = w[0], a1 = w[1], a2 = w[2], a3 = w[3], a4 = w[4];
    return make_uint4(__funnelshift_r(a0, a1, sh), __funnelshift_r(a1, a2, sh), __funnelshift_r(a2, a3, sh),
                      __funnelshift_r(a3, a4, sh));
}

__global__ void __launch_bounds__(SR_THREADS) search_kernel(SearchArgs a) {
    __shared__ SearchSmem sm;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) sm.tile = atomicAdd(a.ticket, 1u);
    __syncthreads();
    const uint32_t tile = sm.tile;
    const uint64_t t0 = (uint64_t)tile * kSearchTile;
    const uint64_t N = a.text_len;
    const uint32_t m = a.pat_len;
    const bool staged = m <= kSearchMaxStagedPattern;
    const uint32_t halo = staged ? ((m - 1 + 15) & ~15u) : 0u;  // bytes past the tile
    const uint32_t pat_staged = staged ? m : kSearchMaxStagedPattern;

    uint4 v[SR_STEPS];
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) v[k] = ld_stream16(a.text + t0 + k * 4096 + tid * 16);
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) *reinterpret_cast<uint4 *>(&sm.text[k * 4096 + tid * 16]) = v[k];
    for (uint32_t o = tid * 16; o < halo; o += SR_THREADS * 16)
        *reinterpret_cast<uint4 *>(&sm.text[kSearchTile + o]) = ld_stream16(a.text + t0 + kSearchTile + o);
    // Stage 4 words past the halo as well (unaligned 16-byte reads may touch them).
    if (tid < 1) *reinterpret_cast<uint4 *>(&sm.text[kSearchTile + halo]) = make_uint4(0, 0, 0, 0);
    for (uint32_t o = tid; o < pat_staged; o += SR_THREADS) sm.pat[o] = a.pattern[o];
    __syncthreads();

    const uint8_t p0 = sm.pat[0];
    const uint8_t pl = staged ? sm.pat[m - 1] : a.pattern[m - 1];
    const uint32_t F4 = p0 * 0x01010101u, L4 = pl * 0x01010101u;
    const uint64_t stage_end = t0 + kSearchTile + halo;
    const uint8_t *gtext = a.text;
    const uint8_t *gpat = a.pattern;
    auto tat = [&](uint64_t pos) -> uint8_t { return pos < stage_end ? sm.text[pos - t0] : __ldg(gtext + pos); };
    auto pat = [&](uint32_t i) -> uint8_t { return i < kSearchMaxStagedPattern ? sm.pat[i] : __ldg(gpat + i); };

    uint32_t match[SR_STEPS];
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) {
        const uint32_t off = k * 4096 + tid * 16;
        const uint64_t p0g = t0 + off;
        uint32_t cand = eq_mask16(v[k], F4);
        // only starts whose occurrence fits in the text: p + m <= N
        if (N < m) {
            cand = 0;
        } else {
            uint64_t last_ok = N - m;  // largest valid start
            if (p0g > last_ok) cand = 0;
            else if (p0g + 15 > last_ok) cand &= (1u << (uint32_t)(last_ok - p0g + 1)) - 1u;
        }
        if (cand && m > 1) {
            uint4 w;
            if (staged) {
                w = lds16_unaligned(sm.text, off + m - 1);
            } else {
                // Only candidate starts (all < N - m + 1) are read: in bounds.
                uint8_t b[16];
#pragma unroll
                for (int r = 0; r < 16; r++) b[r] = (cand >> r) & 1u ? __ldg(gtext + p0g + m - 1 + r) : (uint8_t)~pl;
                w = *reinterpret_cast<uint4 *>(b);
            }
            cand &= eq_mask16(w, L4);
        }
        uint32_t mk = 0;
        while (cand) {
            uint32_t b = __ffs(cand) - 1;
            cand &= cand - 1;
            uint64_t p = p0g + b;
            bool ok = true;
            for (uint32_t i = 1; i + 1 < m; i++) {
                if (tat(p + i) != pat(i)) {
                    ok = false;
                    break;
                }
            }
            if (ok) mk |= 1u << b;
        }
        match[k] = mk;
    }

    // Rank the matches in position order: (step, warp, lane, bit).
    uint32_t rank[SR_STEPS];
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) {
        uint32_t c = __popc(match[k]), inc = c;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += t;
        }
        rank[k] = inc - c;
        if (lane == 31) sm.warp_tot[k][warp] = inc;
    }
    __syncthreads();
    if (warp == 0) {
        uint32_t c = sm.warp_tot[lane >> 3][lane & 7], inc = c;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += t;
        }
        sm.warp_base[lane >> 3][lane & 7] = inc - c;
        uint32_t total = __shfl_sync(0xFFFFFFFFu, inc, 31);
        if (lane == 0) st_relaxed_u64(a.tile_status + tile, (uint64_t)total | (tile == 0 ? LB_PREFIX : LB_AGGREGATE));
        uint32_t base = tile == 0 ? 0u : lb_sum_exclusive(a.tile_status, tile, a.error);
        if (lane == 0) {
            sm.base = base;
            if (tile != 0) st_relaxed_u64(a.tile_status + tile, (uint64_t)(base + total) | LB_PREFIX);
            if (tile == a.n_tiles - 1) *a.total = base + total;
        }
    }
    __syncthreads();
    const uint32_t base = sm.base;
#pragma unroll
    for (uint32_t k = 0; k < SR_STEPS; k++) {
        uint32_t r = base + sm.warp_base[k][warp] + rank[k];
        uint32_t mk = match[k];
        while (mk && r < a.max_out) {
            uint32_t b = __ffs(mk) - 1;
            mk &= mk - 1;
            a.out[r++] = (uint32_t)(t0 + k * 4096 + tid * 16 + b);
        }
    }
}

cudaError_t launch_search(const SearchArgs &a, cudaStream_t st) {
    if (a.n_tiles == 0) return cudaSuccess;
    search_kernel<<<a.n_tiles, SR_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace ol
