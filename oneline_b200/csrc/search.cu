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

// High bit of each byte of x that is zero; may also flag a 0x01 byte right
// above a zero byte (candidates are verified, so that costs nothing).
__device__ __forceinline__ uint32_t zero_bytes_loose(uint32_t x) { return (x - 0x01010101u) & ~x & 0x80808080u; }

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

    const uint32_t stage_len = kSearchTile + halo;  // tile-local bytes held in shared memory
    const uint8_t *gtext = a.text;

    // Phase A: for each pattern, the 16-bit match mask of each of my pieces.
#pragma unroll 1
    for (uint32_t p = 0; p < a.np; p++) {
        const uint32_t m = a.pat_len[p];
        const uint8_t *pat = a.pat[p];
        const uint8_t pf = __ldg(pat), pl = __ldg(pat + m - 1);
        const uint32_t F4 = pf * 0x01010101u;
        // largest tile-local start whose occurrence ends inside the text
        const int64_t last_ok = (int64_t)N - (int64_t)m - (int64_t)t0;
#pragma unroll
        for (uint32_t k = 0; k < SR_STEPS; k++) {
            const uint32_t lo = k * 4096 + tid * 16;
            uint32_t zw[4] = {zero_bytes_loose(v[k].x ^ F4), zero_bytes_loose(v[k].y ^ F4),
                              zero_bytes_loose(v[k].z ^ F4), zero_bytes_loose(v[k].w ^ F4)};
            uint32_t mk = 0;
            if ((zw[0] | zw[1] | zw[2] | zw[3]) && (int64_t)lo <= last_ok) {
#pragma unroll
                for (uint32_t i = 0; i < 4; i++) {
                    uint32_t zz = zw[i];
                    while (zz) {
                        uint32_t b = 4 * i + ((__ffs(zz) - 8) >> 3);
                        zz &= zz - 1;
                        uint32_t ls = lo + b;  // tile-local start
                        if ((int64_t)ls > last_ok) break;
                        if (sm.text[ls] != pf) continue;  // loose SWAR false positive
                        bool ok;
                        if (ls + m <= stage_len) {
                            ok = sm.text[ls + m - 1] == pl;
                            for (uint32_t j = 1; ok && j + 1 < m; j++) ok = sm.text[ls + j] == __ldg(pat + j);
                        } else {
                            ok = __ldg(gtext + t0 + ls + m - 1) == pl;
                            for (uint32_t j = 1; ok && j + 1 < m; j++) {
                                uint32_t q = ls + j;
                                uint8_t t = q < stage_len ? sm.text[q] : __ldg(gtext + t0 + q);
                                ok = t == __ldg(pat + j);
                            }
                        }
                        if (ok) mk |= 1u << b;
                    }
                }
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
