// Kernel (a)+(b): newline scan fused with per-line classification.
//
// One pass over the text. Each CTA takes the next 16 KiB tile from a ticket
// counter (so every predecessor tile is already running when a tile looks
// back), loads it with 16-byte coalesced vector loads, finds its newlines with
// byte SWAR, compacts their positions in order (warp popc scans), takes its
// global line base from a single-pass decoupled look-back over tile newline
// counts, and classifies every line that starts after one of its newlines while
// the bytes are still in shared memory. A line that runs past the tile plus a
// 256-byte halo is queued for a small fix-up kernel, which reads it from global
// memory once the offsets array is complete.
//
// Replaces crates/oneline-gpu/src/scan.wgsl:20-237 (three passes + a host read
// of the line count) and shader.wgsl:34-134 (one thread per line, byte loads
// from global memory). Semantics: crates/oneline-simd/src/lib.rs:49-66 (line
// starts) and crates/oneline-simd/src/line.rs:8-81 (classification).
#include <cuda_runtime.h>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

constexpr uint32_t PT_THREADS = 256;
constexpr uint32_t PT_STEPS = 4;                          // 16-byte pieces per thread
constexpr uint32_t PT_TILE = PT_THREADS * 16 * PT_STEPS;  // 16384
constexpr uint32_t PT_HALO = 256;

static_assert(PT_TILE == kParseTile && PT_HALO == kParseHalo, "tile geometry");

struct ParseSmem {
    alignas(16) uint8_t text[PT_TILE + PT_HALO];
    uint16_t nl[PT_TILE];            // local newline positions, ascending
    uint32_t warp_tot[PT_STEPS][8];  // newline count per (step, warp)
    uint32_t warp_base[PT_STEPS][8];
    uint32_t halo_first;             // first newline in the halo (local), or NONE
    uint32_t tile;
    uint32_t nl_base;                // newlines before this tile
    uint32_t n_nl;                   // newlines in this tile
    uint32_t max_depth;
};

__global__ void __launch_bounds__(PT_THREADS) parse_tiles_kernel(ParseArgs a) {
    extern __shared__ __align__(16) uint8_t parse_smem_raw[];
    ParseSmem &sm = *reinterpret_cast<ParseSmem *>(parse_smem_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) {
        sm.tile = atomicAdd(&a.stats->ticket, 1u);
        sm.halo_first = NONE;
        sm.max_depth = 0;
    }
    __syncthreads();
    const uint32_t tile = sm.tile;
    const uint64_t t0 = (uint64_t)tile * PT_TILE;
    const uint64_t N = a.text_len;

    // 1. Coalesced 16-byte loads: step k covers [t0 + k*4096, +4096), lane-major.
    uint4 v[PT_STEPS];
#pragma unroll
    for (uint32_t k = 0; k < PT_STEPS; k++) v[k] = ld_stream16(a.text + t0 + k * 4096 + tid * 16);
    uint4 vh = make_uint4(0, 0, 0, 0);
    if (tid < PT_HALO / 16) vh = ld_stream16(a.text + t0 + PT_TILE + tid * 16);

#pragma unroll
    for (uint32_t k = 0; k < PT_STEPS; k++) *reinterpret_cast<uint4 *>(&sm.text[k * 4096 + tid * 16]) = v[k];
    if (tid < PT_HALO / 16) *reinterpret_cast<uint4 *>(&sm.text[PT_TILE + tid * 16]) = vh;

    // 2. Newline masks, only for positions < N.
    const uint32_t NL4 = 0x0A0A0A0Au;
    uint32_t m[PT_STEPS];
#pragma unroll
    for (uint32_t k = 0; k < PT_STEPS; k++) {
        uint64_t p0 = t0 + k * 4096 + tid * 16;
        uint32_t mk = eq_mask16(v[k], NL4);
        if (p0 + 16 > N) mk &= p0 >= N ? 0u : ((1u << (uint32_t)(N - p0)) - 1u);
        m[k] = mk;
    }
    if (tid < PT_HALO / 16) {
        uint64_t p0 = t0 + PT_TILE + tid * 16;
        uint32_t mh = eq_mask16(vh, NL4);
        if (p0 + 16 > N) mh &= p0 >= N ? 0u : ((1u << (uint32_t)(N - p0)) - 1u);
        uint32_t first = mh ? PT_TILE + tid * 16 + __ffs(mh) - 1 : NONE;
        // lanes 0..15 of warp 0
        for (int o = 8; o > 0; o >>= 1) first = min(first, __shfl_xor_sync(0x0000FFFFu, first, o));
        if (tid == 0) sm.halo_first = first;
    }

    // 3. Per-(step, warp) exclusive scans of the newline counts.
    uint32_t rank[PT_STEPS];
#pragma unroll
    for (uint32_t k = 0; k < PT_STEPS; k++) {
        uint32_t c = __popc(m[k]), inc = c;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += t;
        }
        rank[k] = inc - c;
        if (lane == 31) sm.warp_tot[k][warp] = inc;
    }
    __syncthreads();
    if (warp == 0) {
        // 32 (step, warp) totals in position order: index = k*8 + w.
        uint32_t c = sm.warp_tot[lane >> 3][lane & 7], inc = c;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += t;
        }
        sm.warp_base[lane >> 3][lane & 7] = inc - c;
        uint32_t total = __shfl_sync(0xFFFFFFFFu, inc, 31);
        if (lane == 0) {
            sm.n_nl = total;
            // Publish the aggregate (tile 0 publishes its prefix at once).
            st_relaxed_u64(a.tile_status + tile, (uint64_t)total | (tile == 0 ? LB_PREFIX : LB_AGGREGATE));
        }
    }
    __syncthreads();

    // 4. Ordered list of newline positions.
#pragma unroll
    for (uint32_t k = 0; k < PT_STEPS; k++) {
        uint32_t r = sm.warp_base[k][warp] + rank[k];
        uint32_t mk = m[k];
        while (mk) {
            uint32_t b = __ffs(mk) - 1;
            mk &= mk - 1;
            sm.nl[r++] = (uint16_t)(k * 4096 + tid * 16 + b);
        }
    }

    // 5. Look-back for the number of newlines before this tile.
    if (warp == 0) {
        uint32_t base = tile == 0 ? 0u : lb_sum_exclusive(a.tile_status, tile, &a.stats->error);
        if (lane == 0) {
            sm.nl_base = base;
            if (tile != 0) st_relaxed_u64(a.tile_status + tile, (uint64_t)(base + sm.n_nl) | LB_PREFIX);
            if (tile == a.n_tiles - 1) {
                // L = 1 + newlines before the last byte.
                uint32_t total_nl = base + sm.n_nl;
                uint32_t last_is_nl = a.text[N - 1] == '\n';
                a.stats->line_count = 1u + total_nl - last_is_nl;
            }
        }
    }
    __syncthreads();

    // 6. Classify the lines that start in this tile (after one of its newlines,
    //    plus line 0 for tile 0).
    const uint32_t n_nl = sm.n_nl, off = tile == 0 ? 1u : 0u;
    const uint32_t n_lines = n_nl + off;
    const uint64_t stage_end = t0 + PT_TILE + PT_HALO;
    const uint32_t halo_first = sm.halo_first;
    uint32_t my_max = 0;
    auto at = [&](uint32_t pos) -> uint8_t { return sm.text[pos - t0]; };
    for (uint32_t j = tid; j < n_lines; j += PT_THREADS) {
        int32_t q = (int32_t)j - (int32_t)off;  // newline that precedes the line (-1: none)
        uint64_t s = q < 0 ? 0 : t0 + sm.nl[q] + 1;
        if (s >= N) continue;  // the final '\n' starts no line
        uint32_t idx = sm.nl_base + j + 1 - off;
        uint64_t e;
        if ((uint32_t)(q + 1) < n_nl) e = t0 + sm.nl[q + 1];
        else if (halo_first != NONE) e = t0 + halo_first;
        else if (N <= stage_end) e = N;
        else {
            // Runs past the halo: classified by the fix-up kernel.
            uint32_t slot = atomicAdd(&a.stats->fixup_count, 1u);
            if (slot < a.fixup_cap) a.fixup[slot] = make_uint2(idx, (uint32_t)s);
            else atomicOr(&a.stats->error, OL_DEVERR_FIXUP);
            if (idx < a.line_cap) a.offsets[idx] = (uint32_t)s;
            else atomicOr(&a.stats->error, OL_DEVERR_CAPACITY);
            continue;
        }
        FlatNode nd = classify_line((uint32_t)s, (uint32_t)e, at);
        if (idx >= a.line_cap) {
            atomicOr(&a.stats->error, OL_DEVERR_CAPACITY);
            continue;
        }
        a.offsets[idx] = (uint32_t)s;
        a.kinds[idx] = (uint8_t)nd.kind;
        a.depth8[idx] = (uint8_t)min(nd.depth, 255u);
        if (nd.kind != KIND_BLANK) my_max = max(my_max, nd.depth);
        if (a.nodes) a.nodes[idx] = nd;
    }
    for (int o = 16; o > 0; o >>= 1) my_max = max(my_max, __shfl_xor_sync(0xFFFFFFFFu, my_max, o));
    if (lane == 0 && my_max) atomicMax(&a.stats->max_content_depth, my_max);
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
        if (a.nodes) a.nodes[idx] = nd;
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
    cudaError_t e0 = cudaFuncSetAttribute(parse_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)sizeof(ParseSmem));
    if (e0 != cudaSuccess) return e0;
    parse_tiles_kernel<<<a.n_tiles, PT_THREADS, sizeof(ParseSmem), st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    uint32_t blocks = a.fixup_cap < 64 ? 8 : 64;
    parse_fixup_kernel<<<blocks, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_classify_lines(const uint8_t *text, uint64_t N, const uint32_t *offsets, uint32_t L, FlatNode *nodes,
                                  uint32_t *depth32, cudaStream_t st) {
    if (L == 0) return cudaSuccess;
    classify_lines_kernel<<<(L + 255) / 256, 256, 0, st>>>(text, N, offsets, L, nodes, depth32);
    return cudaGetLastError();
}

}  // namespace ol
