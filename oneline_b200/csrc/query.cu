// Node query filter: the lines of a range whose kind and depth match, in
// ascending order. Replaces filter_nodes / filter_fused
// (crates/oneline-gpu/src/shader.wgsl:136-193) and their slot atomics with a
// count pass, a column scan and a writing pass, so a truncated answer is the
// lowest max_out lines rather than an arbitrary subset.
//
// Filter semantics (shader.wgsl:152-160, query.rs:138-139): target_kind 0
// accepts every kind (so the reference cannot ask for Blank lines either), and
// target_depth 0xFFFFFFFF accepts every depth.
#include <cuda_runtime.h>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

constexpr uint32_t QY_THREADS = 256;
constexpr uint32_t QY_PER_THREAD = 16;
constexpr uint32_t QY_LINES = QY_THREADS * QY_PER_THREAD;  // lines per block

uint32_t query_blocks(uint32_t lines) { return (lines + QY_LINES - 1) / QY_LINES; }

__device__ __forceinline__ bool query_match(const QueryArgs &a, uint32_t i) {
    uint32_t kind, depth8;
    if (a.nodes) {
        FlatNode nd = a.nodes[i];
        if (a.target_kind != 0 && nd.kind != a.target_kind) return false;
        return a.target_depth == NONE || nd.depth == a.target_depth;
    }
    kind = a.kinds[i];
    if (a.target_kind != 0 && kind != a.target_kind) return false;
    if (a.target_depth == NONE) return true;
    depth8 = a.depth8[i];
    if (depth8 < 255) return depth8 == a.target_depth;
    if (a.target_depth < 255) return false;
    // 255 or deeper: the exact depth from the text
    const uint32_t s = a.offsets[i];
    const uint32_t last_end = a.text[a.text_len - 1] == '\n' ? (uint32_t)(a.text_len - 1) : (uint32_t)a.text_len;
    const uint32_t e = i + 1 < a.lines ? a.offsets[i + 1] - 1 : last_end;
    FlatNode nd = classify_line(s, e, [&](uint32_t p) -> uint8_t { return __ldg(a.text + p); });
    return nd.depth == a.target_depth;
}

// 16 consecutive lines of the range per thread: bit j = line lo + 16t + j matches.
__device__ __forceinline__ uint32_t query_mask(const QueryArgs &a, uint32_t first) {
    uint32_t m = 0;
    for (uint32_t j = 0; j < QY_PER_THREAD; j++) {
        uint32_t i = first + j;
        if (i < a.hi && query_match(a, i)) m |= 1u << j;
    }
    return m;
}

__device__ __forceinline__ uint32_t qy_block_exclusive(uint32_t x, uint32_t *warp_sum, uint32_t *total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if ((int)lane >= o) inc += t;
    }
    if (lane == 31) warp_sum[warp] = inc;
    __syncthreads();
    uint32_t before = 0, all = 0;
#pragma unroll
    for (uint32_t w = 0; w < QY_THREADS / 32; w++) {
        before += w < warp ? warp_sum[w] : 0u;
        all += warp_sum[w];
    }
    if (total) *total = all;
    return before + inc - x;
}

__global__ void __launch_bounds__(QY_THREADS) query_count_kernel(QueryArgs a) {
    __shared__ uint32_t warp_sum[QY_THREADS / 32];
    const uint32_t first = a.lo + blockIdx.x * QY_LINES + threadIdx.x * QY_PER_THREAD;
    const uint32_t m = first < a.hi ? query_mask(a, first) : 0u;
    uint32_t total;
    qy_block_exclusive(__popc(m), warp_sum, &total);
    if (threadIdx.x == 0) a.counts[blockIdx.x] = total;
}

__global__ void __launch_bounds__(QY_THREADS) query_write_kernel(QueryArgs a) {
    __shared__ uint32_t warp_sum[QY_THREADS / 32];
    if (a.counts[blockIdx.x] == 0 || a.bases[blockIdx.x] >= a.max_out) return;  // uniform per block
    const uint32_t first = a.lo + blockIdx.x * QY_LINES + threadIdx.x * QY_PER_THREAD;
    uint32_t m = first < a.hi ? query_mask(a, first) : 0u;
    uint32_t r = a.bases[blockIdx.x] + qy_block_exclusive(__popc(m), warp_sum, nullptr);
    while (m && r < a.max_out) {
        uint32_t j = __ffs(m) - 1;
        m &= m - 1;
        a.out[r++] = first + j;
    }
}

cudaError_t launch_query(const QueryArgs &a, cudaStream_t st) {
    if (a.hi <= a.lo) return cudaSuccess;
    const uint32_t blocks = query_blocks(a.hi - a.lo);
    query_count_kernel<<<blocks, QY_THREADS, 0, st>>>(a); OL_LAUNCHED();
    cudaError_t e = launch_scan_columns(a.counts, a.bases, a.total, blocks, 1, scan_ld(blocks), st);
    if (e != cudaSuccess) return e;
    query_write_kernel<<<blocks, QY_THREADS, 0, st>>>(a); OL_LAUNCHED();
    return cudaGetLastError();
}

}  // namespace ol
