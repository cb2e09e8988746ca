// Kernel (c): tree links from the per-line depth sequence.
//
//   parent[i]       nearest previous content line with a smaller depth (PSV)
//   subtree_end[i]  nearest next content line with depth <= depth[i], else L
//   first_child[i]  next content line j if depth[j] > depth[i], else NONE
//   next_sibling[i] j = subtree_end[i] when parent[j] == parent[i], else NONE
// Blank lines: parent NONE, subtree_end i+1, no children, no sibling.
// Semantics: crates/oneline-core/src/links.rs:52-82 (sequential stack) and
// crates/oneline-simd/src/links.rs:135-180; first_child / next_sibling are
// derived from those links.
//
// Fast path (every content line has depth < 32): two single-pass kernels with
// a per-level decoupled look-back.
//   forward : each thread owns 16 consecutive lines; per level k it records the
//             last line of depth k in its run; a per-level max-scan over the
//             threads and a per-level look-back over tiles give every thread the
//             last line of each depth before its run, from which it rebuilds the
//             ancestor stack as a 32-bit level mask and resolves parents in O(1)
//             per line. It also stores each line's parent depth (1 byte).
//   backward: the mirror image (tiles taken from the end, per-level min of the
//             first line of each depth after a run) gives subtree_end, the next
//             content line (first_child) and, with the parent depth from the
//             forward pass, next_sibling: j = subtree_end[i] shares i's parent
//             exactly when i has no parent or its parent is shallower than j.
// Replaces crates/oneline-gpu/src/tree.wgsl:128-375 (seven passes).
//
// Any-depth path: 32-ary min tree over the depths; each line searches left
// (strictly smaller) and right (smaller or equal) through it.
#include <cuda_runtime.h>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

constexpr uint32_t TR_THREADS = 256;
constexpr uint32_t TR_RUN = 16;
static_assert(TR_THREADS * TR_RUN == kTreeTile, "tree tile");

struct TreeSmem {
    uint32_t lvl[kTreeLevels][TR_THREADS];  // run summary, then exclusive scan, then the stack
    uint32_t in[kTreeLevels];               // look-back result per level
    uint32_t agg[kTreeLevels];
    uint32_t tile;
};

__device__ __forceinline__ uint32_t mask_below(uint32_t d) { return d >= 32 ? 0xFFFFFFFFu : ((1u << d) - 1u); }
__device__ __forceinline__ uint32_t mask_le(uint32_t d) { return d >= 31 ? 0xFFFFFFFFu : ((2u << d) - 1u); }

__device__ __forceinline__ void load16(const uint8_t *p, uint64_t first, uint32_t L, uint8_t out[16]) {
    if (first + 16 <= L) {
        uint4 v = *reinterpret_cast<const uint4 *>(p + first);
        const uint8_t *b = reinterpret_cast<const uint8_t *>(&v);
#pragma unroll
        for (int r = 0; r < 16; r++) out[r] = b[r];
    } else {
#pragma unroll
        for (int r = 0; r < 16; r++) out[r] = first + r < L ? p[first + r] : 0;
    }
}

__device__ __forceinline__ void store16_u32(uint32_t *p, uint64_t first, uint32_t L, const uint32_t v[16]) {
    if (first + 16 <= L) {
#pragma unroll
        for (int q = 0; q < 4; q++)
            *reinterpret_cast<uint4 *>(p + first + 4 * q) = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else {
#pragma unroll
        for (int r = 0; r < 16; r++)
            if (first + r < L) p[first + r] = v[r];
    }
}

// Warp inclusive scan with max (forward) or min (backward).
template <bool MAX>
__device__ __forceinline__ uint32_t warp_scan(uint32_t x, uint32_t lane, bool reverse) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = reverse ? __shfl_down_sync(0xFFFFFFFFu, x, o) : __shfl_up_sync(0xFFFFFFFFu, x, o);
        bool ok = reverse ? (lane + o < 32) : ((int)lane >= o);
        if (ok) x = MAX ? max(x, t) : min(x, t);
    }
    return x;
}

__global__ void __launch_bounds__(TR_THREADS) tree_forward_kernel(TreeArgs a) {
    __shared__ TreeSmem sm;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) sm.tile = atomicAdd(&a.stats->tree_ticket_fwd, 1u);
    __syncthreads();
    const uint32_t tile = sm.tile;
    const uint64_t first = (uint64_t)tile * kTreeTile + tid * TR_RUN;

    uint8_t kd[16], dp[16];
    load16(a.kinds, first, a.L, kd);
    load16(a.depth8, first, a.L, dp);

    // Run summary: last line (+1) of each depth in my run; 0 = none.
#pragma unroll
    for (uint32_t k = 0; k < kTreeLevels; k++) sm.lvl[k][tid] = 0;
#pragma unroll
    for (int r = 0; r < 16; r++)
        if (first + r < a.L && kd[r] != KIND_BLANK) sm.lvl[min((uint32_t)dp[r], kTreeLevels - 1)][tid] = (uint32_t)(first + r + 1);
    __syncthreads();

    // Exclusive max-scan across the threads, per level; warp w owns levels w, w+8, ...
    for (uint32_t k = warp; k < kTreeLevels; k += 8) {
        uint32_t run = 0;
        for (uint32_t j = 0; j < TR_THREADS / 32; j++) {
            uint32_t x = sm.lvl[k][j * 32 + lane];
            uint32_t inc = warp_scan<true>(x, lane, false);
            uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, inc, 1);
            sm.lvl[k][j * 32 + lane] = max(run, lane == 0 ? 0u : prev);
            run = max(run, __shfl_sync(0xFFFFFFFFu, inc, 31));
        }
        if (lane == 0) sm.agg[k] = run;
    }
    __syncthreads();

    // Per-level look-back (lane k carries level k).
    if (warp == 0) {
        uint64_t *st = a.status_fwd + (uint64_t)tile * kTreeLevels;
        uint32_t agg = sm.agg[lane];
        st_relaxed_u64(st + lane, (uint64_t)agg | (tile == 0 ? LB_PREFIX : LB_AGGREGATE));
        uint32_t in = 0;
        if (tile > 0)
            in = lb_lane_exclusive(a.status_fwd, tile, kTreeLevels, 0u, &a.stats->error,
                                   [](uint32_t v, uint32_t acc) { return max(v, acc); });
        if (tile > 0) st_relaxed_u64(st + lane, (uint64_t)max(in, agg) | LB_PREFIX);
        sm.in[lane] = in;
    }
    __syncthreads();

    // Rebuild the ancestor stack before my run: level k is on it iff the last
    // line of depth k comes after every line of smaller depth.
    uint32_t M = 0, runmax = 0;
#pragma unroll
    for (uint32_t k = 0; k < kTreeLevels; k++) {
        uint32_t v = max(sm.in[k], sm.lvl[k][tid]);
        if (v > runmax) {
            M |= 1u << k;
            runmax = v;
        }
        sm.lvl[k][tid] = v;  // my column now holds the stack entries (line + 1)
    }

    uint32_t par[16];
    uint8_t pd[16];
#pragma unroll
    for (int r = 0; r < 16; r++) {
        uint64_t i = first + r;
        par[r] = NONE;
        pd[r] = 0xFF;
        if (i >= a.L || kd[r] == KIND_BLANK) continue;
        uint32_t d = dp[r];
        if (d >= kTreeLevels) {
            atomicOr(&a.stats->error, OL_DEVERR_DEEP);
            d = kTreeLevels - 1;
        }
        uint32_t low = M & mask_below(d);
        if (low) {
            uint32_t top = 31 - __clz(low);
            par[r] = sm.lvl[top][tid] - 1;
            pd[r] = (uint8_t)top;
        }
        M = low | (1u << d);
        sm.lvl[d][tid] = (uint32_t)(i + 1);
    }
    store16_u32(a.parent, first, a.L, par);
    if (first + 16 <= a.L) {
        uint4 v;
        uint8_t *b = reinterpret_cast<uint8_t *>(&v);
#pragma unroll
        for (int r = 0; r < 16; r++) b[r] = pd[r];
        *reinterpret_cast<uint4 *>(a.pdepth + first) = v;
    } else {
#pragma unroll
        for (int r = 0; r < 16; r++)
            if (first + r < a.L) a.pdepth[first + r] = pd[r];
    }
}

__global__ void __launch_bounds__(TR_THREADS) tree_backward_kernel(TreeArgs a) {
    __shared__ TreeSmem sm;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) sm.tile = atomicAdd(&a.stats->tree_ticket_bwd, 1u);
    __syncthreads();
    const uint32_t order = sm.tile;             // processing order: from the end
    const uint32_t tile = a.n_tiles - 1 - order;  // line range of this block
    const uint64_t first = (uint64_t)tile * kTreeTile + tid * TR_RUN;

    uint8_t kd[16], dp[16], pd[16];
    load16(a.kinds, first, a.L, kd);
    load16(a.depth8, first, a.L, dp);
    load16(a.pdepth, first, a.L, pd);

    // Run summary: first line of each depth in my run; NONE = none.
#pragma unroll
    for (uint32_t k = 0; k < kTreeLevels; k++) sm.lvl[k][tid] = NONE;
#pragma unroll
    for (int r = 15; r >= 0; r--)
        if (first + r < a.L && kd[r] != KIND_BLANK) sm.lvl[min((uint32_t)dp[r], kTreeLevels - 1)][tid] = (uint32_t)(first + r);
    __syncthreads();

    // Exclusive suffix min-scan across the threads, per level.
    for (uint32_t k = warp; k < kTreeLevels; k += 8) {
        uint32_t run = NONE;
        for (int j = TR_THREADS / 32 - 1; j >= 0; j--) {
            uint32_t x = sm.lvl[k][j * 32 + lane];
            uint32_t inc = warp_scan<false>(x, lane, true);
            uint32_t next = __shfl_down_sync(0xFFFFFFFFu, inc, 1);
            sm.lvl[k][j * 32 + lane] = min(run, lane == 31 ? NONE : next);
            run = min(run, __shfl_sync(0xFFFFFFFFu, inc, 0));
        }
        if (lane == 0) sm.agg[k] = run;
    }
    __syncthreads();

    if (warp == 0) {
        uint64_t *st = a.status_bwd + (uint64_t)order * kTreeLevels;
        uint32_t agg = sm.agg[lane];
        st_relaxed_u64(st + lane, (uint64_t)agg | (order == 0 ? LB_PREFIX : LB_AGGREGATE));
        uint32_t in = NONE;
        if (order > 0)
            in = lb_lane_exclusive(a.status_bwd, order, kTreeLevels, NONE, &a.stats->error,
                                   [](uint32_t v, uint32_t acc) { return min(v, acc); });
        if (order > 0) st_relaxed_u64(st + lane, (uint64_t)min(in, agg) | LB_PREFIX);
        sm.in[lane] = in;
    }
    __syncthreads();

    // Stack of the lines after my run: level k is on it iff the first line of
    // depth k comes before every line of smaller depth.
    uint32_t M = 0, runmin = NONE;
#pragma unroll
    for (uint32_t k = 0; k < kTreeLevels; k++) {
        uint32_t v = min(sm.in[k], sm.lvl[k][tid]);
        if (v < runmin) {
            M |= 1u << k;
            runmin = v;
        }
        sm.lvl[k][tid] = v;
    }

    uint32_t se[16], fc[16], ns[16];
#pragma unroll
    for (int r = 15; r >= 0; r--) {
        uint64_t i = first + r;
        se[r] = (uint32_t)(i + 1);
        fc[r] = NONE;
        ns[r] = NONE;
        if (i >= a.L || kd[r] == KIND_BLANK) continue;
        uint32_t d = min((uint32_t)dp[r], kTreeLevels - 1);
        if (M) {
            uint32_t nb = 31 - __clz(M);  // nearest following content line
            if (nb > d) fc[r] = sm.lvl[nb][tid];
        }
        uint32_t le = M & mask_le(d);
        if (le) {
            uint32_t top = 31 - __clz(le);
            uint32_t j = sm.lvl[top][tid];
            se[r] = j;
            if (pd[r] == 0xFF || pd[r] < top) ns[r] = j;
        } else {
            se[r] = a.L;
        }
        M = (M & mask_below(d)) | (1u << d);
        sm.lvl[d][tid] = (uint32_t)i;
    }
    if (a.subtree_end) store16_u32(a.subtree_end, first, a.L, se);
    store16_u32(a.first_child, first, a.L, fc);
    store16_u32(a.next_sibling, first, a.L, ns);
}

cudaError_t launch_tree_fast(const TreeArgs &a, cudaStream_t st) {
    if (a.n_tiles == 0) return cudaSuccess;
    tree_forward_kernel<<<a.n_tiles, TR_THREADS, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    tree_backward_kernel<<<a.n_tiles, TR_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

// ------------------------------------------------------------ any depth ----

__global__ void min_level_kernel(const uint32_t *__restrict__ src, uint32_t n, uint32_t *__restrict__ dst, uint32_t m) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= m) return;
    uint32_t v = NONE;
    uint64_t b = (uint64_t)g * 32;
    for (uint32_t c = 0; c < 32 && b + c < n; c++) v = min(v, src[b + c]);
    dst[g] = v;
}

__device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

// Nearest j < i with levels[0][j] < d, through the 32-ary min tree.
__device__ uint32_t deep_prev_less(const TreeDeepArgs &a, uint32_t i, uint32_t d) {
    int64_t pos = i;
    for (uint32_t lv = 0; lv < a.n_levels; lv++) {
        const uint32_t *v = a.levels[lv];
        int64_t g0 = (pos >> 5) << 5;
        for (int64_t j = pos - 1; j >= g0; j--) {
            if (v[j] < d) {
                uint64_t node = (uint64_t)j;
                for (int64_t l = (int64_t)lv - 1; l >= 0; l--) {
                    const uint32_t *c = a.levels[l];
                    uint64_t lo = node * 32, hi = umin64(lo + 32, a.level_len[l]);
                    for (uint64_t x = hi; x-- > lo;) {
                        if (c[x] < d) {
                            node = x;
                            break;
                        }
                    }
                }
                return (uint32_t)node;
            }
        }
        pos >>= 5;
    }
    return NONE;
}

// Nearest j > i with levels[0][j] <= d.
__device__ uint32_t deep_next_le(const TreeDeepArgs &a, uint32_t i, uint32_t d) {
    uint64_t pos = (uint64_t)i + 1;
    for (uint32_t lv = 0; lv < a.n_levels; lv++) {
        const uint32_t *v = a.levels[lv];
        uint64_t gend = umin64(((pos >> 5) + 1) << 5, a.level_len[lv]);
        for (uint64_t j = pos; j < gend; j++) {
            if (v[j] <= d) {
                uint64_t node = j;
                for (int64_t l = (int64_t)lv - 1; l >= 0; l--) {
                    const uint32_t *c = a.levels[l];
                    uint64_t lo = node * 32, hi = umin64(lo + 32, a.level_len[l]);
                    for (uint64_t x = lo; x < hi; x++) {
                        if (c[x] <= d) {
                            node = x;
                            break;
                        }
                    }
                }
                return (uint32_t)node;
            }
        }
        pos = (pos >> 5) + 1;
    }
    return NONE;
}

__global__ void deep_links_kernel(TreeDeepArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.L) return;
    uint32_t d = a.keys[i];
    if (d == NONE) {
        a.parent[i] = NONE;
        if (a.subtree_end) a.subtree_end[i] = i + 1;
        return;
    }
    a.parent[i] = d == 0 ? NONE : deep_prev_less(a, i, d);
    uint32_t e = deep_next_le(a, i, d);
    if (a.subtree_end) a.subtree_end[i] = e == NONE ? a.L : e;
}

__global__ void deep_children_kernel(TreeDeepArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.L) return;
    uint32_t d = a.keys[i];
    if (d == NONE) {
        a.first_child[i] = NONE;
        a.next_sibling[i] = NONE;
        return;
    }
    uint32_t nb = deep_next_le(a, i, NONE - 1);  // next content line
    a.first_child[i] = (nb != NONE && a.keys[nb] > d) ? nb : NONE;
    uint32_t e = deep_next_le(a, i, d);
    a.next_sibling[i] = (e != NONE && a.parent[e] == a.parent[i]) ? e : NONE;
}

cudaError_t launch_tree_deep(const TreeDeepArgs &a, cudaStream_t st) {
    if (a.L == 0) return cudaSuccess;
    for (uint32_t l = 1; l < a.n_levels; l++) {
        uint32_t m = a.level_len[l];
        min_level_kernel<<<(m + 255) / 256, 256, 0, st>>>(a.levels[l - 1], a.level_len[l - 1], a.levels[l], m);
    }
    deep_links_kernel<<<(a.L + 255) / 256, 256, 0, st>>>(a);
    deep_children_kernel<<<(a.L + 255) / 256, 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace ol
