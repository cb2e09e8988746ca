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
// Fast path (every content line has depth < 32; D = max depth + 1 levels),
// three kernels over tiles of 4096 lines (256 threads x 16 consecutive lines):
//   summary : per tile and level k, the last and the first line of depth k;
//   scan    : per level, the exclusive prefix max (last line before the tile)
//             and suffix min (first line after it) over the tiles;
//   resolve : per level, the same scans over the threads of the tile give
//             every thread the last line of each depth before its run and the
//             first line of each depth after it. From these it rebuilds the
//             ancestor stack as a 32-bit level mask and walks its 16 lines
//             forward (parent in O(1) per line, the parent's depth kept in
//             registers), then the stack of following lines and walks backward
//             (subtree_end, next content line = first_child candidate, and
//             next_sibling: j = subtree_end[i] shares i's parent exactly when i
//             has no parent or its parent is shallower than j).
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

__device__ __forceinline__ uint32_t mask_below(uint32_t d) { return d >= 32 ? 0xFFFFFFFFu : ((1u << d) - 1u); }
__device__ __forceinline__ uint32_t mask_le(uint32_t d) { return d >= 31 ? 0xFFFFFFFFu : ((2u << d) - 1u); }

// The 16 lines of thread `tid` of tile `tile`: kinds and depths packed four per word.
struct Run {
    uint4 kd, dp;
    uint64_t first;
};

__device__ __forceinline__ Run load_run(const TreeArgs &a, uint32_t tile, uint32_t tid) {
    Run r;
    r.first = (uint64_t)tile * kTreeTile + tid * TR_RUN;
    if (r.first + 16 <= a.L) {
        r.kd = *reinterpret_cast<const uint4 *>(a.kinds + r.first);
        r.dp = *reinterpret_cast<const uint4 *>(a.depth8 + r.first);
    } else {
        uint8_t k[16], d[16];
#pragma unroll
        for (int i = 0; i < 16; i++) {
            bool in = r.first + i < a.L;
            k[i] = in ? a.kinds[r.first + i] : (uint8_t)KIND_BLANK;  // past the end: blank
            d[i] = in ? a.depth8[r.first + i] : (uint8_t)0;
        }
        r.kd = *reinterpret_cast<uint4 *>(k);
        r.dp = *reinterpret_cast<uint4 *>(d);
    }
    return r;
}

__device__ __forceinline__ uint32_t byte_of(const uint4 &v, int i) {
    uint32_t w = i < 4 ? v.x : i < 8 ? v.y : i < 12 ? v.z : v.w;
    return (w >> (8 * (i & 3))) & 0xFF;
}

// Level of a line for the tree, or 0xFF for a blank line. Depths >= levels
// cannot reach this path (the host picks the any-depth path for them).
__device__ __forceinline__ uint32_t level_of(const Run &r, int i, uint32_t levels) {
    if (byte_of(r.kd, i) == KIND_BLANK) return 0xFF;
    return min(byte_of(r.dp, i), levels - 1);
}

// Dynamic shared memory of the summary and resolve kernels: D levels x 256
// threads of "last line + 1" (forward) followed by the same of "first line"
// (backward).
struct TreeSmem {
    uint32_t *fa, *fb;
    uint32_t D;
    __device__ uint32_t &a(uint32_t k, uint32_t t) { return fa[k * TR_THREADS + t]; }
    __device__ uint32_t &b(uint32_t k, uint32_t t) { return fb[k * TR_THREADS + t]; }
};
extern __shared__ __align__(16) uint32_t tree_dyn_smem[];

__device__ __forceinline__ TreeSmem tree_smem(uint32_t D) {
    TreeSmem s;
    s.fa = tree_dyn_smem;
    s.fb = tree_dyn_smem + D * TR_THREADS;
    s.D = D;
    return s;
}

// Pass 1: per tile and level, the last line (+1) and the first line of that depth.
__global__ void __launch_bounds__(TR_THREADS) tree_summary_kernel(TreeArgs a) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, tile = blockIdx.x;
    const uint32_t D = a.levels;
    TreeSmem sm = tree_smem(D);
    Run r = load_run(a, tile, tid);
    for (uint32_t k = 0; k < D; k++) {
        sm.a(k, tid) = 0;
        sm.b(k, tid) = NONE;
    }
#pragma unroll
    for (int i = 0; i < 16; i++) {
        uint32_t d = level_of(r, i, D);
        if (d != 0xFF) sm.a(d, tid) = (uint32_t)(r.first + i + 1);
    }
#pragma unroll
    for (int i = 15; i >= 0; i--) {
        uint32_t d = level_of(r, i, D);
        if (d != 0xFF) sm.b(d, tid) = (uint32_t)(r.first + i);
    }
    __syncthreads();
    for (uint32_t k = warp; k < D; k += 8) {
        uint32_t mx = 0, mn = NONE;
#pragma unroll
        for (int j = 0; j < TR_THREADS / 32; j++) {
            mx = max(mx, sm.a(k, j * 32 + lane));
            mn = min(mn, sm.b(k, j * 32 + lane));
        }
        mx = __reduce_max_sync(0xFFFFFFFFu, mx);
        mn = __reduce_min_sync(0xFFFFFFFFu, mn);
        if (lane == 0) {
            a.tile_last[(size_t)tile * kTreeLevels + k] = mx;
            a.tile_first[(size_t)tile * kTreeLevels + k] = mn;
        }
    }
}

// Pass 2: for each level (one block per level), exclusive prefix max of
// tile_last and exclusive suffix min of tile_first over the tiles.
__global__ void __launch_bounds__(1024) tree_scan_kernel(TreeArgs a) {
    __shared__ uint32_t s_max[32], s_min[32];
    const uint32_t k = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t T = a.n_tiles;
    const uint32_t per = (T + 1023) / 1024;
    const uint32_t lo = min(T, tid * per), hi = min(T, lo + per);
    // Up to kHeld tiles per thread (documents of up to 2^25 lines) are read
    // once, all loads in flight together, and kept in registers for the walks
    // below.
    constexpr uint32_t kHeld = 8;
    const bool held = per <= kHeld;  // uniform
    uint32_t vl[kHeld], vf[kHeld];
    uint32_t mx = 0, mn = NONE;
    if (held) {
#pragma unroll
        for (uint32_t i = 0; i < kHeld; i++) {
            const bool in = lo + i < hi;
            vl[i] = in ? a.tile_last[(size_t)(lo + i) * kTreeLevels + k] : 0u;
            vf[i] = in ? a.tile_first[(size_t)(lo + i) * kTreeLevels + k] : NONE;
        }
#pragma unroll
        for (uint32_t i = 0; i < kHeld; i++) {
            mx = max(mx, vl[i]);
            mn = min(mn, vf[i]);
        }
    } else {
        for (uint32_t t = lo; t < hi; t++) {
            mx = max(mx, a.tile_last[(size_t)t * kTreeLevels + k]);
            mn = min(mn, a.tile_first[(size_t)t * kTreeLevels + k]);
        }
    }
    // inclusive scans over threads: max forward, min backward
    uint32_t imx = mx, imn = mn;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t1 = __shfl_up_sync(0xFFFFFFFFu, imx, o);
        uint32_t t2 = __shfl_down_sync(0xFFFFFFFFu, imn, o);
        if ((int)lane >= o) imx = max(imx, t1);
        if (lane + o < 32) imn = min(imn, t2);
    }
    if (lane == 31) s_max[warp] = imx;
    if (lane == 0) s_min[warp] = imn;
    __syncthreads();
    uint32_t before = 0, after = NONE;  // warps before / after mine
    for (uint32_t w = 0; w < warp; w++) before = max(before, s_max[w]);
    for (uint32_t w = warp + 1; w < 32; w++) after = min(after, s_min[w]);
    // every lane takes part in both shuffles; lanes 0 / 31 discard the result
    const uint32_t up = __shfl_up_sync(0xFFFFFFFFu, imx, 1);
    const uint32_t down = __shfl_down_sync(0xFFFFFFFFu, imn, 1);
    uint32_t ex_mx = max(before, lane == 0 ? 0u : up);
    uint32_t ex_mn = min(after, lane == 31 ? NONE : down);
    // walk my tiles: forward exclusive max, then backward exclusive min
    if (held) {
        uint32_t run = ex_mx;
#pragma unroll
        for (uint32_t i = 0; i < kHeld; i++) {
            if (lo + i < hi) a.in_last[(size_t)(lo + i) * kTreeLevels + k] = run;
            run = max(run, vl[i]);
        }
        run = ex_mn;
#pragma unroll
        for (int i = kHeld - 1; i >= 0; i--) {
            if (lo + i < hi) a.in_first[(size_t)(lo + i) * kTreeLevels + k] = run;
            run = min(run, vf[i]);
        }
        return;
    }
    uint32_t run = ex_mx;
    for (uint32_t t = lo; t < hi; t++) {
        a.in_last[(size_t)t * kTreeLevels + k] = run;
        run = max(run, a.tile_last[(size_t)t * kTreeLevels + k]);
    }
    run = ex_mn;
    for (uint32_t t = hi; t-- > lo;) {
        a.in_first[(size_t)t * kTreeLevels + k] = run;
        run = min(run, a.tile_first[(size_t)t * kTreeLevels + k]);
    }
}

// Pass 3: every thread rebuilds the ancestor stack before its 16 lines and
// the stack of the lines after them, walks forward for parent (and the
// parent's depth, kept in registers) and backward for subtree_end,
// first_child and next_sibling.
__global__ void __launch_bounds__(TR_THREADS, 5) tree_resolve_kernel(TreeArgs a) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, tile = blockIdx.x;
    const uint32_t D = a.levels;
    TreeSmem sm = tree_smem(D);
    Run r = load_run(a, tile, tid);
    for (uint32_t k = 0; k < D; k++) {
        sm.a(k, tid) = 0;
        sm.b(k, tid) = NONE;
    }
#pragma unroll
    for (int i = 0; i < 16; i++) {
        uint32_t d = level_of(r, i, D);
        if (d != 0xFF) sm.a(d, tid) = (uint32_t)(r.first + i + 1);
    }
#pragma unroll
    for (int i = 15; i >= 0; i--) {
        uint32_t d = level_of(r, i, D);
        if (d != 0xFF) sm.b(d, tid) = (uint32_t)(r.first + i);
    }
    __syncthreads();
    // Per level: exclusive max over the threads before mine (seeded with the
    // tiles before this one) and exclusive min over the threads after mine
    // (seeded with the tiles after this one).
    // One warp per level; lane L holds the entries of threads 8L .. 8L+7 (two
    // 16-byte loads), reduces them, and one warp scan of the 32 lane values
    // gives each lane its seed.
    for (uint32_t k = warp; k < D; k += 8) {
        uint4 *ra = reinterpret_cast<uint4 *>(&sm.a(k, 8 * lane));
        uint4 *rb = reinterpret_cast<uint4 *>(&sm.b(k, 8 * lane));
        {
            const uint4 q0 = ra[0], q1 = ra[1];
            uint32_t v[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
            uint32_t inc = 0;
#pragma unroll
            for (int i = 0; i < 8; i++) inc = max(inc, v[i]);
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
                if ((int)lane >= o) inc = max(inc, t);
            }
            const uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, inc, 1);
            uint32_t run = max(a.in_last[(size_t)tile * kTreeLevels + k], lane == 0 ? 0u : prev);
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const uint32_t t = v[i];
                v[i] = run;
                run = max(run, t);
            }
            ra[0] = make_uint4(v[0], v[1], v[2], v[3]);
            ra[1] = make_uint4(v[4], v[5], v[6], v[7]);
        }
        {
            const uint4 q0 = rb[0], q1 = rb[1];
            uint32_t v[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
            uint32_t inc = NONE;
#pragma unroll
            for (int i = 0; i < 8; i++) inc = min(inc, v[i]);
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_down_sync(0xFFFFFFFFu, inc, o);
                if (lane + o < 32) inc = min(inc, t);
            }
            const uint32_t next = __shfl_down_sync(0xFFFFFFFFu, inc, 1);
            uint32_t run = min(a.in_first[(size_t)tile * kTreeLevels + k], lane == 31 ? NONE : next);
#pragma unroll
            for (int i = 7; i >= 0; i--) {
                const uint32_t t = v[i];
                v[i] = run;
                run = min(run, t);
            }
            rb[0] = make_uint4(v[0], v[1], v[2], v[3]);
            rb[1] = make_uint4(v[4], v[5], v[6], v[7]);
        }
    }
    __syncthreads();

    // Forward: level k is on the ancestor stack iff its last line comes after
    // every line of smaller depth.
    uint32_t M = 0, runmax = 0;
    for (uint32_t k = 0; k < D; k++) {
        uint32_t v = sm.a(k, tid);
        if (v > runmax) {
            M |= 1u << k;
            runmax = v;
        }
    }
    uint32_t pdw[4] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};  // parent depth bytes, 0xFF = none
    uint32_t par[4];
#pragma unroll
    for (int i = 0; i < 16; i++) {
        uint32_t d = level_of(r, i, D);
        uint32_t pv = NONE;
        if (d != 0xFF) {
            uint32_t low = M & mask_below(d);
            if (low) {
                uint32_t top = 31 - __clz(low);
                pv = sm.a(top, tid) - 1;
                pdw[i >> 2] = (pdw[i >> 2] & ~(0xFFu << (8 * (i & 3)))) | (top << (8 * (i & 3)));
            }
            M = low | (1u << d);
            sm.a(d, tid) = (uint32_t)(r.first + i + 1);
        }
        par[i & 3] = pv;
        if ((i & 3) == 3) {
            uint64_t at = r.first + (i - 3);
            if (at + 4 <= a.L) *reinterpret_cast<uint4 *>(a.parent + at) = make_uint4(par[0], par[1], par[2], par[3]);
            else
                for (int q = 0; q < 4; q++)
                    if (at + q < a.L) a.parent[at + q] = par[q];
        }
    }

    // Backward: level k is on the stack of following lines iff its first line
    // comes before every line of smaller depth; the highest level on it is the
    // next content line.
    M = 0;
    uint32_t runmin = NONE;
    for (uint32_t k = 0; k < D; k++) {
        uint32_t v = sm.b(k, tid);
        if (v < runmin) {
            M |= 1u << k;
            runmin = v;
        }
    }
    uint32_t se[4], fc[4], ns[4];
#pragma unroll
    for (int i = 15; i >= 0; i--) {
        uint64_t line = r.first + i;
        uint32_t d = level_of(r, i, D);
        uint32_t vse = (uint32_t)(line + 1), vfc = NONE, vns = NONE;
        if (d != 0xFF) {
            if (M) {
                uint32_t nb = 31 - __clz(M);
                if (nb > d) vfc = sm.b(nb, tid);
            }
            uint32_t le = M & mask_le(d);
            if (le) {
                uint32_t top = 31 - __clz(le);
                uint32_t j = sm.b(top, tid);
                vse = j;
                uint32_t pd = (pdw[i >> 2] >> (8 * (i & 3))) & 0xFF;
                if (pd == 0xFF || pd < top) vns = j;
            } else {
                vse = a.L;
            }
            M = (M & mask_below(d)) | (1u << d);
            sm.b(d, tid) = (uint32_t)line;
        }
        se[i & 3] = vse;
        fc[i & 3] = vfc;
        ns[i & 3] = vns;
        if ((i & 3) == 0) {
            uint64_t at = line;
            if (at + 4 <= a.L) {
                if (a.subtree_end) *reinterpret_cast<uint4 *>(a.subtree_end + at) = make_uint4(se[0], se[1], se[2], se[3]);
                *reinterpret_cast<uint4 *>(a.first_child + at) = make_uint4(fc[0], fc[1], fc[2], fc[3]);
                *reinterpret_cast<uint4 *>(a.next_sibling + at) = make_uint4(ns[0], ns[1], ns[2], ns[3]);
            } else {
                for (int q = 0; q < 4; q++) {
                    if (at + q >= a.L) continue;
                    if (a.subtree_end) a.subtree_end[at + q] = se[q];
                    a.first_child[at + q] = fc[q];
                    a.next_sibling[at + q] = ns[q];
                }
            }
        }
    }
}

cudaError_t launch_tree_fast(const TreeArgs &a, cudaStream_t st) {
    if (a.n_tiles == 0) return cudaSuccess;
    size_t smem = (size_t)a.levels * TR_THREADS * 4 * 2;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(tree_summary_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(tree_resolve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    tree_summary_kernel<<<a.n_tiles, TR_THREADS, smem, st>>>(a); OL_LAUNCHED();
    tree_scan_kernel<<<a.levels, 1024, 0, st>>>(a); OL_LAUNCHED();
    tree_resolve_kernel<<<a.n_tiles, TR_THREADS, smem, st>>>(a); OL_LAUNCHED();
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
        min_level_kernel<<<(m + 255) / 256, 256, 0, st>>>(a.levels[l - 1], a.level_len[l - 1], a.levels[l], m); OL_LAUNCHED();
    }
    deep_links_kernel<<<(a.L + 255) / 256, 256, 0, st>>>(a); OL_LAUNCHED();
    deep_children_kernel<<<(a.L + 255) / 256, 256, 0, st>>>(a); OL_LAUNCHED();
    return cudaGetLastError();
}

}  // namespace ol
