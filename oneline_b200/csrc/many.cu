// Kernel (e): dictionary search. Every (pattern, offset) at which one of a set
// of patterns (4..64 bytes, up to 65,536 of them) occurs, ordered by
// (pattern, offset) like ManyPatterns::find_all_par
// (crates/oneline-simd/src/search.rs:259-282). Replaces the reference's
// window-filter kernels and host sort (crates/oneline-gpu/src/many.rs:391-646).
//
// The compiled set (runtime_many.cu) deduplicates the patterns and builds a
// trie over the unique ones; its depth-4 nodes are reached through a hash
// table keyed by a position's first four bytes, and a two-hash filter of those
// keys (16 KiB) sits in shared memory, copied there once per block with a bulk
// TMA copy (cp.async.bulk, no multicast).
//
// dict_match_kernel: persistent blocks walk 16 KiB tiles staged in shared
// memory. Each warp takes 32 consecutive positions at a time (lane = position):
// filter, table probe, then all lanes walk the trie one depth per iteration.
// A unique pattern u of length d is met at depth d by every lane where it
// occurs, so `__match_any_sync` on u at that depth groups exactly those lanes:
//   * heavy patterns (chosen per search from a sample of the text) get one
//     bitmap word per 32 positions, the group's lane mask, written without
//     atomics through a per-warp staging area, sector by sector;
//   * light patterns append (u << 32 | offset) keys with one warp-aggregated
//     atomic per depth, and their counts with one atomic per group.
// Then: popcounts of the bitmaps and a column scan give every heavy hit its
// rank; a stable radix sort orders the light keys; a single-block pass gives
// every pattern id its first output slot; the emit kernels write each hit
// once per id that holds the same bytes (duplicates are reported once per id).
#include <cuda_runtime.h>

#include <algorithm>

#include "ol_common.cuh"
#include "ol_kernels.h"

namespace ol {

constexpr uint32_t DM_THREADS = 256;
constexpr uint32_t DM_WARPS = DM_THREADS / 32;
constexpr uint32_t DM_QCAP = 64;                          // per-warp candidate queue
constexpr uint32_t DM_FILTER_WORDS = 1u << (kDictFilterBits - 5);
constexpr uint32_t kMbarSpins = 1u << 24;
// A warp's work item: SLICE text positions (staged with the longest pattern
// after them) and their SLICE / 32 heavy-bitmap words per heavy pattern.
template <uint32_t SLICE>
struct DictSmem {
    static constexpr uint32_t kWords = SLICE / 32;
    static constexpr uint32_t kText = SLICE + kDictHalo;
    static_assert(kText % 16 == 0 && kDictWordsPerTile % kWords == 0 && kDictTile % SLICE == 0, "slice geometry");
    uint32_t filter[DM_FILTER_WORDS];
    alignas(16) uint8_t text[DM_WARPS][kText];
    uint32_t hmask[DM_WARPS][SLICE];  // per slice position: bit h = heavy pattern h starts there
    uint16_t queue[DM_WARPS][DM_QCAP];
    alignas(8) unsigned long long bar;
};

// ---------------------------------------------------------------- TMA bulk --

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Global -> shared bulk copy (16-byte aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, unsigned long long *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity) {
    for (uint32_t i = 0; i < kMbarSpins; i++) {
        uint32_t ok;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(ok)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// ------------------------------------------------------------ trie walk ----

__device__ __forceinline__ uint32_t dict_child(const DictSet &s, const uint4 &nd, uint32_t b) {
    if (nd.y & kDictDenseFlag) return __ldg(s.dense + (size_t)nd.w * 256 + b);
    const uint32_t n = nd.y;
    if (n == 0) return NONE;
    uint32_t e0 = nd.z & 0xFFu;
    if (e0 == b) return nd.z >> 8;
    if (n == 1 || b < e0) return NONE;
    if (n == 2) return (nd.w & 0xFFu) == b ? nd.w >> 8 : NONE;
    for (uint32_t i = 0; i < n - 1; i++) {
        uint32_t e = __ldg(s.extra + nd.w + i);
        uint32_t eb = e & 0xFFu;
        if (eb == b) return e >> 8;
        if (eb > b) break;
    }
    return NONE;
}

__device__ __forceinline__ uint32_t dict_probe(const DictSet &s, uint32_t key) {
    const uint32_t mask = (1u << s.table_bits) - 1u;
    uint32_t slot = dict_table_h(key, s.table_bits);
    for (uint32_t i = 0; i <= s.max_probe; i++) {
        uint2 e = __ldg(s.table + slot);
        if (e.y == NONE) return NONE;
        if (e.x == key) return e.y;
        slot = (slot + 1) & mask;
    }
    return NONE;
}

// ------------------------------------------------------------- matching ----

// Emits unique pattern u at absolute offset pos: counts (count mode), a bit of
// the walk's heavy mask, or a light key.
__device__ __forceinline__ void dict_emit(const DictMatchArgs &a, uint32_t &hm, uint32_t u, uint64_t pos) {
    if (a.count_only) {
        const uint32_t peers = __match_any_sync(__activemask(), u);
        if ((peers & ((1u << (threadIdx.x & 31)) - 1u)) == 0) atomicAdd(a.counts + u, (uint32_t)__popc(peers));
        return;
    }
    const uint32_t hv = __ldg(a.heavy_of_u + u);
    if (hv != 0xFFu) {
        hm |= 1u << hv;
    } else {
        atomicAdd(a.counts + u, 1u);
        const uint32_t slot = atomicAdd(a.light_n, 1u);
        if (slot < a.light_cap) a.light_keys[slot] = ((unsigned long long)u << 32) | (uint32_t)pos;
    }
}

// Every unique pattern starting at slice position p: probe the table with the
// position's first four bytes, then walk the trie byte by byte. Hits must end
// by `lim` (the end of the text, or of the position's document in a batch).
// Returns the heavy patterns found (bit h: heavy pattern h).
__device__ __forceinline__ uint32_t dict_walk(const DictMatchArgs &a, const uint8_t *text, uint32_t p, uint64_t pos,
                                              uint64_t lim, uint32_t &levels) {
    const uint32_t key = (uint32_t)text[p] | ((uint32_t)text[p + 1] << 8) | ((uint32_t)text[p + 2] << 16) |
                         ((uint32_t)text[p + 3] << 24);
    uint32_t v = pos + kDictMinLen <= lim ? dict_probe(a.set, key) : NONE;
    uint32_t d = kDictMinLen, hm = 0;
    if (v != NONE && a.n_chains && key == (key & 0xFFu) * 0x01010101u) {
        // The position starts a run of one byte c: if c has a chain, jump to
        // the chain node of depth D = min(run, chain, max length, document
        // end), taking every pattern c^4..c^D at once, then walk on from it.
        const uint32_t c = key & 0xFFu;
        uint32_t j = 0;
        while (j < a.n_chains && ((a.chain_bytes >> (8 * j)) & 0xFFu) != c) j++;
        if (j < a.n_chains) {
            const DictChain *ch = a.chains + j;
            uint32_t cap = min(__ldg(&ch->K), kDictMaxLen);
            if (lim - pos < cap) cap = (uint32_t)(lim - pos);  // >= kDictMinLen: the probe ran
            const uint32_t *tw = reinterpret_cast<const uint32_t *>(text);
            const uint32_t C4 = c * 0x01010101u;
            uint32_t run = kDictMinLen;
            while (run < cap) {  // 4 bytes per step; the staged halo covers p + 67
                const uint32_t q = p + run;
                const uint32_t w = __funnelshift_r(tw[q >> 2], tw[(q >> 2) + 1], (q & 3) * 8);
                const uint32_t z = zero_bytes(w ^ C4);
                if (z == 0x80808080u) {
                    run += 4;
                    continue;
                }
                run += (__ffs(~z & 0x80808080u) - 8) >> 3;
                break;
            }
            const uint32_t D = min(run, cap);
            levels++;
            hm = __ldg(&ch->cum[D]);
            const uint32_t nl = __ldg(&ch->n_light);
            for (uint32_t i = 0; i < nl; i++) {
                const uint32_t e = __ldg(&ch->light[i]);
                if ((e >> 24) > D) break;
                dict_emit(a, hm, e & 0xFFFFFFu, pos);
            }
            if (D >= kDictMaxLen || pos + D >= lim) return hm;
            v = dict_child(a.set, __ldg(a.set.nodes + __ldg(&ch->node[D])), text[p + D]);
            d = D + 1;
        }
    }
    while (v != NONE) {
        const uint4 nd = __ldg(a.set.nodes + v);
        levels++;
        if (nd.x != NONE) dict_emit(a, hm, nd.x, pos);
        if (d >= kDictMaxLen || pos + d >= lim) break;
        v = dict_child(a.set, nd, text[p + d]);
        d++;
    }
    return hm;
}

// End of the document holding pos (pos itself when pos lies between
// documents), searching forward from hint, the first document ending after the
// slice start.
__device__ __forceinline__ uint64_t dict_limit(const DictMatchArgs &a, uint64_t pos, uint32_t hint) {
    if (!a.seg_end) return a.text_len;
    uint32_t i = hint;
    while (i < a.n_seg && a.seg_end[i] <= pos) i++;
    if (i == a.n_seg || a.seg_start[i] > pos) return pos;
    return a.seg_end[i];
}

// Each warp takes slices of SLICE positions in turn: it stages the slice (plus
// the longest pattern) in its own shared memory, filters all positions 32 at a
// time, queues the candidates and walks them 32 at a time (one per lane), so
// walks run on full warps. A walk returns the heavy patterns of its position as
// a 32-bit mask (no atomics); after the slice, ballots over each 32 positions'
// masks transpose them into the heavy patterns' bitmap words, which lane h
// stores for heavy pattern h. Warps never wait for one another.
template <uint32_t SLICE>
__global__ void __launch_bounds__(DM_THREADS) dict_match_kernel(DictMatchArgs a) {
    using Smem = DictSmem<SLICE>;
    constexpr uint32_t DM_SLICE = SLICE, DM_SLICE_WORDS = Smem::kWords, DM_TEXT_BYTES = Smem::kText;
    constexpr uint32_t DM_SLICES_PER_TILE = kDictTile / SLICE;
    extern __shared__ __align__(16) uint8_t dyn_smem[];
    Smem &sm = *reinterpret_cast<Smem *>(dyn_smem);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t lt = (1u << lane) - 1u;

    // The filter, once per block, by a bulk copy.
    if (tid == 0) mbar_init(&sm.bar, 1);
    __syncthreads();
    if (tid == 0) {
        mbar_expect_tx(&sm.bar, DM_FILTER_WORDS * 4);
        bulk_copy_g2s(sm.filter, a.set.filter, DM_FILTER_WORDS * 4, &sm.bar);
    }
    bool ok = mbar_wait(&sm.bar, 0);
    // (A separate statement: folded into the wait's result, the test hook
    // made the whole match kernel 47% slower, 19.8 against 13.5 ms per GiB.)
    if (a.force_timeout) ok = false;
    if (!__syncthreads_and(ok)) {
        if (tid == 0) atomicOr(a.error, OL_DEVERR_TIMEOUT);
        mbar_wait(&sm.bar, 0);  // let the copy land before the block exits
        return;
    }

    const uint64_t N = a.text_len;
    const uint32_t n_words = a.n_tiles * kDictWordsPerTile;
    const uint32_t n_items = ((a.n_tiles + a.tile_stride - 1) / a.tile_stride) * DM_SLICES_PER_TILE;
    const uint32_t H = a.count_only ? 0u : a.n_heavy;
    uint8_t *text = sm.text[warp];
    uint32_t *hmask = sm.hmask[warp];
    uint32_t cands = 0, levels = 0;  // per lane, for the search statistics
    uint16_t *queue = sm.queue[warp];

    for (uint32_t item = blockIdx.x * DM_WARPS + warp; item < n_items; item += gridDim.x * DM_WARPS) {
        const uint32_t slice = (item / DM_SLICES_PER_TILE) * a.tile_stride * DM_SLICES_PER_TILE + item % DM_SLICES_PER_TILE;
        const uint64_t s0 = (uint64_t)slice * DM_SLICE;  // slices past the text only write zero words
        __syncwarp();
        for (uint32_t o = lane * 16; o < DM_TEXT_BYTES; o += 32 * 16)
            *reinterpret_cast<uint4 *>(&text[o]) = ld_stream16(a.text + s0 + o);
        if (H)
            for (uint32_t f = lane; f < DM_SLICE; f += 32) hmask[f] = 0;
        __syncwarp();
        const uint32_t *tw = reinterpret_cast<const uint32_t *>(text);
        uint32_t hint = 0;
        if (a.seg_end) {  // first document ending after the slice start
            uint32_t lo = 0, hi = a.n_seg;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (a.seg_end[mid] <= s0)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            hint = lo;
        }
        uint32_t qn = 0;
        for (uint32_t step = 0; step < DM_SLICE / 32; step++) {
            const uint32_t p = step * 32 + lane;
            const uint64_t pos = s0 + p;
            bool cand = false;
            if (pos + kDictMinLen <= N) {
                const uint32_t key = __funnelshift_r(tw[p >> 2], tw[(p >> 2) + 1], (p & 3) * 8);
                const uint32_t h1 = dict_filter_h1(key), h2 = dict_filter_h2(key);
                cand = ((sm.filter[h1 >> 5] >> (h1 & 31)) & (sm.filter[h2 >> 5] >> (h2 & 31)) & 1u) != 0;
            }
            const uint32_t cm = __ballot_sync(0xFFFFFFFFu, cand);
            if (cand) queue[qn + __popc(cm & lt)] = (uint16_t)p;
            qn += __popc(cm);
            __syncwarp();
            if (qn >= 32) {  // walk 32 candidates, one per lane
                const uint32_t q = queue[lane];
                const uint32_t hm = dict_walk(a, text, q, s0 + q, dict_limit(a, s0 + q, hint), levels);
                if (hm) hmask[q] = hm;
                cands++;
                __syncwarp();
                const uint16_t keep = lane + 32 < qn ? queue[lane + 32] : (uint16_t)0;
                __syncwarp();
                if (lane + 32 < qn) queue[lane] = keep;
                qn -= 32;
                __syncwarp();
            }
        }
        if (lane < qn) {
            const uint32_t q = queue[lane];
            const uint32_t hm = dict_walk(a, text, q, s0 + q, dict_limit(a, s0 + q, hint), levels);
            if (hm) hmask[q] = hm;
            cands++;
        }
        __syncwarp();
        if (H) {
            // transpose: word w of heavy pattern h holds bit h of positions
            // 32w..32w+31. Lane q has position 32w+q's mask (a row of a 32x32
            // bit matrix); five butterfly rounds swap ever smaller off-diagonal
            // blocks between lanes, after which lane h holds column h.
            uint32_t words[DM_SLICE_WORDS];
#pragma unroll
            for (uint32_t w = 0; w < DM_SLICE_WORDS; w++) {
                uint32_t x = hmask[w * 32 + lane];
                if (__any_sync(0xFFFFFFFFu, x != 0)) {
#pragma unroll
                    for (uint32_t j = 16; j > 0; j >>= 1) {
                        const uint32_t left = j == 16 ? 0x0000FFFFu : j == 8 ? 0x00FF00FFu : j == 4 ? 0x0F0F0F0Fu
                                              : j == 2 ? 0x33333333u : 0x55555555u;  // bits i with (i & j) == 0
                        const uint32_t y = __shfl_xor_sync(0xFFFFFFFFu, x, j);
                        x = (lane & j) ? (x & ~left) | ((y & ~left) >> j) : (x & left) | ((y & left) << j);
                    }
                }
                words[w] = x;
            }
            // lane h stores heavy pattern h's words of the slice (contiguous, 16-byte stores)
            if (lane < H) {
                uint4 *dst = reinterpret_cast<uint4 *>(a.bitmap + (size_t)lane * n_words + (size_t)slice * DM_SLICE_WORDS);
#pragma unroll
                for (uint32_t w = 0; w < DM_SLICE_WORDS; w += 4)
                    dst[w / 4] = make_uint4(words[w], words[w + 1], words[w + 2], words[w + 3]);
            }
        }
    }
    if (a.stats) {  // candidates walked and trie nodes visited
        const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, cands), l = __reduce_add_sync(0xFFFFFFFFu, levels);
        if (lane == 0) {
            atomicAdd(a.stats, (unsigned long long)c);
            atomicAdd(a.stats + 1, (unsigned long long)l);
        }
    }
}

template <uint32_t SLICE>
static cudaError_t launch_match(const DictMatchArgs &a, int sm_count, uint32_t blocks_per_sm, cudaStream_t st) {
    const size_t smem = sizeof(DictSmem<SLICE>);
    cudaError_t e = cudaFuncSetAttribute(dict_match_kernel<SLICE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dict_match_kernel<SLICE>, DM_THREADS, smem);
    if (e != cudaSuccess) return e;
    if (blocks_per_sm) per_sm = std::min<int>(per_sm, (int)blocks_per_sm);
    const uint64_t n_items = (uint64_t)((a.n_tiles + a.tile_stride - 1) / a.tile_stride) * (kDictTile / SLICE);
    const uint32_t grid = (uint32_t)std::min<uint64_t>((n_items + DM_WARPS - 1) / DM_WARPS,
                                                       (uint64_t)std::max(per_sm, 1) * sm_count);
    dict_match_kernel<SLICE><<<grid, DM_THREADS, smem, st>>>(a); OL_LAUNCHED();
    return cudaGetLastError();
}

// slice: text positions per warp work item (256, 512 or 1024); blocks_per_sm:
// resident blocks per SM of the persistent grid (0: as many as fit).
cudaError_t launch_dict_match(const DictMatchArgs &a, int sm_count, cudaStream_t st, uint32_t slice,
                              uint32_t blocks_per_sm) {
    if (a.n_tiles == 0) return cudaSuccess;
    switch (slice) {
        case 256: return launch_match<256>(a, sm_count, blocks_per_sm, st);
        case 1024: return launch_match<1024>(a, sm_count, blocks_per_sm, st);
        default: return launch_match<512>(a, sm_count, blocks_per_sm, st);
    }
}

// ------------------------------------------------------------ heavy ranks --

constexpr uint32_t DH_THREADS = 256;
constexpr uint32_t DH_WORDS_PER_THREAD = 16;
constexpr uint32_t DH_WORDS = DH_THREADS * DH_WORDS_PER_THREAD;  // 4096 words per block

uint32_t dict_heavy_blocks(uint32_t n_words) { return (n_words + DH_WORDS - 1) / DH_WORDS; }

// Block sum / exclusive scan helpers for 256 threads.
__device__ __forceinline__ uint32_t block_exclusive_256(uint32_t x, uint32_t *warp_sum, uint32_t *total) {
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
    for (uint32_t w = 0; w < DH_THREADS / 32; w++) {
        uint32_t ws = warp_sum[w];
        before += w < warp ? ws : 0u;
        all += ws;
    }
    __syncthreads();
    if (total) *total = all;
    return before + inc - x;
}

__global__ void __launch_bounds__(DH_THREADS) dict_heavy_count_kernel(const uint32_t *__restrict__ bitmap,
                                                                       uint32_t n_words, uint32_t *counts,
                                                                       uint32_t ld) {
    __shared__ uint32_t warp_sum[DH_THREADS / 32];
    const uint32_t h = blockIdx.y, b = blockIdx.x;
    const uint32_t w0 = b * DH_WORDS + threadIdx.x * DH_WORDS_PER_THREAD;
    const uint32_t *col = bitmap + (size_t)h * n_words;
    uint32_t c = 0;
    if (w0 < n_words) {  // n_words is a multiple of 512: a thread's 16 words are all in range
#pragma unroll
        for (uint32_t i = 0; i < DH_WORDS_PER_THREAD; i += 4) {
            uint4 q = __ldg(reinterpret_cast<const uint4 *>(col + w0 + i));
            c += __popc(q.x) + __popc(q.y) + __popc(q.z) + __popc(q.w);
        }
    }
    uint32_t total;
    block_exclusive_256(c, warp_sum, &total);
    if (threadIdx.x == 0) counts[(size_t)h * ld + b] = total;
}

cudaError_t launch_dict_heavy_count(const uint32_t *bitmap, uint32_t n_words, uint32_t n_heavy, uint32_t *counts,
                                    uint32_t ld, cudaStream_t st) {
    if (n_heavy == 0 || n_words == 0) return cudaSuccess;
    dim3 grid(dict_heavy_blocks(n_words), n_heavy);
    dict_heavy_count_kernel<<<grid, DH_THREADS, 0, st>>>(bitmap, n_words, counts, ld); OL_LAUNCHED();
    return cudaGetLastError();
}

// ---------------------------------------------------- light-key radix sort --

constexpr uint32_t DS_THREADS = 256;
constexpr uint32_t DS_WARPS = DS_THREADS / 32;
constexpr uint32_t DS_PER_LANE = kDictSortChunk / 32;

uint32_t dict_sort_chunks(uint32_t n) { return (n + kDictSortChunk - 1) / kDictSortChunk; }

// Per-warp digit histograms: chunk c (one warp) holds keys [512c, 512c + 512).
__global__ void __launch_bounds__(DS_THREADS) dict_sort_hist_kernel(const unsigned long long *__restrict__ keys,
                                                                     uint32_t n, uint32_t shift, uint32_t *hist,
                                                                     uint32_t ld, uint32_t chunks) {
    __shared__ uint32_t sh[DS_WARPS][256];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t c = blockIdx.x * DS_WARPS + warp;
    for (uint32_t d = lane; d < 256; d += 32) sh[warp][d] = 0;
    __syncwarp();
    if (c < chunks) {
#pragma unroll 4
        for (uint32_t i = 0; i < DS_PER_LANE; i++) {
            uint32_t idx = c * kDictSortChunk + i * 32 + lane;
            if (idx < n) atomicAdd(&sh[warp][(uint32_t)(keys[idx] >> shift) & 255u], 1u);
        }
        __syncwarp();
        for (uint32_t d = lane; d < 256; d += 32) hist[(size_t)d * ld + c] = sh[warp][d];
    }
}

// Stable scatter: each warp walks its chunk in order, 32 keys at a time; lanes
// with the same digit take consecutive slots in lane order.
__global__ void __launch_bounds__(DS_THREADS) dict_sort_scatter_kernel(const unsigned long long *__restrict__ in,
                                                                        unsigned long long *__restrict__ out,
                                                                        uint32_t n, uint32_t shift,
                                                                        const uint32_t *__restrict__ base,
                                                                        const uint32_t *__restrict__ totals,
                                                                        uint32_t ld, uint32_t chunks) {
    __shared__ uint32_t start[256];
    __shared__ uint32_t warp_sum[DS_WARPS];
    __shared__ uint32_t cursor[DS_WARPS][256];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // digit starts: exclusive scan of the 256 digit totals
    start[tid] = block_exclusive_256(totals[tid], warp_sum, nullptr);
    __syncthreads();
    const uint32_t c = blockIdx.x * DS_WARPS + warp;
    if (c >= chunks) return;
    for (uint32_t d = lane; d < 256; d += 32) cursor[warp][d] = start[d] + base[(size_t)d * ld + c];
    __syncwarp();
    const uint32_t lt = (1u << lane) - 1u;
    unsigned long long nkey = c * kDictSortChunk + lane < n ? in[c * kDictSortChunk + lane] : 0ull;  // a step ahead
    for (uint32_t i = 0; i < DS_PER_LANE; i++) {
        const uint32_t idx = c * kDictSortChunk + i * 32 + lane;
        const bool valid = idx < n;
        const uint32_t vm = __ballot_sync(0xFFFFFFFFu, valid);
        if (!vm) break;
        const unsigned long long key = nkey;
        if (i + 1 < DS_PER_LANE) nkey = idx + 32 < n ? in[idx + 32] : 0ull;
        uint32_t d = 0, peers = 0;
        if (valid) {
            d = (uint32_t)(key >> shift) & 255u;
            peers = __match_any_sync(vm, d);
            out[cursor[warp][d] + __popc(peers & lt)] = key;
        }
        __syncwarp();
        if (valid && (peers & lt) == 0) cursor[warp][d] += __popc(peers);
        __syncwarp();
    }
}

cudaError_t launch_dict_sort(unsigned long long *keys, unsigned long long *tmp, uint32_t n, uint32_t key_bits,
                             uint32_t *hist, uint32_t *totals, cudaStream_t st) {
    if (n < 2) return cudaSuccess;
    const uint32_t chunks = dict_sort_chunks(n);
    const uint32_t ld = scan_ld(chunks);
    uint32_t *counts = hist, *bases = hist + (size_t)256 * ld;
    const uint32_t blocks = (chunks + DS_WARPS - 1) / DS_WARPS;
    unsigned long long *src = keys, *dst = tmp;
    uint32_t passes = (key_bits + 7) / 8;
    passes += passes & 1;  // an even number of passes leaves the result in keys
    for (uint32_t p = 0; p < passes; p++) {
        const uint32_t shift = 8 * p;
        dict_sort_hist_kernel<<<blocks, DS_THREADS, 0, st>>>(src, n, shift, counts, ld, chunks); OL_LAUNCHED();
        cudaError_t e = launch_scan_columns(counts, bases, totals, chunks, 256, ld, st);
        if (e != cudaSuccess) return e;
        dict_sort_scatter_kernel<<<blocks, DS_THREADS, 0, st>>>(src, dst, n, shift, bases, totals, ld, chunks); OL_LAUNCHED();
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        unsigned long long *t = src;
        src = dst;
        dst = t;
    }
    return cudaSuccess;
}

// ------------------------------------------------------------------ ids ----

constexpr uint32_t DI_THREADS = 1024;

// One block: per id its count and first output slot (u64 exclusive scan in id
// order), the total, and per unique pattern the start of its light keys.
__global__ void __launch_bounds__(DI_THREADS) dict_ids_kernel(DictEmitArgs a) {
    __shared__ unsigned long long wsum64[DI_THREADS / 32];
    __shared__ uint32_t wsum32[DI_THREADS / 32];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    auto count_of_u = [&](uint32_t u) -> uint32_t {
        uint32_t h = a.heavy_of_u[u];
        return h == 0xFFu ? a.light_count[u] : a.heavy_totals[h];
    };
    // ids
    {
        const uint32_t per = (a.n_ids + DI_THREADS - 1) / DI_THREADS;
        const uint32_t lo = min(a.n_ids, tid * per), hi = min(a.n_ids, lo + per);
        unsigned long long sum = 0;
        for (uint32_t i = lo; i < hi; i++) sum += count_of_u(a.u_of_id[i]);
        unsigned long long inc = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += t;
        }
        if (lane == 31) wsum64[warp] = inc;
        __syncthreads();
        unsigned long long before = 0, all = 0;
        for (uint32_t w = 0; w < DI_THREADS / 32; w++) {
            before += w < warp ? wsum64[w] : 0ull;
            all += wsum64[w];
        }
        unsigned long long run = before + inc - sum;
        for (uint32_t i = lo; i < hi; i++) {
            uint32_t c = count_of_u(a.u_of_id[i]);
            a.id_counts[i] = c;
            a.id_base[i] = run;
            run += c;
        }
        if (tid == 0) *a.total = all;
    }
    __syncthreads();
    // light key starts per unique pattern
    {
        const uint32_t per = (a.n_u + DI_THREADS - 1) / DI_THREADS;
        const uint32_t lo = min(a.n_u, tid * per), hi = min(a.n_u, lo + per);
        uint32_t sum = 0;
        for (uint32_t u = lo; u < hi; u++) sum += a.heavy_of_u[u] == 0xFFu ? a.light_count[u] : 0u;
        uint32_t inc = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += t;
        }
        if (lane == 31) wsum32[warp] = inc;
        __syncthreads();
        uint32_t before = 0;
        for (uint32_t w = 0; w < warp; w++) before += wsum32[w];
        uint32_t run = before + inc - sum;
        for (uint32_t u = lo; u < hi; u++) {
            a.light_base[u] = run;
            run += a.heavy_of_u[u] == 0xFFu ? a.light_count[u] : 0u;
        }
    }
}

cudaError_t launch_dict_ids(const DictEmitArgs &a, cudaStream_t st) {
    dict_ids_kernel<<<1, DI_THREADS, 0, st>>>(a); OL_LAUNCHED();
    return cudaGetLastError();
}

// ----------------------------------------------------------------- emit ----

// One hit into output slot `slot`: a ManyHit {pattern, offset u32}, or the
// (pattern u32, offset u64) pair of arrays. Streaming stores: the emission
// never reads them back.
__device__ __forceinline__ void put_hit(const DictEmitArgs &a, unsigned long long slot, uint32_t id, uint32_t off) {
    if (slot >= a.max_hits) return;
    if (a.hit_off) {
        __stcs(a.hit_pat + slot, id);
        __stcs(a.hit_off + slot, (unsigned long long)off);
    } else {
        __stcs(&a.hits[slot], make_uint2(id, off));
    }
}

// Heavy hits: block (b, h) expands words [4096b, 4096b + 4096) of bitmap h,
// warp w the 512 words [4096b + 512w, ...), 32 words per round. Each lane
// lists its word's hits, at their ranks from a warp scan of the popcounts, in
// the warp's shared buffer; the warp then writes the round's hits to
// consecutive slots, so every store instruction covers 32 consecutive hits.
// The ids of a unique pattern and their first output slots are read once per
// block into shared memory (up to DH_MAX_DUPS of them), not once per 32 hits.
constexpr uint32_t DH_MAX_DUPS = 64;

__global__ void __launch_bounds__(DH_THREADS) dict_emit_heavy_kernel(DictEmitArgs a) {
    __shared__ uint32_t warp_tot[DH_THREADS / 32];
    __shared__ uint32_t dup_id[DH_MAX_DUPS];
    __shared__ unsigned long long dup_base[DH_MAX_DUPS];
    __shared__ uint32_t hit_buf[DH_THREADS / 32][32 * 32];  // per warp: one round's hit offsets, in order
    const uint32_t h = blockIdx.y, b = blockIdx.x;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *buf = hit_buf[warp];
    const uint32_t *col = a.bitmap + (size_t)h * a.n_words;
    const uint32_t u = a.heavy_u[h];
    const uint32_t d0 = a.dup_start[u], d1 = a.dup_start[u + 1];
    const uint32_t n_dup = d1 - d0;
    const bool cached = n_dup <= DH_MAX_DUPS;
    if (cached && threadIdx.x < n_dup) {
        const uint32_t id = __ldg(a.dup_ids + d0 + threadIdx.x);
        dup_id[threadIdx.x] = id;
        dup_base[threadIdx.x] = a.id_base[id];
    }
    const uint32_t w0 = b * DH_WORDS + warp * (DH_WORDS / (DH_THREADS / 32));
    constexpr uint32_t kRounds = DH_WORDS / (DH_THREADS / 32) / 32;  // 16
    uint32_t c = 0;
    for (uint32_t r = 0; r < kRounds; r++) {
        const uint32_t idx = w0 + r * 32 + lane;
        c += idx < a.n_words ? __popc(__ldg(col + idx)) : 0u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if (lane == 0) warp_tot[warp] = c;
    __syncthreads();
    uint32_t rank = a.heavy_bases[(size_t)h * a.ld + b];
    for (uint32_t w = 0; w < warp; w++) rank += warp_tot[w];
    if (c == 0) return;  // uniform over the warp
    // each round's bitmap word is loaded a round ahead, so its latency hides
    // behind the previous round's listing and stores
    uint32_t nxt = w0 + lane < a.n_words ? __ldg(col + w0 + lane) : 0u;
    for (uint32_t r = 0; r < kRounds; r++) {
        const uint32_t idx = w0 + r * 32 + lane;
        const uint32_t word = nxt;
        if (r + 1 < kRounds) nxt = idx + 32 < a.n_words ? __ldg(col + idx + 32) : 0u;
        const uint32_t cnt = __popc(word);
        uint32_t inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if ((int)lane >= o) inc += t;
        }
        const uint32_t excl = inc - cnt;
        const uint32_t T = __shfl_sync(0xFFFFFFFFu, inc, 31);  // <= 1024
        // each lane lists its word's hit offsets at their ranks in the warp's
        // buffer; then the warp writes them, 32 consecutive hits per store
        {
            uint32_t bits = word, r2 = excl;
            const uint32_t wbase = idx * 32;
            while (bits) {
                const uint32_t bb = __ffs(bits) - 1;
                bits &= bits - 1;
                buf[r2++] = wbase + bb;
            }
        }
        __syncwarp();
        for (uint32_t base = 0; base < T; base += 32) {
            const uint32_t j = base + lane;
            if (j < T) {
                const uint32_t off = buf[j];
                if (cached) {
                    for (uint32_t d = 0; d < n_dup; d++) put_hit(a, dup_base[d] + rank + j, dup_id[d], off);
                } else {
                    for (uint32_t d = d0; d < d1; d++) {
                        const uint32_t id = __ldg(a.dup_ids + d);
                        put_hit(a, a.id_base[id] + rank + j, id, off);
                    }
                }
            }
        }
        __syncwarp();  // the buffer is refilled by the next round
        rank += T;
    }
}

__global__ void dict_emit_light_kernel(DictEmitArgs a) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.light_n) return;
    const unsigned long long key = a.light_keys[k];
    const uint32_t u = (uint32_t)(key >> 32), off = (uint32_t)key;
    const uint32_t rank = k - a.light_base[u];
    const uint32_t d0 = a.dup_start[u], d1 = a.dup_start[u + 1];
    for (uint32_t d = d0; d < d1; d++) {
        const uint32_t id = a.dup_ids[d];
        put_hit(a, a.id_base[id] + rank, id, off);
    }
}

cudaError_t launch_dict_emit(const DictEmitArgs &a, cudaStream_t st) {
    if (a.max_hits == 0) return cudaSuccess;
    if (a.n_heavy && a.n_words) {
        dim3 grid(dict_heavy_blocks(a.n_words), a.n_heavy);
        dict_emit_heavy_kernel<<<grid, DH_THREADS, 0, st>>>(a); OL_LAUNCHED();
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (a.light_n) {
        dict_emit_light_kernel<<<(a.light_n + 255) / 256, 256, 0, st>>>(a); OL_LAUNCHED();
        return cudaGetLastError();
    }
    return cudaSuccess;
}

}  // namespace ol
