// ol_search_noalloc: substring search that allocates nothing.
//
// Some callers cannot call cudaMalloc: a serving process whose allocator
// reserved the GPU's memory up front and hands out every byte itself, or a
// latency-critical loop where cudaMalloc/cudaFree would stall the device with
// an implicit synchronisation or fail for lack of free memory. This entry
// point runs the same three search launches as ol_search_async (count, column
// scan, write) on buffers the caller owns; the per-tile counts and output
// bases those launches need, and the device copy of the pattern, live in one
// fixed array below that every GPU which loads this library holds until the
// process exits.
//
// The pattern reaches the device inside the arguments of a one-block kernel
// that writes it into the array, so the call reads the caller's pattern
// buffer only while it runs: the caller may overwrite that buffer (pageable or
// pinned) as soon as the call returns.
//
// The array is shared by every call on a device and keeps what the last call
// left in it. Nothing a call reads from it is left over from an earlier call:
// the pattern is written in, the count launch writes every tile's count and
// the scan writes every base and the total, before anything reads them. Two
// calls whose work overlaps on the GPU (different streams, no ordering between
// them) race on the array and may both return wrong results.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/oneline_cuda.h"
#include "ol_kernels.h"

namespace {

constexpr uint64_t kMaxTiles = (OL_NOALLOC_MAX_TEXT_LEN + ol::kSearchTile - 1) / ol::kSearchTile;
constexpr size_t kPatternBytes = 256;                                       // OL_MAX_PATTERN_LEN, rounded up
constexpr size_t kColumnWords = kMaxTiles * ol::kSearchMaxPatterns;          // counts, then bases
constexpr size_t kScratchBytes = kPatternBytes + 2 * kColumnWords * sizeof(uint32_t);  // 1 MiB + 256 B
constexpr int kMaxDevices = 64;

static_assert(OL_MAX_PATTERN_LEN <= kPatternBytes, "pattern area");
static_assert(((OL_MAX_PATTERN_LEN - 1 + 15) & ~15u) <= ol::kSearchMaxStagedPattern, "patterns are staged");

// Device scratch. Host code must not pass this name to a kernel: on the host
// it is only a stand-in for the symbol. Its device address comes from
// cudaGetSymbolAddress, once per device (and again if the device's context is
// ever created anew).
static __device__ __align__(256) uint8_t g_noalloc_scratch[kScratchBytes];

// The pattern bytes, passed by value as a kernel argument.
struct PatternBytes {
    uint8_t b[OL_MAX_PATTERN_LEN];
};

__global__ void noalloc_put_pattern_kernel(PatternBytes p, uint32_t len, uint8_t *dst) {
    if (threadIdx.x < len) dst[threadIdx.x] = p.b[threadIdx.x];
}

// The scratch array's device address per device, with the CUDA context it was
// looked up in: a device whose primary context was destroyed and created again
// (cudaDeviceReset) gets a new set-up instead of a stale address.
struct ScratchSetup {
    void *context = nullptr;
    uint8_t *ptr = nullptr;
};
std::mutex g_setup_mu;
ScratchSetup g_setup[kMaxDevices];

typedef int (*CtxGetCurrentFn)(void **);
CtxGetCurrentFn g_ctx_get_current = nullptr;

ol_status fail(char *err, uint32_t err_cap, ol_status s, const char *fmt, unsigned long long a = 0,
               unsigned long long b = 0) {
    if (err && err_cap) snprintf(err, err_cap, fmt, a, b);
    return s;
}

}  // namespace

extern "C" ol_status ol_search_noalloc(const uint8_t *d_text, uint64_t text_len, uint64_t text_cap,
                                       const uint8_t *pattern, uint32_t pat_len, uint32_t max_matches,
                                       uint32_t *d_total, uint32_t *d_out, void *stream, char *err,
                                       uint32_t err_cap) {
    if (err && err_cap) err[0] = 0;
    if (text_len > OL_NOALLOC_MAX_TEXT_LEN)
        return fail(err, err_cap, OL_ERR_INPUT_TOO_LARGE,
                    "ol_search_noalloc: text of %llu bytes exceeds its fixed maximum of %llu bytes",
                    (unsigned long long)text_len, (unsigned long long)OL_NOALLOC_MAX_TEXT_LEN);
    if (pat_len == 0 || !pattern)
        return fail(err, err_cap, OL_ERR_BAD_PATTERN, "ol_search_noalloc: pattern must not be empty");
    if (pat_len > OL_MAX_PATTERN_LEN)
        return fail(err, err_cap, OL_ERR_BAD_PATTERN,
                    "ol_search_noalloc: pattern of %llu bytes exceeds the %llu-byte maximum", pat_len,
                    OL_MAX_PATTERN_LEN);
    if (!d_total || ((uintptr_t)d_total & 3))
        return fail(err, err_cap, OL_ERR_INVALID_ARG, "ol_search_noalloc: d_total must be a 4-byte aligned device pointer");
    if (max_matches && (!d_out || ((uintptr_t)d_out & 3)))
        return fail(err, err_cap, OL_ERR_INVALID_ARG, "ol_search_noalloc: d_out must be a 4-byte aligned device pointer");
    if (text_len && (!d_text || ((uintptr_t)d_text & 15)))
        return fail(err, err_cap, OL_ERR_INVALID_ARG, "ol_search_noalloc: d_text must be a 16-byte aligned device pointer");
    if (text_len && text_cap < OL_NOALLOC_TEXT_CAP(text_len))
        return fail(err, err_cap, OL_ERR_INVALID_ARG,
                    "ol_search_noalloc: text buffer of %llu bytes is too small; OL_NOALLOC_TEXT_CAP(len) = %llu",
                    (unsigned long long)text_cap, (unsigned long long)OL_NOALLOC_TEXT_CAP(text_len));

    // Set-up, once per device, with that device current: the device address of
    // the scratch array.
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return fail(err, err_cap, OL_ERR_CUDA, "ol_search_noalloc: cudaGetDevice failed (error %llu)", (unsigned)e);
    if (dev < 0 || dev >= kMaxDevices)
        return fail(err, err_cap, OL_ERR_INVALID_ARG, "ol_search_noalloc: device %llu is beyond the %llu supported",
                    (unsigned)dev, kMaxDevices);
    uint8_t *scratch;
    {
        std::lock_guard<std::mutex> g(g_setup_mu);
        if (!g_ctx_get_current) {
            void *fn = nullptr;
            cudaDriverEntryPointQueryResult q;
            e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
            if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
                return fail(err, err_cap, OL_ERR_CUDA,
                            "ol_search_noalloc: the driver's cuCtxGetCurrent is unavailable (error %llu)", (unsigned)e);
            g_ctx_get_current = (CtxGetCurrentFn)fn;
        }
        // cudaSetDevice makes the device's primary context current (CUDA 12+)
        e = cudaSetDevice(dev);
        void *cur = nullptr;
        if (e != cudaSuccess || g_ctx_get_current(&cur) != 0 || !cur)
            return fail(err, err_cap, OL_ERR_CUDA, "ol_search_noalloc: no current CUDA context (error %llu)",
                        (unsigned)e);
        ScratchSetup &su = g_setup[dev];
        if (!su.ptr || su.context != cur) {
            uint8_t *p = nullptr;
            e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return fail(err, err_cap, OL_ERR_CUDA,
                            "ol_search_noalloc: cudaGetSymbolAddress of the scratch array failed (error %llu)",
                            (unsigned)e);
            su.context = cur;
            su.ptr = p;
        }
        scratch = su.ptr;
    }

    cudaStream_t st = (cudaStream_t)stream;
    // An empty text, or a pattern longer than the text, has no matches.
    if (text_len == 0 || pat_len > text_len) {
        e = cudaMemsetAsync(d_total, 0, sizeof(uint32_t), st);
        return e == cudaSuccess ? OL_OK
                                : fail(err, err_cap, OL_ERR_CUDA, "ol_search_noalloc: cudaMemsetAsync failed (error %llu)",
                                       (unsigned)e);
    }
    // The pattern goes into the array through a kernel argument: its bytes are
    // taken from the caller's buffer here, before this call returns.
    PatternBytes pb{};
    memcpy(pb.b, pattern, pat_len);
    noalloc_put_pattern_kernel<<<1, OL_MAX_PATTERN_LEN, 0, st>>>(pb, pat_len, scratch);
    OL_LAUNCHED();
    e = cudaGetLastError();
    if (e != cudaSuccess)
        return fail(err, err_cap, OL_ERR_CUDA, "ol_search_noalloc: pattern write failed (error %llu)", (unsigned)e);

    ol::SearchArgs a{};
    a.text = d_text;
    a.text_len = text_len;
    a.n_tiles = (uint32_t)((text_len + ol::kSearchTile - 1) / ol::kSearchTile);
    a.halo = (pat_len - 1 + 15u) & ~15u;
    ol::search_add_pattern(a, pattern, scratch, pat_len, d_out, max_matches);
    a.ld = ol::scan_ld(a.n_tiles);
    a.counts = reinterpret_cast<uint32_t *>(scratch + kPatternBytes);
    a.bases = a.counts + kColumnWords;
    a.totals = d_total;
    e = ol::launch_search(a, st);
    if (e != cudaSuccess)
        return fail(err, err_cap, OL_ERR_CUDA, "ol_search_noalloc: launch failed (error %llu)", (unsigned)e);
    return OL_OK;
}
