// The `.olb` binary container of a parsed document, and loading one straight
// into a resident document without parsing the text again. The layout is the
// one planned in the reference (.agents/tasks/phase4-zero-copy-binary-
// serialization.md:13-36), all integers little-endian:
//
//   0x00  magic "ONELINE\0"            0x08  version u32 (1)   0x0C  flags u32 (0)
//   0x10  text_len u64                 0x18  line_count u64
//   0x20  text_offset u64              0x28  nodes_offset u64
//   0x30  line_offsets_offset u64      0x38  crc32 u64
//   text_offset:          the UTF-8 text (text_len bytes)
//   nodes_offset:         FlatNode[line_count], 16 bytes each
//   line_offsets_offset:  u32[line_count]
//
// Sections start on 64-byte boundaries (zero padding between them). crc32 is
// the CRC-32 (IEEE 802.3, reflected polynomial 0xEDB88320, the zlib CRC) of the
// file's bytes from text_offset to its end.
//
// Loading maps the file, registers its pages for DMA where the driver allows
// (read-only host registration, else the pinned staging ring), copies text,
// offsets and nodes to the device and derives the resident kinds and depths
// from the nodes with one kernel that also checks the offsets against the text.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "runtime.h"

using namespace ol;

namespace {

constexpr uint64_t kHeader = 64;
constexpr uint32_t kVersion = 1;
const char kMagic[8] = {'O', 'N', 'E', 'L', 'I', 'N', 'E', '\0'};

struct OlbHeader {
    char magic[8];
    uint32_t version, flags;
    uint64_t text_len, line_count;
    uint64_t text_offset, nodes_offset, offsets_offset, crc32;
};
static_assert(sizeof(OlbHeader) == kHeader, "header layout");

uint64_t align64(uint64_t x) { return (x + 63) & ~63ull; }

// CRC-32 by slicing eight bytes per step (tables built once).
struct Crc32 {
    uint32_t t[8][256];
    Crc32() {
        for (uint32_t i = 0; i < 256; i++) {
            uint32_t c = i;
            for (int k = 0; k < 8; k++) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            t[0][i] = c;
        }
        for (uint32_t i = 0; i < 256; i++)
            for (int s = 1; s < 8; s++) t[s][i] = (t[s - 1][i] >> 8) ^ t[0][t[s - 1][i] & 0xFF];
    }
    uint32_t update(uint32_t crc, const uint8_t *p, uint64_t n) const {
        crc = ~crc;
        while (n >= 8) {
            uint32_t a, b;
            memcpy(&a, p, 4);
            memcpy(&b, p + 4, 4);
            a ^= crc;
            crc = t[7][a & 0xFF] ^ t[6][(a >> 8) & 0xFF] ^ t[5][(a >> 16) & 0xFF] ^ t[4][a >> 24] ^ t[3][b & 0xFF] ^
                  t[2][(b >> 8) & 0xFF] ^ t[1][(b >> 16) & 0xFF] ^ t[0][b >> 24];
            p += 8;
            n -= 8;
        }
        while (n--) crc = t[0][(crc ^ *p++) & 0xFF] ^ (crc >> 8);
        return ~crc;
    }
};

const Crc32 &crc_tables() {
    static const Crc32 tables;
    return tables;
}

// kinds and depth8 of every line from its node; error bit 1 when an offset is
// not inside the text or not after the previous line's, bit 2 when a kind is
// not a NodeKind code.
__global__ void olb_nodes_kernel(const FlatNode *__restrict__ nodes, const uint32_t *__restrict__ offsets, uint32_t L,
                                 uint64_t text_len, uint8_t *__restrict__ kinds, uint8_t *__restrict__ depth8,
                                 DocStats *stats) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t deepest = 0, bad = 0;
    if (i < L) {
        const FlatNode n = nodes[i];
        const uint32_t o = offsets[i];
        if ((uint64_t)o >= text_len || (i == 0 && o != 0) || (i > 0 && o <= offsets[i - 1])) bad |= 1;
        if (n.kind > KIND_COMMENT) bad |= 2;
        kinds[i] = (uint8_t)(n.kind & 7);
        depth8[i] = (uint8_t)min(n.depth, 255u);
        if (n.kind != KIND_BLANK) deepest = n.depth;
    }
    for (int o = 16; o > 0; o >>= 1) {
        deepest = max(deepest, __shfl_xor_sync(0xFFFFFFFFu, deepest, o));
        bad |= __shfl_xor_sync(0xFFFFFFFFu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (deepest) atomicMax(&stats->max_content_depth, deepest);
        if (bad) atomicOr(&stats->error, bad << 8);
    }
}

// An open, mapped file; unmapped and closed by the destructor.
struct Mapped {
    int fd = -1;
    uint8_t *p = nullptr;
    uint64_t size = 0;
    ~Mapped() {
        if (p) munmap(p, size);
        if (fd >= 0) close(fd);
    }
};

}  // namespace

extern "C" ol_status ol_doc_save_olb(ol_ctx *ctx, const ol_doc *d, const char *path) {
    if (!ctx || !d || !path) return OL_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const uint64_t N = d->text_len, L = d->line_count;
    OlbHeader h{};
    memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.text_len = N;
    h.line_count = L;
    h.text_offset = kHeader;
    h.nodes_offset = align64(h.text_offset + N);
    h.offsets_offset = align64(h.nodes_offset + L * 16);
    const uint64_t file_len = h.offsets_offset + L * 4;
    std::vector<uint8_t> body(file_len - kHeader, 0);
    cudaError_t e = cudaSuccess;
    if (N) e = cudaMemcpyAsync(body.data(), d->text, N, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && L) {
        e = ctx->scratch_c.reserve(L * sizeof(FlatNode), st);
        if (e == cudaSuccess)
            e = launch_classify_lines(d->text, N, d->offsets, (uint32_t)L, (FlatNode *)ctx->scratch_c.ptr, nullptr, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(body.data() + (h.nodes_offset - kHeader), ctx->scratch_c.ptr, L * 16,
                                cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(body.data() + (h.offsets_offset - kHeader), d->offsets, L * 4, cudaMemcpyDeviceToHost,
                                st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return ctx_cuda(ctx, e, "save .olb");
    h.crc32 = crc_tables().update(0, body.data(), body.size());
    FILE *f = fopen(path, "wb");
    if (!f) return ctx_fail(ctx, OL_ERR_INVALID_ARG, std::string("cannot create ") + path);
    const bool ok = fwrite(&h, kHeader, 1, f) == 1 && (body.empty() || fwrite(body.data(), body.size(), 1, f) == 1);
    const bool closed = fclose(f) == 0;
    if (!ok || !closed) return ctx_fail(ctx, OL_ERR_INVALID_ARG, std::string("cannot write ") + path);
    return OL_OK;
}

extern "C" ol_status ol_doc_load_olb(ol_ctx *ctx, const char *path, uint32_t flags, ol_doc **out) {
    if (!ctx || !path || !out || (flags & ~(uint32_t)OL_OLB_VERIFY)) return OL_ERR_INVALID_ARG;
    *out = nullptr;
    Mapped m;
    m.fd = open(path, O_RDONLY);
    if (m.fd < 0) return ctx_fail(ctx, OL_ERR_NOT_FOUND, std::string("cannot open ") + path);
    struct stat sb;
    if (fstat(m.fd, &sb) != 0) return ctx_fail(ctx, OL_ERR_INVALID_ARG, std::string("cannot stat ") + path);
    m.size = (uint64_t)sb.st_size;
    auto bad = [&](const std::string &why) { return ctx_fail(ctx, OL_ERR_INVALID_ARG, std::string(path) + ": " + why); };
    if (m.size < kHeader) return bad("shorter than the 64-byte .olb header");
    void *p = mmap(nullptr, m.size, PROT_READ, MAP_PRIVATE, m.fd, 0);
    if (p == MAP_FAILED) return bad("cannot be mapped");
    m.p = (uint8_t *)p;
    OlbHeader h;
    memcpy(&h, m.p, kHeader);
    if (memcmp(h.magic, kMagic, 8) != 0) return bad("not an .olb file (magic)");
    if (h.version != kVersion) return bad("unsupported .olb version " + std::to_string(h.version));
    if (h.text_len > OL_MAX_GPU_INPUT_LEN) return bad("text longer than the GPU path addresses");
    if (h.line_count > h.text_len + 1 || h.text_offset < kHeader || h.text_offset > m.size ||
        h.text_len > m.size - h.text_offset || h.nodes_offset < h.text_offset + h.text_len || h.nodes_offset > m.size ||
        h.line_count * 16 > m.size - h.nodes_offset || h.offsets_offset < h.nodes_offset + h.line_count * 16 ||
        h.offsets_offset > m.size || h.line_count * 4 > m.size - h.offsets_offset)
        return bad("sections do not fit the file");
    if ((h.text_len == 0) != (h.line_count == 0)) return bad("line count does not match the text");
    if (flags & OL_OLB_VERIFY) {
        const uint32_t crc = crc_tables().update(0, m.p + h.text_offset, m.size - h.text_offset);
        if (crc != (uint32_t)h.crc32) return bad("checksum mismatch");
    }
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    ol_doc *d = nullptr;
    ol_status s = new_doc(ctx, h.text_len, &d);
    if (s != OL_OK) return s;
    if (h.text_len == 0) {
        *out = d;
        return OL_OK;
    }
    const uint64_t L = h.line_count;
    s = alloc_lines(ctx, d, L);
    if (s != OL_OK) {
        ol_doc_free(d);
        return s;
    }
    // The mapped pages go to the device by DMA when they can be registered
    // (read-only); otherwise through the pinned staging ring.
    bool registered = cudaHostRegister(m.p, m.size, cudaHostRegisterReadOnly) == cudaSuccess;
    if (!registered) cudaGetLastError();
    cudaError_t e;
    {
        GpuPass pass(ctx, "load .olb: copy to device");
        e = registered ? cudaMemcpyAsync(d->text, m.p + h.text_offset, h.text_len, cudaMemcpyHostToDevice, st)
                       : h2d(ctx, d->text, m.p + h.text_offset, h.text_len);
        if (e == cudaSuccess) e = ctx->scratch_c.reserve(L * sizeof(FlatNode), st);
        if (e == cudaSuccess)
            e = registered ? cudaMemcpyAsync(ctx->scratch_c.ptr, m.p + h.nodes_offset, L * 16, cudaMemcpyHostToDevice, st)
                           : h2d(ctx, (uint8_t *)ctx->scratch_c.ptr, m.p + h.nodes_offset, L * 16);
        if (e == cudaSuccess)
            e = registered ? cudaMemcpyAsync(d->offsets, m.p + h.offsets_offset, L * 4, cudaMemcpyHostToDevice, st)
                           : h2d(ctx, (uint8_t *)d->offsets, m.p + h.offsets_offset, L * 4);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(d->stats, 0, sizeof(DocStats), st);
    if (e == cudaSuccess) {
        GpuPass pass(ctx, "load .olb: kinds and depths");
        olb_nodes_kernel<<<(uint32_t)((L + 255) / 256), 256, 0, st>>>((const FlatNode *)ctx->scratch_c.ptr, d->offsets,
                                                                      (uint32_t)L, h.text_len, d->kinds, d->depth8,
                                                                      d->stats);
        OL_LAUNCHED();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&d->host_stats, d->stats, sizeof(DocStats), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (registered) cudaHostUnregister(m.p);
    prof_mark(ctx, "load .olb");
    if (e != cudaSuccess) {
        ol_doc_free(d);
        return ctx_cuda(ctx, e, "load .olb");
    }
    if (d->host_stats.error >> 8) {
        ol_doc_free(d);
        return bad((d->host_stats.error >> 8) & 1 ? "line offsets are not increasing inside the text"
                                                   : "a node has no NodeKind code");
    }
    d->line_count = (uint32_t)L;
    d->max_depth = d->host_stats.max_content_depth;
    d->host_stats.line_count = (uint32_t)L;
    const uint32_t l32 = (uint32_t)L;  // the device counters as a parse leaves them
    e = cudaMemcpy(&d->stats->line_count, &l32, 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        ol_doc_free(d);
        return ctx_cuda(ctx, e, "load .olb");
    }
    *out = d;
    return OL_OK;
}
