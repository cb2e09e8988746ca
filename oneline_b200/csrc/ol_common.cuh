// Device-side building blocks shared by the oneline sm_100a kernels.
//
// * NodeKind codes and FlatNode layout (crates/oneline-core/src/lib.rs:39-96).
// * Device status words: a kernel never traps or spins forever; the one
//   bounded wait (the dictionary kernel's bulk-copy barrier) sets
//   OL_DEVERR_TIMEOUT when it runs out and the host discards the results.
// * Byte SWAR helpers and the line classifier.
#pragma once
#include <cstdint>

namespace ol {

constexpr uint32_t NONE = 0xFFFFFFFFu;

enum Kind : uint8_t {
    KIND_BLANK = 0,
    KIND_TEXT = 1,
    KIND_HEADING = 2,
    KIND_ELEMENT = 3,
    KIND_LIST = 4,
    KIND_CONNECT = 5,
    KIND_ORDERED = 6,
    KIND_COMMENT = 7,
};

struct FlatNode {
    uint32_t depth, kind, span_start, span_len;
};

// Device status bits (DocStats::error and friends).
constexpr uint32_t OL_DEVERR_TIMEOUT = 1u << 0;   // a bounded wait ran out
constexpr uint32_t OL_DEVERR_CAPACITY = 1u << 1;  // an output buffer was too small
constexpr uint32_t OL_DEVERR_FIXUP = 1u << 2;     // fix-up list overflow (cannot happen by construction)
constexpr uint32_t OL_DEVERR_DEEP = 1u << 3;      // a content line deeper than the fast tree path handles

// Per-launch counters that live in device memory next to a document.
struct DocStats {
    uint32_t line_count;        // lines in the document
    uint32_t max_content_depth; // deepest non-blank line (saturates at 0xFFFFFFFF)
    uint32_t fixup_count;       // lines classified by the fix-up kernel
    uint32_t error;             // OL_DEVERR_* bits
    uint32_t pad[12];
};

// ---------------------------------------------------------- memory access --

// Asks L2 to fetch [p, p + bytes) from device memory ahead of its use: one
// bulk prefetch that returns no data and that nothing waits on. p 16-byte
// aligned, bytes a multiple of 16, the range inside one allocation.
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// How far ahead (in tiles) a one-tile-per-block kernel prefetches its text:
// about the blocks resident at once over the GPU (148 SMs, 5-7 blocks each),
// so the prefetched tile is one that a block starting soon reads.
constexpr uint32_t kPrefetchTilesAhead = 1024;

// Streaming 16-byte load (read once: do not keep in L1).
__device__ __forceinline__ uint4 ld_stream16(const void *p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

// ------------------------------------------------------------ byte SWAR ----

// High bit of each byte of x set exactly where that byte is zero.
__device__ __forceinline__ uint32_t zero_bytes(uint32_t x) {
    uint32_t y = (x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu;
    return ~(y | x | 0x7F7F7F7Fu);
}

// 4-bit mask (bit i = byte i) of bytes of w equal to c4's byte.
__device__ __forceinline__ uint32_t eq_mask4(uint32_t w, uint32_t c4) {
    uint32_t z = zero_bytes(w ^ c4);  // bits 7,15,23,31
    // gather bits 7,15,23,31 into 0..3
    return ((z >> 7) & 1u) | ((z >> 14) & 2u) | ((z >> 21) & 4u) | ((z >> 28) & 8u);
}

// 16-bit mask of the bytes of a 16-byte vector equal to byte c.
__device__ __forceinline__ uint32_t eq_mask16(uint4 v, uint32_t c4) {
    return eq_mask4(v.x, c4) | (eq_mask4(v.y, c4) << 4) | (eq_mask4(v.z, c4) << 8) | (eq_mask4(v.w, c4) << 12);
}

// 16-bit mask (bit i = byte i) from the high bits of four SWAR words. One
// multiply gathers two words: the high bits of c0 (moved to bits 0, 8, 16,
// 24) and of c1 (bits 4, 12, 20, 28) land, shifted by 21, 14, 7 and 0, on bits
// 21..28 in byte order; no two partial products meet, so nothing carries.
__device__ __forceinline__ uint32_t gather16(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3) {
    auto g2 = [](uint32_t lo, uint32_t hi) { return ((((lo >> 7) | (hi >> 3)) * 0x00204081u) >> 21) & 0xFFu; };
    return g2(c0, c1) | (g2(c2, c3) << 8);
}

__device__ __forceinline__ bool is_blank(uint8_t b) { return b == ' ' || b == '\t'; }

// classify_line (crates/oneline-simd/src/line.rs:57-81) on the first content
// bytes c0, c1, c2; n = content length (bytes at index >= n do not exist).
__device__ __forceinline__ uint8_t classify3(uint8_t c0, uint8_t c1, uint8_t c2, uint32_t n) {
    switch (c0) {
    case '=': return KIND_HEADING;
    case ':': return KIND_CONNECT;
    case '@': return KIND_ELEMENT;
    case '/': return (n > 1 && c1 == '/') ? KIND_COMMENT : KIND_TEXT;
    case '-':
        if (n > 1 && is_blank(c1)) return KIND_LIST;
        if (n > 2 && c1 == '.' && is_blank(c2)) return KIND_ORDERED;
        return KIND_TEXT;
    default: return KIND_TEXT;
    }
}

// One line [s, e) where e is the position of its terminating '\n' or the text
// end, read through `at(pos)`. Implements parse_line (line.rs:8-44):
//   * the trailing run of '\r' before e is dropped (e itself is '\n' or end);
//   * a line starting with '|' has a prefix made of the maximal run of '|' and
//     blanks; its depth is the number of '|' in it, the content starts after it;
//   * otherwise the depth is 0 and the content starts after leading blanks;
//   * empty content gives Blank with the depth kept.
template <class At>
__device__ __forceinline__ FlatNode classify_line(uint32_t s, uint32_t e, At at) {
    uint32_t eff = e;
    while (eff > s && at(eff - 1) == '\r') eff--;
    uint32_t c = s, depth = 0;
    if (c < eff && at(c) == '|') {
        while (c < eff) {
            uint8_t b = at(c);
            if (b == '|') depth++;
            else if (!is_blank(b)) break;
            c++;
        }
    } else {
        while (c < eff && is_blank(at(c))) c++;
    }
    FlatNode nd;
    nd.depth = depth;
    nd.span_start = c;
    if (c == eff) {
        nd.kind = KIND_BLANK;
        nd.span_len = 0;
        return nd;
    }
    uint32_t n = eff - c;
    uint8_t c0 = at(c);
    uint8_t c1 = n > 1 ? at(c + 1) : 0;
    uint8_t c2 = n > 2 ? at(c + 2) : 0;
    nd.kind = classify3(c0, c1, c2, n);
    nd.span_len = n;
    return nd;
}

}  // namespace ol
