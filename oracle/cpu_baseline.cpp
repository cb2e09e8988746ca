// ORACLE — test infrastructure only (timed CPU baseline).
//
// A multi-threaded C++ restatement of the reference's CPU engine (crates/
// oneline-simd), used as the CPU baseline that bench.py times on the host's
// cores and as a second checker in tests. The product never links or calls it.
// The reference itself is Rust and cannot be built here, and its memchr /
// aho-corasick dependencies are not vendored, so this is a port ("kind": "port"):
//
//   olb_parse_par     lib.rs:30-43,115-137,189-244 two-pass count/fill over
//                     line-aligned chunks, newline flattening per 16 KiB tile
//                     (scan.rs:91-183) and parse_line (line.rs:8-81)
//   olb_build_links   links.rs:27-180 three-phase ANSV (local stacks, persistent
//                     global stack combine, resolve) for parent and subtree_end
//   olb_children      first_child / next_sibling derived from the links
//   olb_find_all_par  search.rs:28-60,88-99 overlapping chunks (pattern-1 bytes
//                     of overlap), every overlapping hit; the per-chunk searcher
//                     is a first/last-byte AVX2 filter plus memcmp (the
//                     published "SIMD-friendly substring search" method), in
//                     place of memchr::memmem
//   olb_many_*        search.rs:206-282 dictionary search with an Aho-Corasick
//                     DFA (standard goto/failure/output construction, byte
//                     classes, full transition table), overlapping iteration
//                     over chunks with longest-1 bytes of overlap, hits ordered
//                     by (pattern, offset)
#include <immintrin.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;

struct Node {
    uint32_t depth, kind, span_start, span_len;
};

template <class F>
void parallel_for(int threads, size_t n, F f) {
    if (threads <= 1 || n <= 1) {
        for (size_t i = 0; i < n; i++) f(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    int t = std::min<size_t>(threads, n);
    for (int k = 0; k < t; k++)
        pool.emplace_back([&] {
            for (;;) {
                size_t i = next.fetch_add(1);
                if (i >= n) break;
                f(i);
            }
        });
    for (auto &th : pool) th.join();
}

inline bool blank(uint8_t b) { return b == ' ' || b == '\t'; }

// parse_line (line.rs:8-81).
inline Node parse_line(const uint8_t *line, size_t len, uint32_t start) {
    size_t eff = len;
    while (eff > 0 && (line[eff - 1] == '\r' || line[eff - 1] == '\n')) eff--;
    if (eff == 0) return Node{0, 0, start, 0};
    size_t depth = 0;
    while (depth < eff && line[depth] == '|') depth++;
    size_t pos = depth, bl = 0;
    while (pos + bl < eff && blank(line[pos + bl])) bl++;
    while (depth > 0 && pos + bl < eff && line[pos + bl] == '|') {
        pos += bl;
        size_t run = 0;
        while (pos + run < eff && line[pos + run] == '|') run++;
        depth += run;
        pos += run;
        bl = 0;
        while (pos + bl < eff && blank(line[pos + bl])) bl++;
    }
    size_t cs = pos + bl;
    if (cs == eff) return Node{(uint32_t)depth, 0, start + (uint32_t)cs, 0};
    const uint8_t *c = line + cs;
    size_t n = eff - cs;
    uint32_t k = 1;
    switch (c[0]) {
    case '=': k = 2; break;
    case ':': k = 5; break;
    case '@': k = 3; break;
    case '/': k = (n > 1 && c[1] == '/') ? 7 : 1; break;
    case '-':
        if (n > 1 && blank(c[1])) k = 4;
        else if (n > 2 && c[1] == '.' && blank(c[2])) k = 6;
        break;
    default: break;
    }
    return Node{(uint32_t)depth, k, start + (uint32_t)cs, (uint32_t)n};
}

__attribute__((target("avx2,popcnt"))) size_t count_newlines_avx2(const uint8_t *b, size_t len) {
    const __m256i nl = _mm256_set1_epi8('\n');
    size_t i = 0, total = 0;
    for (; i + 32 <= len; i += 32) {
        __m256i v = _mm256_loadu_si256((const __m256i *)(b + i));
        total += __builtin_popcount((uint32_t)_mm256_movemask_epi8(_mm256_cmpeq_epi8(v, nl)));
    }
    for (; i < len; i++) total += b[i] == '\n';
    return total;
}

size_t count_newlines(const uint8_t *b, size_t len) {
    if (__builtin_cpu_supports("avx2")) return count_newlines_avx2(b, len);
    size_t n = 0;
    for (size_t i = 0; i < len; i++) n += b[i] == '\n';
    return n;
}

size_t lines_in_chunk(const uint8_t *b, size_t len) { return len == 0 ? 0 : count_newlines(b, len) + (b[len - 1] != '\n'); }

// flatten_newlines (scan.rs:91-183): positions of '\n' in a tile, written in
// fixed groups so that the count, not a branch per newline, advances.
__attribute__((target("avx2,popcnt,bmi"))) size_t flatten_avx2(const uint8_t *b, size_t len, uint32_t base, uint32_t *out) {
    const __m256i nl = _mm256_set1_epi8('\n');
    size_t n = 0, i = 0;
    for (; i + 64 <= len; i += 64) {
        uint64_t lo = (uint32_t)_mm256_movemask_epi8(_mm256_cmpeq_epi8(_mm256_loadu_si256((const __m256i *)(b + i)), nl));
        uint64_t hi = (uint32_t)_mm256_movemask_epi8(_mm256_cmpeq_epi8(_mm256_loadu_si256((const __m256i *)(b + i + 32)), nl));
        uint64_t m = lo | (hi << 32);
        size_t cnt = (size_t)__builtin_popcountll(m);
        uint32_t at = base + (uint32_t)i;
        for (int g = 0; g < 8; g++) {
            out[n + g] = at + (uint32_t)__builtin_ctzll(m | (1ull << 63));
            m &= m - 1;
        }
        if (cnt > 8) {
            for (size_t g = 8; g < cnt; g++) {
                out[n + g] = at + (uint32_t)__builtin_ctzll(m);
                m &= m - 1;
            }
        }
        n += cnt;
    }
    for (; i < len; i++)
        if (b[i] == '\n') out[n++] = base + (uint32_t)i;
    return n;
}

size_t flatten(const uint8_t *b, size_t len, uint32_t base, uint32_t *out) {
    if (__builtin_cpu_supports("avx2") && __builtin_cpu_supports("bmi")) return flatten_avx2(b, len, base, out);
    size_t n = 0;
    for (size_t i = 0; i < len; i++)
        if (b[i] == '\n') out[n++] = base + (uint32_t)i;
    return n;
}

constexpr size_t TILE = 16 * 1024;
constexpr size_t MIN_CHUNK = 128 * 1024;

// fill_chunk (lib.rs:73-112).
void fill_chunk(const uint8_t *bytes, size_t start, size_t end, Node *nodes, uint32_t *offsets) {
    const uint8_t *chunk = bytes + start;
    size_t len = end - start, k = 0, line_start = 0;
    std::vector<uint32_t> pos(TILE + 64);
    for (size_t t = 0; t < len; t += TILE) {
        size_t tl = std::min(TILE, len - t);
        size_t n = flatten(chunk + t, tl, (uint32_t)t, pos.data());
        for (size_t j = 0; j < n; j++) {
            size_t line_end = pos[j] + 1;
            uint32_t abs = (uint32_t)(start + line_start);
            if (offsets) offsets[k] = abs;
            if (nodes) nodes[k] = parse_line(chunk + line_start, line_end - line_start, abs);
            k++;
            line_start = line_end;
        }
    }
    if (line_start < len) {
        uint32_t abs = (uint32_t)(start + line_start);
        if (offsets) offsets[k] = abs;
        if (nodes) nodes[k] = parse_line(chunk + line_start, len - line_start, abs);
    }
}

// partition_chunks (lib.rs:115-137).
std::vector<std::pair<size_t, size_t>> partition(const uint8_t *b, size_t len, size_t target) {
    std::vector<std::pair<size_t, size_t>> out;
    if (len == 0) return out;
    target = std::max<size_t>(1, std::min(target, len / MIN_CHUNK));
    size_t approx = len / target;
    std::vector<size_t> bounds{0};
    for (size_t k = 1; k < target; k++) {
        size_t pos = k * approx;
        const void *nl = memchr(b + pos, '\n', len - pos);
        if (!nl) break;
        pos = (size_t)((const uint8_t *)nl - b) + 1;
        if (pos < len && pos > bounds.back()) bounds.push_back(pos);
    }
    bounds.push_back(len);
    for (size_t i = 0; i + 1 < bounds.size(); i++) out.push_back({bounds[i], bounds[i + 1]});
    return out;
}

// ANSV (links.rs:27-131): for each line the nearest line before it in scan
// order (j < i when FORWARD, j > i otherwise) whose key is smaller (or, with
// OR_EQUAL, smaller or equal); NONE if there is none. A line's key is its
// depth, NONE for a blank line. Three phases, as the reference: each block of
// BLOCK lines runs a stack (key and position together, so the keys are read
// once, in order, from the nodes), the blocks' remaining stacks are chained in
// scan order, and each block resolves its pending lines against the chain.
constexpr size_t BLOCK = 1 << 15;
constexpr uint32_t PENDING = NONE - 1;

inline uint32_t node_key(const Node &nd) { return nd.kind == 0 ? NONE : std::min(nd.depth, NONE - 1); }

template <bool OR_EQUAL, bool FORWARD>
void nearest_before(const Node *nodes, size_t n, uint32_t *res, int threads) {
    if (n == 0) return;
    auto ok = [](uint32_t v, uint32_t x) { return OR_EQUAL ? v <= x : v < x; };
    auto at = [n](size_t v) { return FORWARD ? v : n - 1 - v; };  // scan step -> line
    struct KeyAt {
        uint32_t key, idx;
    };
    size_t nb = (n + BLOCK - 1) / BLOCK;
    std::vector<std::vector<KeyAt>> summaries(nb);
    parallel_for(threads, nb, [&](size_t b) {
        size_t base = b * BLOCK, end = std::min(n, base + BLOCK);
        std::vector<KeyAt> stack;
        stack.reserve(256);
        for (size_t v = base; v < end; v++) {
            const size_t j = at(v);
            const uint32_t x = node_key(nodes[j]);
            while (!stack.empty() && !ok(stack.back().key, x)) stack.pop_back();
            res[j] = stack.empty() ? PENDING : stack.back().idx;
            stack.push_back(KeyAt{x, (uint32_t)j});
        }
        auto &s = summaries[b];
        for (size_t i = 0; i < stack.size(); i++) {
            bool next_same = i + 1 < stack.size() && stack[i + 1].key == stack[i].key;
            if (!next_same) s.push_back(stack[i]);
        }
    });
    struct Entry {
        uint32_t key, idx, link;
    };
    std::vector<Entry> pool;
    std::vector<uint32_t> heads(nb);
    uint32_t head = NONE;
    for (size_t b = 0; b < nb; b++) {
        heads[b] = head;
        auto &s = summaries[b];
        if (!s.empty()) {
            uint32_t min_key = s[0].key;
            while (head != NONE && !ok(pool[head].key, min_key)) head = pool[head].link;
            for (const KeyAt &e : s) {
                pool.push_back(Entry{e.key, e.idx, head});
                head = (uint32_t)(pool.size() - 1);
            }
        }
    }
    parallel_for(threads, nb, [&](size_t b) {
        size_t base = b * BLOCK, end = std::min(n, base + BLOCK);
        uint32_t p = heads[b];
        for (size_t v = base; v < end; v++) {
            const size_t j = at(v);
            if (res[j] != PENDING) continue;
            const uint32_t x = node_key(nodes[j]);
            while (p != NONE && !ok(pool[p].key, x)) p = pool[p].link;
            res[j] = p == NONE ? NONE : pool[p].idx;
        }
    });
}

// Equality of n bytes; n <= 8 as one masked 64-bit compare (the caller
// guarantees 8 readable bytes at both addresses), longer ones with memcmp.
inline bool same_bytes(const uint8_t *a, const uint8_t *b, size_t n) {
    if (n <= 8) {
        uint64_t x, y;
        memcpy(&x, a, 8);
        memcpy(&y, b, 8);
        uint64_t mask = n == 8 ? ~0ull : ((1ull << (8 * n)) - 1);
        return ((x ^ y) & mask) == 0;
    }
    return memcmp(a, b, n) == 0;
}

// First/last-byte AVX2 filter + memcmp: every overlapping occurrence of p in
// hay[0..len), reported as base + i.
__attribute__((target("avx2,bmi"))) void find_chunk_avx2(const uint8_t *hay, size_t len, const uint8_t *p, size_t m,
                                                         size_t base, std::vector<uint32_t> &out) {
    if (m == 0 || len < m) return;
    size_t last = len - m;  // last valid start
    size_t i = 0;
    if (m >= 2) {
        const __m256i f = _mm256_set1_epi8((char)p[0]);
        const __m256i l = _mm256_set1_epi8((char)p[m - 1]);
        // pattern bytes 1..m-2, padded so that the short compare may read 8
        uint8_t mid[8] = {0};
        memcpy(mid, p + 1, std::min<size_t>(m - 2, 8));
        const bool short_mid = m - 2 <= 8;
        for (; i + 32 <= last + 1; i += 32) {
            __m256i a = _mm256_loadu_si256((const __m256i *)(hay + i));
            __m256i b = _mm256_loadu_si256((const __m256i *)(hay + i + m - 1));
            uint32_t mask = (uint32_t)_mm256_movemask_epi8(_mm256_and_si256(_mm256_cmpeq_epi8(a, f), _mm256_cmpeq_epi8(b, l)));
            while (mask) {
                size_t k = i + (size_t)__builtin_ctz(mask);
                // 8 bytes from k + 1 stay inside hay when k + 1 + 8 <= len
                bool eq = short_mid && k + 9 <= len ? same_bytes(hay + k + 1, mid, m - 2)
                                                    : memcmp(hay + k + 1, p + 1, m - 2) == 0;
                if (eq) out.push_back((uint32_t)(base + k));
                mask &= mask - 1;
            }
        }
    } else {
        const __m256i f = _mm256_set1_epi8((char)p[0]);
        for (; i + 32 <= last + 1; i += 32) {
            uint32_t mask = (uint32_t)_mm256_movemask_epi8(_mm256_cmpeq_epi8(_mm256_loadu_si256((const __m256i *)(hay + i)), f));
            while (mask) {
                out.push_back((uint32_t)(base + i + (size_t)__builtin_ctz(mask)));
                mask &= mask - 1;
            }
        }
    }
    for (; i <= last; i++)
        if (hay[i] == p[0] && memcmp(hay + i, p, m) == 0) out.push_back((uint32_t)(base + i));
}

void find_chunk(const uint8_t *hay, size_t len, const uint8_t *p, size_t m, size_t base, std::vector<uint32_t> &out) {
    if (__builtin_cpu_supports("avx2")) return find_chunk_avx2(hay, len, p, m, base, out);
    if (m == 0 || len < m) return;
    for (size_t i = 0; i + m <= len; i++)
        if (memcmp(hay + i, p, m) == 0) out.push_back((uint32_t)(base + i));
}

// ---- Aho-Corasick DFA ------------------------------------------------------

struct AcDfa {
    uint32_t n_classes = 0;
    uint8_t cls[256];
    std::vector<uint32_t> trans;     // state * n_classes + class -> state
    std::vector<uint32_t> out_first; // first pattern id recognised in the state (own), or NONE
    std::vector<uint32_t> out_link;  // nearest state on the failure chain with own outputs, or NONE
    std::vector<uint32_t> pid_next;  // next pattern id with the same end state
    std::vector<uint32_t> lens;
    uint32_t longest = 0;
    uint32_t n_states = 0;
};

}  // namespace

extern "C" {

// Parse: line offsets + 16-byte nodes, multi-threaded (try_parse_par_with_buffers
// TwoPass, lib.rs:189-244, 445-469). Returns the line count; writes at most cap.
uint64_t olb_parse_par(const uint8_t *text, uint64_t len, uint32_t *offsets, Node *nodes, uint64_t cap, int threads) {
    if (len == 0) return 0;
    auto chunks = partition(text, len, (size_t)threads * 4);
    std::vector<size_t> counts(chunks.size());
    parallel_for(threads, chunks.size(), [&](size_t i) { counts[i] = lines_in_chunk(text + chunks[i].first, chunks[i].second - chunks[i].first); });
    std::vector<size_t> base(chunks.size() + 1, 0);
    for (size_t i = 0; i < chunks.size(); i++) base[i + 1] = base[i] + counts[i];
    uint64_t total = base.back();
    if (total > cap) return total;
    parallel_for(threads, chunks.size(), [&](size_t i) {
        fill_chunk(text, chunks[i].first, chunks[i].second, nodes ? nodes + base[i] : nullptr, offsets ? offsets + base[i] : nullptr);
    });
    return total;
}

// build_links (links.rs:135-180): parent + subtree_end. The nearest smaller
// line before each line is its parent; the nearest smaller-or-equal line after
// it ends its subtree (the document's end when there is none).
void olb_build_links(const Node *nodes, uint64_t n, uint32_t *parent, uint32_t *subtree_end, int threads) {
    nearest_before<false, true>(nodes, n, parent, threads);
    nearest_before<true, false>(nodes, n, subtree_end, threads);
    size_t step = std::max<size_t>(1, (n + threads - 1) / std::max(threads, 1));
    size_t parts = (n + step - 1) / step;
    parallel_for(threads, parts, [&](size_t p) {
        for (size_t i = p * step; i < std::min<size_t>(n, (p + 1) * step); i++) {
            if (nodes[i].kind == 0) {
                parent[i] = NONE;
                subtree_end[i] = (uint32_t)i + 1;
            } else if (subtree_end[i] == NONE) {
                subtree_end[i] = (uint32_t)n;
            }
        }
    });
}

// first_child / next_sibling from the links, in parallel chunks.
void olb_children(const Node *nodes, uint64_t n, const uint32_t *parent, const uint32_t *subtree_end, uint32_t *first_child,
                  uint32_t *next_sibling, int threads) {
    size_t step = std::max<size_t>(1, (n + threads - 1) / std::max(threads, 1));
    size_t parts = (n + step - 1) / step;
    parallel_for(threads, parts, [&](size_t p) {
        size_t lo = p * step, hi = std::min<size_t>(n, (p + 1) * step);
        uint32_t next_nb = NONE;
        for (size_t j = hi; j < n; j++)
            if (nodes[j].kind != 0) {
                next_nb = (uint32_t)j;
                break;
            }
        for (size_t i = hi; i-- > lo;) {
            if (nodes[i].kind == 0) {
                first_child[i] = NONE;
                next_sibling[i] = NONE;
                continue;
            }
            uint32_t e = subtree_end[i];
            first_child[i] = (next_nb != NONE && next_nb < e) ? next_nb : NONE;
            next_sibling[i] = (e < n && parent[e] == parent[i]) ? e : NONE;
            next_nb = (uint32_t)i;
        }
    });
}

// find_all_par (search.rs:28-52). Writes at most cap offsets; returns the total.
uint64_t olb_find_all_par(const uint8_t *text, uint64_t len, const uint8_t *pat, uint64_t m, uint32_t *out, uint64_t cap,
                          int threads) {
    if (m == 0 || len < m) return 0;
    size_t chunk = std::max<size_t>(len / ((size_t)threads * 4), 1 << 20);
    size_t nch = (len + chunk - 1) / chunk;
    std::vector<std::vector<uint32_t>> parts(nch);
    parallel_for(threads, nch, [&](size_t c) {
        size_t start = c * chunk, end = std::min<size_t>(start + chunk, len);
        size_t wend = std::min<size_t>(end + m - 1, len);
        find_chunk(text + start, wend - start, pat, m, start, parts[c]);
    });
    // chunks in order; each copies its hits to its place in parallel
    std::vector<uint64_t> at(nch + 1, 0);
    for (size_t c = 0; c < nch; c++) at[c + 1] = at[c] + parts[c].size();
    parallel_for(threads, nch, [&](size_t c) {
        if (at[c] >= cap || parts[c].empty()) return;
        size_t k = (size_t)std::min<uint64_t>(parts[c].size(), cap - at[c]);
        memcpy(out + at[c], parts[c].data(), k * 4);
    });
    return at[nch];
}

// ManyPatterns::new (search.rs:214-227): Aho-Corasick automaton, MatchKind::Standard.
void *olb_many_new(const uint8_t *pats, const uint32_t *lens, uint32_t n) {
    auto *d = new AcDfa();
    d->lens.assign(lens, lens + n);
    bool used[256] = {false};
    uint64_t at = 0;
    for (uint32_t i = 0; i < n; i++) {
        for (uint32_t k = 0; k < lens[i]; k++) used[pats[at + k]] = true;
        at += lens[i];
        d->longest = std::max(d->longest, lens[i]);
    }
    uint32_t nc = 1;  // class 0 = bytes in no pattern
    for (int b = 0; b < 256; b++) d->cls[b] = used[b] ? (uint8_t)(nc++ & 0xFF) : 0;
    // more than 255 used bytes: classes are the bytes themselves
    if (nc > 256) {
        nc = 256;
        for (int b = 0; b < 256; b++) d->cls[b] = (uint8_t)b;
    }
    d->n_classes = nc;
    // Trie (goto function).
    std::vector<uint32_t> &tr = d->trans;
    tr.assign(nc, NONE);
    d->out_first.assign(1, NONE);
    d->pid_next.assign(n, NONE);
    uint32_t states = 1;
    at = 0;
    std::vector<uint32_t> endstate(n);
    for (uint32_t i = 0; i < n; i++) {
        uint32_t s = 0;
        for (uint32_t k = 0; k < lens[i]; k++) {
            uint32_t c = d->cls[pats[at + k]];
            uint32_t nx = tr[(size_t)s * nc + c];
            if (nx == NONE) {
                nx = states++;
                tr.resize((size_t)states * nc, NONE);
                d->out_first.push_back(NONE);
                tr[(size_t)s * nc + c] = nx;
            }
            s = nx;
        }
        endstate[i] = s;
        at += lens[i];
    }
    // Pattern ids per end state, ascending.
    for (uint32_t ii = n; ii-- > 0;) {
        if (lens[ii] == 0) continue;
        d->pid_next[ii] = d->out_first[endstate[ii]];
        d->out_first[endstate[ii]] = ii;
    }
    // BFS: failure links, output links, full DFA transitions.
    std::vector<uint32_t> fail(states, 0);
    d->out_link.assign(states, NONE);
    std::vector<uint32_t> queue;
    queue.reserve(states);
    for (uint32_t c = 0; c < nc; c++) {
        uint32_t nx = tr[c];
        if (nx == NONE) {
            tr[c] = 0;
        } else {
            fail[nx] = 0;
            queue.push_back(nx);
        }
    }
    for (size_t qi = 0; qi < queue.size(); qi++) {
        uint32_t s = queue[qi];
        uint32_t f = fail[s];
        d->out_link[s] = d->out_first[f] != NONE ? f : d->out_link[f];
        for (uint32_t c = 0; c < nc; c++) {
            uint32_t nx = tr[(size_t)s * nc + c];
            if (nx == NONE) {
                tr[(size_t)s * nc + c] = tr[(size_t)f * nc + c];
            } else {
                fail[nx] = tr[(size_t)f * nc + c];
                queue.push_back(nx);
            }
        }
    }
    d->n_states = states;
    return d;
}

void olb_many_free(void *p) { delete (AcDfa *)p; }
uint32_t olb_many_states(void *p) { return ((AcDfa *)p)->n_states; }

// ManyPatterns::find_all_par (search.rs:259-282): every hit, sorted by
// (pattern, offset). Writes at most cap hits; per-pattern counts into counts.
uint64_t olb_many_find_all_par(void *p, const uint8_t *text, uint64_t len, uint64_t *counts, uint32_t *hit_pat, uint32_t *hit_off,
                               uint64_t cap, int threads) {
    const AcDfa &d = *(const AcDfa *)p;
    uint32_t np = (uint32_t)d.lens.size();
    for (uint32_t i = 0; i < np; i++) counts[i] = 0;
    if (len == 0 || np == 0) return 0;
    size_t chunk = std::max<size_t>(len / ((size_t)threads * 4), 1 << 20);
    size_t nch = (len + chunk - 1) / chunk;
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> parts(nch);
    const uint32_t nc = d.n_classes;
    parallel_for(threads, nch, [&](size_t c) {
        size_t start = c * chunk, end = std::min<size_t>(start + chunk, len);
        size_t wend = std::min<size_t>(end + d.longest - 1, len);
        auto &out = parts[c];
        uint32_t s = 0;
        const uint32_t *tr = d.trans.data();
        for (size_t i = start; i < wend; i++) {
            s = tr[(size_t)s * nc + d.cls[text[i]]];
            uint32_t st = d.out_first[s] != NONE ? s : d.out_link[s];
            while (st != NONE) {
                for (uint32_t id = d.out_first[st]; id != NONE; id = d.pid_next[id]) {
                    size_t mstart = i + 1 - d.lens[id];
                    if (mstart >= start && mstart < end) out.push_back({id, (uint32_t)mstart});
                }
                st = d.out_link[st];
            }
        }
    });
    // Counting sort by pattern; chunks are visited in order and each chunk's
    // hits ascend by end position, so sort each chunk's hits by offset first.
    parallel_for(threads, nch, [&](size_t c) {
        std::sort(parts[c].begin(), parts[c].end(), [](auto a, auto b) { return a.second < b.second || (a.second == b.second && a.first < b.first); });
    });
    std::vector<uint64_t> cnt(np, 0);
    for (auto &v : parts)
        for (auto &h : v) cnt[h.first]++;
    std::vector<uint64_t> base(np);
    uint64_t total = 0;
    for (uint32_t i = 0; i < np; i++) {
        base[i] = total;
        total += cnt[i];
        counts[i] = cnt[i];
    }
    if (cap > 0) {
        for (auto &v : parts)
            for (auto &h : v) {
                uint64_t slot = base[h.first]++;
                if (slot < cap) {
                    hit_pat[slot] = h.first;
                    hit_off[slot] = h.second;
                }
            }
    }
    return total;
}

// Order-checking digest of the whole sorted hit list, without building it:
// the sum over every hit of hit_digest(slot, pattern, offset), where slot is
// the hit's index in the (pattern, offset) order of ManyPatterns::find_all_par
// (search.rs:259-282). Two passes over the same chunks: the first counts each
// pattern's hits per chunk; the second walks again and, since a chunk meets a
// pattern's hits in ascending offset order, gives each its slot from the
// running per-(chunk, pattern) base. counts[i] receives pattern i's hits.
// Returns the digest; *total the number of hits.
uint64_t olb_hit_digest(uint64_t slot, uint32_t pattern, uint32_t offset) {
    uint64_t x = (((uint64_t)pattern << 32) | offset) ^ (slot * 0x9E3779B97F4A7C15ull);
    x ^= x >> 30;
    x *= 0xBF58476D1CE4E5B9ull;
    x ^= x >> 27;
    x *= 0x94D049BB133111EBull;
    x ^= x >> 31;
    return x;
}

uint64_t olb_many_digest_par(void *p, const uint8_t *text, uint64_t len, uint64_t *counts, uint64_t *total_out,
                             int threads) {
    const AcDfa &d = *(const AcDfa *)p;
    const uint32_t np = (uint32_t)d.lens.size();
    for (uint32_t i = 0; i < np; i++) counts[i] = 0;
    *total_out = 0;
    if (len == 0 || np == 0) return 0;
    size_t chunk = std::max<size_t>(len / ((size_t)threads * 4), 1 << 20);
    size_t nch = (len + chunk - 1) / chunk;
    const uint32_t nc = d.n_classes;
    // walk(c, f): f(pattern, offset) for every hit starting in chunk c, in the
    // order the automaton meets them
    auto walk = [&](size_t c, auto &&f) {
        size_t start = c * chunk, end = std::min<size_t>(start + chunk, len);
        size_t wend = std::min<size_t>(end + d.longest - 1, len);
        uint32_t s = 0;
        const uint32_t *tr = d.trans.data();
        for (size_t i = start; i < wend; i++) {
            s = tr[(size_t)s * nc + d.cls[text[i]]];
            uint32_t st = d.out_first[s] != NONE ? s : d.out_link[s];
            while (st != NONE) {
                for (uint32_t id = d.out_first[st]; id != NONE; id = d.pid_next[id]) {
                    size_t mstart = i + 1 - d.lens[id];
                    if (mstart >= start && mstart < end) f(id, (uint32_t)mstart);
                }
                st = d.out_link[st];
            }
        }
    };
    std::vector<std::vector<uint64_t>> per(nch, std::vector<uint64_t>(np, 0));
    parallel_for(threads, nch, [&](size_t c) {
        auto &cnt = per[c];
        walk(c, [&](uint32_t id, uint32_t) { cnt[id]++; });
    });
    // per-(chunk, pattern) first slot: patterns in order, chunks in order within each
    uint64_t at = 0;
    for (uint32_t i = 0; i < np; i++) {
        for (size_t c = 0; c < nch; c++) {
            uint64_t k = per[c][i];
            per[c][i] = at;
            at += k;
            counts[i] += k;
        }
    }
    *total_out = at;
    std::vector<uint64_t> sums(nch, 0);
    parallel_for(threads, nch, [&](size_t c) {
        auto &next = per[c];
        uint64_t sum = 0;
        walk(c, [&](uint32_t id, uint32_t off) { sum += olb_hit_digest(next[id]++, id, off); });
        sums[c] = sum;
    });
    uint64_t digest = 0;
    for (uint64_t v : sums) digest += v;
    return digest;
}

}  // extern "C"
