/* ORACLE — test infrastructure only.
 *
 * A plain-C restatement of the reference's CPU algorithms for the oneline
 * parse-and-search path (tomet-lang/oneline, crates oneline-core and
 * oneline-simd). It is the checker: only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load it. The product (oneline_b200) never
 * links or calls it, and has no CPU fallback.
 *
 * Pinning: the reference is Rust and cannot be built in this environment (no
 * cargo/rustc, and its memchr / aho-corasick dependencies are not vendored), so
 * this restatement is pinned against the reference's own known-answer tests and
 * differential tests (tests/golden/reference_kat.json, transcribed from the
 * reference's test modules with file:line citations), including its
 * byte-loop classifier oracle (line.rs:89-142), restated below and checked
 * exhaustively against the fast form the way line.rs:145-181 does.
 *
 * Functions (all extern "C", plain pointers):
 *   olo_parse_line            crates/oneline-simd/src/line.rs:8-81
 *   olo_parse_line_bytewise   crates/oneline-simd/src/line.rs:89-142
 *   olo_scan_line_offsets     crates/oneline-simd/src/lib.rs:49-66
 *   olo_parse                 crates/oneline-simd/src/lib.rs:493-513 (reference())
 *   olo_tree                  crates/oneline-core/src/links.rs:52-82
 *   olo_tree_children         first_child / next_sibling derived from the links
 *   olo_find_all              crates/oneline-simd/src/search.rs:106-114 (naive)
 *   olo_find_many             crates/oneline-simd/src/search.rs:259-282 semantics:
 *                             every (pattern, offset), duplicates once per id,
 *                             sorted by (pattern, offset)
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OLO_NONE 0xFFFFFFFFu

typedef struct {
    uint32_t depth, kind, span_start, span_len;
} olo_node;

enum { K_BLANK = 0, K_TEXT = 1, K_HEADING = 2, K_ELEMENT = 3, K_LIST = 4, K_CONNECT = 5, K_ORDERED = 6, K_COMMENT = 7 };

static int is_blank(uint8_t b) { return b == ' ' || b == '\t'; }

/* classify_line (line.rs:57-81): the content's first byte decides; '-' needs a
 * blank after it (or ". " for an ordered item), '/' needs a second '/'. */
static uint32_t classify(const uint8_t *c, uint64_t n) {
    switch (c[0]) {
    case '=': return K_HEADING;
    case ':': return K_CONNECT;
    case '@': return K_ELEMENT;
    case '/': return (n > 1 && c[1] == '/') ? K_COMMENT : K_TEXT;
    case '-':
        if (n > 1 && is_blank(c[1])) return K_LIST;
        if (n > 1 && c[1] == '.' && n > 2 && is_blank(c[2])) return K_ORDERED;
        return K_TEXT;
    default: return K_TEXT;
    }
}

/* parse_line (line.rs:8-44). */
void olo_parse_line(const uint8_t *line, uint64_t len, uint32_t line_start, olo_node *out) {
    uint64_t eff = len;
    while (eff > 0 && (line[eff - 1] == '\r' || line[eff - 1] == '\n')) eff--;
    if (eff == 0) {
        out->depth = 0;
        out->kind = K_BLANK;
        out->span_start = line_start;
        out->span_len = 0;
        return;
    }
    uint64_t depth = 0;
    while (depth < eff && line[depth] == '|') depth++;
    uint64_t pos = depth;
    uint64_t blanks = 0;
    while (pos + blanks < eff && is_blank(line[pos + blanks])) blanks++;
    while (depth > 0 && pos + blanks < eff && line[pos + blanks] == '|') {
        pos += blanks;
        uint64_t run = 0;
        while (pos + run < eff && line[pos + run] == '|') run++;
        depth += run;
        pos += run;
        blanks = 0;
        while (pos + blanks < eff && is_blank(line[pos + blanks])) blanks++;
    }
    uint64_t cs = pos + blanks;
    out->depth = (uint32_t)depth;
    out->span_start = line_start + (uint32_t)cs;
    if (cs == eff) {
        out->kind = K_BLANK;
        out->span_len = 0;
        return;
    }
    out->kind = classify(line + cs, eff - cs);
    out->span_len = (uint32_t)(eff - cs);
}

/* The older byte-loop classifier the reference keeps as its test oracle
 * (line.rs:89-142): remembers where the last '|' was; a blank run belongs to
 * the prefix only if another '|' follows it. */
void olo_parse_line_bytewise(const uint8_t *b, uint64_t len, uint32_t line_start, olo_node *out) {
    out->depth = 0;
    out->kind = K_BLANK;
    out->span_start = line_start;
    out->span_len = 0;
    if (len == 0) return;
    uint64_t eff = len;
    while (eff > 0 && (b[eff - 1] == '\r' || b[eff - 1] == '\n')) eff--;
    if (eff == 0) return;
    uint64_t depth = 0, prefix_end = 0, i = 0;
    while (i < eff) {
        if (b[i] == '|') {
            depth++;
            i++;
            prefix_end = i;
        } else if (is_blank(b[i]) && depth > 0) {
            i++;
        } else {
            break;
        }
    }
    uint64_t cs = prefix_end;
    while (cs < eff && is_blank(b[cs])) cs++;
    out->depth = (uint32_t)depth;
    out->span_start = line_start + (uint32_t)cs;
    if (eff == cs) return;
    const uint8_t *r = b + cs;
    uint64_t n = eff - cs;
    uint32_t k = K_TEXT;
    if (r[0] == '=') k = K_HEADING;
    else if (r[0] == ':') k = K_CONNECT;
    else if (r[0] == '@') k = K_ELEMENT;
    else if (r[0] == '-' && n > 1 && is_blank(r[1])) k = K_LIST;
    else if (r[0] == '-' && n > 2 && r[1] == '.' && is_blank(r[2])) k = K_ORDERED;
    else if (r[0] == '/' && n > 1 && r[1] == '/') k = K_COMMENT;
    out->kind = k;
    out->span_len = (uint32_t)n;
}

/* Number of lines: one per '\n' whose successor exists, plus the first line
 * (lib.rs:36-43 / reference() at lib.rs:496-504). 0 for empty text. */
uint64_t olo_count_lines(const uint8_t *t, uint64_t len) {
    if (len == 0) return 0;
    uint64_t n = 1;
    for (uint64_t i = 0; i + 1 < len; i++) n += t[i] == '\n';
    return n;
}

/* scan_line_offsets (lib.rs:49-66): 0, then p+1 for every '\n' at p with
 * p+1 < len. Writes at most cap entries; returns the line count. */
uint64_t olo_scan_line_offsets(const uint8_t *t, uint64_t len, uint32_t *out, uint64_t cap) {
    if (len == 0) return 0;
    uint64_t n = 0;
    if (cap > 0) out[0] = 0;
    n = 1;
    for (uint64_t i = 0; i + 1 < len; i++) {
        if (t[i] == '\n') {
            if (n < cap) out[n] = (uint32_t)(i + 1);
            n++;
        }
    }
    return n;
}

/* reference() (lib.rs:493-513): split after every '\n', parse each piece.
 * Either output may be NULL. Returns the line count. */
uint64_t olo_parse(const uint8_t *t, uint64_t len, uint32_t *offsets, olo_node *nodes, uint64_t cap) {
    if (len == 0) return 0;
    uint64_t n = 0, s = 0;
    for (uint64_t i = 0; i < len; i++) {
        if (t[i] == '\n' || i + 1 == len) {
            uint64_t e = i + 1;
            if (n < cap) {
                if (offsets) offsets[n] = (uint32_t)s;
                if (nodes) olo_parse_line(t + s, e - s, (uint32_t)s, &nodes[n]);
            }
            n++;
            s = e;
        }
    }
    return n;
}

/* Kinds only (u8), the compact form of the parse. */
void olo_kinds(const olo_node *nodes, uint64_t n, uint8_t *kinds) {
    for (uint64_t i = 0; i < n; i++) kinds[i] = (uint8_t)nodes[i].kind;
}

/* TreeLinks::from_nodes_sequential (core links.rs:52-82): monotonic stack over
 * the non-blank lines. parent = nearest previous content line with a smaller
 * depth; subtree_end = nearest next content line with depth <= own, else n.
 * Blank lines: parent NONE, subtree_end i+1. */
void olo_tree(const olo_node *nodes, uint64_t n, uint32_t *parent, uint32_t *subtree_end) {
    uint32_t *stack = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    uint64_t sp = 0;
    for (uint64_t i = 0; i < n; i++) {
        parent[i] = OLO_NONE;
        subtree_end[i] = (uint32_t)(i + 1);
    }
    for (uint64_t i = 0; i < n; i++) {
        if (nodes[i].kind == K_BLANK) continue;
        while (sp > 0 && nodes[stack[sp - 1]].depth >= nodes[i].depth) {
            subtree_end[stack[sp - 1]] = (uint32_t)i;
            sp--;
        }
        parent[i] = sp > 0 ? stack[sp - 1] : OLO_NONE;
        stack[sp++] = (uint32_t)i;
    }
    for (uint64_t k = 0; k < sp; k++) subtree_end[stack[k]] = (uint32_t)n;
    free(stack);
}

/* first_child / next_sibling (not a reference output; derived from the links):
 *   first_child[i]  = first non-blank line j > i if j < subtree_end[i], else NONE
 *   next_sibling[i] = j = subtree_end[i] if j < n and parent[j] == parent[i], else NONE
 * Blank lines get NONE for both. */
void olo_tree_children(const olo_node *nodes, uint64_t n, const uint32_t *parent, const uint32_t *subtree_end,
                       uint32_t *first_child, uint32_t *next_sibling) {
    uint32_t next_nb = OLO_NONE; /* first non-blank line after i */
    for (uint64_t ii = n; ii-- > 0;) {
        if (nodes[ii].kind == K_BLANK) {
            first_child[ii] = OLO_NONE;
            next_sibling[ii] = OLO_NONE;
            continue;
        }
        uint32_t e = subtree_end[ii];
        first_child[ii] = (next_nb != OLO_NONE && next_nb < e) ? next_nb : OLO_NONE;
        next_sibling[ii] = (e < n && parent[e] == parent[ii]) ? e : OLO_NONE;
        next_nb = (uint32_t)ii;
    }
}

/* naive (search.rs:106-114): every overlapping occurrence, ascending. An empty
 * pattern or a text shorter than the pattern gives nothing. Writes at most cap
 * offsets; returns the total. */
uint64_t olo_find_all(const uint8_t *t, uint64_t len, const uint8_t *p, uint64_t m, uint32_t *out, uint64_t cap) {
    if (m == 0 || len < m) return 0;
    uint64_t n = 0;
    const uint8_t *cur = t;
    const uint8_t *last = t + (len - m);
    while (cur <= last) {
        const uint8_t *hit = (const uint8_t *)memchr(cur, p[0], (size_t)(last - cur) + 1);
        if (!hit) break;
        if (memcmp(hit, p, m) == 0) {
            if (n < cap) out[n] = (uint32_t)(hit - t);
            n++;
        }
        cur = hit + 1;
    }
    return n;
}

/* ---- dictionary: a byte trie walked from every text position ------------
 * Every (pattern id, offset) with text[offset..offset+len) == pattern[id] is an
 * occurrence (search.rs:259-282 with MatchKind::Standard overlapping iteration;
 * the reference's tests pin it to per-pattern find_all, search.rs:291-312 and
 * crates/oneline-gpu/src/tests.rs:754-802). Walking a plain trie from each
 * start position finds exactly that set; sorting by (pattern, offset) gives the
 * reference's order (search.rs:280, PatternHit derives Ord pattern-then-offset). */

typedef struct {
    uint32_t first_child, next_sibling, first_term;
    uint8_t byte;
} trie_node;

typedef struct {
    trie_node *nodes;
    uint32_t n, cap;
    uint32_t *term_next; /* per pattern: next pattern id ending at the same node */
} trie;

static uint32_t trie_new_node(trie *tr, uint8_t byte) {
    if (tr->n == tr->cap) {
        tr->cap = tr->cap ? tr->cap * 2 : 1024;
        tr->nodes = (trie_node *)realloc(tr->nodes, tr->cap * sizeof(trie_node));
    }
    trie_node *nd = &tr->nodes[tr->n];
    nd->first_child = OLO_NONE;
    nd->next_sibling = OLO_NONE;
    nd->first_term = OLO_NONE;
    nd->byte = byte;
    return tr->n++;
}

static uint32_t trie_child(const trie *tr, uint32_t node, uint8_t byte) {
    for (uint32_t c = tr->nodes[node].first_child; c != OLO_NONE; c = tr->nodes[c].next_sibling)
        if (tr->nodes[c].byte == byte) return c;
    return OLO_NONE;
}

/* pats: all patterns back to back; lens[i] their lengths. counts[n_pats] gets
 * per-pattern totals (may be NULL). Hits are written sorted by (pattern,
 * offset), at most cap of them; returns the total number of hits. */
uint64_t olo_find_many(const uint8_t *t, uint64_t len, const uint8_t *pats, const uint32_t *lens, uint32_t n_pats,
                       uint64_t *counts, uint32_t *hit_pat, uint32_t *hit_off, uint64_t cap) {
    trie tr = {0};
    tr.term_next = (uint32_t *)malloc((n_pats ? n_pats : 1) * sizeof(uint32_t));
    uint32_t root = trie_new_node(&tr, 0);
    uint64_t at = 0;
    /* Attach pattern ids in descending order so each node's list is ascending. */
    uint64_t *starts = (uint64_t *)malloc((n_pats ? n_pats : 1) * sizeof(uint64_t));
    for (uint32_t i = 0; i < n_pats; i++) {
        starts[i] = at;
        at += lens[i];
    }
    for (uint32_t ii = n_pats; ii-- > 0;) {
        tr.term_next[ii] = OLO_NONE;
        if (lens[ii] == 0) continue;
        uint32_t node = root;
        for (uint32_t k = 0; k < lens[ii]; k++) {
            uint8_t b = pats[starts[ii] + k];
            uint32_t c = trie_child(&tr, node, b);
            if (c == OLO_NONE) {
                c = trie_new_node(&tr, b);
                tr.nodes[c].next_sibling = tr.nodes[node].first_child;
                tr.nodes[node].first_child = c;
            }
            node = c;
        }
        tr.term_next[ii] = tr.nodes[node].first_term;
        tr.nodes[node].first_term = ii;
    }
    /* Count pass. */
    uint64_t *cnt = (uint64_t *)calloc(n_pats ? n_pats : 1, sizeof(uint64_t));
    for (uint64_t p = 0; p < len; p++) {
        uint32_t node = root;
        for (uint64_t q = p; q < len; q++) {
            node = trie_child(&tr, node, t[q]);
            if (node == OLO_NONE) break;
            for (uint32_t id = tr.nodes[node].first_term; id != OLO_NONE; id = tr.term_next[id]) cnt[id]++;
        }
    }
    uint64_t total = 0;
    uint64_t *base = (uint64_t *)malloc((n_pats ? n_pats : 1) * sizeof(uint64_t));
    for (uint32_t i = 0; i < n_pats; i++) {
        base[i] = total;
        total += cnt[i];
        if (counts) counts[i] = cnt[i];
    }
    /* Fill pass: positions ascend, so each pattern's bucket fills in offset order. */
    if (cap > 0 && total > 0) {
        uint64_t *fill = (uint64_t *)calloc(n_pats, sizeof(uint64_t));
        for (uint64_t p = 0; p < len; p++) {
            uint32_t node = root;
            for (uint64_t q = p; q < len; q++) {
                node = trie_child(&tr, node, t[q]);
                if (node == OLO_NONE) break;
                for (uint32_t id = tr.nodes[node].first_term; id != OLO_NONE; id = tr.term_next[id]) {
                    uint64_t slot = base[id] + fill[id]++;
                    if (slot < cap) {
                        hit_pat[slot] = id;
                        hit_off[slot] = (uint32_t)p;
                    }
                }
            }
        }
        free(fill);
    }
    free(base);
    free(cnt);
    free(starts);
    free(tr.term_next);
    free(tr.nodes);
    return total;
}
