/* Seeded synthetic oneline documents and pattern sets.
 *
 * Two families of generators live here:
 *
 *  1. The reference's own test-document generator, restated so that tests can
 *     use the same document shapes the reference's tests use:
 *       crates/oneline-core/src/datagen.rs:53-82   xorshift64* Rng
 *       crates/oneline-core/src/datagen.rs:110-122 prose_vocabulary()
 *       crates/oneline-core/src/datagen.rs:143-157 push_prefix / eol
 *       crates/oneline-core/src/datagen.rs:159-253 generate(profile, bytes, seed)
 *
 *  2. The benchmark-document generator for the parse+search workloads (new: the
 *     reference publishes no benchmark corpus). Per line: the depth does a +-1
 *     random walk clamped to 0..16 and is rendered as depth x '|' plus one space
 *     (oneline's depth is the number of '|' prefix bytes, crates/oneline-simd/
 *     src/line.rs:19-32; leading spaces would always give depth 0); 5% of lines
 *     are empty; of the rest 70% start with one of the six markers the classifier
 *     recognises ("=", ":", "@", "- ", "-. ", "//", crates/oneline-simd/src/
 *     line.rs:47-81) and 30% are plain text; payloads are printable ASCII with a
 *     geometric length of mean 40; LF endings; the document ends with '\n'.
 *
 * Everything is deterministic for a given seed on every machine: the only
 * floating point is IEEE double arithmetic plus log/exp/pow from libm, used the
 * same way each run.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- rng ---- */

typedef struct {
    uint64_t s;
} olg_rng;

/* Rng::new: seed * 0x9E3779B97F4A7C15 | 1 (datagen.rs:56-58). */
static void rng_init(olg_rng *r, uint64_t seed) { r->s = (seed * 0x9E3779B97F4A7C15ull) | 1ull; }

/* xorshift 12/25/27 then multiply (datagen.rs:60-67). */
static uint64_t rng_next(olg_rng *r) {
    uint64_t x = r->s;
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    r->s = x;
    return x * 0x2545F4914F6CDD1Dull;
}

/* below(n) = (next >> 11) % n (datagen.rs:70-72). */
static uint64_t rng_below(olg_rng *r, uint64_t n) { return (rng_next(r) >> 11) % n; }
static uint64_t rng_range(olg_rng *r, uint64_t lo, uint64_t hi) { return lo + rng_below(r, hi - lo); }
static int rng_chance(olg_rng *r, uint64_t percent) { return rng_below(r, 100) < percent; }
/* Uniform double in [0, 1) with 53 bits. */
static double rng_unit(olg_rng *r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }

/* Exposed so that Python code can draw from the very same stream. */
uint64_t olg_rng_seed_state(uint64_t seed) {
    olg_rng r;
    rng_init(&r, seed);
    return r.s;
}
uint64_t olg_rng_next(uint64_t *state) {
    olg_rng r = {*state};
    uint64_t v = rng_next(&r);
    *state = r.s;
    return v;
}

/* -------------------------------------------------------- byte buffer ---- */

typedef struct {
    uint8_t *p;
    uint64_t len, cap;
    int overflow;
} olg_buf;

static void put(olg_buf *b, const void *src, uint64_t n) {
    if (b->len + n > b->cap) {
        b->overflow = 1;
        n = b->cap > b->len ? b->cap - b->len : 0;
    }
    memcpy(b->p + b->len, src, n);
    b->len += n;
}
static void putc_(olg_buf *b, uint8_t c) { put(b, &c, 1); }
static void puts_(olg_buf *b, const char *s) { put(b, s, strlen(s)); }

/* --------------------------------------------- reference test documents -- */

enum { P_REPEAT = 0, P_SHORT = 1, P_MIXED = 2, P_LONG = 3, P_PROSE = 4, P_NESTED = 5 };

static const char *const WORDS[23] = {
    "lorem", "ipsum", "dolor", "sit", "amet", "parse", "line", "node",
    "depth", "tomet", "SIMD", "GPU",
    "\xe7\xb8\xa6\xe6\xa3\x92",             /* 縦棒 */
    "\xe9\x9a\x8e\xe5\xb1\xa4",             /* 階層 */
    "\xe6\xa7\x8b\xe6\x96\x87",             /* 構文 */
    "\xe8\xa7\xa3\xe6\x9e\x90",             /* 解析 */
    "na\xc3\xafve",                         /* naïve */
    "caf\xc3\xa9",                          /* café */
    "\xe3\x83\x87\xe3\x83\xbc\xe3\x82\xbf", /* データ */
    "|pipe|", "a", "of", "the"};

#define VOCAB_N 4096
static char g_vocab[VOCAB_N][11];
static uint8_t g_vocab_len[VOCAB_N];
static int g_vocab_ready = 0;

/* prose_vocabulary(): 4096 words of 2..=10 lowercase letters from Rng(0xC0FFEE). */
static void vocab_init(void) {
    if (g_vocab_ready) return;
    olg_rng r;
    rng_init(&r, 0xC0FFEEull);
    for (int i = 0; i < VOCAB_N; i++) {
        uint64_t len = rng_range(&r, 2, 11);
        for (uint64_t k = 0; k < len; k++) g_vocab[i][k] = (char)('a' + rng_below(&r, 26));
        g_vocab[i][len] = 0;
        g_vocab_len[i] = (uint8_t)len;
    }
    g_vocab_ready = 1;
}

/* Writes word `i` of the prose vocabulary into out (>= 11 bytes); returns its length. */
uint32_t olg_prose_word(uint32_t i, char *out) {
    vocab_init();
    memcpy(out, g_vocab[i % VOCAB_N], g_vocab_len[i % VOCAB_N] + 1);
    return g_vocab_len[i % VOCAB_N];
}

static void push_text(olg_buf *b, olg_rng *r, uint64_t target_len, int prose) {
    uint64_t start = b->len;
    while (b->len - start < target_len && !b->overflow) {
        if (b->len > start) putc_(b, ' ');
        if (prose) {
            double u = (double)rng_below(r, 1u << 20) / (double)(1u << 20);
            uint64_t idx = (uint64_t)((u * u * u) * (double)VOCAB_N) % VOCAB_N;
            put(b, g_vocab[idx], g_vocab_len[idx]);
        } else {
            puts_(b, WORDS[rng_below(r, 23)]);
        }
    }
}

static void push_prefix(olg_buf *b, uint32_t depth) {
    for (uint32_t i = 0; i < depth; i++) putc_(b, '|');
    if (depth > 0) putc_(b, ' ');
}

static void eol(olg_buf *b, olg_rng *r, uint64_t crlf_percent) {
    if (rng_chance(r, crlf_percent)) putc_(b, '\r');
    putc_(b, '\n');
}

/* generate(profile, target_bytes, seed) (datagen.rs:159-253). Writes into out
 * (capacity cap; target + 16 KiB is always enough) and returns the length, or
 * UINT64_MAX if cap was too small. */
uint64_t olg_generate_profile(int profile, uint64_t target, uint64_t seed, uint8_t *out, uint64_t cap) {
    olg_buf b = {out, 0, cap, 0};
    olg_rng r;
    rng_init(&r, seed);
    if (profile == P_REPEAT) {
        static const char *sample =
            "|=[ Header ]\n| Is this syntax necessary?\n||@card(title: \"x\")\n"
            "||:rule(allow:list(card))\n|| Content.\n|||- Item A\n|||- Item B\n";
        while (b.len < target && !b.overflow) puts_(&b, sample);
        return b.overflow ? UINT64_MAX : b.len;
    }
    int prose = profile == P_PROSE;
    if (prose) vocab_init();
    uint64_t until_heading = 0, section = 0;
    uint32_t depth = 1;
    while (b.len < target && !b.overflow) {
        uint64_t roll = rng_below(&r, 10);
        if (roll <= 1 && depth > 0) {
            depth -= 1;
        } else if (roll >= 2 && roll <= 3 && depth < 7) {
            depth += 1;
        } else if (roll == 4 && rng_chance(&r, 2)) {
            depth = (uint32_t)rng_below(&r, 3);
        }
        if (profile == P_NESTED) {
            if (until_heading == 0) {
                section += 1;
                char head[64];
                int n = 0;
                /* "=[ Section {section} ]" */
                char digits[24];
                int nd = 0;
                uint64_t s = section;
                do {
                    digits[nd++] = (char)('0' + s % 10);
                    s /= 10;
                } while (s);
                memcpy(head, "=[ Section ", 11);
                n = 11;
                while (nd) head[n++] = digits[--nd];
                head[n++] = ' ';
                head[n++] = ']';
                put(&b, head, (uint64_t)n);
                eol(&b, &r, 0);
                double u = (double)rng_below(&r, 1u << 20) / (double)(1u << 20);
                until_heading = (uint64_t)pow(10.0, 1.0 + 5.0 * u);
                continue;
            }
            until_heading -= 1;
            if (depth < 1) depth = 1;
        }
        uint64_t body;
        if (profile == P_SHORT) body = rng_range(&r, 4, 24);
        else if (profile == P_LONG) body = rng_range(&r, 200, 1500);
        else if (rng_chance(&r, 1)) body = rng_range(&r, 800, 4000);
        else body = rng_range(&r, 5, 120);
        uint64_t crlf = profile == P_MIXED ? 2 : 0;
        uint64_t kind = rng_below(&r, 100);
        if (kind <= 4) {
            if (rng_chance(&r, 30)) push_prefix(&b, depth);
        } else if (kind <= 9) {
            push_prefix(&b, depth);
            puts_(&b, "=[ ");
            push_text(&b, &r, body < 60 ? body : 60, prose);
            puts_(&b, " ]");
        } else if (kind <= 14) {
            push_prefix(&b, depth);
            puts_(&b, ":rule(");
            push_text(&b, &r, body < 60 ? body : 60, prose);
            puts_(&b, ")");
        } else if (kind <= 22) {
            push_prefix(&b, depth);
            puts_(&b, "@card(title: \"");
            push_text(&b, &r, body < 30 ? body : 30, prose);
            puts_(&b, "\")");
        } else if (kind <= 37) {
            push_prefix(&b, depth);
            if (rng_chance(&r, 70)) puts_(&b, "- ");
            else puts_(&b, "-. ");
            push_text(&b, &r, body, prose);
        } else {
            push_prefix(&b, depth);
            push_text(&b, &r, body, prose);
        }
        eol(&b, &r, crlf);
    }
    return b.overflow ? UINT64_MAX : b.len;
}

/* --------------------------------------------------- benchmark corpus ---- */

static const char *const MARKERS[6] = {"=", ":", "@", "- ", "-. ", "//"};

/* Geometric length with mean 40: P(k) = (1-q) q^k, q = 40/41, by inversion. */
static uint64_t geometric40(olg_rng *r) {
    double u = rng_unit(r);
    return (uint64_t)floor(log1p(-u) / log(40.0 / 41.0));
}

/* Printable ASCII 0x20..0x7E, four bytes per draw (16-bit chunks scaled to 95). */
static void printable(olg_buf *b, olg_rng *r, uint64_t n) {
    if (b->len + n > b->cap) {
        b->overflow = 1;
        n = b->cap - b->len;
    }
    uint8_t *dst = b->p + b->len;
    b->len += n;
    while (n > 0) {
        uint64_t x = rng_next(r);
        int k = n < 4 ? (int)n : 4;
        for (int i = 0; i < k; i++) {
            uint32_t c = (uint32_t)((x >> (16 * i)) & 0xFFFF);
            *dst++ = (uint8_t)(0x20 + ((c * 95u) >> 16));
        }
        n -= (uint64_t)k;
    }
}

/* Plain-text lines must not start with a blank, a '|' or a marker byte, so the
 * intended kind holds (the classifier still decides). */
static int plain_first_ok(uint8_t c) {
    return !(c == ' ' || c == '\t' || c == '|' || c == '=' || c == ':' || c == '@' || c == '-' || c == '/');
}

/* Exactly `target` bytes of benchmark document for `seed`; the last byte is '\n'.
 * Returns target, or UINT64_MAX when cap < target. */
uint64_t olg_generate_corpus(uint64_t target, uint64_t seed, uint8_t *out, uint64_t cap) {
    if (cap < target) return UINT64_MAX;
    /* Generate into the buffer with 8 KiB of slack beyond target, then cut. */
    uint8_t tail[8192];
    olg_buf b = {out, 0, target, 0};
    olg_rng r;
    rng_init(&r, seed);
    uint32_t depth = 0;
    while (b.len < target) {
        if (rng_below(&r, 2) == 0) {
            if (depth > 0) depth--;
        } else if (depth < 16) {
            depth++;
        }
        /* Lines are at most ~4.1 KiB: far from the end they are written in
         * place, near the end into a scratch buffer that is then clipped. */
        int direct = b.len + sizeof tail <= target;
        olg_buf line = direct ? (olg_buf){out + b.len, 0, sizeof tail, 0} : (olg_buf){tail, 0, sizeof tail, 0};
        if (rng_below(&r, 100) < 5) {
            putc_(&line, '\n');
        } else {
            push_prefix(&line, depth);
            uint64_t len = geometric40(&r);
            if (len > 4000) len = 4000;
            if (rng_below(&r, 100) < 70) {
                puts_(&line, MARKERS[rng_below(&r, 6)]);
                printable(&line, &r, len);
            } else {
                uint8_t c;
                do {
                    c = (uint8_t)(0x20 + rng_below(&r, 95));
                } while (!plain_first_ok(c));
                putc_(&line, c);
                printable(&line, &r, len);
            }
            putc_(&line, '\n');
        }
        if (direct) b.len += line.len;
        else put(&b, line.p, line.len); /* clipped at target */
    }
    out[target - 1] = '\n';
    return target;
}

/* Pattern set of a benchmark config, packed back to back into `pat_bytes` with
 * lengths in `lens`. `kind`:
 *   0: one 12-byte pattern sampled from the text (parse + one search)
 *   1: 8 patterns of 4..1024 B; even indices sampled from the text, odd
 *      indices random bytes 0x00..0xFF (parse + 8 searches)
 *   2: `n` patterns of U[4,64] B; 60% text substrings, 40% random printable
 *      ASCII (dictionary)
 * Returns the total number of bytes written, or UINT64_MAX on bad arguments. */
uint64_t olg_generate_patterns(int kind, const uint8_t *text, uint64_t text_len, uint64_t seed,
                               uint32_t n, uint8_t *pat_bytes, uint64_t cap, uint32_t *lens) {
    olg_rng r;
    rng_init(&r, seed ^ 0x5EED0F0A11CEull);
    static const uint32_t L1[8] = {4, 8, 16, 32, 64, 128, 256, 1024};
    uint64_t w = 0;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t len;
        int from_text;
        if (kind == 0) {
            len = 12;
            from_text = 1;
        } else if (kind == 1) {
            len = L1[i % 8];
            from_text = (i % 2) == 0;
        } else {
            len = (uint32_t)rng_range(&r, 4, 65);
            from_text = rng_below(&r, 100) < 60;
        }
        if (w + len > cap) return UINT64_MAX;
        if (from_text) {
            if (text_len < len) return UINT64_MAX;
            uint64_t at = rng_below(&r, text_len - len + 1);
            memcpy(pat_bytes + w, text + at, len);
        } else if (kind == 1) {
            for (uint32_t k = 0; k < len; k++) pat_bytes[w + k] = (uint8_t)(rng_next(&r) >> 56);
        } else {
            for (uint32_t k = 0; k < len; k++) pat_bytes[w + k] = (uint8_t)(0x20 + rng_below(&r, 95));
        }
        lens[i] = len;
        w += len;
    }
    return w;
}

/* Log-normal document sizes: median * exp(sigma * z), z ~ N(0,1) by Box-Muller,
 * clamped to [lo, hi]. */
void olg_lognormal_sizes(uint64_t seed, uint32_t n, double median, double sigma, uint64_t lo, uint64_t hi,
                         uint64_t *out) {
    olg_rng r;
    rng_init(&r, seed ^ 0x10C0A11ull);
    for (uint32_t i = 0; i < n; i++) {
        double u1 = rng_unit(&r), u2 = rng_unit(&r);
        if (u1 < 1e-300) u1 = 1e-300;
        double z = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
        double v = median * exp(sigma * z);
        uint64_t s = v < (double)lo ? lo : (v > (double)hi ? hi : (uint64_t)v);
        out[i] = s;
    }
}

/* Poisson arrival times (seconds) at `rate` per second: exponential gaps. */
void olg_poisson_arrivals(uint64_t seed, uint32_t n, double rate, double *out) {
    olg_rng r;
    rng_init(&r, seed ^ 0xA441A1ull);
    double t = 0.0;
    for (uint32_t i = 0; i < n; i++) {
        double u = rng_unit(&r);
        t += -log1p(-u) / rate;
        out[i] = t;
    }
}
