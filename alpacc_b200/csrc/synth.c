/*
 * Seeded synthetic inputs for the benchmark grammars (host code, gcc).
 *
 *   alp_synth_json   -- JSON documents for json.alp: values are object 25% /
 *                       array 20% / string 25% / number 20% / true,false,null
 *                       10%; 0-12 members per container; strings of
 *                       geometric length (mean 12) of printable ASCII with 2%
 *                       escapes and 1% UTF-8 multibyte characters; numbers are
 *                       an optional '-', 1-6 digits and an optional fraction
 *                       (json.alp has no exponent); 0-3 whitespace bytes
 *                       between tokens.  A string never ends its content with
 *                       a backslash: json.alp reads backslash-quote as part of
 *                       the string, so such a string would not close.
 *   alp_synth_arith  -- arithmetic.alp expressions by random derivation.
 *   alp_synth_sexp   -- sexp.alp lists of atoms (1-10 alphanumerics).
 *
 * Every generator writes exactly `target` bytes (trailing whitespace pads a
 * document that closed early) and is deterministic in `seed`.
 */
#include <stdint.h>
#include <string.h>

typedef struct { uint64_t s[4]; } rng_t;

static uint64_t splitmix(uint64_t *x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static void rng_seed(rng_t *r, uint64_t seed) {
    for (int i = 0; i < 4; ++i) r->s[i] = splitmix(&seed);
}
static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static inline uint64_t rnext(rng_t *r) { /* xoshiro256** */
    uint64_t *s = r->s, res = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45);
    return res;
}
static inline uint32_t rint_(rng_t *r, uint32_t n) { return (uint32_t)(((rnext(r) >> 32) * (uint64_t)n) >> 32); }
static inline double runif(rng_t *r) { return (double)(rnext(r) >> 11) * (1.0 / 9007199254740992.0); }

typedef struct { uint8_t *p; int64_t n, cap; } buf_t;
static inline void put(buf_t *b, uint8_t c) { if (b->n < b->cap) b->p[b->n] = c; b->n++; }
static inline void puts_(buf_t *b, const char *s) { while (*s) put(b, (uint8_t)*s++); }

static const char WS[4] = {' ', '\n', '\t', '\r'};
static void ws03(buf_t *b, rng_t *r) { uint32_t k = rint_(r, 4); for (uint32_t i = 0; i < k; ++i) put(b, (uint8_t)WS[rint_(r, 4)]); }

static void json_string(buf_t *b, rng_t *r, uint32_t max_len) {
    put(b, '"');
    uint32_t len = 0;
    while (runif(r) >= 1.0 / 13.0 && len < max_len) ++len; /* geometric, mean 12 */
    int last_bs = 0;
    for (uint32_t i = 0; i < len; ++i) {
        double u = runif(r);
        last_bs = 0;
        if (u < 0.02) {
            static const char esc[6] = {'"', '\\', '/', 'n', 't', 'u'};
            char e = esc[rint_(r, 6)];
            put(b, '\\');
            if (e == 'u') { puts_(b, "u00e9"); }
            else { put(b, (uint8_t)e); last_bs = (e == '\\'); }
        } else if (u < 0.03) {
            if (rint_(r, 2)) { put(b, 0xC3); put(b, (uint8_t)(0xA0 + rint_(r, 16))); }
            else { put(b, 0xE2); put(b, 0x82); put(b, 0xAC); }
        } else {
            uint8_t c;
            do { c = (uint8_t)(0x20 + rint_(r, 95)); } while (c == '"' || c == '\\');
            put(b, c);
        }
    }
    if (last_bs) put(b, 'x');
    put(b, '"');
}

static void json_number(buf_t *b, rng_t *r) {
    if (rint_(r, 10) < 3) put(b, '-');
    uint32_t d = 1 + rint_(r, 6);
    put(b, (uint8_t)(d == 1 ? '0' + rint_(r, 10) : '1' + rint_(r, 9)));
    for (uint32_t i = 1; i < d; ++i) put(b, (uint8_t)('0' + rint_(r, 10)));
    if (rint_(r, 10) < 4) {
        put(b, '.');
        uint32_t f = 1 + rint_(r, 6);
        for (uint32_t i = 0; i < f; ++i) put(b, (uint8_t)('0' + rint_(r, 10)));
    }
}

typedef struct { uint8_t obj; int32_t left; uint8_t first; } frame_t;

/* One JSON document of exactly `target` bytes.  The root is an array (or an
 * object when root_obj) that keeps taking members while the remaining room
 * can hold one more member plus the closing brackets of every open container;
 * string lengths are capped by that room, so nothing is ever cut. */
static int64_t json_doc(rng_t *r, uint8_t *out, int64_t target, int max_depth, int root_obj) {
    if (target < 2) target = 2;
    buf_t b = {out, 0, target};
    frame_t st[64];
    if (max_depth > 60) max_depth = 60;
    if (max_depth < 1) max_depth = 1;
    int sp = 0;
    put(&b, root_obj ? '{' : '[');
    st[sp].obj = (uint8_t)root_obj; st[sp].left = 0x7fffffff; st[sp].first = 1; ++sp;
    while (sp > 0) {
        frame_t *f = &st[sp - 1];
        int64_t room = target - b.n - 4 * (int64_t)sp - 8;
        if (f->left == 0 || room < 64) {
            put(&b, f->obj ? '}' : ']');
            --sp;
            if (sp > 0 && target - b.n - 4 * (int64_t)sp > 3) ws03(&b, r);
            continue;
        }
        int64_t ml = (room - 40) / 12;
        uint32_t max_len = ml > 200 ? 200 : (uint32_t)ml;
        if (!f->first) { put(&b, ','); ws03(&b, r); }
        else ws03(&b, r);
        f->first = 0;
        f->left--;
        if (f->obj) { json_string(&b, r, max_len); ws03(&b, r); put(&b, ':'); ws03(&b, r); }
        uint32_t u = rint_(r, 100);
        int depth = sp; /* containers open above this value */
        if (u < 45 && depth < max_depth) {
            int obj = u < 25;
            put(&b, obj ? '{' : '[');
            st[sp].obj = (uint8_t)obj; st[sp].left = (int32_t)rint_(r, 13); st[sp].first = 1; ++sp;
            continue;
        }
        if (u < 45) u = 45 + rint_(r, 55); /* at the depth limit: a scalar */
        if (u < 70) json_string(&b, r, max_len);
        else if (u < 90) json_number(&b, r);
        else { uint32_t k = rint_(r, 3); puts_(&b, k == 0 ? "true" : (k == 1 ? "false" : "null")); }
        ws03(&b, r);
    }
    while (b.n < target) put(&b, ' ');
    return b.n;
}

int64_t alp_synth_json(uint64_t seed, int64_t target, int max_depth, uint8_t *out) {
    rng_t r;
    rng_seed(&r, seed);
    return json_doc(&r, out, target, max_depth, 0);
}

/* Many documents back to back: sizes[i] bytes each, offsets written to
 * off[0..n] (off[0] = 0).  Roots alternate between arrays and objects. */
int64_t alp_synth_json_batch(uint64_t seed, const int64_t *sizes, int64_t n, int max_depth, uint8_t *out,
                             int64_t *off) {
    rng_t r;
    rng_seed(&r, seed);
    int64_t p = 0;
    off[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t t = sizes[i] < 2 ? 2 : sizes[i];
        json_doc(&r, out + p, t, max_depth, (int)(rnext(&r) & 1));
        p += t;
        off[i + 1] = p;
    }
    return p;
}

/* ------------------------------------------------------------- arithmetic -- */

static void ar_ws(buf_t *b, rng_t *r) { if (rint_(r, 10) == 0) put(b, (uint8_t)WS[rint_(r, 3)]); }

/* pending: a binary '-' was just written, so a digit must not follow it */
static void ar_num(buf_t *b, rng_t *r, int *pending) {
    int neg = rint_(r, 4) == 0;
    if (*pending && !neg) put(b, ' ');
    *pending = 0;
    if (neg) put(b, '-');
    uint32_t d = 1 + rint_(r, 6);
    put(b, (uint8_t)(d == 1 ? '0' + rint_(r, 10) : '1' + rint_(r, 9)));
    for (uint32_t i = 1; i < d; ++i) put(b, (uint8_t)('0' + rint_(r, 10)));
}
static void ar_var(buf_t *b, rng_t *r, int *pending) {
    *pending = 0;
    uint32_t d = 1 + rint_(r, 8);
    for (uint32_t i = 0; i < d; ++i) put(b, (uint8_t)('a' + rint_(r, 26)));
}
static void ar_e0(buf_t *b, rng_t *r, int depth, int max_depth, int *pending);
static void ar_e2(buf_t *b, rng_t *r, int depth, int max_depth, int *pending) {
    if (depth < max_depth && runif(r) < 0.2) {
        *pending = 0;
        put(b, '(');
        ar_ws(b, r);
        ar_e0(b, r, depth + 1, max_depth, pending);
        put(b, ')');
    } else if (rint_(r, 2)) ar_num(b, r, pending);
    else ar_var(b, r, pending);
    ar_ws(b, r);
}
static void ar_e1(buf_t *b, rng_t *r, int depth, int max_depth, int *pending) {
    ar_e2(b, r, depth, max_depth, pending);
    uint32_t k = rint_(r, 3);
    for (uint32_t i = 0; i < k; ++i) {
        put(b, rint_(r, 2) ? '*' : '/');
        *pending = 0;
        ar_ws(b, r);
        ar_e2(b, r, depth, max_depth, pending);
    }
}
static void ar_e0(buf_t *b, rng_t *r, int depth, int max_depth, int *pending) {
    ar_e1(b, r, depth, max_depth, pending);
    uint32_t k = rint_(r, 3);
    for (uint32_t i = 0; i < k; ++i) {
        if (rint_(r, 2)) { put(b, '+'); *pending = 0; }
        else { put(b, '-'); *pending = 1; }
        if (rint_(r, 10) == 0) { put(b, ' '); *pending = 0; }
        ar_e1(b, r, depth, max_depth, pending);
    }
}

/* Whole top-level expressions joined by '+' until `target` is nearly reached;
 * trailing whitespace pads to exactly `target` bytes. */
int64_t alp_synth_arith(uint64_t seed, int64_t target, int max_depth, uint8_t *out) {
    rng_t r;
    rng_seed(&r, seed);
    buf_t b = {out, 0, target};
    if (target < 1) return 0;
    int pending = 0;
    int64_t guard = 1 << 16;
    if (target < guard + 16) guard = target / 2;
    int first = 1;
    while (first || b.n < target - guard) {
        int64_t save = b.n;
        if (!first) { put(&b, '+'); pending = 0; }
        ar_e0(&b, &r, 0, max_depth, &pending);
        if (b.n > target) { b.n = save; break; }
        first = 0;
    }
    if (b.n == 0) put(&b, (uint8_t)('0' + rint_(&r, 10)));  /* nothing fitted: one digit */
    while (b.n < target) put(&b, ' ');
    return b.n;
}

/* ------------------------------------------------------------------- sexp -- */

static void sx_atom(buf_t *b, rng_t *r) {
    static const char AL[] = "abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789";
    uint32_t d = 1 + rint_(r, 10);
    for (uint32_t i = 0; i < d; ++i) put(b, (uint8_t)AL[rint_(r, 62)]);
}
static void sx_ws(buf_t *b, rng_t *r) { uint32_t k = 1 + rint_(r, 2); for (uint32_t i = 0; i < k; ++i) put(b, (uint8_t)WS[rint_(r, 4)]); }

static int64_t sexp_doc(rng_t *r, uint8_t *out, int64_t target, int max_depth) {
    if (target < 2) target = 2;
    buf_t b = {out, 0, target};
    int32_t left[64];
    if (max_depth > 60) max_depth = 60;
    int sp = 0;
    int64_t reserve = 2 * 64 + 64;
    if (target < reserve + 4) {
        put(&b, '(');
        while (b.n + 12 < target) { sx_atom(&b, r); put(&b, ' '); }
        put(&b, ')');
        while (b.n < target) put(&b, ' ');
        return target;
    }
    put(&b, '(');
    left[sp++] = 0x7fffffff;
    while (sp > 0) {
        if (left[sp - 1] == 0 || b.n > target - reserve) {
            put(&b, ')');
            --sp;
            if (sp > 0) sx_ws(&b, r);
            continue;
        }
        left[sp - 1]--;
        if (sp < max_depth && rint_(r, 10) < 3) {
            put(&b, '(');
            left[sp++] = (int32_t)rint_(r, 9);
            continue;
        }
        sx_atom(&b, r);
        sx_ws(&b, r);
    }
    while (b.n < target) put(&b, ' ');
    return b.n;
}

int64_t alp_synth_sexp(uint64_t seed, int64_t target, int max_depth, uint8_t *out) {
    rng_t r;
    rng_seed(&r, seed);
    return sexp_doc(&r, out, target, max_depth);
}

int64_t alp_synth_sexp_batch(uint64_t seed, const int64_t *sizes, int64_t n, int max_depth, uint8_t *out,
                             int64_t *off) {
    rng_t r;
    rng_seed(&r, seed);
    int64_t p = 0;
    off[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        int64_t t = sizes[i] < 2 ? 2 : sizes[i];
        sexp_doc(&r, out + p, t, max_depth);
        p += t;
        off[i + 1] = p;
    }
    return p;
}
