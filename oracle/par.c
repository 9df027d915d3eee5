/*
 * Data-parallel CPU restatement of the reference's generated lexer and
 * parser, for one document on all host cores (OpenMP).
 *
 * TEST INFRASTRUCTURE ONLY: it is the timed CPU baseline of the benchmark
 * (the reference's own CPU path is Futhark `multicore` output of a Haskell
 * generator, neither of which exists on these machines) and is checked
 * against the sequential oracle (oracle.c) by the tests.  The product path
 * never calls it.
 *
 * It follows the data-parallel formulation of the templates, with each
 * parallel map/scan/scatter cut into one block of elements per task:
 *
 *   lexer  (futhark/lexer.fut:67-172)
 *     fold         map bytes to endomorphisms and reduce each block with the
 *                  composition (lines 67-81: `compose`, `trans_to_state`)
 *     (serial)     exclusive scan of the block endomorphisms with the same
 *                  composition table, applied to the initial state
 *     count        per block: produce flags and the ignore filter
 *                  (lines 103-107) counted, last kept start (take_right,
 *                  lines 83-84, 112-120)
 *     (serial)     exclusive scan of (count, last start)
 *     emit         the compaction scatter (lines 108-133)
 *   parser (futhark/parser.fut:110-332)
 *     pairs        keys over ⊢ tokens ⊣ (get_key, lines 117-122, 235-240) and
 *                  the pair lookup (lines 130-148), summed per block
 *     (serial)     exclusive scan of the block sums (stack and production
 *                  offsets, depth, exscan(arity - 1), terminal count)
 *     expand       segmented copies of brackets and productions (lines
 *                  216-233) with depth values and exscan(arity - 1) values
 *     prev_leq     "previous smaller-or-equal" (find_previous over a min tree,
 *                  lines 72-108) for bracket matching (lines 153-184) and
 *                  parents (lines 286-298): a stack per block, then the
 *                  elements no block-local answer serves search the earlier
 *                  blocks' remaining stacks (ascending values: binary search)
 *     terminals    the k-th terminal production takes the k-th token's span
 *                  (lines 305-332)
 *
 * Tables derived once per context from the reference tables: the pair lookup
 * indexes a direct table over the key space (the template probes an FNV-1a
 * open-addressing table; both give each key's pair or a miss), and each DFA
 * transition carries its produce flag and the ignore filter of the states on
 * both sides.  The byte passes run two blocks per task in lockstep, so that
 * two independent table chains are in flight on each core.
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define NONE64 INT64_MIN

/* transition entry: next state | a kept token ends before this byte (the
 * state left is not ignore) | a kept token starts here (the state entered is
 * not ignore); both only on produce transitions */
#define E_NEXT 0xffffu
#define E_END (1u << 16)
#define E_START (1u << 17)

/* Buffers grow and are kept from call to call (the outputs of a call stay
 * valid until the next call on the context), as the GPU library keeps its
 * scratch and outputs: steady-state calls touch no fresh pages. */
enum { B_TERM, B_TSTART, B_TEND, B_BF, B_BS, B_BC, B_BL, B_PAIR, B_BSUM, B_BR, B_DS, B_VV, B_PARENT, B_TAG, B_KIND,
       B_NST, B_NEN, B_PV, B_STK, B_LEN, B_COUNT };

typedef struct {
    const orc_tables *t;
    uint32_t *ent;       /* [S][256] */
    uint16_t *key_index; /* [T^(q+k)] pair id + 1, 0 = no pair */
    int64_t key_space;
    uint32_t T;
    int threads;
    void *buf[B_COUNT];
    size_t cap[B_COUNT];
} par_ctx;

static void *need(par_ctx *c, int i, size_t bytes) {
    if (bytes < 64) bytes = 64;
    if (c->cap[i] < bytes) {
        free(c->buf[i]);
        c->buf[i] = malloc(bytes);
        c->cap[i] = c->buf[i] ? bytes : 0;
    }
    return c->buf[i];
}

void par_free(par_ctx *c) {
    if (c) {
        for (int i = 0; i < B_COUNT; ++i) free(c->buf[i]);
        free(c->ent);
        free(c->key_index);
        free(c);
    }
}

par_ctx *par_create(const orc_tables *t, int threads) {
    par_ctx *c = (par_ctx *)calloc(1, sizeof(par_ctx));
    if (!c) return NULL;
    c->t = t;
    c->threads = threads > 0 ? threads : omp_get_max_threads();
    if (t->has_lexer) {
        c->ent = (uint32_t *)malloc((size_t)t->S * 256 * 4);
        if (!c->ent) { par_free(c); return NULL; }
        for (uint32_t st = 0; st < t->S; ++st)
            for (uint32_t b = 0; b < 256; ++b) {
                const uint32_t nx = orc_nxt(t, st, (uint8_t)b);
                uint32_t e = nx;
                if (orc_prod(t, st, (uint8_t)b)) {
                    if (!orc_is_ignore(t, t->token[st])) e |= E_END;
                    if (!orc_is_ignore(t, t->token[nx])) e |= E_START;
                }
                c->ent[(size_t)st * 256 + b] = e;
            }
    }
    if (t->has_parser) {
        uint32_t T = t->n_term_syms, W = t->q + t->k;
        int64_t space = 1;
        for (uint32_t j = 0; j < W; ++j) {
            space *= T;
            if (space > (1ll << 26)) { par_free(c); return NULL; }
        }
        c->T = T;
        c->key_space = space;
        c->key_index = (uint16_t *)calloc((size_t)space, 2);
        if (!c->key_index) { par_free(c); return NULL; }
        for (uint32_t i = 0; i < t->n_keys; ++i) {
            int64_t x = 0;
            for (uint32_t j = 0; j < W; ++j) x = x * T + t->keys[(size_t)i * W + j];
            c->key_index[x] = (uint16_t)(t->key_pair[i] + 1);
        }
    }
    return c;
}

int par_threads(const par_ctx *c) { return c->threads; }

/* Blocks: a multiple of 16 per thread, at least min_block elements each, even. */
static int64_t nblocks(const par_ctx *c, int64_t n, int64_t min_block) {
    int64_t b = (int64_t)c->threads * 16;
    if (n / b < min_block) b = n / min_block;
    if (b < 2) b = 2;
    return b + (b & 1);
}

/* ------------------------------------------------------------------ lexer */

typedef struct {
    uint32_t st;       /* DFA state */
    int64_t cnt, last; /* tokens ended, last kept start */
} lexrun;

static inline void count_byte(const uint32_t *ent, lexrun *r, const uint8_t *s, int64_t j) {
    const uint32_t e = ent[(size_t)r->st * 256 + s[j]];
    if ((e & E_END) && j >= 1) ++r->cnt;
    if (e & E_START) r->last = j;
    r->st = e & E_NEXT;
}

typedef struct {
    uint32_t st;
    int64_t k, cur; /* next slot, start of the token in progress */
} emitrun;

static inline void emit_byte(const orc_tables *t, const uint32_t *ent, emitrun *r, const uint8_t *s, int64_t j,
                             uint32_t *term, int64_t *start, int64_t *end) {
    const uint32_t e = ent[(size_t)r->st * 256 + s[j]];
    if ((e & E_END) && j >= 1) {
        term[r->k] = t->token[r->st];
        start[r->k] = r->cur;
        end[r->k] = j;
        ++r->k;
    }
    if (e & E_START) r->cur = j;
    r->st = e & E_NEXT;
}

/* Lex one document into the context's token buffers (valid until the next
 * call).  Returns 1 accepted, 0 rejected (no tokens). */
int par_lex(par_ctx *c, const uint8_t *s, int64_t n, uint32_t **o_term, int64_t **o_start, int64_t **o_end,
            int64_t *ntok) {
    const orc_tables *t = c->t;
    const uint32_t *ent = c->ent;
    *ntok = 0;
    *o_term = NULL; *o_start = NULL; *o_end = NULL;
    if (n == 0) return t->accept[INIT_STATE] ? 1 : 0;
    const int64_t B = nblocks(c, n, 1 << 16);
    const uint32_t C1 = t->C + 1, S = t->S;
    uint16_t *bf = (uint16_t *)need(c, B_BF, B * sizeof(uint16_t));    /* block endomorphism */
    uint32_t *bs = (uint32_t *)need(c, B_BS, B * sizeof(uint32_t));    /* state entering the block */
    int64_t *bc = (int64_t *)need(c, B_BC, (B + 1) * sizeof(int64_t)); /* token ends in the block, then before it */
    int64_t *bl = (int64_t *)need(c, B_BL, (B + 1) * sizeof(int64_t)); /* last kept start in / before the block */
    if (!bf || !bs || !bc || !bl) return -1;
    /* map + per-block reduce with the composition (endo 0 is the identity) */
#pragma omp parallel for schedule(static) num_threads(c->threads)
    for (int64_t h = 0; h < B / 2; ++h) {
        const int64_t a0 = n * (2 * h) / B, a1 = n * (2 * h + 1) / B, a2 = n * (2 * h + 2) / B;
        const int64_t len = (a1 - a0) < (a2 - a1) ? (a1 - a0) : (a2 - a1);
        uint32_t f = 0, g = 0;
        for (int64_t i = 0; i < len; ++i) {
            f = t->endo_step[(size_t)f * C1 + t->cls[s[a0 + i]]];
            g = t->endo_step[(size_t)g * C1 + t->cls[s[a1 + i]]];
        }
        for (int64_t j = a0 + len; j < a1; ++j) f = t->endo_step[(size_t)f * C1 + t->cls[s[j]]];
        for (int64_t j = a1 + len; j < a2; ++j) g = t->endo_step[(size_t)g * C1 + t->cls[s[j]]];
        bf[2 * h] = (uint16_t)f;
        bf[2 * h + 1] = (uint16_t)g;
    }
    /* exclusive scan of the block endomorphisms, applied to the initial state */
    uint32_t pre = 0;
    for (int64_t b = 0; b < B; ++b) {
        bs[b] = t->endo_app[(size_t)pre * S + INIT_STATE];
        pre = t->endo_comp[(size_t)pre * t->E + bf[b]];
    }
    const uint32_t final_state = t->endo_app[(size_t)pre * S + INIT_STATE];
    if (!t->accept[final_state]) return 0;
    /* token ends (a flag at byte j >= 1 closes the token that ends at j) and
     * the last kept token start of each block */
#pragma omp parallel for schedule(static) num_threads(c->threads)
    for (int64_t h = 0; h < B / 2; ++h) {
        const int64_t a0 = n * (2 * h) / B, a1 = n * (2 * h + 1) / B, a2 = n * (2 * h + 2) / B;
        const int64_t len = (a1 - a0) < (a2 - a1) ? (a1 - a0) : (a2 - a1);
        lexrun x = {bs[2 * h], 0, NONE64}, y = {bs[2 * h + 1], 0, NONE64};
        for (int64_t i = 0; i < len; ++i) {
            count_byte(ent, &x, s, a0 + i);
            count_byte(ent, &y, s, a1 + i);
        }
        for (int64_t j = a0 + len; j < a1; ++j) count_byte(ent, &x, s, j);
        for (int64_t j = a1 + len; j < a2; ++j) count_byte(ent, &y, s, j);
        bc[2 * h] = x.cnt;
        bl[2 * h] = x.last;
        bc[2 * h + 1] = y.cnt;
        bl[2 * h + 1] = y.last;
    }
    /* exclusive scan of (count, last start) */
    int64_t total = 0, lastall = NONE64;
    for (int64_t b = 0; b < B; ++b) {
        const int64_t cb = bc[b], lb = bl[b];
        bc[b] = total;
        bl[b] = lastall;
        total += cb;
        if (lb != NONE64) lastall = lb;
    }
    const uint32_t lt = t->token[final_state];
    const int64_t m = total + (orc_is_ignore(t, lt) ? 0 : 1);
    uint32_t *term = (uint32_t *)need(c, B_TERM, (m + 1) * sizeof(uint32_t));
    int64_t *start = (int64_t *)need(c, B_TSTART, (m + 1) * sizeof(int64_t));
    int64_t *end = (int64_t *)need(c, B_TEND, (m + 1) * sizeof(int64_t));
    if (!term || !start || !end) return -1;
    /* scatter every token into its slot */
#pragma omp parallel for schedule(static) num_threads(c->threads)
    for (int64_t h = 0; h < B / 2; ++h) {
        const int64_t a0 = n * (2 * h) / B, a1 = n * (2 * h + 1) / B, a2 = n * (2 * h + 2) / B;
        const int64_t len = (a1 - a0) < (a2 - a1) ? (a1 - a0) : (a2 - a1);
        emitrun x = {bs[2 * h], bc[2 * h], bl[2 * h] == NONE64 ? 0 : bl[2 * h]};
        emitrun y = {bs[2 * h + 1], bc[2 * h + 1], bl[2 * h + 1] == NONE64 ? 0 : bl[2 * h + 1]};
        for (int64_t i = 0; i < len; ++i) {
            emit_byte(t, ent, &x, s, a0 + i, term, start, end);
            emit_byte(t, ent, &y, s, a1 + i, term, start, end);
        }
        for (int64_t j = a0 + len; j < a1; ++j) emit_byte(t, ent, &x, s, j, term, start, end);
        for (int64_t j = a1 + len; j < a2; ++j) emit_byte(t, ent, &y, s, j, term, start, end);
    }
    if (m > total) {
        term[total] = lt;
        start[total] = lastall == NONE64 ? 0 : lastall;
        end[total] = n;
    }
    *o_term = term; *o_start = start; *o_end = end;
    *ntok = m;
    return 1;
}

/* ------------------------------------------------ previous smaller-or-equal */

/* out[i] = largest j < i with v[j] <= v[i], or -1.  A stack per block; the
 * block's final stack (ascending values, kept in `stk` at the block's start)
 * answers the later blocks' elements that found nothing in their own block. */
static int par_prev_leq(par_ctx *c, const int32_t *v, int64_t n, int64_t *out) {
    if (n == 0) return 0;
    const int64_t B = nblocks(c, n, 1 << 14);
    uint32_t *stk = (uint32_t *)need(c, B_STK, n * sizeof(uint32_t));
    int64_t *len = (int64_t *)need(c, B_LEN, B * sizeof(int64_t));
    if (!stk || !len) return -1;
#pragma omp parallel for schedule(static) num_threads(c->threads)
    for (int64_t b = 0; b < B; ++b) {
        const int64_t lo = n * b / B, hi = n * (b + 1) / B;
        uint32_t *sk = stk + lo;
        int64_t top = 0;
        for (int64_t i = lo; i < hi; ++i) {
            while (top > 0 && v[sk[top - 1]] > v[i]) --top;
            out[i] = top > 0 ? (int64_t)sk[top - 1] : -1;
            sk[top++] = (uint32_t)i;
        }
        len[b] = top;
    }
#pragma omp parallel for schedule(dynamic, 4) num_threads(c->threads)
    for (int64_t b = 1; b < B; ++b) {
        const int64_t lo = n * b / B, hi = n * (b + 1) / B;
        for (int64_t i = lo; i < hi; ++i) {
            if (out[i] >= 0) continue;
            const int32_t x = v[i];
            for (int64_t u = b - 1; u >= 0; --u) {
                const uint32_t *sk = stk + n * u / B;
                if (len[u] == 0 || v[sk[0]] > x) continue;
                int64_t a = 0, z = len[u] - 1; /* last k with v[sk[k]] <= x */
                while (a < z) {
                    const int64_t mid = (a + z + 1) >> 1;
                    if (v[sk[mid]] <= x) a = mid; else z = mid - 1;
                }
                out[i] = sk[a];
                break;
            }
        }
    }
    return 0;
}

/* ----------------------------------------------------------------- parser */

typedef struct {
    int64_t nb, np, nt;   /* brackets, productions, terminal productions */
    int64_t depth, mind;  /* depth change; least depth reached inside, relative */
    int64_t v;            /* sum of (arity - 1) */
    int64_t miss;         /* keys without a pair */
} psum;

static inline uint32_t pos_sym(const orc_tables *t, const uint32_t *ters, int64_t n, int64_t x) {
    if (x < 0 || x >= n) return t->empty;
    if (x == 0) return t->start;
    if (x == n - 1) return t->end;
    return ters[x - 1];
}

/* parse_int over a token array (futhark/parser.fut:286-332) into the
 * context's node buffers (valid until the next call).  Returns 1 valid,
 * 0 rejected, -1 out of memory. */
int par_parse(par_ctx *c, const uint32_t *ters, const int64_t *tstart, const int64_t *tend, int64_t m,
              int64_t **o_parent, uint32_t **o_tag, uint8_t **o_kind, int64_t **o_start, int64_t **o_end,
              int64_t *nnode) {
    const orc_tables *t = c->t;
    *nnode = 0;
    *o_parent = NULL; *o_tag = NULL; *o_kind = NULL; *o_start = NULL; *o_end = NULL;
    const int64_t n = m + 2;
    const uint32_t W = t->q + t->k, T = c->T;
    const int64_t B = nblocks(c, n, 1 << 14);
    uint16_t *pair = (uint16_t *)need(c, B_PAIR, n * sizeof(uint16_t));
    psum *bsum = (psum *)need(c, B_BSUM, (B + 1) * sizeof(psum));
    if (!pair || !bsum) return -1;
    /* keys, lookup, block sums */
#pragma omp parallel for schedule(static) num_threads(c->threads)
    for (int64_t b = 0; b < B; ++b) {
        const int64_t lo = n * b / B, hi = n * (b + 1) / B;
        psum a = {0, 0, 0, 0, 0, 0, 0};
        for (int64_t i = lo; i < hi; ++i) {
            int64_t x = 0;
            for (uint32_t j = 0; j < W; ++j) x = x * T + pos_sym(t, ters, n, i + (int64_t)j - (int64_t)t->q);
            const uint32_t p = c->key_index[x];
            if (!p) { a.miss = 1; pair[i] = 0; continue; }
            pair[i] = (uint16_t)(p - 1);
            const uint32_t *pp = t->pairs + 4 * (size_t)(p - 1);
            for (uint32_t j = pp[0]; j < pp[1]; ++j) {
                a.depth += (t->stack[j] >> 31) ? 1 : -1;
                if (a.depth < a.mind) a.mind = a.depth;
            }
            a.nb += pp[1] - pp[0];
            for (uint32_t j = pp[2]; j < pp[3]; ++j) {
                a.v += (int64_t)t->arity[t->pseq[j]] - 1;
                if (t->prod_term[t->pseq[j]] >= 0) ++a.nt;
            }
            a.np += pp[3] - pp[2];
        }
        bsum[b] = a;
    }
    /* exclusive scan of the block sums; depth never below zero, zero at the end */
    int ok = 1;
    psum tot = {0, 0, 0, 0, 0, 0, 0};
    for (int64_t b = 0; b < B; ++b) {
        const psum a = bsum[b];
        if (a.miss || tot.depth + a.mind < 0) ok = 0;
        bsum[b] = tot;
        tot.nb += a.nb; tot.np += a.np; tot.nt += a.nt; tot.depth += a.depth; tot.v += a.v;
    }
    if (tot.nb != 0 && tot.depth != 0) ok = 0;
    if (!ok) return 0;
    const int64_t NB = tot.nb, NP = tot.np;
    uint32_t *br = (uint32_t *)need(c, B_BR, (NB + 1) * sizeof(uint32_t));
    int32_t *ds = (int32_t *)need(c, B_DS, (NB + 1) * sizeof(int32_t));
    int32_t *vv = (int32_t *)need(c, B_VV, (NP + 1) * sizeof(int32_t));
    int64_t *parent = (int64_t *)need(c, B_PARENT, (NP + 1) * sizeof(int64_t));
    uint32_t *tag = (uint32_t *)need(c, B_TAG, (NP + 1) * sizeof(uint32_t));
    uint8_t *kind = (uint8_t *)need(c, B_KIND, NP + 1);
    int64_t *nst = (int64_t *)need(c, B_NST, (NP + 1) * sizeof(int64_t));
    int64_t *nen = (int64_t *)need(c, B_NEN, (NP + 1) * sizeof(int64_t));
    int64_t *pv = (int64_t *)need(c, B_PV, (NB + 1) * sizeof(int64_t));
    if (!br || !ds || !vv || !parent || !tag || !kind || !nst || !nen || !pv) return -1;
    const int subst = tot.nt == m; /* futhark/parser.fut:305-332 */
    /* segmented copies: brackets with their depth values, productions with
     * exscan(arity - 1), terminal productions with their token's span */
#pragma omp parallel for schedule(static) num_threads(c->threads)
    for (int64_t b = 0; b < B; ++b) {
        const int64_t lo = n * b / B, hi = n * (b + 1) / B;
        int64_t ob = bsum[b].nb, op = bsum[b].np, kk = bsum[b].nt, dep = bsum[b].depth, v = bsum[b].v;
        for (int64_t i = lo; i < hi; ++i) {
            const uint32_t *pp = t->pairs + 4 * (size_t)pair[i];
            for (uint32_t j = pp[0]; j < pp[1]; ++j, ++ob) {
                const uint32_t sym = t->stack[j];
                const int left = (sym >> 31) & 1;
                dep += left ? 1 : -1;
                br[ob] = sym;
                ds[ob] = (int32_t)(dep - left);
            }
            for (uint32_t j = pp[2]; j < pp[3]; ++j, ++op) {
                const uint32_t pr = t->pseq[j];
                const int32_t ptm = t->prod_term[pr];
                vv[op] = (int32_t)v;
                v += (int64_t)t->arity[pr] - 1;
                tag[op] = pr;
                kind[op] = 0;
                nst[op] = 0;
                nen[op] = 0;
                if (ptm >= 0 && subst) {
                    kind[op] = 1;
                    tag[op] = (uint32_t)ptm;
                    nst[op] = tstart[kk];
                    nen[op] = tend[kk];
                }
                if (ptm >= 0) ++kk;
            }
        }
    }
    /* bracket matching: every right's previous smaller-or-equal is a left of
     * the same symbol */
    if (par_prev_leq(c, ds, NB, pv)) return -1;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad) num_threads(c->threads)
    for (int64_t i = 0; i < NB; ++i) {
        if ((br[i] >> 31) & 1) continue;
        const int64_t j = pv[i];
        if (j < 0 || (br[i] & 0x7fffffffu) != (br[j] & 0x7fffffffu)) bad = 1;
    }
    if (bad) return 0;
    if (par_prev_leq(c, vv, NP, parent)) return -1;
    if (NP > 0) parent[0] = 0;
    *o_parent = parent; *o_tag = tag; *o_kind = kind; *o_start = nst; *o_end = nen;
    *nnode = NP;
    return 1;
}

/* lex+parse of one document (the generated parse_int on bytes). */
int par_lex_parse(par_ctx *c, const uint8_t *s, int64_t n, int64_t **o_parent, uint32_t **o_tag, uint8_t **o_kind,
                  int64_t **o_start, int64_t **o_end, int64_t *nnode) {
    uint32_t *term;
    int64_t *ts, *te, m = 0;
    *nnode = 0;
    *o_parent = NULL; *o_tag = NULL; *o_kind = NULL; *o_start = NULL; *o_end = NULL;
    const int r = par_lex(c, s, n, &term, &ts, &te, &m);
    if (r != 1) return r;
    return par_parse(c, term, ts, te, m, o_parent, o_tag, o_kind, o_start, o_end, nnode);
}
