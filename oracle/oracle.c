/*
 * CPU oracle for the alpacc lex/parse hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only the tests, the smoke check and the CPU
 * baseline leg of the benchmark load this library, and only as the checker.
 * The product path (alpacc_b200/) never calls it.
 *
 * It restates, in plain sequential C, the reference algorithms for the path:
 *
 *   orc_tokenize       -- tokenize            src/Alpacc/Lexer/DFA.hs:415-447
 *   orc_lex_futhark    -- lex_step/lex_int    futhark/lexer.fut:91-178
 *                         (including its chunk loop, lines 144-172)
 *   orc_parse_futhark  -- parse_int_flag      futhark/parser.fut:110-332
 *   orc_parse_glue     -- llpParse + glue + llpParseTree/flattenTree
 *                                            src/Alpacc/LLP.hs:595-727
 *
 * It reads the same table blob as the product library (layout documented
 * in alpacc_b200/tables.py), but only the plain forms: the 256-column DFA,
 * the token map and the admissible-pair list.  The sequential functions here
 * never read the endomorphism forms; par.c (the data-parallel restatement)
 * does.
 */
#include "oracle.h"

static const uint8_t *rd32(const uint8_t *p, const uint8_t *e, uint32_t *v) {
    if (!p || p + 4 > e) return NULL;
    memcpy(v, p, 4);
    return p + 4;
}

static const uint8_t *skip(const uint8_t *p, const uint8_t *e, size_t n) {
    if (!p || p + n > e) return NULL;
    return p + ((n + 3) & ~(size_t)3) <= e ? p + ((n + 3) & ~(size_t)3) : e;
}

void orc_free(orc_tables *t) {
    if (t) {
        free(t->copy);
        free(t);
    }
}

orc_tables *orc_load(const void *blob, size_t len) {
    orc_tables *t = (orc_tables *)calloc(1, sizeof(orc_tables));
    if (!t) return NULL;
    t->copy = (uint8_t *)malloc(len + 4);
    if (!t->copy) { free(t); return NULL; }
    memcpy(t->copy, blob, len);
    const uint8_t *p = t->copy, *e = t->copy + len;
    uint32_t magic, ver, hl, hp;
    p = rd32(p, e, &magic); p = rd32(p, e, &ver); p = rd32(p, e, &hl); p = rd32(p, e, &hp);
    if (!p || magic != ORC_MAGIC) { orc_free(t); return NULL; }
    t->has_lexer = (int)hl;
    t->has_parser = (int)hp;
    if (hl) {
        p = rd32(p, e, &t->S); p = rd32(p, e, &t->C); p = rd32(p, e, &t->E);
        p = rd32(p, e, &t->ignore_term); p = rd32(p, e, &t->dead_term); p = rd32(p, e, &t->n_terms);
        if (!p) { orc_free(t); return NULL; }
        uint32_t S = t->S, C = t->C, E = t->E;
        t->cls = p; p = skip(p, e, 256);                       /* byte classes */
        t->delta256 = (const uint16_t *)p; p = skip(p, e, (size_t)S * 256 * 2);
        p = skip(p, e, (size_t)S * (C + 1) * 2);               /* class table */
        t->token = (const uint32_t *)p; p = skip(p, e, (size_t)S * 4);
        t->accept = p; p = skip(p, e, S);
        t->endo_step = (const uint16_t *)p; p = skip(p, e, (size_t)E * (C + 1) * 2);
        t->endo_comp = (const uint16_t *)p; p = skip(p, e, (size_t)E * E * 2);
        t->endo_app = (const uint16_t *)p; p = skip(p, e, (size_t)E * S * 2);
        if (!p) { orc_free(t); return NULL; }
    }
    if (hp) {
        p = rd32(p, e, &t->q); p = rd32(p, e, &t->k); p = rd32(p, e, &t->n_term_syms);
        p = rd32(p, e, &t->empty); p = rd32(p, e, &t->start); p = rd32(p, e, &t->end);
        p = rd32(p, e, &t->n_prods);
        uint32_t nt; p = rd32(p, e, &nt);
        if (!p) { orc_free(t); return NULL; }
        if (!hl) t->n_terms = nt;
        t->arity = (const uint32_t *)p; p = skip(p, e, (size_t)t->n_prods * 4);
        t->prod_term = (const int32_t *)p; p = skip(p, e, (size_t)t->n_prods * 4);
        p = rd32(p, e, &t->n_pairs);
        t->pairs = (const uint32_t *)p; p = skip(p, e, (size_t)t->n_pairs * 16);
        p = rd32(p, e, &t->n_stack);
        t->stack = (const uint32_t *)p; p = skip(p, e, (size_t)t->n_stack * 4);
        p = rd32(p, e, &t->n_pseq);
        t->pseq = (const uint32_t *)p; p = skip(p, e, (size_t)t->n_pseq * 4);
        p = rd32(p, e, &t->n_keys);
        t->keys = (const uint32_t *)p; p = skip(p, e, (size_t)t->n_keys * (t->q + t->k) * 4);
        t->key_pair = (const uint32_t *)p; p = skip(p, e, (size_t)t->n_keys * 4);
        if (!p) { orc_free(t); return NULL; }
    }
    return t;
}

int orc_info(const orc_tables *t, uint32_t *out /* [8] */) {
    out[0] = t->has_lexer; out[1] = t->has_parser; out[2] = t->S; out[3] = t->n_terms;
    out[4] = t->q; out[5] = t->k; out[6] = t->n_prods; out[7] = t->n_pairs;
    return 0;
}

/* ---------------------------------------------------------------- lexer -- */

#define nxt orc_nxt
#define prod orc_prod
#define is_ignore orc_is_ignore

/* tokenize (src/Alpacc/Lexer/DFA.hs:415-447).  Returns 1 (valid), 0
 * (rejected: no tokens), -1 (capacity exceeded). */
int orc_tokenize(const orc_tables *t, const uint8_t *s, int64_t n, uint32_t *term, int64_t *start,
                 int64_t *end, int64_t cap, int64_t *ntok) {
    *ntok = 0;
    if (n == 0) return t->accept[INIT_STATE] ? 1 : 0;
    uint32_t st = INIT_STATE;
    int64_t i0 = 0, m = 0;
    for (int64_t j = 0; j < n; ++j) {
        uint32_t s2 = nxt(t, st, s[j]);
        if (s2 == 0) { *ntok = 0; return 0; }
        if (j == n - 1) {
            if (!t->accept[s2]) { *ntok = 0; return 0; }
            uint32_t k = t->token[s2];
            if (!is_ignore(t, k)) {
                if (m >= cap) return -1;
                term[m] = k; start[m] = i0; end[m] = j + 1; ++m;
            }
        } else if (prod(t, s2, s[j + 1])) {
            uint32_t k = t->token[s2];
            if (!is_ignore(t, k)) {
                if (m >= cap) return -1;
                term[m] = k; start[m] = i0; end[m] = j + 1; ++m;
            }
            i0 = j + 1;
        }
        st = s2;
    }
    *ntok = m;
    return 1;
}

/* lex_int_flag (futhark/lexer.fut:91-172) restated with the DFA: the scan
 * "compose" of byte endomorphisms applied to the initial state is the DFA run,
 * the produce bit of a position is that of the transition into it and the
 * terminal of a position is the token of the state reached.  chunk <= 0 means
 * one chunk.  The loop keeps the template's exact chunk arithmetic: a chunk
 * reads one byte past its end, the next chunk starts from the state that
 * already includes that byte, and after every chunk the span map is applied to
 * the whole result array. */
typedef struct { uint32_t t; int64_t s, e; } orc_tok;

int orc_lex_futhark(const orc_tables *t, const uint8_t *str, int64_t n, int64_t chunk, uint32_t *term,
                    int64_t *start, int64_t *end, int64_t cap, int64_t *ntok) {
    *ntok = 0;
    if (chunk <= 0) chunk = n > 0 ? n : 1;
    int64_t dcap = 1;
    orc_tok *dest = (orc_tok *)calloc(1, sizeof(orc_tok));
    uint32_t state = INIT_STATE; /* identity endo applied to the initial state */
    int64_t pstart = 0, size = 0;
    uint32_t *st = NULL;
    uint8_t *pr = NULL;
    int64_t *starts = NULL;
    for (int64_t off = 0; off < n; off += chunk) {
        int64_t m = off + chunk + 1 < n ? off + chunk + 1 : n;
        int64_t L = m - off;
        st = (uint32_t *)realloc(st, L * sizeof(uint32_t));
        pr = (uint8_t *)realloc(pr, L);
        starts = (int64_t *)realloc(starts, L * sizeof(int64_t));
        uint32_t cur = state;
        for (int64_t i = 0; i < L; ++i) {
            uint8_t b = str[off + i];
            st[i] = nxt(t, cur, b);
            pr[i] = (uint8_t)prod(t, cur, b);
            cur = st[i];
        }
        int64_t cnt = 0;
        for (int64_t i = 0; i + 1 < L; ++i)
            if (pr[i + 1] && !is_ignore(t, t->token[st[i]])) ++cnt;
        for (int64_t i = 0; i < L; ++i) {
            int64_t v;
            if (pr[i] && !is_ignore(t, t->token[st[i]])) v = i;
            else if (i == 0) v = pstart - off; /* take_right (prev_start - offset) highest */
            else v = HIGHEST;
            if (i > 0 && v == HIGHEST) v = starts[i - 1];
            starts[i] = v;
        }
        int64_t extra = size + cnt + 1;
        if (dcap <= extra) {
            orc_tok *nd = (orc_tok *)calloc(2 * extra, sizeof(orc_tok));
            memcpy(nd, dest, dcap * sizeof(orc_tok));
            free(dest);
            dest = nd;
            dcap = 2 * extra;
        }
        int64_t o = size;
        for (int64_t i = 0; i + 1 < L; ++i)
            if (pr[i + 1] && !is_ignore(t, t->token[st[i]])) {
                dest[o].t = t->token[st[i]];
                dest[o].s = starts[i];
                dest[o].e = i;
                ++o;
            }
        for (int64_t i = 0; i < dcap; ++i) { dest[i].s += off; dest[i].e += 1 + off; }
        state = st[L - 1];
        pstart = starts[L - 1] != HIGHEST ? off + starts[L - 1] : pstart;
        size += cnt;
    }
    int valid;
    if (n == 0) valid = t->accept[INIT_STATE];
    else valid = t->accept[state];
    uint32_t lt = n == 0 ? t->dead_term : t->token[state];
    if (!is_ignore(t, lt)) {
        if (size >= dcap) {
            orc_tok *nd = (orc_tok *)calloc(size + 1, sizeof(orc_tok));
            memcpy(nd, dest, dcap * sizeof(orc_tok));
            free(dest);
            dest = nd;
            dcap = size + 1;
        }
        dest[size].t = lt; dest[size].s = pstart; dest[size].e = n;
        ++size;
    }
    int rc = 0;
    if (valid) {
        if (size > cap) rc = -1;
        else {
            for (int64_t i = 0; i < size; ++i) { term[i] = dest[i].t; start[i] = dest[i].s; end[i] = dest[i].e; }
            *ntok = size;
            rc = 1;
        }
    }
    free(dest); free(st); free(pr); free(starts);
    return rc;
}

/* --------------------------------------------------------------- parser -- */

static int64_t key_lookup(const orc_tables *t, const uint32_t *key) {
    /* binary search in the sorted key list (same answers as the template's
     * FNV-1a open-addressing probe, futhark/parser.fut:110-142) */
    uint32_t w = t->q + t->k;
    int64_t lo = 0, hi = (int64_t)t->n_keys - 1;
    while (lo <= hi) {
        int64_t mid = (lo + hi) / 2;
        int c = 0;
        for (uint32_t j = 0; j < w && !c; ++j) {
            uint32_t a = t->keys[(size_t)mid * w + j], b = key[j];
            c = a < b ? -1 : (a > b ? 1 : 0);
        }
        if (c == 0) return t->key_pair[mid];
        if (c < 0) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

/* nearest previous index j < i with v[j] <= v[i], or -1
 * (find_previous (<=) over mk_tree, futhark/parser.fut:72-108) */
static void prev_leq(const int64_t *v, int64_t n, int64_t *out) {
    int64_t *stk = (int64_t *)malloc((n + 1) * sizeof(int64_t));
    int64_t top = 0;
    for (int64_t i = 0; i < n; ++i) {
        while (top > 0 && v[stk[top - 1]] > v[i]) --top;
        out[i] = top > 0 ? stk[top - 1] : -1;
        stk[top++] = i;
    }
    free(stk);
}

/* pre_productions_int_flag (futhark/parser.fut:235-271).  Writes the
 * production sequence; returns 1 valid, 0 rejected, -1 capacity. */
int orc_pre_productions(const orc_tables *t, const uint32_t *ters, int64_t m, uint32_t *prods, int64_t cap,
                        int64_t *nprod) {
    *nprod = 0;
    int64_t n = m + 2;
    uint32_t w = t->q + t->k;
    uint32_t key[64];
    if (w > 64) return -1;
    int64_t *pair = (int64_t *)malloc(n * sizeof(int64_t));
    int ok = 1;
    int64_t nb = 0, np = 0;
    for (int64_t i = 0; i < n && ok; ++i) {
        for (uint32_t j = 0; j < w; ++j) {
            int64_t x = i + (int64_t)j - (int64_t)t->q; /* arr'[i+j-q] */
            uint32_t v;
            if (x < 0 || x >= n) v = t->empty;
            else if (x == 0) v = t->start;
            else if (x == n - 1) v = t->end;
            else v = ters[x - 1];
            key[j] = v;
        }
        pair[i] = key_lookup(t, key);
        if (pair[i] < 0) ok = 0;
        else {
            const uint32_t *p = t->pairs + 4 * pair[i];
            nb += p[1] - p[0];
            np += p[3] - p[2];
        }
    }
    if (!ok) { free(pair); return 0; }
    /* brackets_matches: depth scan then previous <= match (parser.fut:153-184) */
    uint32_t *br = (uint32_t *)malloc((nb + 1) * sizeof(uint32_t));
    int64_t b = 0;
    for (int64_t i = 0; i < n; ++i) {
        const uint32_t *p = t->pairs + 4 * pair[i];
        for (uint32_t j = p[0]; j < p[1]; ++j) br[b++] = t->stack[j];
    }
    int64_t *ds = (int64_t *)malloc((nb + 1) * sizeof(int64_t));
    int64_t sc = 0;
    for (int64_t i = 0; i < nb && ok; ++i) {
        int left = (br[i] >> 31) & 1;
        sc += left ? 1 : -1;
        if (sc < 0) ok = 0;
        ds[i] = sc - left;
    }
    if (ok && nb != 0 && sc != 0) ok = 0;
    if (ok) {
        int64_t *pv = (int64_t *)malloc((nb + 1) * sizeof(int64_t));
        prev_leq(ds, nb, pv);
        for (int64_t i = 0; i < nb && ok; ++i) {
            if ((br[i] >> 31) & 1) continue;
            int64_t j = pv[i];
            if (j < 0 || (br[i] & 0x7fffffffu) != (br[j] & 0x7fffffffu)) ok = 0;
        }
        free(pv);
    }
    free(ds); free(br);
    if (!ok) { free(pair); return 0; }
    if (np > cap) { free(pair); return -1; }
    int64_t o = 0;
    for (int64_t i = 0; i < n; ++i) {
        const uint32_t *p = t->pairs + 4 * pair[i];
        for (uint32_t j = p[2]; j < p[3]; ++j) prods[o++] = t->pseq[j];
    }
    free(pair);
    *nprod = np;
    return 1;
}

/* parse_int_flag (futhark/parser.fut:286-332): parents from the exclusive
 * scan of (arity-1), terminal productions replaced by the token spans. */
int orc_parse_futhark(const orc_tables *t, const uint32_t *ters, const int64_t *tstart, const int64_t *tend,
                      int64_t m, int64_t *parent, uint32_t *tag, uint8_t *kind, int64_t *nstart,
                      int64_t *nend, int64_t cap, int64_t *nnode) {
    *nnode = 0;
    int64_t np = 0;
    int rc = orc_pre_productions(t, ters, m, tag, cap, &np);
    if (rc != 1) return rc;
    int64_t *v = (int64_t *)malloc((np + 1) * sizeof(int64_t));
    int64_t acc = 0;
    for (int64_t i = 0; i < np; ++i) { v[i] = acc; acc += (int64_t)t->arity[tag[i]] - 1; }
    prev_leq(v, np, parent);
    if (np > 0) parent[0] = 0;
    free(v);
    int64_t nterm = 0;
    for (int64_t i = 0; i < np; ++i) if (t->prod_term[tag[i]] >= 0) ++nterm;
    int64_t kk = 0;
    for (int64_t i = 0; i < np; ++i) {
        int32_t pt = t->prod_term[tag[i]];
        kind[i] = 0; nstart[i] = 0; nend[i] = 0;
        if (pt >= 0 && nterm == m) {
            kind[i] = 1;
            tag[i] = (uint32_t)pt;
            nstart[i] = tstart[kk];
            nend[i] = tend[kk];
            ++kk;
        }
    }
    *nnode = np;
    return 1;
}

/* Sequential LLP parse: pairLookup + glue (src/Alpacc/LLP.hs:595-650) over the
 * homomorphic images, i.e. a stack machine that pops the right brackets and
 * pushes the left brackets of every admissible pair; the tree is rebuilt from
 * the derivation and arities in preorder (llpParseTree/flattenTree,
 * src/Alpacc/LLP.hs:670-727).  Independent of the scan-based formulation. */
int orc_parse_glue(const orc_tables *t, const uint32_t *ters, const int64_t *tstart, const int64_t *tend,
                   int64_t m, int64_t *parent, uint32_t *tag, uint8_t *kind, int64_t *nstart, int64_t *nend,
                   int64_t cap, int64_t *nnode) {
    *nnode = 0;
    int64_t n = m + 2;
    uint32_t w = t->q + t->k, key[64];
    if (w > 64) return -1;
    int64_t scap = 64, sp = 0, np = 0;
    uint32_t *stk = (uint32_t *)malloc(scap * sizeof(uint32_t));
    int ok = 1;
    for (int64_t i = 0; i < n && ok; ++i) {
        for (uint32_t j = 0; j < w; ++j) {
            int64_t x = i + (int64_t)j - (int64_t)t->q;
            key[j] = (x < 0 || x >= n) ? t->empty : (x == 0 ? t->start : (x == n - 1 ? t->end : ters[x - 1]));
        }
        int64_t pi = key_lookup(t, key);
        if (pi < 0) { ok = 0; break; }
        const uint32_t *p = t->pairs + 4 * pi;
        for (uint32_t j = p[0]; j < p[1] && ok; ++j) {
            uint32_t s = t->stack[j];
            if ((s >> 31) & 1) {
                if (sp == scap) { scap *= 2; stk = (uint32_t *)realloc(stk, scap * sizeof(uint32_t)); }
                stk[sp++] = s & 0x7fffffffu;
            } else if (sp > 0) {
                /* glue: a pop below the known stack joins the composed alpha */
                if (stk[sp - 1] != s) ok = 0;
                else --sp;
            }
        }
        for (uint32_t j = p[2]; j < p[3] && ok; ++j) {
            if (np >= cap) { free(stk); return -1; }
            tag[np++] = t->pseq[j];
        }
    }
    free(stk);
    if (!ok) return 0;
    /* preorder rebuild: each production node waits for arity children */
    int64_t *open_node = (int64_t *)malloc((np + 1) * sizeof(int64_t));
    int64_t *open_left = (int64_t *)malloc((np + 1) * sizeof(int64_t));
    int64_t top = 0, kk = 0;
    for (int64_t i = 0; i < np; ++i) {
        while (top > 0 && open_left[top - 1] == 0) --top;
        parent[i] = top > 0 ? open_node[top - 1] : 0;
        if (top > 0) open_left[top - 1]--;
        uint32_t a = t->arity[tag[i]];
        int32_t pt = t->prod_term[tag[i]];
        kind[i] = 0; nstart[i] = 0; nend[i] = 0;
        if (pt >= 0) {
            if (kk >= m) { free(open_node); free(open_left); return 0; }
            kind[i] = 1; tag[i] = (uint32_t)pt; nstart[i] = tstart[kk]; nend[i] = tend[kk]; ++kk;
        }
        if (a > 0) { open_node[top] = i; open_left[top] = a; ++top; }
    }
    free(open_node); free(open_left);
    *nnode = np;
    return 1;
}

/* Maximum productions per admissible pair (sizes node buffers). */
int64_t orc_max_pair_prods(const orc_tables *t) {
    int64_t mx = 0;
    for (uint32_t i = 0; i < t->n_pairs; ++i) {
        int64_t d = (int64_t)t->pairs[4 * i + 3] - t->pairs[4 * i + 2];
        if (d > mx) mx = d;
    }
    return mx;
}
