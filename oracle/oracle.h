/*
 * Table view shared by the CPU oracle (oracle.c, sequential) and its
 * data-parallel restatement (par.c).  TEST INFRASTRUCTURE ONLY.
 */
#ifndef ALPACC_ORACLE_H
#define ALPACC_ORACLE_H
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAGIC 0x42504C41u
#define HIGHEST INT64_MAX
#define INIT_STATE 1u

typedef struct {
    /* lexer */
    int has_lexer;
    uint32_t S, C, E, ignore_term, dead_term, n_terms;
    const uint16_t *delta256; /* [S][256]: next | produce<<15 */
    const uint32_t *token;    /* [S] */
    const uint8_t *accept;    /* [S] */
    /* the endomorphism forms of the same DFA (futhark/lexer.fut:8-27), read
     * only by the data-parallel restatement: byte classes, one more byte of a
     * class after endo e, composition (a then b), and the state after endo e */
    const uint8_t *cls;        /* [256] */
    const uint16_t *endo_step; /* [E][C+1] */
    const uint16_t *endo_comp; /* [E][E] */
    const uint16_t *endo_app;  /* [E][S] */
    /* parser */
    int has_parser;
    uint32_t q, k, n_term_syms, empty, start, end, n_prods;
    const uint32_t *arity;
    const int32_t *prod_term;
    uint32_t n_pairs;
    const uint32_t *pairs; /* [n_pairs][4] */
    uint32_t n_stack;
    const uint32_t *stack;
    uint32_t n_pseq;
    const uint32_t *pseq;
    uint32_t n_keys;
    const uint32_t *keys;     /* [n_keys][q+k], sorted */
    const uint32_t *key_pair; /* [n_keys] */
    uint8_t *copy;            /* private copy of the blob */
} orc_tables;

orc_tables *orc_load(const void *blob, size_t len);
void orc_free(orc_tables *t);

static inline uint32_t orc_nxt(const orc_tables *t, uint32_t s, uint8_t b) { return t->delta256[(size_t)s * 256 + b] & 0x7fffu; }
static inline int orc_prod(const orc_tables *t, uint32_t s, uint8_t b) { return (t->delta256[(size_t)s * 256 + b] >> 15) & 1; }
static inline int orc_is_ignore(const orc_tables *t, uint32_t term) { return t->ignore_term != 0xffffffffu && term == t->ignore_term; }

#endif
