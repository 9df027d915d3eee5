/*
 * alpacc_b200 -- B200-native lexer/parser for alpacc grammars: the C ABI.
 *
 * The reference's de-facto C ABI for this path is the library that the
 * Futhark compiler makes from alpacc's generated program: the entry points
 * `lex_int`/`lex` (src/Alpacc/Generator/Futhark/Generator.hs:63-75),
 * `parse_int`/`parse` (src/Alpacc/Generator/Futhark/Generator.hs:24-44) and,
 * for the parser-only generator, `parse_int` over a token array and
 * `pre_productions_int` (futhark/parser.fut:41-44, futhark/test.fut:75-119),
 * all called through one context (Futhark's futhark_context).  Every function
 * below replaces one of them; the comment names which.
 *
 * Conventions
 *   - Return value: ALP_OK (0) or an ALP_ERR_* code; alp_last_error() gives
 *     the message.  A grammar REJECTING the input is not an error: it is
 *     `*valid = 0` with zero outputs, exactly the reference's `#none` (and the
 *     empty arrays of the lexer-only `lex_int` entry point).
 *   - `d_` pointers are device memory on the context's device; `h_` pointers
 *     are host memory.  Calls are ordered on the context's stream and return
 *     after the results are known (they synchronise that stream once).
 *   - Outputs returned through `**` pointers are owned by the context and stay
 *     valid until the next call on it.  `_into` variants write to caller
 *     buffers of `cap` elements and fail with ALP_ERR_CAPACITY (setting the
 *     needed count) when too small.
 *   - Terminal and production ids are widened to uint32 and positions to
 *     int64.  Spans are [start, end) byte offsets.  A tree node is
 *     (parent, tag, kind, start, end): kind 0 = production (tag = production
 *     id, span 0,0), kind 1 = terminal (tag = terminal id, the token's span).
 *     Nodes are in preorder and the root is its own parent.
 *   - A context is not thread safe, like a Futhark context.
 */
#ifndef ALPACC_B200_H
#define ALPACC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ALP_OK = 0,
    ALP_ERR_ARG = 1,       /* bad argument (null pointer, size out of range) */
    ALP_ERR_CUDA = 2,      /* a CUDA call failed */
    ALP_ERR_TIMEOUT = 3,   /* a kernel's bounded wait gave up */
    ALP_ERR_TABLE = 4,     /* malformed table blob, or tables too large */
    ALP_ERR_CAPACITY = 5,  /* caller buffer too small */
    ALP_ERR_MODE = 6       /* the tables have no lexer / no parser */
};

typedef struct alp_ctx alp_ctx;

/* futhark_context_new + the generated table constants: load one grammar's
 * tables (the blob written by alpacc_b200.tables) onto `device`. */
int alp_ctx_create(const void* blob, size_t len, int device, alp_ctx** out);
void alp_ctx_destroy(alp_ctx* ctx);
const char* alp_last_error(const alp_ctx* ctx);
/* Order every later call on this CUDA stream (a cudaStream_t; NULL = legacy default). */
int alp_set_stream(alp_ctx* ctx, void* stream);
/* Grammar facts: out[0] has_lexer, [1] has_parser, [2] n_terminals,
 * [3] n_productions, [4] lookback q, [5] lookahead k, [6] max productions per
 * admissible pair, [7] max brackets per pair; counts of the last call on this
 * context: [8] tokens, [9] parser positions (tokens + 2 per document),
 * [10] brackets, [11] brackets left for the bracket-matching search after
 * the pairs closed between adjacent positions are removed; [12] device
 * allocations (cudaMalloc calls) this context has made so far; [13], [14]
 * data bytes the last host-buffer call (alp_parse_host, alp_parse_batch_host,
 * alp_lex_host, alp_lex_host_stream) moved to the device (input) and to the
 * host (tree or tokens).  No reference counterpart (measurement support). */
int alp_ctx_info(const alp_ctx* ctx, int64_t* out, int n_out);

/* Per-kernel timing (no reference counterpart; measurement support): when on,
 * every later call records a CUDA event after each kernel; alp_ctx_timings
 * writes "kernel_name milliseconds" lines for the recorded calls and clears them. */
int alp_ctx_profile(alp_ctx* ctx, int on);
int alp_ctx_timings(alp_ctx* ctx, char* buf, size_t len);

/* Failure detection (no reference counterpart): every wait inside a kernel of
 * this library is bounded, and a wait that runs out records the fact and lets
 * the call return ALP_ERR_TIMEOUT with the context still usable.  This runs
 * one such wait on a status word that nothing sets; it returns ALP_ERR_TIMEOUT
 * after about a second when the bounds work. */
int alp_check_bounded_wait(alp_ctx* ctx);

/* Autotuning (no reference counterpart).  A context carries launch shapes:
 * cfg[0] the tile shape of the previous-smaller-or-equal kernel (an index into
 * the list alp_tune_shapes writes as (threads, elements per thread) pairs),
 * cfg[1] and cfg[2] the CTAs per SM of the persistent pair and expand kernels
 * (0: as many as fit); with n >= 4, cfg[3] the boundary-MLP inference kernel
 * (0: tcgen05 tensor-memory kernel, the default; 1: mma.sync kernel, whose
 * predictions may differ where two logits are within rounding); with n >= 5,
 * cfg[4] the lexer's token pass (0: one fused pass that counts, looks back
 * over tiles and writes tokens; 1: a count pass, a tile scan and a token
 * pass, the default); with n >= 6, cfg[5] the parser's position pass (0: one
 * fused pass that looks up the pairs, looks back over tiles and expands, sized
 * from the previous parse on the context; 1: a pair pass and a scan of its
 * tile sums before the expansion, the default); with n >= 7, cfg[6] the lexer state
 * scan's chunks per lane (8, 16 or 32; 0 or 16 the default).  The tuner tries
 * the lexer's knobs first, then the parser's.
 * alp_tune_parse times alp_parse on a sample (the median
 * of `reps` calls per candidate, CUDA events), one knob at a time, keeps the
 * fastest setting in the context and writes "knob value ms" lines to
 * `report`.  Every setting gives the same outputs; only speed differs. */
int alp_tune_parse(alp_ctx* ctx, const uint8_t* d_in, int64_t n, int reps, char* report, size_t report_len);
int alp_tune_get(const alp_ctx* ctx, int32_t* cfg, int n);
int alp_tune_set(alp_ctx* ctx, const int32_t* cfg, int n);
int alp_tune_shapes(int32_t* out, int n);

/* Copy `bytes` between any two addresses (device or host) on the context's
 * stream and wait for it; lets bindings move context-owned outputs. */
int alp_memcpy(alp_ctx* ctx, void* dst, const void* src, size_t bytes);

/* lex_int: bytes -> tokens (futhark/lexer.fut:174-178 through
 * src/Alpacc/Generator/Futhark/Generator.hs:70-75). */
int alp_lex(alp_ctx* ctx, const uint8_t* d_in, int64_t n, uint32_t** d_term, int64_t** d_start,
            int64_t** d_end, int64_t* n_tok, int* valid);
int alp_lex_into(alp_ctx* ctx, const uint8_t* d_in, int64_t n, uint32_t* d_term, int64_t* d_start,
                 int64_t* d_end, int64_t cap, int64_t* n_tok, int* valid);
/* Same as alp_lex_into with host buffers: copies in, lexes, copies out.  The
 * spans of an input shorter than 2^31 bytes cross PCIe as 32-bit values and
 * are widened on the host as they land (12 bytes a token instead of 20), as in
 * alp_parse_host. */
int alp_lex_host(alp_ctx* ctx, const uint8_t* h_in, int64_t n, uint32_t* h_term, int64_t* h_start,
                 int64_t* h_end, int64_t cap, int64_t* n_tok, int* valid);

/* lex_int without any device allocation (no counterpart in the reference).
 * For callers that cannot allocate device memory when they lex: a caller whose
 * own pool reserved all device memory up front (a serving process that owns
 * the GPU), or a path where cudaMalloc/cudaFree would synchronise the device
 * and stall its other streams.  Same results as alp_lex_into.
 *   - Input is limited to 128 MiB (134217728 bytes); larger inputs fail with
 *     ALP_ERR_ARG and a message naming the limit.
 *   - Scratch is one fixed 393,472-byte array compiled into the library; every
 *     GPU that loads the library holds it until the process exits.  The
 *     outputs are the caller's buffers of `cap` tokens.
 *   - Every call looks up the array's device address (cudaGetSymbolAddress,
 *     which allocates nothing); the first call on a device may load the
 *     library's kernels there, so make it before any stream capture.
 *   - All calls share the one array, which keeps the last call's contents (the
 *     call clears the part it uses first): calls that overlap on the GPU
 *     (other streams, other contexts on the same device) race and must not
 *     overlap.
 *   - The call blocks on the context stream until the token count is back.
 *   - It makes no cudaMalloc/cudaFree and no allocating library call; only its
 *     error paths write the context's host-side message. */
int alp_lex_noalloc(alp_ctx* ctx, const uint8_t* d_in, int64_t n, uint32_t* d_term, int64_t* d_start,
                    int64_t* d_end, int64_t cap, int64_t* n_tok, int* valid);

/* Token streams: input that arrives in pieces, lexed as it comes.  Replaces the
 * reference's chunk loop, which carries (last state, last start, size) from one
 * chunk to the next (futhark/lexer.fut:148-160; cuda/lexer.cu:452-543
 * lexer_stream).  The tokens equal alp_lex on the concatenation of all pieces,
 * with positions counted from the stream's first byte.
 *   - begin: tokens will go to the caller's device buffers of `cap` tokens.
 *   - push: lexes one piece of device bytes (any size, empty included) and
 *     writes the tokens that end inside it.  Stream-ordered on the context's
 *     stream, no wait; the piece must stay unchanged until the work is done.
 *   - tokens: waits for the pushed pieces; *n_tok = tokens written so far.
 *   - end: writes the last token, waits; *valid and *n_tok as alp_lex (a
 *     rejected stream: *valid = 0, *n_tok = 0).  With a buffer too small,
 *     ALP_ERR_CAPACITY and *n_tok = the tokens needed.
 *   - window: later tokens go to these buffers, stream token `first` at
 *     element 0 (tokens before it are not stored).  With first = the count
 *     from alp_lex_stream_tokens, one piece-sized buffer serves a stream of
 *     any length, as the reference's per-chunk output arrays do.
 * Tokens are final once written: a stream that turns out rejected at its end
 * has already written the tokens before the point of rejection.  Needs a DFA
 * of at most 32 states (ALP_ERR_TABLE otherwise).  One stream per context at
 * a time. */
typedef struct alp_lex_stream alp_lex_stream;
int alp_lex_stream_begin(alp_ctx* ctx, uint32_t* d_term, int64_t* d_start, int64_t* d_end, int64_t cap,
                         alp_lex_stream** out);
int alp_lex_stream_push(alp_lex_stream* s, const uint8_t* d_piece, int64_t n);
int alp_lex_stream_tokens(alp_lex_stream* s, int64_t* n_tok);
int alp_lex_stream_end(alp_lex_stream* s, int64_t* n_tok, int* valid);
int alp_lex_stream_window(alp_lex_stream* s, uint32_t* d_term, int64_t* d_start, int64_t* d_end, int64_t cap,
                          int64_t first);
void alp_lex_stream_free(alp_lex_stream* s);

/* One document lexed by several GPUs (no reference counterpart: the
 * reference's chunk loop runs its chunks one after another).  Each GPU holds
 * one byte range; the ranks exchange two small records (by any collective)
 * and each writes the tokens that end in its range, with document positions.
 * The union over the ranges equals alp_lex on the whole document.
 *   - begin: `pos` = the range's first byte in the document, is_last for the
 *     range that ends it; writes the range's state function to h_fn[32]
 *     (h_fn[s] = state after the range from entry state s).  Entry state of
 *     range r: start from 1 (the initial state) and apply h_fn of ranges
 *     0 .. r-1 in order.
 *   - count: from that entry state, *n_tok = tokens that end in the range and
 *     *last_start = document position of its last token start (-1: none).
 *     Range r's first token index is the sum of n_tok over ranges before it;
 *     its carried start is the last last_start >= 0 among them, else 0.
 *   - emit: writes the range's *n_tok tokens (token k of the range at element
 *     k); on the last range *valid as alp_lex (1 elsewhere).
 * Needs a DFA of at most 32 states.  One shard per context at a time. */
typedef struct alp_lex_shard alp_lex_shard;
int alp_lex_shard_begin(alp_ctx* ctx, const uint8_t* d_in, int64_t n, int64_t pos, int is_last, uint8_t* h_fn,
                        alp_lex_shard** out);
int alp_lex_shard_count(alp_lex_shard* s, uint32_t entry_state, int64_t* n_tok, int64_t* last_start);
int alp_lex_shard_emit(alp_lex_shard* s, int64_t carried_start, uint32_t* d_term, int64_t* d_start,
                       int64_t* d_end, int64_t cap, int64_t* n_tok, int* valid);
void alp_lex_shard_free(alp_lex_shard* s);

/* One document parsed by several GPUs (no counterpart in the reference, whose
 * API parses one document per call; it splits the scans of
 * futhark/parser.fut:110-332 at slice edges).  Rank r holds a contiguous slice
 * of the document's tokens (as alp_lex_shard gives them, spans in document
 * positions); the first slice's positions start with ⊢ and the last's end
 * with ⊣.  Three small all-gathers join the ranks:
 *   - begin: the slice's positions; h_edge[0..15] the terminals of its first
 *     16 positions and h_edge[16..31] of its last 16 (the parser's empty
 *     terminal where the slice is shorter), *n_pos its position count.
 *     Gather (h_edge, n_pos) from every rank.
 *   - sums: halo_l[16] / halo_r[16] the terminals of the 16 positions before
 *     and after the slice (empty past the document), from the gathered edges.
 *     sums[10]: nodes, brackets, depth, sum of (arity - 1), terminal
 *     productions, document heads, the last head's position (-1: none),
 *     bracket pairs closed between adjacent positions, those closed at the
 *     slice's first position with the slice before, the first position's
 *     pair id.  Gather sums from every rank.
 *   - expand: pre[8] the first eight sums combined over the slices before
 *     (depth, v and terminal counts restart after a head), pos_base the
 *     positions before the slice, closed_next the next slice's sums[8] (0 on
 *     the last).  Writes the slice's nodes (parents within the slice, spans
 *     and tags final) and matches its brackets; gives the sizes of its two
 *     staircases (node values and bracket depths strictly below everything
 *     after them in the slice).
 *   - stairs: copies the staircases out (values; global node index or bracket
 *     symbol).  Gather them from every rank.
 *   - resolve: the staircases of the slices before, concatenated in rank
 *     order with offsets n_off / b_off [n_prev + 1]; answers what had no
 *     answer in the slice; *valid this slice's verdict (the document is
 *     accepted iff every slice's is 1).
 *   - tree: the slice's nodes (context-owned, until the next call on the
 *     context) and the global index of its first node.
 * One shard per context at a time. */
typedef struct alp_parse_shard alp_parse_shard;
int alp_parse_shard_begin(alp_ctx* ctx, const uint32_t* d_term, const int64_t* d_start, const int64_t* d_end,
                          int64_t m, int is_first, int is_last, uint32_t* h_edge, int64_t* n_pos,
                          alp_parse_shard** out);
int alp_parse_shard_sums(alp_parse_shard* s, const uint32_t* halo_l, const uint32_t* halo_r, int64_t* sums);
int alp_parse_shard_expand(alp_parse_shard* s, const int64_t* pre, int64_t pos_base, int64_t closed_next,
                           int64_t* n_node, int64_t* n_stair_nodes, int64_t* n_stair_brackets);
int alp_parse_shard_stairs(alp_parse_shard* s, int32_t* h_nval, int64_t* h_nidx, int32_t* h_bval, uint32_t* h_bsym);
int alp_parse_shard_resolve(alp_parse_shard* s, int n_prev, const int64_t* n_off, const int32_t* nval,
                            const int64_t* nidx, const int64_t* b_off, const int32_t* bval, const uint32_t* bsym,
                            int* valid);
int alp_parse_shard_tree(alp_parse_shard* s, int64_t** d_parent, uint32_t** d_tag, uint8_t** d_kind,
                         int64_t** d_start, int64_t** d_end, int64_t* n_node, int64_t* first_node);
void alp_parse_shard_free(alp_parse_shard* s);

/* alp_lex_host over a stream of `piece`-byte pieces (0: 16 MiB): the copy of
 * one piece in, the lexing of the one before and the copy of the tokens of the
 * one before that out overlap on three CUDA streams.  Same results as
 * alp_lex_host, for inputs of any size; host buffers should be pinned
 * (cudaHostAlloc) for the copies to overlap.  Below 2^31 bytes the spans cross
 * as 32-bit values, widened on the host as they land. */
int alp_lex_host_stream(alp_ctx* ctx, const uint8_t* h_in, int64_t n, int64_t piece, uint32_t* h_term,
                        int64_t* h_start, int64_t* h_end, int64_t cap, int64_t* n_tok, int* valid);

/* parse_int of the lexer+parser generator: bytes -> preorder tree
 * (src/Alpacc/Generator/Futhark/Generator.hs:35-44, futhark/parser.fut:316-336). */
int alp_parse(alp_ctx* ctx, const uint8_t* d_in, int64_t n, int64_t** d_parent, uint32_t** d_tag,
              uint8_t** d_kind, int64_t** d_start, int64_t** d_end, int64_t* n_node, int* valid);
int alp_parse_into(alp_ctx* ctx, const uint8_t* d_in, int64_t n, int64_t* d_parent, uint32_t* d_tag,
                   uint8_t* d_kind, int64_t* d_start, int64_t* d_end, int64_t cap, int64_t* n_node,
                   int* valid);
/* The same from and into host memory.  Parents and spans cross PCIe as 32-bit
 * values (17 bytes a node instead of 29) into a 64 MiB ring of pinned slots,
 * and host threads sign-extend each landed 1 Mi-value chunk into the caller's
 * arrays while later chunks are still in flight; the call returns when every
 * output is written.  The threads: the CPUs the process may run on, less the
 * calling thread, at most eight; or ALP_HOST_THREADS when that is set (read once
 * per context). */
int alp_parse_host(alp_ctx* ctx, const uint8_t* h_in, int64_t n, int64_t* h_parent, uint32_t* h_tag,
                   uint8_t* h_kind, int64_t* h_start, int64_t* h_end, int64_t cap, int64_t* n_node,
                   int* valid);

/* parse_int of the parser-only generator: tokens -> tree (futhark/parser.fut:334-336). */
int alp_parse_tokens(alp_ctx* ctx, const uint32_t* d_term, const int64_t* d_tstart, const int64_t* d_tend,
                     int64_t m, int64_t** d_parent, uint32_t** d_tag, uint8_t** d_kind, int64_t** d_start,
                     int64_t** d_end, int64_t* n_node, int* valid);

/* pre_productions_int: token ids -> production sequence (futhark/parser.fut:269-271). */
int alp_pre_productions(alp_ctx* ctx, const uint32_t* d_term, int64_t m, uint32_t** d_prod,
                        int64_t* n_prod, int* valid);

/* Learned boundary-state speculation (no reference counterpart).
 *
 * alp_lex_states: the exact DFA state entering byte 16*i, for every i with
 * 16*i < n (the composition scan's own states; training labels).
 *
 * The MLP (64-byte window -> 16-d byte embedding -> 128 -> 128 -> state
 * logits, BF16 weights, FP32 accumulation) lives in caller memory:
 *   params / grads / adam_m / adam_v: FP32 blocks of 155936 floats laid out
 *     emb[256*16] w1[1024*128] b1[128] w2[128*128] b2[128] w3[128*32] b3[32];
 *   wbf: the BF16 copies of emb, w1, w2, w3, back to back (155648 values).
 * alp_mlp_train_step runs forward + backward (+ AdamW when `update`) on one
 * batch of windows [batch][64] with labels [batch]; batch % 16 == 0.
 * alp_mlp_predict writes the argmax state for the window ending before each
 * position in d_pos.
 *
 * alp_lex_speculative: lex_int with chunk starts predicted by the MLP and
 * verified by re-running mispredicted chunks until every start state is
 * exact -- the same tokens as alp_lex for any weights.  stats (4 values):
 * chunks, first-round mismatches, chunks re-run, verification rounds (-1:
 * more than 64 rounds were needed and the plain scan produced the tokens). */
int alp_lex_states(alp_ctx* ctx, const uint8_t* d_in, int64_t n, uint8_t* d_states);
int alp_mlp_train_step(alp_ctx* ctx, float* params, uint16_t* wbf, float* grads, float* adam_m, float* adam_v,
                       int n_states, const uint8_t* d_win, const uint8_t* d_lab, int batch, float lr, float wd,
                       int step, int update, float* h_loss, float* h_acc);
int alp_mlp_predict(alp_ctx* ctx, const uint16_t* wbf, const float* wf32, int n_states, const uint8_t* d_in,
                    int64_t n, const int64_t* d_pos, int64_t count, uint8_t* d_pred);
int alp_lex_speculative(alp_ctx* ctx, const uint16_t* wbf, const float* wf32, int n_states, const uint8_t* d_in,
                        int64_t n, int64_t chunk, uint32_t** d_term, int64_t** d_start, int64_t** d_end,
                        int64_t* n_tok, int* valid, int64_t* stats);

/* Batched documents (no reference counterpart: the reference parses one
 * document per call; this is that call applied to every document).
 * d_in holds the documents back to back, d_off[0..n_docs] their byte offsets.
 * Per document i: d_valid[i], and its outputs in [d_out_off[i], d_out_off[i+1]).
 * Positions and parents are relative to the document. */
int alp_lex_batch(alp_ctx* ctx, const uint8_t* d_in, const int64_t* d_off, int64_t n_docs,
                  uint32_t** d_term, int64_t** d_start, int64_t** d_end, int64_t** d_tok_off,
                  uint8_t** d_valid, int64_t* n_tok_total);
int alp_parse_batch(alp_ctx* ctx, const uint8_t* d_in, const int64_t* d_off, int64_t n_docs,
                    int64_t** d_parent, uint32_t** d_tag, uint8_t** d_kind, int64_t** d_start,
                    int64_t** d_end, int64_t** d_node_off, uint8_t** d_valid, int64_t* n_node_total);
/* alp_parse_batch from and into host memory: h_off[0..n_docs] (starting at 0, not
 * decreasing) on the host, the trees' nodes into arrays of capacity cap (the
 * node total is set, with ALP_ERR_CAPACITY, when cap is short), h_node_off[n_docs
 * + 1] and h_valid[n_docs].  Parents and spans cross PCIe as 32-bit values widened
 * on the host, as in alp_parse_host. */
int alp_parse_batch_host(alp_ctx* ctx, const uint8_t* h_in, const int64_t* h_off, int64_t n_docs,
                         int64_t* h_parent, uint32_t* h_tag, uint8_t* h_kind, int64_t* h_start,
                         int64_t* h_end, int64_t* h_node_off, uint8_t* h_valid, int64_t cap,
                         int64_t* n_node_total);

/* The reference's test wire format, written from batch results in host memory
 * (host code only, no GPU work): the `.outputs` files that `alpacc test`
 * generates and compares, big-endian u64 counts and fields, one boolean byte
 * per input (src/Alpacc/Test/Lexer.hs:59-85, src/Alpacc/Test/LexerParser.hs:54-99,
 * src/Alpacc/Test/Parser.hs:41-56).  A C, cgo or JNI caller that holds
 * alp_lex_batch / alp_parse_batch / alp_pre_productions results can write the
 * file these tools diff without a second serialiser.
 *   ALP_WIRE_LEXER     per accepted input: u64 n, then n x (u64 term, u64 start,
 *                      u64 end) from id / start / end;
 *   ALP_WIRE_LEXPARSE  n x (u8 kind, u64 parent, u64 id, u64 start, u64 end) from
 *                      kind / parent / id / start / end (spans written as 0 for
 *                      production nodes, kind 0);
 *   ALP_WIRE_PARSER    n x u64 production from id.
 * Input i's elements are [off[i], off[i+1]); valid[i] = 0 writes only its
 * boolean.  Arrays a mode does not read may be NULL.  *len receives the size of
 * the file; with out == NULL that is all (a size query, ALP_OK), with cap < *len
 * nothing is written and ALP_ERR_CAPACITY is returned.  ALP_ERR_ARG for an unknown
 * mode, a missing array, offsets that decrease, or a kind other than 0 or 1. */
#define ALP_WIRE_LEXER 0
#define ALP_WIRE_LEXPARSE 1
#define ALP_WIRE_PARSER 2
int alp_write_reference_format(int mode, int64_t n_docs, const uint8_t* valid, const int64_t* off,
                               const uint32_t* id, const int64_t* parent, const uint8_t* kind,
                               const int64_t* start, const int64_t* end, uint8_t* out, size_t cap,
                               size_t* len);

/* The comparison `alpacc test compare` makes (src/Alpacc/Test/Lexer.hs:181-231,
 * LexerParser.hs:342-392, Parser.hs:140-167), on two such files held in host
 * memory (host code only): *first_diff = -1 when every input has the same
 * result, else the first input whose result differs (accepted in one file and
 * rejected in the other, a different element count, or a different element);
 * files with different numbers of results differ at the first input only one
 * of them has, whatever the shared ones hold.  *field names the first
 * differing field of the first differing element, in record order (lexer:
 * term, start, end; lexer+parser: kind, parent, id, start, end; parser: the
 * production), else -1.  ALP_ERR_ARG for an unknown mode or a malformed file
 * (truncated, a boolean or kind byte other than 0 or 1, bytes after the last
 * input). */
int alp_compare_reference_format(int mode, const uint8_t* a, size_t a_len, const uint8_t* b, size_t b_len,
                                 int64_t* first_diff, int* field);

/* The batched parse as a CUDA graph (no reference counterpart).  alp_parse_batch
 * waits on the host three times (input size, token total, node and bracket
 * totals) to size its outputs; for a fixed batch shape this set-up captures the
 * same kernels, sized by the capacities given here and reading the actual
 * counts from device memory, in one CUDA graph, so that a batch costs one
 * cudaGraphLaunch and no host round trip.
 *   - create: the device buffers and sizes are fixed: d_in (n bytes),
 *     d_off (n_docs + 1 offsets, d_off[n_docs] = n), node outputs of cap_nodes
 *     elements, d_node_off (n_docs + 1), d_valid (n_docs), d_counts (4 int64:
 *     nodes, brackets, positions, error bits).  The contents of d_in and d_off
 *     may change between launches (same n and n_docs).  Runs the batch once
 *     uncaptured to size the graph's own scratch, then captures it.
 *   - launch: enqueues one run on `stream` (a cudaStream_t; NULL: the legacy
 *     default stream), ordered after the work already on it; no wait.
 *   - result: waits for the last launch; *n_nodes = nodes of the batch;
 *     ALP_ERR_CAPACITY when cap_nodes or cap_brackets was too small (then the
 *     outputs are incomplete and *n_nodes is the count needed).
 * Outputs and their layout are those of alp_parse_batch.  The graph keeps its
 * own scratch and shares only the tables with `ctx`, which stays usable; the
 * graph must be destroyed before `ctx`.  Needs a DFA of at most 32 states. */
typedef struct alp_parse_graph alp_parse_graph;
int alp_parse_graph_create(alp_ctx* ctx, const uint8_t* d_in, int64_t n, const int64_t* d_off, int64_t n_docs,
                           int64_t cap_nodes, int64_t cap_brackets, int64_t* d_parent, uint32_t* d_tag,
                           uint8_t* d_kind, int64_t* d_start, int64_t* d_end, int64_t* d_node_off, uint8_t* d_valid,
                           int64_t* d_counts, alp_parse_graph** out);
int alp_parse_graph_launch(alp_parse_graph* g, void* stream);
int alp_parse_graph_result(alp_parse_graph* g, int64_t* n_nodes);
const char* alp_parse_graph_error(const alp_parse_graph* g);
void alp_parse_graph_destroy(alp_parse_graph* g);

#ifdef __cplusplus
}
#endif
#endif /* ALPACC_B200_H */
