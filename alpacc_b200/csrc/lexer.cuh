// Single-pass lexer kernel (sm_100a).
//
// Restates the data-parallel lexer of futhark/lexer.fut:73-172 for one whole
// input in one launch (no 16 MiB host chunk loop):
//   * byte -> endomorphism and the inclusive "compose" scan
//     (futhark/lexer.fut:67-81): each thread folds its bytes with the step
//     table f' = f . class(byte) held in shared memory, the block combines
//     thread functions with the composition table, and tiles chain through a
//     decoupled look-back whose inclusive value is the DFA state itself;
//   * token-end flags, ignore filtering, the take_right start scan and the
//     compaction (futhark/lexer.fut:103-133): each thread re-runs the DFA
//     from its now-known start state; a second look-back carries
//     (token count, last token start) across tiles;
//   * the final token and the accept test (futhark/lexer.fut:161-172).
#pragma once
#include "common.cuh"

namespace alp {

constexpr int LEX_THREADS = 256;

// tokinfo bits
constexpr uint32_t TOK_IGNORE = 1u << 31;
constexpr uint32_t TOK_ACCEPT = 1u << 30;
constexpr uint32_t TOK_TERM_MASK = (1u << 30) - 1;

struct LexTables {
    const uint8_t* cls;       // [256] byte -> class
    const uint16_t* cdelta;   // [S][C1] next | produce<<15 (class C1-1 = identity pad)
    const uint32_t* tokinfo;  // [S] terminal | TOK_ACCEPT | TOK_IGNORE
    const uint16_t* step;     // [E][C1] endo after one more byte of the class
    const uint16_t* comp;     // [E][E]  comp[a*E+b] = a then b
    const uint16_t* apply;    // [E][S]  endo applied to a state
    int S, C1, E;
};

struct LexArgs {
    const uint8_t* in;
    long long n;
    int aligned16;                 // `in` is 16-byte aligned: vector loads allowed
    LexTables t;
    uint32_t* stA;                 // [tiles] endo / state look-back
    unsigned long long* stB;       // [tiles] (count, start) look-back
    unsigned int* ticket;
    void* out_term;
    void* out_start;
    void* out_end;
    long long cap;
    AlpResult* res;
    unsigned int num_tiles;        // tiles of the input; CTAs loop over tickets until done
    uint8_t* state_out;            // optional: DFA state entering each ITEMS-byte chunk (exact)
};

__host__ __device__ inline size_t lex_smem_bytes(int S, int C1, int E) {
    size_t b = 256 + 4 * (size_t)S + 2 * (size_t)S * C1;
    b = (b + 15) & ~(size_t)15;
    b += 2 * (size_t)E * C1;
    return (b + 15) & ~(size_t)15;
}

template <int ITEMS, typename TermT, typename PosT>
__global__ void __launch_bounds__(LEX_THREADS) lex_kernel(LexArgs a) {
    constexpr int TILE = LEX_THREADS * ITEMS;
    extern __shared__ __align__(16) uint8_t smem[];
    const int S = a.t.S, C1 = a.t.C1, E = a.t.E;
    uint8_t* s_cls = smem;
    uint32_t* s_tok = reinterpret_cast<uint32_t*>(smem + 256);
    uint16_t* s_cd = reinterpret_cast<uint16_t*>(smem + 256 + 4 * S);
    size_t off_step = (256 + 4 * (size_t)S + 2 * (size_t)S * C1 + 15) & ~(size_t)15;
    uint16_t* s_step = reinterpret_cast<uint16_t*>(smem + off_step);

    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_wagg[LEX_THREADS / 32];
    __shared__ uint32_t s_wexc[LEX_THREADS / 32];
    __shared__ uint32_t s_sin;
    __shared__ uint32_t s_wc[LEX_THREADS / 32], s_wp[LEX_THREADS / 32];
    __shared__ uint32_t s_xc, s_xp;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < 256; i += LEX_THREADS) s_cls[i] = a.t.cls[i];
    for (int i = tid; i < S; i += LEX_THREADS) s_tok[i] = a.t.tokinfo[i];
    for (int i = tid; i < S * C1; i += LEX_THREADS) s_cd[i] = a.t.cdelta[i];
    for (int i = tid; i < E * C1; i += LEX_THREADS) s_step[i] = a.t.step[i];
    const long long n = a.n;
    for (;;) {
    if (tid == 0) s_tile = atomicAdd(a.ticket, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= a.num_tiles) break;
    const long long my = (long long)tile * TILE + (long long)tid * ITEMS;
    const uint8_t PAD = (uint8_t)(C1 - 1);

    // ---- load ITEMS bytes as classes --------------------------------------
    uint8_t c[ITEMS];
    if (a.aligned16 && my + ITEMS <= n) {
#pragma unroll
        for (int v = 0; v < ITEMS / 16; ++v) {
            uint4 w = __ldg(reinterpret_cast<const uint4*>(a.in + my) + v);
            uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int j = 0; j < 16; ++j) c[v * 16 + j] = s_cls[(ws[j >> 2] >> (8 * (j & 3))) & 0xff];
        }
    } else {
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) c[j] = (my + j < n) ? s_cls[a.in[my + j]] : PAD;
    }

    // ---- phase A: this thread's endomorphism ------------------------------
    uint32_t f = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) f = s_step[f * C1 + c[j]];

    // block scan of endomorphisms (inclusive in warp, then across warps)
    uint32_t incl = f;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t o = __shfl_up_sync(ALP_FULL_MASK, incl, d);
        if (lane >= d) incl = __ldg(&a.t.comp[o * E + incl]);
    }
    uint32_t excl = __shfl_up_sync(ALP_FULL_MASK, incl, 1);
    if (lane == 0) excl = 0;
    if (lane == 31) s_wagg[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < LEX_THREADS / 32 ? s_wagg[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int d = 1; d < LEX_THREADS / 32; d <<= 1) {
            uint32_t o = __shfl_up_sync(ALP_FULL_MASK, wi, d);
            if (lane >= d) wi = __ldg(&a.t.comp[o * E + wi]);
        }
        uint32_t we = __shfl_up_sync(ALP_FULL_MASK, wi, 1);
        if (lane == 0) we = 0;
        if (lane < LEX_THREADS / 32) s_wexc[lane] = we;
        const uint32_t F = __shfl_sync(ALP_FULL_MASK, wi, LEX_THREADS / 32 - 1);

        // ---- look-back A: the DFA state entering this tile ----------------
        uint32_t sin;
        if (tile == 0) {
            sin = 1u;  // initial state
            if (lane == 0) st_volatile32(&a.stA[0], (ST_P << 30) | __ldg(&a.t.apply[F * S + sin]));
        } else {
            if (lane == 0) st_volatile32(&a.stA[tile], (ST_A << 30) | F);
            uint32_t acc = 0;
            long long end = tile;
            while (true) {
                long long idx = end - 32 + lane;
                uint32_t w2 = idx >= 0 ? wait32(&a.stA[idx], &a.res->error) : ((ST_P << 30) | 1u);
                uint32_t flag = w2 >> 30, val = w2 & 0x3fffffffu;
                uint32_t pm = __ballot_sync(ALP_FULL_MASK, flag == ST_P);
                if (pm) {
                    int p = 31 - __clz(pm);
                    uint32_t s = __shfl_sync(ALP_FULL_MASK, val, p);
                    for (int j = p + 1; j < 32; ++j) {
                        uint32_t aj = __shfl_sync(ALP_FULL_MASK, val, j);
                        s = __ldg(&a.t.apply[aj * S + s]);
                    }
                    sin = acc ? __ldg(&a.t.apply[acc * S + s]) : s;
                    break;
                }
                uint32_t g = 0;
                for (int j = 0; j < 32; ++j) {
                    uint32_t aj = __shfl_sync(ALP_FULL_MASK, val, j);
                    g = __ldg(&a.t.comp[g * E + aj]);
                }
                acc = __ldg(&a.t.comp[g * E + acc]);
                end -= 32;
            }
            if (lane == 0) st_volatile32(&a.stA[tile], (ST_P << 30) | __ldg(&a.t.apply[F * S + sin]));
        }
        if (lane == 0) s_sin = sin;
    }
    __syncthreads();
    const uint32_t fexc = __ldg(&a.t.comp[s_wexc[warp] * E + excl]);
    const uint32_t s0 = __ldg(&a.t.apply[fexc * S + s_sin]);
    if (a.state_out && my < n) a.state_out[my / ITEMS] = (uint8_t)s0;

    // ---- phase B: run the DFA once, recording token ends and starts -------
    // bit j of emit: a token ends just before byte j (its terminal in tk[j]);
    // bit j of stt: a token starts at byte j.
    uint32_t cnt = 0, lastp = ALP_NONE32, emit = 0, stt = 0;
    uint32_t tk[ITEMS];
    uint32_t s_last;
    {
        uint32_t s = s0;
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            uint32_t e = s_cd[s * C1 + c[j]];
            uint32_t s2 = e & 0x7fffu;
            tk[j] = 0;
            if (e & 0x8000u) {
                const uint32_t ti = s_tok[s];
                if (!(ti & TOK_IGNORE)) { ++cnt; emit |= 1u << j; tk[j] = ti & TOK_TERM_MASK; }
                if (!(s_tok[s2] & TOK_IGNORE)) { lastp = (uint32_t)(my + j); stt |= 1u << j; }
            }
            s = s2;
        }
        s_last = s;
    }
    uint32_t ic = cnt, ip = lastp;
    warp_scan_cs(ic, ip, lane);
    uint32_t ec = __shfl_up_sync(ALP_FULL_MASK, ic, 1), ep = __shfl_up_sync(ALP_FULL_MASK, ip, 1);
    if (lane == 0) { ec = 0; ep = ALP_NONE32; }
    if (lane == 31) { s_wc[warp] = ic; s_wp[warp] = ip; }
    __syncthreads();
    if (warp == 0) {
        uint32_t wc = lane < LEX_THREADS / 32 ? s_wc[lane] : 0u;
        uint32_t wp = lane < LEX_THREADS / 32 ? s_wp[lane] : ALP_NONE32;
        uint32_t bc = wc, bp = wp;
        warp_scan_cs(bc, bp, lane);
        uint32_t xc = __shfl_up_sync(ALP_FULL_MASK, bc, 1), xp = __shfl_up_sync(ALP_FULL_MASK, bp, 1);
        if (lane == 0) { xc = 0; xp = ALP_NONE32; }
        if (lane < LEX_THREADS / 32) { s_wc[lane] = xc; s_wp[lane] = xp; }
        const uint32_t Bc = __shfl_sync(ALP_FULL_MASK, bc, LEX_THREADS / 32 - 1);
        const uint32_t Bp = __shfl_sync(ALP_FULL_MASK, bp, LEX_THREADS / 32 - 1);

        // ---- look-back B: tokens and token start before this tile ---------
        uint32_t Xc, Xp;
        if (tile == 0) {
            Xc = 0; Xp = 0;  // the input starts a token at position 0
            if (lane == 0) st_volatile64(&a.stB[0], cs_pack(ST_P, Bc, Bp != ALP_NONE32 ? Bp : 0u));
        } else {
            if (lane == 0) st_volatile64(&a.stB[tile], cs_pack(ST_A, Bc, Bp));
            uint32_t acc_c = 0, acc_p = ALP_NONE32;
            long long end = tile;
            while (true) {
                long long idx = end - 32 + lane;
                unsigned long long w2 = idx >= 0 ? wait64(&a.stB[idx], &a.res->error) : cs_pack(ST_P, 0, 0);
                uint32_t flag = (uint32_t)(w2 >> 62);
                uint32_t pm = __ballot_sync(ALP_FULL_MASK, flag == ST_P);
                int p = pm ? 31 - __clz(pm) : -1;
                uint32_t vc = lane >= p ? cs_count(w2) : 0u;
                uint32_t vp = lane >= p ? cs_pos(w2) : ALP_NONE32;
                // reduce lanes in order: sum, take-right
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    uint32_t oc = __shfl_down_sync(ALP_FULL_MASK, vc, d);
                    uint32_t op = __shfl_down_sync(ALP_FULL_MASK, vp, d);
                    if (lane + d < 32) {
                        vc += oc;
                        if (op != ALP_NONE32) vp = op;
                    }
                }
                vc = __shfl_sync(ALP_FULL_MASK, vc, 0);
                vp = __shfl_sync(ALP_FULL_MASK, vp, 0);
                acc_c += vc;
                if (acc_p == ALP_NONE32) acc_p = vp;
                if (pm) break;
                end -= 32;
            }
            Xc = acc_c; Xp = acc_p;
            if (lane == 0) st_volatile64(&a.stB[tile], cs_pack(ST_P, Xc + Bc, Bp != ALP_NONE32 ? Bp : Xp));
        }
        if (lane == 0) { s_xc = Xc; s_xp = Xp; }
    }
    __syncthreads();

    // ---- phase B, pass 2: emit tokens -------------------------------------
    const uint32_t wxc = s_wc[warp], wxp = s_wp[warp];
    uint32_t tcount = s_xc + wxc + ec;
    uint32_t cur = ep != ALP_NONE32 ? ep : (wxp != ALP_NONE32 ? wxp : s_xp);
    TermT* o_term = reinterpret_cast<TermT*>(a.out_term);
    PosT* o_start = reinterpret_cast<PosT*>(a.out_start);
    PosT* o_end = reinterpret_cast<PosT*>(a.out_end);
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        if (emit & (1u << j)) {
            if ((long long)tcount < a.cap) {
                o_term[tcount] = (TermT)tk[j];
                o_start[tcount] = (PosT)cur;
                o_end[tcount] = (PosT)(my + j);
            } else {
                atomicOr(&a.res->error, ALP_DEV_ERR_CAPACITY);
            }
            ++tcount;
        }
        if (stt & (1u << j)) cur = (uint32_t)(my + j);
    }
    const uint32_t s = s_last;
    // ---- the final token and the accept test ------------------------------
    if (my <= n - 1 && n - 1 < my + ITEMS) {
        uint32_t ti = s_tok[s];
        long long total = tcount;
        if (!(ti & TOK_IGNORE)) {
            if (total < a.cap) {
                o_term[total] = (TermT)(ti & TOK_TERM_MASK);
                o_start[total] = (PosT)cur;
                o_end[total] = (PosT)n;
            } else {
                atomicOr(&a.res->error, ALP_DEV_ERR_CAPACITY);
            }
            ++total;
        }
        a.res->count = total;
        a.res->valid = (ti & TOK_ACCEPT) ? 1 : 0;
    }
    __syncthreads();  // shared words are rewritten by the next tile
    }
}

}  // namespace alp

namespace alp {

// ---------------------------------------------------------------------------
// Segmented lexer: many documents back to back in one launch.
//
// Each document is lexed exactly as the single-document kernel lexes one
// input (the reference API lexes one document per call): at a document's
// first byte the DFA restarts from the initial state and a token start is
// forced; at its last byte its final token is appended and its accept bit is
// its validity.  In the endomorphism scan a restart is a constant function,
// encoded as id E + state (ext_* below), so the same scan and look-backs
// carry it across threads and tiles.
//
// Outputs: tokens compacted in document order with spans relative to their
// document, tok_off[d] = index of document d's first token, valid[d].  With
// `sentinels` the tokens are laid out for the parser instead: document d
// occupies [tok_off[d] + 2d, tok_off[d+1] + 2d + 2) as ⊢, its tokens, ⊣.
// ---------------------------------------------------------------------------
struct LexSeg {
    const long long* doc_off;  // [n_docs + 1], doc_off[n_docs] = n
    long long n_docs;
    long long* tok_off;        // [n_docs + 1] out
    uint8_t* valid;            // [n_docs] out
    int sentinels;
    uint32_t sent_l, sent_r;   // ⊢ and ⊣ terminal ids
    int cont;                  // document 0 continues a stream: no head at byte 0 (lex3 only)
    long long end1;            // with doc_off null (one document): doc_off[1] (lex3 only)
};

// doc_off[d], or (0, end1) for a single document given without an offsets array
__device__ __forceinline__ long long seg_off(const LexSeg& sg, long long d) {
    return sg.doc_off ? sg.doc_off[d] : (d == 0 ? 0 : sg.end1);
}

__device__ __forceinline__ uint32_t ext_apply(const LexTables& t, uint32_t f, uint32_t s) {
    return f >= (uint32_t)t.E ? f - t.E : __ldg(&t.apply[f * t.S + s]);
}
__device__ __forceinline__ uint32_t ext_comp(const LexTables& t, uint32_t a, uint32_t b) {
    if (b >= (uint32_t)t.E) return b;
    if (a >= (uint32_t)t.E) return t.E + __ldg(&t.apply[b * t.S + (a - t.E)]);
    return __ldg(&t.comp[a * t.E + b]);
}

// largest d in [lo, hi] with off[d] <= p
__device__ __forceinline__ long long doc_upper(const long long* off, long long lo, long long hi, long long p) {
    while (lo < hi) {
        const long long mid = (lo + hi + 1) >> 1;
        if (off[mid] <= p) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Bytes of a thread live in four uint4 registers; byte j of the 64.
__device__ __forceinline__ uint32_t raw_byte(const uint4 (&w)[4], int j) {
    const uint4 v = w[j >> 4];
    const int q = (j >> 2) & 3;
    const uint32_t x = q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
    return (x >> (8 * (j & 3))) & 0xffu;
}

constexpr int SEG_ITEMS = 64;                      // bytes per thread
constexpr int SEG_TILE = LEX_THREADS * SEG_ITEMS;  // 16 KiB per tile

// One tile = 256 threads x 64 bytes.  Three short passes over the bytes held
// in registers: the endomorphism fold, a counting run of the DFA (token
// count and last start for the second look-back) and the emitting run.
template <typename TermT, typename PosT>
__global__ void __launch_bounds__(LEX_THREADS, 4) lex_seg_kernel(LexArgs a, LexSeg sg) {
    constexpr int ITEMS = SEG_ITEMS;
    constexpr int TILE = SEG_TILE;
    extern __shared__ __align__(16) uint8_t smem[];
    const int S = a.t.S, C1 = a.t.C1, E = a.t.E;
    uint8_t* s_cls = smem;
    uint32_t* s_tok = reinterpret_cast<uint32_t*>(smem + 256);
    uint16_t* s_cd = reinterpret_cast<uint16_t*>(smem + 256 + 4 * S);
    size_t off_step = (256 + 4 * (size_t)S + 2 * (size_t)S * C1 + 15) & ~(size_t)15;
    uint16_t* s_step = reinterpret_cast<uint16_t*>(smem + off_step);

    __shared__ uint32_t s_tile;
    __shared__ long long s_d0, s_d1;
    __shared__ uint32_t s_wagg[LEX_THREADS / 32];
    __shared__ uint32_t s_wexc[LEX_THREADS / 32];
    __shared__ uint32_t s_sin;
    __shared__ uint32_t s_wc[LEX_THREADS / 32], s_wp[LEX_THREADS / 32];
    __shared__ uint32_t s_xc, s_xp;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < 256; i += LEX_THREADS) s_cls[i] = a.t.cls[i];
    for (int i = tid; i < S; i += LEX_THREADS) s_tok[i] = a.t.tokinfo[i];
    for (int i = tid; i < S * C1; i += LEX_THREADS) s_cd[i] = a.t.cdelta[i];
    for (int i = tid; i < E * C1; i += LEX_THREADS) s_step[i] = a.t.step[i];
    const long long n = a.n;
    const long long ND = sg.n_docs;
    const uint32_t INIT = 1u;
    for (;;) {
        if (tid == 0) {
            s_tile = atomicAdd(a.ticket, 1u);
            if (s_tile < a.num_tiles) {
                const long long t0 = (long long)s_tile * TILE;
                const long long t1 = min(t0 + TILE, n) - 1;
                s_d0 = doc_upper(sg.doc_off, 0, ND - 1, t0);
                s_d1 = doc_upper(sg.doc_off, 0, ND - 1, t1);
            }
        }
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= a.num_tiles) break;
        const long long my = (long long)tile * TILE + (long long)tid * ITEMS;
        const long long d0 = s_d0, d1 = s_d1;
        const int lim = (int)max(0ll, min((long long)ITEMS, n - my));  // valid bytes of this thread

        // ---- bytes, document heads and last bytes --------------------------
        uint4 w[4];
        if (a.aligned16 && lim == ITEMS) {
#pragma unroll
            for (int v = 0; v < 4; ++v) w[v] = __ldg(reinterpret_cast<const uint4*>(a.in + my) + v);
        } else {
            uint32_t x[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                uint32_t y = 0;
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    if (q * 4 + b < lim) y |= (uint32_t)a.in[my + q * 4 + b] << (8 * b);
                x[q] = y;
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) w[v] = make_uint4(x[4 * v], x[4 * v + 1], x[4 * v + 2], x[4 * v + 3]);
        }
        unsigned long long head = 0, last = 0;
        long long mydoc = 0;
        if (lim > 0) {
            mydoc = doc_upper(sg.doc_off, d0, d1, my);
            if (sg.doc_off[mydoc] == my) head |= 1ull;
            for (long long d = mydoc + 1; d <= ND; ++d) {
                const long long h = sg.doc_off[d];
                if (h > my + ITEMS || h > n) break;
                if (h - 1 >= my) last |= 1ull << (int)(h - 1 - my);
                if (h < n && h < my + ITEMS) head |= 1ull << (int)(h - my);
            }
        }

        // ---- phase A: the endomorphism of this thread's bytes --------------
        uint32_t f = 0;
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            if (j < lim) {
                const uint32_t c = s_cls[raw_byte(w, j)];
                if ((head >> j) & 1ull) f = E + (s_cd[INIT * C1 + c] & 0x7fffu);
                else if (f >= (uint32_t)E) f = E + (s_cd[(f - E) * C1 + c] & 0x7fffu);
                else f = s_step[f * C1 + c];
            }
        }
        uint32_t incl = f;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t o = __shfl_up_sync(ALP_FULL_MASK, incl, d);
            if (lane >= d) incl = ext_comp(a.t, o, incl);
        }
        uint32_t excl = __shfl_up_sync(ALP_FULL_MASK, incl, 1);
        if (lane == 0) excl = 0;
        if (lane == 31) s_wagg[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t wv = lane < LEX_THREADS / 32 ? s_wagg[lane] : 0u;
            uint32_t wi = wv;
#pragma unroll
            for (int d = 1; d < LEX_THREADS / 32; d <<= 1) {
                uint32_t o = __shfl_up_sync(ALP_FULL_MASK, wi, d);
                if (lane >= d) wi = ext_comp(a.t, o, wi);
            }
            uint32_t we = __shfl_up_sync(ALP_FULL_MASK, wi, 1);
            if (lane == 0) we = 0;
            if (lane < LEX_THREADS / 32) s_wexc[lane] = we;
            const uint32_t F = __shfl_sync(ALP_FULL_MASK, wi, LEX_THREADS / 32 - 1);
            uint32_t sin;
            if (tile == 0) {
                sin = INIT;
                if (lane == 0) st_volatile32(&a.stA[0], (ST_P << 30) | ext_apply(a.t, F, sin));
            } else {
                if (lane == 0) st_volatile32(&a.stA[tile], (ST_A << 30) | F);
                uint32_t acc = 0;
                long long end = tile;
                while (true) {
                    long long idx = end - 32 + lane;
                    uint32_t w2 = idx >= 0 ? wait32(&a.stA[idx], &a.res->error) : ((ST_P << 30) | INIT);
                    uint32_t flag = w2 >> 30, val = w2 & 0x3fffffffu;
                    uint32_t pm = __ballot_sync(ALP_FULL_MASK, flag == ST_P);
                    if (pm) {
                        int p = 31 - __clz(pm);
                        uint32_t st = __shfl_sync(ALP_FULL_MASK, val, p);
                        for (int j = p + 1; j < 32; ++j) {
                            uint32_t aj = __shfl_sync(ALP_FULL_MASK, val, j);
                            st = ext_apply(a.t, aj, st);
                        }
                        sin = acc ? ext_apply(a.t, acc, st) : st;
                        break;
                    }
                    uint32_t gg = 0;
                    for (int j = 0; j < 32; ++j) {
                        uint32_t aj = __shfl_sync(ALP_FULL_MASK, val, j);
                        gg = ext_comp(a.t, gg, aj);
                    }
                    acc = ext_comp(a.t, gg, acc);
                    end -= 32;
                }
                if (lane == 0) st_volatile32(&a.stA[tile], (ST_P << 30) | ext_apply(a.t, F, sin));
            }
            if (lane == 0) s_sin = sin;
        }
        __syncthreads();
        const uint32_t s0 = ext_apply(a.t, ext_comp(a.t, s_wexc[warp], excl), s_sin);

        // ---- phase B, pass 1: tokens ending here and the last start --------
        uint32_t cnt = 0, lastp = ALP_NONE32;
        {
            uint32_t st = s0;
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                if (j < lim) {
                    if ((head >> j) & 1ull) { st = INIT; lastp = (uint32_t)(my + j); }
                    const uint32_t e = s_cd[st * C1 + s_cls[raw_byte(w, j)]];
                    const uint32_t s2 = e & 0x7fffu;
                    if (e & 0x8000u) {
                        if (!(s_tok[st] & TOK_IGNORE)) ++cnt;
                        if (!(s_tok[s2] & TOK_IGNORE)) lastp = (uint32_t)(my + j);
                    }
                    st = s2;
                    if (((last >> j) & 1ull) && !(s_tok[st] & TOK_IGNORE)) ++cnt;
                }
            }
        }
        uint32_t ic = cnt, ip = lastp;
        warp_scan_cs(ic, ip, lane);
        uint32_t ec = __shfl_up_sync(ALP_FULL_MASK, ic, 1), ep = __shfl_up_sync(ALP_FULL_MASK, ip, 1);
        if (lane == 0) { ec = 0; ep = ALP_NONE32; }
        if (lane == 31) { s_wc[warp] = ic; s_wp[warp] = ip; }
        __syncthreads();
        if (warp == 0) {
            uint32_t wc = lane < LEX_THREADS / 32 ? s_wc[lane] : 0u;
            uint32_t wp = lane < LEX_THREADS / 32 ? s_wp[lane] : ALP_NONE32;
            uint32_t bc = wc, bp = wp;
            warp_scan_cs(bc, bp, lane);
            uint32_t xc = __shfl_up_sync(ALP_FULL_MASK, bc, 1), xp = __shfl_up_sync(ALP_FULL_MASK, bp, 1);
            if (lane == 0) { xc = 0; xp = ALP_NONE32; }
            if (lane < LEX_THREADS / 32) { s_wc[lane] = xc; s_wp[lane] = xp; }
            const uint32_t Bc = __shfl_sync(ALP_FULL_MASK, bc, LEX_THREADS / 32 - 1);
            const uint32_t Bp = __shfl_sync(ALP_FULL_MASK, bp, LEX_THREADS / 32 - 1);
            uint32_t Xc, Xp;
            if (tile == 0) {
                Xc = 0; Xp = 0;
                if (lane == 0) st_volatile64(&a.stB[0], cs_pack(ST_P, Bc, Bp != ALP_NONE32 ? Bp : 0u));
            } else {
                if (lane == 0) st_volatile64(&a.stB[tile], cs_pack(ST_A, Bc, Bp));
                uint32_t acc_c = 0, acc_p = ALP_NONE32;
                long long end = tile;
                while (true) {
                    long long idx = end - 32 + lane;
                    unsigned long long w2 = idx >= 0 ? wait64(&a.stB[idx], &a.res->error) : cs_pack(ST_P, 0, 0);
                    uint32_t flag = (uint32_t)(w2 >> 62);
                    uint32_t pm = __ballot_sync(ALP_FULL_MASK, flag == ST_P);
                    int p = pm ? 31 - __clz(pm) : -1;
                    uint32_t vc = lane >= p ? cs_count(w2) : 0u;
                    uint32_t vp = lane >= p ? cs_pos(w2) : ALP_NONE32;
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        uint32_t oc = __shfl_down_sync(ALP_FULL_MASK, vc, d);
                        uint32_t op = __shfl_down_sync(ALP_FULL_MASK, vp, d);
                        if (lane + d < 32) {
                            vc += oc;
                            if (op != ALP_NONE32) vp = op;
                        }
                    }
                    vc = __shfl_sync(ALP_FULL_MASK, vc, 0);
                    vp = __shfl_sync(ALP_FULL_MASK, vp, 0);
                    acc_c += vc;
                    if (acc_p == ALP_NONE32) acc_p = vp;
                    if (pm) break;
                    end -= 32;
                }
                Xc = acc_c; Xp = acc_p;
                if (lane == 0) st_volatile64(&a.stB[tile], cs_pack(ST_P, Xc + Bc, Bp != ALP_NONE32 ? Bp : Xp));
            }
            if (lane == 0) { s_xc = Xc; s_xp = Xp; }
        }
        __syncthreads();

        // ---- phase B, pass 2: emit -----------------------------------------
        uint32_t tcount = s_xc + s_wc[warp] + ec;
        uint32_t cur = ep != ALP_NONE32 ? ep : (s_wp[warp] != ALP_NONE32 ? s_wp[warp] : s_xp);
        TermT* o_term = reinterpret_cast<TermT*>(a.out_term);
        PosT* o_start = reinterpret_cast<PosT*>(a.out_start);
        PosT* o_end = reinterpret_cast<PosT*>(a.out_end);
        long long doc = mydoc;
        long long base = lim > 0 ? sg.doc_off[doc] : 0;
        const long long sent = sg.sentinels ? 1 : 0;
        auto put = [&](long long idx, uint32_t term, long long st, long long en) {
            if (idx < a.cap) {
                o_term[idx] = (TermT)term;
                o_start[idx] = (PosT)st;
                o_end[idx] = (PosT)en;
            } else {
                atomicOr(&a.res->error, ALP_DEV_ERR_CAPACITY);
            }
        };
        {
            uint32_t st = s0;
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                if (j < lim) {
                    const long long pos = my + j;
                    if ((head >> j) & 1ull) {
                        // every document starting here (empty ones first, then the real one)
                        doc = doc_upper(sg.doc_off, d0, d1, pos);
                        long long dl = doc;  // empty documents that start here too
                        while (dl > 0 && sg.doc_off[dl - 1] >= pos) --dl;
                        base = pos;
                        for (long long e = dl; e <= doc; ++e) {
                            sg.tok_off[e] = tcount;
                            if (sent) put((long long)tcount + 2 * e, sg.sent_l, 0, 0);
                            if (e < doc) {
                                sg.valid[e] = 0;
                                if (sent) put((long long)tcount + 2 * e + 1, sg.sent_r, 0, 0);
                            }
                        }
                        cur = (uint32_t)pos;
                        st = INIT;
                    }
                    const uint32_t e = s_cd[st * C1 + s_cls[raw_byte(w, j)]];
                    const uint32_t s2 = e & 0x7fffu;
                    if (e & 0x8000u) {
                        const uint32_t ti = s_tok[st];
                        if (!(ti & TOK_IGNORE)) {
                            put((long long)tcount + sent * (2 * doc + 1), ti & TOK_TERM_MASK, (long long)cur - base, pos - base);
                            ++tcount;
                        }
                        if (!(s_tok[s2] & TOK_IGNORE)) cur = (uint32_t)pos;
                    }
                    st = s2;
                    if ((last >> j) & 1ull) {
                        const uint32_t ti = s_tok[st];
                        if (!(ti & TOK_IGNORE)) {
                            put((long long)tcount + sent * (2 * doc + 1), ti & TOK_TERM_MASK, (long long)cur - base,
                                pos + 1 - base);
                            ++tcount;
                        }
                        sg.valid[doc] = (ti & TOK_ACCEPT) ? 1 : 0;
                        if (sent) put((long long)tcount + 2 * doc + 1, sg.sent_r, 0, 0);
                    }
                }
            }
        }
        if (my <= n - 1 && n - 1 < my + ITEMS) {
            // documents that start at n (empty, at the end) and the closing offset
            for (long long e = doc + 1; e < ND; ++e) {
                sg.tok_off[e] = tcount;
                sg.valid[e] = 0;
                if (sent) {
                    put((long long)tcount + 2 * e, sg.sent_l, 0, 0);
                    put((long long)tcount + 2 * e + 1, sg.sent_r, 0, 0);
                }
            }
            sg.tok_off[ND] = tcount;
            a.res->count = tcount;
            a.res->valid = 1;
        }
        __syncthreads();
    }
}

}  // namespace alp
