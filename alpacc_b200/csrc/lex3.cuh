// Multi-kernel lexer for DFAs of at most 32 states (sm_100a).
//
// Same results as lex_seg_kernel (futhark/lexer.fut:73-172 per document),
// split so that no step waits on another tile or on table lookups in L2:
//
//   lex3_fold_kernel   every 32-byte chunk -> its endomorphism id, folded with
//                      the step table in shared memory (constant E+s after a
//                      document head).  Two independent chunks per thread.
//   lex3_scan_kernel   the composition scan over chunk endomorphisms.  With
//                      S <= 32 one warp holds a whole function, lane s the
//                      image of state s, so composing two functions is one
//                      shuffle and a tile's aggregate is 32 bytes.  Lanes walk
//                      the chunks of their warp through the apply table in
//                      shared memory; tiles chain through a decoupled look-back
//                      on these vectors.  Output: the state entering each chunk.
//   lex3_count_kernel  the token-end flags and ignore filter (futhark/lexer.fut:
//                      103-107) as counts: each thread runs the DFA over two
//                      chunks from their known states with a 256-column table
//                      whose entries carry the produce/ignore decisions, and
//                      stores the chunk's token count and last token start.
//   lex3_tile_reduce_kernel, lex3_tile_scan_kernel  exclusive (count, last
//                      start) over 8 KiB tiles, the
//                      take_right start scan and the compaction offsets
//                      (futhark/lexer.fut:83-84,108-120) at tile level.
//   lex3_emit_kernel   the compaction (futhark/lexer.fut:121-133): places each
//                      thread from the stored counts, runs the DFA once more,
//                      stages the tile's tokens in shared memory and writes
//                      them with coalesced stores.
#pragma once
#include "common.cuh"
#include "lexer.cuh"

namespace alp {

constexpr int LX_THREADS = 256;
constexpr int LX_CHUNK = 32;                    // bytes per chunk, the unit of the state scan
constexpr int LX_TILE = LX_THREADS * LX_CHUNK;  // 8 KiB emit tile: one chunk per thread
constexpr int LX_WIDE = 2 * LX_TILE;            // 16 KiB fold / count tile: two chunks per thread
constexpr int LX_STAGE = 2048;                  // tokens one emit tile stages in shared memory
constexpr int LS_WARPS = 8;
constexpr int LS_G = 16;                        // chunks per lane in the state scan (default; 8, 16 or 32)
__host__ __device__ constexpr long long ls_tile(int g) { return (long long)LS_WARPS * 32 * g; }  // chunks per scan tile

// ent entries: next state | flags.  Rows are LX_ROW entries apart so that
// lanes reading the same byte in different states hit different banks.
constexpr int LX_ROW = 258;
constexpr uint32_t LX_NEXT = 0x1fu;
constexpr uint32_t LX_START = 1u << 5;  // a kept token starts at this byte
constexpr uint32_t LX_EMIT = 1u << 6;   // a kept token of term(st) ends before this byte
constexpr int LX_TERM_SHIFT = 7;        // with LX_EMIT: term(st), the ended token's terminal (< 512)
constexpr uint32_t LX_NOOFF = 0xffu;    // chunk_c: no token start in the chunk

struct Lex3Tables {
    const uint8_t* cls;       // [256] byte -> class
    const uint16_t* cdelta;   // [S][C1] next | produce<<15
    const uint16_t* step;     // [E][C1] endo after one more byte of the class
    const uint8_t* app8;      // [E+S][32] state after endo f from state s; rows E+s are constant s;
                              // identity beyond S in rows < E
    const uint16_t* ent;      // [S][LX_ROW] next | LX_START | LX_EMIT | term << LX_TERM_SHIFT (columns 256.. unused)
    const uint32_t* tokinfo;  // [S] terminal | TOK_ACCEPT | TOK_IGNORE
    int S, C1, E;
};

// What one piece of a token stream hands to the next, in device memory (the
// reference's chunk loop carries (state, last start, size) the same way:
// futhark/lexer.fut:148-160, cuda/lexer.cu:105-117,397-407).
struct __align__(16) LexCarry {
    long long start;    // stream position where the kept token in progress started
    long long tokens;   // tokens written so far
    long long piece;    // tokens the last piece wrote
    uint32_t state;     // DFA state after the bytes so far
    uint32_t error;     // ALP_DEV_ERR_* bits of all pieces
    int valid;          // set when the stream ends
    int pad;
};

struct Lex3Args {
    const uint8_t* in;
    long long n;
    int aligned16;
    Lex3Tables t;
    long long n_chunks;            // ceil(n / 32)
    uint16_t* chunk_f;             // [n_chunks] endomorphism of each chunk (E + s: constant s)
    uint8_t* chunk_s;              // [n_chunks] state entering each chunk
    uint16_t* chunk_c;             // [n_chunks] tokens ending in the chunk | last start offset << 8
    unsigned long long* tile_cs;   // [tiles] count << 32 | last start; inclusive per tile, then exclusive
    uint32_t* lb_vec;              // [scan tiles][32] state-scan look-back words
    unsigned int* tickets;         // [0] state scan
    const long long* tile_doc;     // [tiles] document holding each 8 KiB tile's first byte (n_docs > 1)
    void* out_term;
    void* out_start;
    void* out_end;
    long long cap;
    AlpResult* res;
    unsigned int num_tiles;        // 8 KiB tiles
    unsigned int num_wide;         // 16 KiB tiles
    unsigned int num_scan_tiles;   // ls_tile(G)-chunk tiles of the state scan
    LexCarry* carry;               // stream piece: entry state and token start (null: plain input)
    long long pos_base;            // stream position of in[0] (added to output positions)
    int carry_tokens;              // outputs start at index carry->tokens - tok_first (else 0)
    long long tok_first;           // stream token stored at element 0 of the outputs
};

__host__ __device__ inline size_t lex3_fold_smem(int S, int C1, int E) {
    size_t b = 256 + 2 * (size_t)S * C1;
    b = (b + 15) & ~(size_t)15;
    b += 2 * (size_t)E * C1;
    return (b + 15) & ~(size_t)15;
}
__host__ __device__ inline size_t lex3_scan_smem(int S, int E) {
    return (32 * ((size_t)E + S) + 15) & ~(size_t)15;
}
__host__ __device__ inline size_t lex3_tok_off(int S) { return (2 * (size_t)S * LX_ROW + 15) & ~(size_t)15; }
__host__ __device__ inline size_t lex3_stage_off(int S) { return (lex3_tok_off(S) + 4 * (size_t)S + 15) & ~(size_t)15; }
__host__ __device__ inline size_t lex3_count_smem(int S) { return lex3_stage_off(S); }
__host__ __device__ inline size_t lex3_emit_smem(int S) { return lex3_stage_off(S) + (size_t)LX_STAGE * 8; }

template <int NV>
__device__ __forceinline__ uint32_t byte_of(const uint4 (&w)[NV], int j) {
    const uint4 v = w[j >> 4];
    const int q = (j >> 2) & 3;
    const uint32_t x = q == 0 ? v.x : (q == 1 ? v.y : (q == 2 ? v.z : v.w));
    return (x >> (8 * (j & 3))) & 0xffu;
}

// tile_doc[t] = the document holding byte t*LX_TILE.  Every tile start lies
// in exactly one non-empty document's [off[d], off[d+1]).
__global__ void lex3_tile_doc_kernel(const long long* off, long long nd, long long* tile_doc, long long tiles) {
    for (long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x; d < nd;
         d += (long long)gridDim.x * blockDim.x) {
        const long long lo = off[d], hi = off[d + 1];
        for (long long t = lo > 0 ? (lo + LX_TILE - 1) / LX_TILE : 0; t < tiles && t * LX_TILE < hi; ++t)
            tile_doc[t] = d;
    }
}

// Document heads and last bytes of tile [t0, t1] as per-chunk bit masks
// (bit j of word c: byte t0 + 32c + j); *s_dmax = the last document with a
// byte at or before t1.
// With s_doff, also s_doff[d - d0] = off[d] for the first LX_DOCS documents.
constexpr int LX_DOCS = 64;
__device__ __forceinline__ void lx_mark_docs(const LexSeg& sg, long long n, long long d0, long long t0, long long t1,
                                             uint32_t* s_head, uint32_t* s_last, unsigned long long* s_dmax,
                                             uint32_t* s_doff = nullptr) {
    for (long long d = d0 + threadIdx.x; d <= sg.n_docs; d += blockDim.x) {
        const long long h = seg_off(sg, d);
        if (h > t1 + 1) break;
        if (s_doff && d - d0 < LX_DOCS) s_doff[d - d0] = (uint32_t)h;
        if (h >= t0 && h <= t1 && h < n && !(sg.cont && d == 0)) {
            const long long r = h - t0;
            atomicOr(&s_head[r >> 5], 1u << (r & 31));
        }
        if (s_last && h - 1 >= t0 && h - 1 <= t1) {
            const long long r = h - 1 - t0;
            atomicOr(&s_last[r >> 5], 1u << (r & 31));
        }
        if (s_dmax && h <= t1 && d < sg.n_docs) atomicMax(s_dmax, (unsigned long long)d);
    }
}

// The (up to) 16*NV bytes starting at `my`.
template <int NV>
__device__ __forceinline__ void lx_load(const Lex3Args& a, long long my, int lim, uint4 (&w)[NV]) {
    if (a.aligned16 && lim == 16 * NV) {
#pragma unroll
        for (int v = 0; v < NV; ++v) w[v] = __ldg(reinterpret_cast<const uint4*>(a.in + my) + v);
    } else {
        uint32_t x[4 * NV];
#pragma unroll
        for (int q = 0; q < 4 * NV; ++q) {
            uint32_t y = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b)
                if (q * 4 + b < lim) y |= (uint32_t)a.in[my + q * 4 + b] << (8 * b);
            x[q] = y;
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) w[v] = make_uint4(x[4 * v], x[4 * v + 1], x[4 * v + 2], x[4 * v + 3]);
    }
}

// ---- kernel 1: chunk endomorphisms ------------------------------------------

// One chunk's endomorphism from bytes in[0, lim), with document heads (a
// compact loop: only chunks at document heads or the input's end).
__device__ __forceinline__ uint32_t lx_fold_slow(const uint8_t* in, int lim, uint32_t head,
                                                 const uint8_t* s_cls, const uint16_t* s_cd, const uint16_t* s_step,
                                                 int C1, uint32_t E) {
    uint32_t f = 0;
#pragma unroll 1
    for (int j = 0; j < lim; ++j) {
        {
            const uint32_t c = s_cls[__ldg(in + j)];
            if ((head >> j) & 1u) f = E + (s_cd[1 * C1 + c] & 0x7fffu);
            else if (f >= E) f = E + (s_cd[(f - E) * C1 + c] & 0x7fffu);
            else f = s_step[f * C1 + c];
        }
    }
    return f;
}

__global__ void __launch_bounds__(LX_THREADS, 4) lex3_fold_kernel(Lex3Args a, LexSeg sg) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int S = a.t.S, C1 = a.t.C1;
    const uint32_t E = (uint32_t)a.t.E;
    uint8_t* s_cls = smem;
    uint16_t* s_cd = reinterpret_cast<uint16_t*>(smem + 256);
    const size_t off_step = (256 + 2 * (size_t)S * C1 + 15) & ~(size_t)15;
    uint16_t* s_step = reinterpret_cast<uint16_t*>(smem + off_step);
    __shared__ uint32_t s_head[LX_WIDE / LX_CHUNK];

    const int tid = threadIdx.x;
    for (int i = tid; i < 256; i += LX_THREADS) s_cls[i] = a.t.cls[i];
    for (int i = tid; i < S * C1; i += LX_THREADS) s_cd[i] = a.t.cdelta[i];
    for (int i = tid; i < (int)E * C1; i += LX_THREADS) s_step[i] = a.t.step[i];
    const long long n = a.n;
    // this thread's 64 bytes of a tile, one tile ahead (in flight while the block folds
    // the tile before)
    uint4 nw[4];
    auto tile_bytes = [&](unsigned ft, uint4 (&w)[4]) {
        const long long my = (long long)ft * LX_WIDE + (long long)tid * (2 * LX_CHUNK);
        const int lim = (int)max(0ll, min((long long)(2 * LX_CHUNK), n - my));
        if (lim > 0) lx_load<4>(a, my, lim, w);
    };
    if (blockIdx.x < a.num_wide) tile_bytes(blockIdx.x, nw);
    for (unsigned ft = blockIdx.x; ft < a.num_wide; ft += gridDim.x) {
        const long long t0 = (long long)ft * LX_WIDE;
        const long long t1 = min(t0 + LX_WIDE, n) - 1;
        uint4 w[4] = {nw[0], nw[1], nw[2], nw[3]};
        if (ft + gridDim.x < a.num_wide) tile_bytes(ft + gridDim.x, nw);
        s_head[tid] = 0;
        s_head[tid + LX_THREADS] = 0;
        __syncthreads();
        lx_mark_docs(sg, n, sg.n_docs > 1 ? a.tile_doc[2 * (size_t)ft] : 0, t0, t1, s_head, nullptr, nullptr);
        __syncthreads();
        const long long my = t0 + (long long)tid * (2 * LX_CHUNK);
        const int lim = (int)max(0ll, min((long long)(2 * LX_CHUNK), n - my));
        if (lim > 0) {
            const uint32_t ha = s_head[2 * tid], hb = s_head[2 * tid + 1];
            const long long c = my / LX_CHUNK;
            if (lim == 2 * LX_CHUNK && (ha | hb) == 0) {
                uint32_t fa = 0, fb = 0;
#pragma unroll
                for (int j = 0; j < LX_CHUNK; ++j) {
                    fa = s_step[fa * C1 + s_cls[byte_of(w, j)]];
                    fb = s_step[fb * C1 + s_cls[byte_of(w, LX_CHUNK + j)]];
                }
                *reinterpret_cast<uint32_t*>(a.chunk_f + c) = fa | (fb << 16);
            } else {
                a.chunk_f[c] = (uint16_t)lx_fold_slow(a.in + my, min(lim, LX_CHUNK), ha, s_cls, s_cd, s_step, C1, E);
                if (lim > LX_CHUNK)
                    a.chunk_f[c + 1] =
                        (uint16_t)lx_fold_slow(a.in + my + LX_CHUNK, lim - LX_CHUNK, hb, s_cls, s_cd, s_step, C1, E);
            }
        }
        __syncthreads();
    }
}

// ---- kernel 2: states entering the chunks -----------------------------------
// G chunks per lane (a tuned launch shape: 8, 16 or 32).
template <int G>
__global__ void __launch_bounds__(LS_WARPS * 32) lex3_scan_kernel(Lex3Args a) {
    static_assert(G == 8 || G == 16 || G == 32, "chunks per lane");
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t rows = (uint32_t)(a.t.E + a.t.S);
    uint8_t* s_app = smem;
    __shared__ uint8_t s_sv[LS_WARPS][32][32];  // [warp][lane segment][start state] -> state
    __shared__ uint8_t s_wagg[LS_WARPS][32];
    __shared__ uint8_t s_wpre[LS_WARPS][32];
    __shared__ uint32_t s_tile, s_sin;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.t.app8);
        uint4* dst = reinterpret_cast<uint4*>(s_app);
        for (uint32_t i = tid; i < rows * 2; i += LS_WARPS * 32) dst[i] = src[i];
    }
    const uint32_t INIT = 1u;
    const long long M = a.n_chunks;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(&a.tickets[0], 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= a.num_scan_tiles) break;
        const long long base = (long long)tile * ls_tile(G) + (long long)warp * (32 * G) + (long long)lane * G;

        // this lane's G chunk endomorphisms, two per word
        uint32_t fr[G / 2];
        if (base + G <= M) {
            const uint4* p = reinterpret_cast<const uint4*>(a.chunk_f + base);
#pragma unroll
            for (int v = 0; v < G / 8; ++v) {
                const uint4 x = p[v];
                fr[4 * v] = x.x; fr[4 * v + 1] = x.y; fr[4 * v + 2] = x.z; fr[4 * v + 3] = x.w;
            }
        } else {
#pragma unroll
            for (int q = 0; q < G / 2; ++q) {
                const uint32_t lo = base + 2 * q < M ? a.chunk_f[base + 2 * q] : 0u;
                const uint32_t hi = base + 2 * q + 1 < M ? a.chunk_f[base + 2 * q + 1] : 0u;
                fr[q] = lo | (hi << 16);
            }
        }

        // lane s follows state s through the warp's 512 chunks
        uint32_t cur = (uint32_t)lane;
        for (int l2 = 0; l2 < 32; ++l2) {
            s_sv[warp][l2][lane] = (uint8_t)cur;
#pragma unroll
            for (int q = 0; q < G / 2; ++q) {
                const uint32_t v = __shfl_sync(ALP_FULL_MASK, fr[q], l2);
                cur = s_app[(v & 0xffffu) * 32 + cur];
                cur = s_app[(v >> 16) * 32 + cur];
            }
        }
        s_wagg[warp][lane] = (uint8_t)cur;
        __syncthreads();

        if (warp == 0) {
            uint32_t x = (uint32_t)lane;
#pragma unroll
            for (int w = 0; w < LS_WARPS; ++w) {
                s_wpre[w][lane] = (uint8_t)x;
                x = s_wagg[w][x];
            }
            // x = the tile's function: lane s -> state after the tile from s
            uint32_t sin = a.carry ? a.carry->state : INIT;
            if (tile > 0) {
                st_volatile32(&a.lb_vec[(size_t)tile * 32 + lane], (ST_A << 30) | x);
                uint32_t acc = (uint32_t)lane;  // composition of the aggregates passed so far
                long long j = (long long)tile - 1;
                bool done = false;
                while (!done) {
                    uint32_t wv[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        wv[q] = j - q >= 0 ? ld_volatile32(&a.lb_vec[(size_t)(j - q) * 32 + lane])
                                           : ((ST_P << 30) | INIT);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (!done) {
                            uint32_t wq = wv[q];
                            if ((wq >> 30) == ST_X) wq = wait32(&a.lb_vec[(size_t)(j - q) * 32 + lane], &a.res->error);
                            const uint32_t val = wq & 0x3fffffffu;
                            const uint32_t pm = __ballot_sync(ALP_FULL_MASK, (wq >> 30) == ST_P);
                            if (pm) {
                                const uint32_t st = __shfl_sync(ALP_FULL_MASK, val, __ffs(pm) - 1) & 31u;
                                sin = __shfl_sync(ALP_FULL_MASK, acc, st);
                                done = true;
                            } else {
                                acc = __shfl_sync(ALP_FULL_MASK, acc, val & 31u);
                            }
                        }
                    }
                    j -= 4;
                }
            }
            const uint32_t out = __shfl_sync(ALP_FULL_MASK, x, sin & 31u);
            st_volatile32(&a.lb_vec[(size_t)tile * 32 + lane], (ST_P << 30) | out);
            if (lane == 0) s_sin = sin;
        }
        __syncthreads();

        const uint32_t win = s_wpre[warp][s_sin & 31u];
        uint32_t st = s_sv[warp][lane][win];
        uint32_t ob[G / 4];
#pragma unroll
        for (int q = 0; q < G / 4; ++q) ob[q] = 0;
#pragma unroll
        for (int q = 0; q < G / 2; ++q) {
            ob[q >> 1] |= st << (16 * (q & 1));
            st = s_app[(fr[q] & 0xffffu) * 32 + st];
            ob[q >> 1] |= st << (16 * (q & 1) + 8);
            st = s_app[(fr[q] >> 16) * 32 + st];
        }
        if (base + G <= M) {
            if constexpr (G == 8) {
                *reinterpret_cast<uint2*>(a.chunk_s + base) = make_uint2(ob[0], ob[1]);
            } else {
#pragma unroll
                for (int v = 0; v < G / 16; ++v)
                    reinterpret_cast<uint4*>(a.chunk_s + base)[v] =
                        make_uint4(ob[4 * v], ob[4 * v + 1], ob[4 * v + 2], ob[4 * v + 3]);
            }
        } else {
#pragma unroll
            for (int g = 0; g < G; ++g)
                if (base + g < M) a.chunk_s[base + g] = (uint8_t)(ob[g >> 2] >> (8 * (g & 3)));
        }
        __syncthreads();
    }
}

// ---- kernel 3: token counts -------------------------------------------------

// Tokens ending in bytes in[0, lim) from state st, with document heads and
// last bytes; *lastoff = offset of the last token start or LX_NOOFF.  A
// compact loop: only chunks at document boundaries or the input's end.
__device__ __forceinline__ uint32_t lx_count_slow(const uint8_t* in, int lim, uint32_t st, uint32_t head,
                                                  uint32_t last, const uint16_t* s_ent, const uint32_t* s_tok,
                                                  uint32_t* lastoff) {
    uint32_t cnt = 0, lo = LX_NOOFF;
#pragma unroll 1
    for (int j = 0; j < lim; ++j) {
        {
            if ((head >> j) & 1u) { st = 1u; lo = (uint32_t)j; }
            const uint32_t e = s_ent[st * LX_ROW + __ldg(in + j)];
            cnt += (e >> 6) & 1u;
            if (e & LX_START) lo = (uint32_t)j;
            st = e & LX_NEXT;
            if (((last >> j) & 1u) && !(s_tok[st] & TOK_IGNORE)) ++cnt;
        }
    }
    *lastoff = lo;
    return cnt;
}

// (count, last position) combine over a warp: counts add, the position takes
// the right operand unless it is NONE.  Lane 0 ends with the total.
__device__ __forceinline__ void cs_reduce_warp(uint32_t& c, uint32_t& p) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t oc = __shfl_down_sync(ALP_FULL_MASK, c, d);
        const uint32_t op = __shfl_down_sync(ALP_FULL_MASK, p, d);
        c += oc;
        if (op != ALP_NONE32) p = op;
    }
}

__global__ void __launch_bounds__(LX_THREADS, 6) lex3_count_kernel(Lex3Args a, LexSeg sg) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int S = a.t.S;
    uint16_t* s_ent = reinterpret_cast<uint16_t*>(smem);
    uint32_t* s_tok = reinterpret_cast<uint32_t*>(smem + lex3_tok_off(S));
    __shared__ uint32_t s_head[LX_WIDE / LX_CHUNK], s_last[LX_WIDE / LX_CHUNK];
    __shared__ uint32_t s_wc[LX_THREADS / 32], s_wp[LX_THREADS / 32];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.t.ent);
        uint4* dst = reinterpret_cast<uint4*>(s_ent);
        for (int i = tid; i < (S * LX_ROW * 2 + 15) / 16; i += LX_THREADS) dst[i] = src[i];
    }
    for (int i = tid; i < S; i += LX_THREADS) s_tok[i] = a.t.tokinfo[i];
    const long long n = a.n;
    for (unsigned ft = blockIdx.x; ft < a.num_wide; ft += gridDim.x) {
        const long long t0 = (long long)ft * LX_WIDE;
        const long long t1 = min(t0 + LX_WIDE, n) - 1;
        s_head[tid] = 0;
        s_head[tid + LX_THREADS] = 0;
        s_last[tid] = 0;
        s_last[tid + LX_THREADS] = 0;
        __syncthreads();
        lx_mark_docs(sg, n, sg.n_docs > 1 ? a.tile_doc[2 * (size_t)ft] : 0, t0, t1, s_head, s_last, nullptr);
        __syncthreads();
        const long long my = t0 + (long long)tid * (2 * LX_CHUNK);
        const int lim = (int)max(0ll, min((long long)(2 * LX_CHUNK), n - my));
        uint32_t cnt = 0, lastp = ALP_NONE32;
        if (lim > 0) {
            uint4 w[4];
            lx_load<4>(a, my, lim, w);
            const long long c = my / LX_CHUNK;
            const uint32_t ha = s_head[2 * tid], hb = s_head[2 * tid + 1];
            const uint32_t la = s_last[2 * tid], lb = s_last[2 * tid + 1];
            uint32_t ca, cb = 0, oa, ob = LX_NOOFF;
            if (lim == 2 * LX_CHUNK && (ha | hb | la | lb) == 0) {
                const uint32_t sab = *reinterpret_cast<const uint16_t*>(a.chunk_s + c);
                uint32_t sa = sab & 0xffu, sb = sab >> 8;
                ca = 0;
                oa = LX_NOOFF;
#pragma unroll
                for (int j = 0; j < LX_CHUNK; ++j) {
                    const uint32_t ea = s_ent[sa * LX_ROW + byte_of(w, j)];
                    const uint32_t eb = s_ent[sb * LX_ROW + byte_of(w, LX_CHUNK + j)];
                    ca += (ea >> 6) & 1u;
                    cb += (eb >> 6) & 1u;
                    if (ea & LX_START) oa = (uint32_t)j;
                    if (eb & LX_START) ob = (uint32_t)j;
                    sa = ea & LX_NEXT;
                    sb = eb & LX_NEXT;
                }
                *reinterpret_cast<uint32_t*>(a.chunk_c + c) = (ca | (oa << 8)) | ((cb | (ob << 8)) << 16);
            } else {
                ca = lx_count_slow(a.in + my, min(lim, LX_CHUNK), a.chunk_s[c], ha, la, s_ent, s_tok, &oa);
                a.chunk_c[c] = (uint16_t)(ca | (oa << 8));
                if (lim > LX_CHUNK) {
                    cb = lx_count_slow(a.in + my + LX_CHUNK, lim - LX_CHUNK, a.chunk_s[c + 1], hb, lb, s_ent, s_tok,
                                       &ob);
                    a.chunk_c[c + 1] = (uint16_t)(cb | (ob << 8));
                }
            }
            cnt = ca + cb;
            lastp = ob != LX_NOOFF ? (uint32_t)(my + LX_CHUNK + ob)
                                   : (oa != LX_NOOFF ? (uint32_t)(my + oa) : ALP_NONE32);
        }
        // per 8 KiB tile (threads 0..127 and 128..255): count and last start
        cs_reduce_warp(cnt, lastp);
        if (lane == 0) { s_wc[warp] = cnt; s_wp[warp] = lastp; }
        __syncthreads();
        if (tid == 0 || tid == LX_THREADS / 2) {
            const int w0 = tid / 32;
            uint32_t c = 0, p = ALP_NONE32;
            for (int w2 = w0; w2 < w0 + LX_THREADS / 64; ++w2) {
                c += s_wc[w2];
                if (s_wp[w2] != ALP_NONE32) p = s_wp[w2];
            }
            const size_t t8 = 2 * (size_t)ft + (tid ? 1 : 0);
            if (t8 < a.num_tiles) a.tile_cs[t8] = ((unsigned long long)c << 32) | p;
        }
        __syncthreads();
    }
}

// ---- kernel 4: exclusive (count, last start) over tiles ---------------------
// Two launches over chunks of LT_CHUNK tiles: the chunk sums, then one CTA per
// chunk scans the chunk sums before its own and its own tiles in place.
// Tile 0 starts from (0, NONE): no token start before the input.
constexpr int LT_CHUNK = 1024;

__device__ __forceinline__ void cs_unpack(unsigned long long v, uint32_t& c, uint32_t& p) {
    c = (uint32_t)(v >> 32);
    p = (uint32_t)v;
}

__global__ void __launch_bounds__(LT_CHUNK) lex3_tile_reduce_kernel(const unsigned long long* tile_cs, long long T,
                                                                    unsigned long long* chunk_cs) {
    __shared__ uint32_t s_c[LT_CHUNK / 32], s_p[LT_CHUNK / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long i = (long long)blockIdx.x * LT_CHUNK + tid;
    uint32_t c = 0, p = ALP_NONE32;
    if (i < T) cs_unpack(tile_cs[i], c, p);
    cs_reduce_warp(c, p);
    if (lane == 0) { s_c[warp] = c; s_p[warp] = p; }
    __syncthreads();
    if (tid == 0) {
        uint32_t tc = 0, tp = ALP_NONE32;
        for (int w = 0; w < LT_CHUNK / 32; ++w) {
            tc += s_c[w];
            if (s_p[w] != ALP_NONE32) tp = s_p[w];
        }
        chunk_cs[blockIdx.x] = ((unsigned long long)tc << 32) | tp;
    }
}

__global__ void __launch_bounds__(LT_CHUNK) lex3_tile_scan_kernel(unsigned long long* tile_cs, long long T,
                                                                  const unsigned long long* chunk_cs) {
    __shared__ uint32_t s_c[LT_CHUNK / 32], s_p[LT_CHUNK / 32];
    __shared__ uint32_t s_cc, s_cp;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long chunk = blockIdx.x;
    if (warp == 0) {
        uint32_t cc = 0, cp = ALP_NONE32;
        for (long long b = 0; b < chunk; b += 32) {
            uint32_t c = 0, p = ALP_NONE32;
            if (b + lane < chunk) cs_unpack(chunk_cs[b + lane], c, p);
            cs_reduce_warp(c, p);
            c = __shfl_sync(ALP_FULL_MASK, c, 0);
            p = __shfl_sync(ALP_FULL_MASK, p, 0);
            cc += c;
            if (p != ALP_NONE32) cp = p;
        }
        if (lane == 0) { s_cc = cc; s_cp = cp; }
    }
    const long long i = chunk * LT_CHUNK + tid;
    uint32_t c = 0, p = ALP_NONE32;
    if (i < T) cs_unpack(tile_cs[i], c, p);
    uint32_t ic = c, ip = p;
    warp_scan_cs(ic, ip, lane);
    if (lane == 31) { s_c[warp] = ic; s_p[warp] = ip; }
    __syncthreads();
    if (warp == 0) {
        uint32_t wc = s_c[lane], wp = s_p[lane];
        warp_scan_cs(wc, wp, lane);
        uint32_t xc = __shfl_up_sync(ALP_FULL_MASK, wc, 1), xp = __shfl_up_sync(ALP_FULL_MASK, wp, 1);
        if (lane == 0) { xc = 0; xp = ALP_NONE32; }
        s_c[lane] = xc;
        s_p[lane] = xp;
    }
    __syncthreads();
    uint32_t ec = __shfl_up_sync(ALP_FULL_MASK, ic, 1), ep = __shfl_up_sync(ALP_FULL_MASK, ip, 1);
    if (lane == 0) { ec = 0; ep = ALP_NONE32; }
    const uint32_t rc = s_cc + s_c[warp] + ec;
    uint32_t rp = ep != ALP_NONE32 ? ep : (s_p[warp] != ALP_NONE32 ? s_p[warp] : s_cp);
    if (i < T) tile_cs[i] = ((unsigned long long)rc << 32) | rp;
}

// ---- kernel 5: tokens ---------------------------------------------------------
template <typename TermT, typename PosT>
__global__ void __launch_bounds__(LX_THREADS, 6) lex3_emit_kernel(Lex3Args a, LexSeg sg) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int S = a.t.S;
    uint16_t* s_ent = reinterpret_cast<uint16_t*>(smem);
    uint32_t* s_tok = reinterpret_cast<uint32_t*>(smem + lex3_tok_off(S));
    uint32_t* s_pk = reinterpret_cast<uint32_t*>(smem + lex3_stage_off(S));  // end - t0 | term << 16
    uint32_t* s_st = s_pk + LX_STAGE;                                        // start (absolute)

    __shared__ unsigned long long s_dmax;
    __shared__ uint32_t s_head[LX_TILE / LX_CHUNK], s_last[LX_TILE / LX_CHUNK];
    __shared__ uint32_t s_wc[LX_THREADS / 32], s_wp[LX_THREADS / 32];
    __shared__ uint32_t s_doff[LX_DOCS];  // offsets of the tile's documents d0.. (up to LX_DOCS)

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.t.ent);
        uint4* dst = reinterpret_cast<uint4*>(s_ent);
        for (int i = tid; i < (S * LX_ROW * 2 + 15) / 16; i += LX_THREADS) dst[i] = src[i];
    }
    for (int i = tid; i < S; i += LX_THREADS) s_tok[i] = a.t.tokinfo[i];
    const long long n = a.n;
    const long long ND = sg.n_docs;
    // document holding position p of this tile: the largest d in [d0, dmax]
    // with off[d] <= p, from the shared offsets when the tile has few documents
    auto doc_of = [&](long long d0, long long dmax, long long p) -> long long {
        if (dmax == d0) return d0;
        if (dmax - d0 < LX_DOCS) {
            int lo = 0, hi = (int)(dmax - d0);
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if ((long long)s_doff[mid] <= p) lo = mid; else hi = mid - 1;
            }
            return d0 + lo;
        }
        return doc_upper(sg.doc_off, d0, dmax, p);
    };
    auto base_of = [&](long long d0, long long dmax, long long d) -> long long {
        return (dmax - d0 < LX_DOCS) ? (long long)s_doff[d - d0] : sg.doc_off[d];
    };
    const uint32_t INIT = 1u;
    TermT* o_term = reinterpret_cast<TermT*>(a.out_term);
    PosT* o_start = reinterpret_cast<PosT*>(a.out_start);
    PosT* o_end = reinterpret_cast<PosT*>(a.out_end);
    const long long sent = sg.sentinels ? 1 : 0;
    // a stream piece places its tokens after the earlier pieces' and maps
    // positions to the stream; a start of NONE is the carried token start
    const long long tbase = (a.carry && a.carry_tokens) ? a.carry->tokens - a.tok_first : 0;
    const long long pb = a.pos_base;
    const long long snone = a.carry ? a.carry->start : 0;
    auto spos = [&](uint32_t st_abs, long long bk) -> long long {
        return st_abs == ALP_NONE32 ? snone : (long long)st_abs - bk + pb;
    };
    auto put = [&](long long idx, uint32_t term, long long st, long long en) {
        idx += tbase;
        if (idx < 0) return;  // before the stream's output window
        if (idx < a.cap) {
            o_term[idx] = (TermT)term;
            o_start[idx] = (PosT)st;
            o_end[idx] = (PosT)en;
        } else {
            atomicOr(&a.res->error, ALP_DEV_ERR_CAPACITY);
        }
    };
    for (unsigned tile = blockIdx.x; tile < a.num_tiles; tile += gridDim.x) {
        const long long t0 = (long long)tile * LX_TILE;
        const long long t1 = min(t0 + LX_TILE, n) - 1;
        const long long d0 = ND > 1 ? a.tile_doc[tile] : 0;
        if (tid == 0) s_dmax = (unsigned long long)d0;
        s_head[tid] = 0;
        s_last[tid] = 0;
        __syncthreads();
        lx_mark_docs(sg, n, d0, t0, t1, s_head, s_last, &s_dmax, s_doff);
        __syncthreads();
        const long long dmax = (long long)s_dmax;
        const long long my = t0 + (long long)tid * LX_CHUNK;
        const int lim = (int)max(0ll, min((long long)LX_CHUNK, n - my));

        uint4 w[2];
        uint32_t s0 = INIT, head = 0, last = 0, cnt = 0, lastp = ALP_NONE32;
        long long mydoc = d0;
        if (lim > 0) {
            lx_load<2>(a, my, lim, w);
            s0 = a.chunk_s[my / LX_CHUNK];
            const uint32_t cc = a.chunk_c[my / LX_CHUNK];
            cnt = cc & 0xffu;
            if ((cc >> 8) != LX_NOOFF) lastp = (uint32_t)(my + (cc >> 8));
            head = s_head[tid];
            last = s_last[tid];
            mydoc = doc_of(d0, dmax, my);
        } else {
            w[0] = w[1] = make_uint4(0, 0, 0, 0);
        }

        // ---- this thread's place: tile prefix + block scan of stored counts --
        const unsigned long long X = a.tile_cs[tile];
        const uint32_t Xc = (uint32_t)(X >> 32), Xp = (uint32_t)X;
        uint32_t ic = cnt, ip = lastp;
        warp_scan_cs(ic, ip, lane);
        uint32_t ec = __shfl_up_sync(ALP_FULL_MASK, ic, 1), ep = __shfl_up_sync(ALP_FULL_MASK, ip, 1);
        if (lane == 0) { ec = 0; ep = ALP_NONE32; }
        if (lane == 31) { s_wc[warp] = ic; s_wp[warp] = ip; }
        __syncthreads();
        uint32_t wc = 0, wp = ALP_NONE32, Bc = 0;
#pragma unroll
        for (int w2 = 0; w2 < LX_THREADS / 32; ++w2) {
            if (w2 < warp) {
                wc += s_wc[w2];
                if (s_wp[w2] != ALP_NONE32) wp = s_wp[w2];
            }
            Bc += s_wc[w2];
        }
        const bool staged = Bc <= (uint32_t)LX_STAGE;
        uint32_t tcount = Xc + wc + ec;
        uint32_t cur = ep != ALP_NONE32 ? ep : (wp != ALP_NONE32 ? wp : Xp);

        // ---- emit ---------------------------------------------------------------
        if (lim > 0) {
            uint32_t st = s0;
            if ((head | last) == 0 && lim == LX_CHUNK && staged) {
                uint32_t k = tcount - Xc;
                const uint32_t rel = (uint32_t)(my - t0);
#pragma unroll
                for (int j = 0; j < LX_CHUNK; ++j) {
                    const uint32_t e = s_ent[st * LX_ROW + byte_of(w, j)];
                    if (e & LX_EMIT) {
                        s_pk[k] = (rel + j) | ((e >> LX_TERM_SHIFT) << 16);
                        s_st[k] = cur;
                        ++k;
                    }
                    if (e & LX_START) cur = (uint32_t)(my + j);
                    st = e & LX_NEXT;
                }
                tcount = Xc + k;
            } else {
                long long doc = mydoc;
                long long base = base_of(d0, dmax, doc);
                auto tok = [&](uint32_t term, uint32_t st_abs, uint32_t en_abs) {
                    if (staged) {
                        const uint32_t k = tcount - Xc;
                        s_pk[k] = (uint32_t)(en_abs - t0) | (term << 16);
                        s_st[k] = st_abs;
                    } else {
                        put((long long)tcount + sent * (2 * doc + 1), term, spos(st_abs, base),
                            (long long)en_abs - base + pb);
                    }
                    ++tcount;
                };
                // a compact loop (bytes through L1): only threads at document
                // boundaries, partial chunks or overflowing tiles come here
#pragma unroll 1
                for (int j = 0; j < lim; ++j) {
                    {
                        const long long pos = my + j;
                        if ((head >> j) & 1u) {
                            // every document starting here (empty ones first, then the real one)
                            doc = doc_of(d0, dmax, pos);
                            long long dl = doc;  // empty documents that start here too
                            while (dl > 0 && sg.doc_off[dl - 1] >= pos) --dl;
                            base = pos;
                            for (long long e2 = dl; e2 <= doc; ++e2) {
                                sg.tok_off[e2] = tcount;
                                if (sent) put((long long)tcount + 2 * e2, sg.sent_l, 0, 0);
                                if (e2 < doc) {
                                    sg.valid[e2] = 0;
                                    if (sent) put((long long)tcount + 2 * e2 + 1, sg.sent_r, 0, 0);
                                }
                            }
                            cur = (uint32_t)pos;
                            st = INIT;
                        }
                        const uint32_t e = s_ent[st * LX_ROW + __ldg(a.in + pos)];
                        if (e & LX_EMIT) tok(e >> LX_TERM_SHIFT, cur, (uint32_t)pos);
                        if (e & LX_START) cur = (uint32_t)pos;
                        st = e & LX_NEXT;
                        if ((last >> j) & 1u) {
                            const uint32_t ti = s_tok[st];
                            if (!(ti & TOK_IGNORE)) tok(ti & TOK_TERM_MASK, cur, (uint32_t)(pos + 1));
                            sg.valid[doc] = (ti & TOK_ACCEPT) ? 1 : 0;
                            if (sent) put((long long)tcount + 2 * doc + 1, sg.sent_r, 0, 0);
                        }
                    }
                }
                mydoc = doc;
            }
        }
        if (my <= n - 1 && n - 1 < my + LX_CHUNK) {
            // documents that start at n (empty, at the end) and the closing offset
            for (long long e2 = mydoc + 1; e2 < ND; ++e2) {
                sg.tok_off[e2] = tcount;
                sg.valid[e2] = 0;
                if (sent) {
                    put((long long)tcount + 2 * e2, sg.sent_l, 0, 0);
                    put((long long)tcount + 2 * e2 + 1, sg.sent_r, 0, 0);
                }
            }
            sg.tok_off[ND] = tcount;
            a.res->count = tcount;
            a.res->valid = 1;
        }
        __syncthreads();

        // ---- coalesced copy of the staged tokens ---------------------------------
        if (staged && dmax == d0) {
            // one document in the tile: every token's index and positions shift alike
            const long long ib = (long long)Xc + sent * (2 * d0 + 1) + tbase;
            const long long off = pb - base_of(d0, dmax, d0);
            for (uint32_t k = tid; k < Bc; k += LX_THREADS) {
                const uint32_t pk = s_pk[k], sv = s_st[k];
                const long long idx = ib + k;
                if (idx < 0) continue;
                if (idx < a.cap) {
                    o_term[idx] = (TermT)(pk >> 16);
                    o_start[idx] = (PosT)(sv == ALP_NONE32 ? snone : (long long)sv + off);
                    o_end[idx] = (PosT)(t0 + (pk & 0xffffu) + off);
                } else {
                    atomicOr(&a.res->error, ALP_DEV_ERR_CAPACITY);
                }
            }
        } else if (staged) {
            const long long b0 = base_of(d0, dmax, d0);
            for (uint32_t k = tid; k < Bc; k += LX_THREADS) {
                const uint32_t pk = s_pk[k];
                const long long en = t0 + (pk & 0xffffu);
                long long dk = d0, bk = b0;
                if (dmax > d0) {
                    dk = doc_of(d0, dmax, en - 1);
                    bk = base_of(d0, dmax, dk);
                }
                put((long long)(Xc + k) + sent * (2 * dk + 1), pk >> 16, spos(s_st[k], bk), en - bk + pb);
            }
        }
        __syncthreads();
    }
}

// ---- kernel 3+4+5 fused: counts, look-back over tiles, tokens ---------------
// One pass over the input for what lex3_count_kernel, the tile scan and
// lex3_emit_kernel do in three: each thread runs the DFA over its chunk once
// from its known state, counting the tokens that end in it and keeping each
// token's place and terminal as a record in shared memory; a block scan places
// the threads in the tile; the tile publishes its (count, last start) and
// finds its exclusive prefix by a decoupled look-back over earlier tiles
// (futhark/lexer.fut:83-84,108-133: the take_right start scan and the
// compaction offsets); the tokens go from the records into the stage and out
// with coalesced stores.  Tiles come in ticket order, so every tile a
// look-back waits for is running or done.  Tiles with document boundaries,
// partial chunks or more tokens than the stage holds take their prefix first
// and write through the compact loop of lex3_emit_kernel.
//
// Look-back word of a tile: [63:62] flag, [61:31] token count, [30:0] last
// kept token start (LX_LB_NONE: none); the inclusive prefix once flagged P.
// Inputs are below 2^31 bytes, so counts and positions fit 31 bits.
constexpr uint32_t LX_LB_NONE = 0x7fffffffu;
constexpr int LX_REC = 16;               // token records a thread keeps from its counting pass
constexpr int LX_REC_ROW = LX_REC + 2;      // u16 per thread row: 9 words, an odd stride across lanes
__host__ __device__ inline size_t lex3_tok_smem(int S) {
    return lex3_stage_off(S) + (size_t)LX_STAGE * 8 + (size_t)LX_THREADS * LX_REC_ROW * 2;
}

__device__ __forceinline__ unsigned long long tk_pack(uint32_t flag, uint32_t c, uint32_t p) {
    return ((unsigned long long)flag << 62) | ((unsigned long long)(c & 0x7fffffffu) << 31) |
           (p == ALP_NONE32 ? LX_LB_NONE : (p & 0x7fffffffu));
}
__device__ __forceinline__ uint32_t tk_count(unsigned long long w) { return (uint32_t)(w >> 31) & 0x7fffffffu; }
__device__ __forceinline__ uint32_t tk_pos(unsigned long long w) {
    const uint32_t p = (uint32_t)w & 0x7fffffffu;
    return p == LX_LB_NONE ? ALP_NONE32 : p;
}

// Warp 0: the (count, last start) of all tiles before `tile`, from the
// look-back words; then publishes this tile's inclusive prefix.
__device__ __forceinline__ void tk_lookback(unsigned long long* lb, unsigned tile, uint32_t Bc, uint32_t Bp,
                                            unsigned int* err, uint32_t* s_xc, uint32_t* s_xp) {
    const int lane = threadIdx.x & 31;
    uint32_t Xc = 0, Xp = ALP_NONE32;
    if (tile > 0) {
        long long end = tile;
        for (;;) {
            const long long idx = end - 32 + lane;
            const unsigned long long w2 = idx >= 0 ? wait64(&lb[idx], err) : tk_pack(ST_P, 0, ALP_NONE32);
            const uint32_t pm = __ballot_sync(ALP_FULL_MASK, (uint32_t)(w2 >> 62) == ST_P);
            const int p = pm ? 31 - __clz(pm) : -1;
            uint32_t vc = lane >= p ? tk_count(w2) : 0u;
            uint32_t vp = lane >= p ? tk_pos(w2) : ALP_NONE32;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {  // lanes in order: sum, take-right
                const uint32_t oc = __shfl_down_sync(ALP_FULL_MASK, vc, d);
                const uint32_t op = __shfl_down_sync(ALP_FULL_MASK, vp, d);
                if (lane + d < 32) {
                    vc += oc;
                    if (op != ALP_NONE32) vp = op;
                }
            }
            Xc += __shfl_sync(ALP_FULL_MASK, vc, 0);
            vp = __shfl_sync(ALP_FULL_MASK, vp, 0);
            if (Xp == ALP_NONE32) Xp = vp;
            if (pm) break;
            end -= 32;
        }
        if (lane == 0) st_volatile64(&lb[tile], tk_pack(ST_P, Xc + Bc, Bp != ALP_NONE32 ? Bp : Xp));
    }
    if (lane == 0) { *s_xc = Xc; *s_xp = Xp; }
}

template <typename TermT, typename PosT>
__global__ void __launch_bounds__(LX_THREADS, 5) lex3_tok_kernel(Lex3Args a, LexSeg sg) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int S = a.t.S;
    uint16_t* s_ent = reinterpret_cast<uint16_t*>(smem);
    uint32_t* s_tok = reinterpret_cast<uint32_t*>(smem + lex3_tok_off(S));
    uint32_t* s_pk = reinterpret_cast<uint32_t*>(smem + lex3_stage_off(S));  // end - t0 | term << 16
    uint32_t* s_st = s_pk + LX_STAGE;                                        // start (absolute; NONE: before the tile)
    uint16_t* s_rec = reinterpret_cast<uint16_t*>(s_st + LX_STAGE);          // [thread][LX_REC_ROW]: j | term << 5

    __shared__ unsigned long long s_dmax;
    __shared__ uint32_t s_head[LX_TILE / LX_CHUNK], s_last[LX_TILE / LX_CHUNK];
    __shared__ uint32_t s_wc[LX_THREADS / 32], s_wp[LX_THREADS / 32];
    __shared__ uint32_t s_doff[LX_DOCS];
    __shared__ uint32_t s_tile, s_xc, s_xp;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.t.ent);
        uint4* dst = reinterpret_cast<uint4*>(s_ent);
        for (int i = tid; i < (S * LX_ROW * 2 + 15) / 16; i += LX_THREADS) dst[i] = src[i];
    }
    for (int i = tid; i < S; i += LX_THREADS) s_tok[i] = a.t.tokinfo[i];
    const long long n = a.n;
    const long long ND = sg.n_docs;
    unsigned long long* lb = a.tile_cs;
    auto doc_of = [&](long long d0, long long dmax, long long p) -> long long {
        if (dmax == d0) return d0;
        if (dmax - d0 < LX_DOCS) {
            int lo = 0, hi = (int)(dmax - d0);
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if ((long long)s_doff[mid] <= p) lo = mid; else hi = mid - 1;
            }
            return d0 + lo;
        }
        return doc_upper(sg.doc_off, d0, dmax, p);
    };
    auto base_of = [&](long long d0, long long dmax, long long d) -> long long {
        return (dmax - d0 < LX_DOCS) ? (long long)s_doff[d - d0] : sg.doc_off[d];
    };
    const uint32_t INIT = 1u;
    TermT* o_term = reinterpret_cast<TermT*>(a.out_term);
    PosT* o_start = reinterpret_cast<PosT*>(a.out_start);
    PosT* o_end = reinterpret_cast<PosT*>(a.out_end);
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
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(&a.tickets[1], 1u);
        __syncthreads();
        const unsigned tile = s_tile;
        if (tile >= a.num_tiles) break;
        const long long t0 = (long long)tile * LX_TILE;
        const long long t1 = min(t0 + LX_TILE, n) - 1;
        const long long d0 = ND > 1 ? a.tile_doc[tile] : 0;
        if (tid == 0) s_dmax = (unsigned long long)d0;
        s_head[tid] = 0;
        s_last[tid] = 0;
        __syncthreads();
        lx_mark_docs(sg, n, d0, t0, t1, s_head, s_last, &s_dmax, s_doff);
        __syncthreads();
        const long long dmax = (long long)s_dmax;
        const long long my = t0 + (long long)tid * LX_CHUNK;
        const int lim = (int)max(0ll, min((long long)LX_CHUNK, n - my));
        const uint32_t rel = (uint32_t)(my - t0);

        uint4 w[2];
        uint32_t s0 = INIT, head = 0, last = 0;
        long long mydoc = d0;
        if (lim > 0) {
            lx_load<2>(a, my, lim, w);
            s0 = a.chunk_s[my / LX_CHUNK];
            head = s_head[tid];
            last = s_last[tid];
            mydoc = doc_of(d0, dmax, my);
        } else {
            w[0] = w[1] = make_uint4(0, 0, 0, 0);
        }
        const bool fast = lim == LX_CHUNK && (head | last) == 0;

        // ---- counting pass: tokens ending in the chunk, its starts, records ----
        uint32_t cnt = 0, lastp = ALP_NONE32, smask = 0;
        if (fast) {
            uint32_t st = s0;
#pragma unroll
            for (int j = 0; j < LX_CHUNK; ++j) {
                const uint32_t e = s_ent[st * LX_ROW + byte_of(w, j)];
                if (e & LX_EMIT) {
                    if (cnt < (uint32_t)LX_REC) s_rec[tid * LX_REC_ROW + cnt] = (uint16_t)(j | ((e >> LX_TERM_SHIFT) << 5));
                    ++cnt;
                }
                if (e & LX_START) smask |= 1u << j;
                st = e & LX_NEXT;
            }
            if (smask) lastp = (uint32_t)(my + 31 - __clz(smask));
        } else if (lim > 0) {
            uint32_t lo;
            cnt = lx_count_slow(a.in + my, lim, s0, head, last, s_ent, s_tok, &lo);
            if (lo != LX_NOOFF) lastp = (uint32_t)(my + lo);
        }

        // ---- place in the tile: block scan of (count, last start) --------------
        uint32_t ic = cnt, ip = lastp;
        warp_scan_cs(ic, ip, lane);
        uint32_t ec = __shfl_up_sync(ALP_FULL_MASK, ic, 1), ep = __shfl_up_sync(ALP_FULL_MASK, ip, 1);
        if (lane == 0) { ec = 0; ep = ALP_NONE32; }
        if (lane == 31) { s_wc[warp] = ic; s_wp[warp] = ip; }
        const int slow_any = __syncthreads_or(lim > 0 && !fast);
        uint32_t wc = 0, wp = ALP_NONE32, Bc = 0, Bp = ALP_NONE32;
#pragma unroll
        for (int w2 = 0; w2 < LX_THREADS / 32; ++w2) {
            const uint32_t c2 = s_wc[w2], p2 = s_wp[w2];
            if (w2 < warp) {
                wc += c2;
                if (p2 != ALP_NONE32) wp = p2;
            }
            Bc += c2;
            if (p2 != ALP_NONE32) Bp = p2;
        }
        const bool staged = Bc <= (uint32_t)LX_STAGE;
        const bool early = slow_any || !staged;  // the tile needs its prefix before it writes tokens
        const uint32_t kx = wc + ec;              // the tile's tokens before this thread
        const uint32_t curx = ep != ALP_NONE32 ? ep : wp;  // last start in the tile before this thread
        if (tid == 0) {
            if (tile == 0) st_volatile64(&lb[0], tk_pack(ST_P, Bc, Bp));
            else st_volatile64(&lb[tile], tk_pack(ST_A, Bc, Bp));
        }
        if (early) {
            if (warp == 0) tk_lookback(lb, tile, Bc, Bp, &a.res->error, &s_xc, &s_xp);
            __syncthreads();
        } else if (warp == 0) {
            // the look-back first, while the other warps move their records to the stage
            tk_lookback(lb, tile, Bc, Bp, &a.res->error, &s_xc, &s_xp);
        }

        // ---- tokens -----------------------------------------------------------------
        if (fast && staged) {
            uint32_t k = kx;
            if (cnt <= (uint32_t)LX_REC) {
                for (uint32_t r = 0; r < cnt; ++r) {
                    const uint32_t rec = s_rec[tid * LX_REC_ROW + r];
                    const uint32_t j = rec & 31u;
                    const uint32_t m = smask & ((1u << j) - 1u);
                    s_pk[k] = (rel + j) | ((rec >> 5) << 16);
                    s_st[k] = m ? (uint32_t)(my + 31 - __clz(m)) : curx;
                    ++k;
                }
            } else {
                uint32_t st = s0, cur = curx;
#pragma unroll
                for (int j = 0; j < LX_CHUNK; ++j) {
                    const uint32_t e = s_ent[st * LX_ROW + byte_of(w, j)];
                    if (e & LX_EMIT) {
                        s_pk[k] = (rel + j) | ((e >> LX_TERM_SHIFT) << 16);
                        s_st[k] = cur;
                        ++k;
                    }
                    if (e & LX_START) cur = (uint32_t)(my + j);
                    st = e & LX_NEXT;
                }
            }
        } else if (lim > 0) {
            // an early tile: every thread's global place is known
            uint32_t tcount = s_xc + kx;
            uint32_t cur = curx != ALP_NONE32 ? curx : s_xp;
            uint32_t st = s0;
            long long doc = mydoc;
            long long base = base_of(d0, dmax, doc);
            auto tok = [&](uint32_t term, uint32_t st_abs, uint32_t en_abs) {
                if (staged) {
                    const uint32_t k = tcount - s_xc;
                    s_pk[k] = (uint32_t)(en_abs - t0) | (term << 16);
                    s_st[k] = st_abs;
                } else {
                    put((long long)tcount + sent * (2 * doc + 1), term, st_abs == ALP_NONE32 ? 0 : (long long)st_abs - base,
                        (long long)en_abs - base);
                }
                ++tcount;
            };
#pragma unroll 1
            for (int j = 0; j < lim; ++j) {
                const long long pos = my + j;
                if ((head >> j) & 1u) {
                    // every document starting here (empty ones first, then the real one)
                    doc = doc_of(d0, dmax, pos);
                    long long dl = doc;
                    while (dl > 0 && sg.doc_off[dl - 1] >= pos) --dl;
                    base = pos;
                    for (long long e2 = dl; e2 <= doc; ++e2) {
                        sg.tok_off[e2] = tcount;
                        if (sent) put((long long)tcount + 2 * e2, sg.sent_l, 0, 0);
                        if (e2 < doc) {
                            sg.valid[e2] = 0;
                            if (sent) put((long long)tcount + 2 * e2 + 1, sg.sent_r, 0, 0);
                        }
                    }
                    cur = (uint32_t)pos;
                    st = INIT;
                }
                const uint32_t e = s_ent[st * LX_ROW + __ldg(a.in + pos)];
                if (e & LX_EMIT) tok(e >> LX_TERM_SHIFT, cur, (uint32_t)pos);
                if (e & LX_START) cur = (uint32_t)pos;
                st = e & LX_NEXT;
                if ((last >> j) & 1u) {
                    const uint32_t ti = s_tok[st];
                    if (!(ti & TOK_IGNORE)) tok(ti & TOK_TERM_MASK, cur, (uint32_t)(pos + 1));
                    sg.valid[doc] = (ti & TOK_ACCEPT) ? 1 : 0;
                    if (sent) put((long long)tcount + 2 * doc + 1, sg.sent_r, 0, 0);
                }
            }
            mydoc = doc;
            if (my <= n - 1 && n - 1 < my + LX_CHUNK) {
                // documents that start at n (empty, at the end) and the closing offset
                for (long long e2 = mydoc + 1; e2 < ND; ++e2) {
                    sg.tok_off[e2] = tcount;
                    sg.valid[e2] = 0;
                    if (sent) {
                        put((long long)tcount + 2 * e2, sg.sent_l, 0, 0);
                        put((long long)tcount + 2 * e2 + 1, sg.sent_r, 0, 0);
                    }
                }
                sg.tok_off[ND] = tcount;
                a.res->count = tcount;
                a.res->valid = 1;
            }
        }
        __syncthreads();

        // ---- coalesced copy of the staged tokens ---------------------------------
        const uint32_t Xc = s_xc, Xp = s_xp;
        auto sres = [&](uint32_t sv) -> uint32_t { return sv != ALP_NONE32 ? sv : Xp; };
        if (staged && dmax == d0) {
            // one document in the tile: every token's index and positions shift alike
            const long long ib = (long long)Xc + sent * (2 * d0 + 1);
            const long long off = -base_of(d0, dmax, d0);
            for (uint32_t k = tid; k < Bc; k += LX_THREADS) {
                const uint32_t pk = s_pk[k], sv = sres(s_st[k]);
                const long long idx = ib + k;
                if (idx < a.cap) {
                    o_term[idx] = (TermT)(pk >> 16);
                    o_start[idx] = (PosT)(sv == ALP_NONE32 ? 0 : (long long)sv + off);
                    o_end[idx] = (PosT)(t0 + (pk & 0xffffu) + off);
                } else {
                    atomicOr(&a.res->error, ALP_DEV_ERR_CAPACITY);
                }
            }
        } else if (staged) {
            const long long b0 = base_of(d0, dmax, d0);
            for (uint32_t k = tid; k < Bc; k += LX_THREADS) {
                const uint32_t pk = s_pk[k], sv = sres(s_st[k]);
                const long long en = t0 + (pk & 0xffffu);
                long long dk = d0, bk = b0;
                if (dmax > d0) {
                    dk = doc_of(d0, dmax, en - 1);
                    bk = base_of(d0, dmax, dk);
                }
                put((long long)(Xc + k) + sent * (2 * dk + 1), pk >> 16, sv == ALP_NONE32 ? 0 : (long long)sv - bk,
                    en - bk);
            }
        }
        __syncthreads();
    }
}

// ---- streams: the carry after a piece, the last token at the end --------------
// After the token pass of one piece (launched with the piece's Lex3Args):
// the DFA state after its last byte, the start of the kept token in progress
// (the last token start in the piece, else unchanged), and the token count.
__global__ void __launch_bounds__(LX_THREADS) lex3_stream_tail_kernel(Lex3Args a) {
    __shared__ long long s_best[LX_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long C = a.n_chunks, T = a.num_tiles;
    long long best = -1;  // last token start in the last tile
    for (long long c = (T - 1) * (LX_TILE / LX_CHUNK) + tid; c < C; c += LX_THREADS) {
        const uint32_t off = a.chunk_c[c] >> 8;
        if (off != LX_NOOFF) best = max(best, c * LX_CHUNK + (long long)off);
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) best = max(best, (long long)__shfl_xor_sync(ALP_FULL_MASK, best, d));
    if (lane == 0) s_best[warp] = best;
    __syncthreads();
    if (tid == 0) {
        for (int w = 0; w < LX_THREADS / 32; ++w) best = max(best, s_best[w]);
        if (best < 0) {
            const uint32_t xp = (uint32_t)a.tile_cs[T - 1];  // exclusive: before the last tile
            if (xp != ALP_NONE32) best = xp;
        }
        LexCarry* c = a.carry;
        if (best >= 0) c->start = a.pos_base + best;
        uint32_t st = a.chunk_s[C - 1];
        for (long long p = (C - 1) * LX_CHUNK; p < a.n; ++p) st = a.t.ent[st * LX_ROW + a.in[p]] & LX_NEXT;
        c->state = st;
        c->piece = a.res->count;
        c->tokens += a.res->count;
        c->error |= a.res->error;
    }
}

// End of a stream of `total` bytes: the last token (futhark/lexer.fut:108-115
// at the input's end) and acceptance, from the carry.  With `global` the token
// goes after all tokens so far (token `first` at element 0), else after the
// last piece's.  An empty stream is judged like an empty input.
__global__ void lex3_stream_end_kernel(LexCarry* c, const uint32_t* tokinfo, long long total, int global,
                                       long long first, uint32_t* term, long long* start, long long* end,
                                       long long cap) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t ti = tokinfo[c->state];
    if (total == 0) {  // the empty input: accepted iff the initial state accepts, no token
        c->valid = (ti & TOK_ACCEPT) ? 1 : 0;
        if (global) c->piece = 0;
        return;
    }
    long long k = 0;
    if (!(ti & TOK_IGNORE)) {
        const long long idx = global ? c->tokens - first : c->piece;
        if (idx < 0) {
            // before the output window: not stored
        } else if (idx < cap) {
            term[idx] = ti & TOK_TERM_MASK;
            start[idx] = c->start;
            end[idx] = total;
        } else {
            c->error |= ALP_DEV_ERR_CAPACITY;
        }
        k = 1;
    }
    c->piece = global ? k : c->piece + k;
    c->tokens += k;
    c->valid = (ti & TOK_ACCEPT) ? 1 : 0;
}

// ---- shards: one byte range of a document lexed on one GPU of several --------
// The state function of a shard: lane s of the result holds the state after
// the shard's bytes from entry state s.  Each block composes a contiguous run
// of chunk endomorphisms (lane-per-state walks through the apply table, one
// warp per sub-run, then the warps in order); lex3_fn_final_kernel composes
// the blocks in order.
constexpr int LF_WARPS = 8;
__global__ void __launch_bounds__(LF_WARPS * 32) lex3_fn_kernel(const uint16_t* chunk_f, long long C,
                                                                const uint8_t* app8, int rows, uint8_t* fn) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint8_t s_w[LF_WARPS][32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const uint4* src = reinterpret_cast<const uint4*>(app8);
        uint4* dst = reinterpret_cast<uint4*>(smem);
        for (int i = tid; i < rows * 2; i += LF_WARPS * 32) dst[i] = src[i];
    }
    __syncthreads();
    const long long per_block = (C + gridDim.x - 1) / gridDim.x;
    const long long b0 = (long long)blockIdx.x * per_block, b1 = min(C, b0 + per_block);
    const long long per_warp = (b1 - b0 + LF_WARPS - 1) / LF_WARPS;
    const long long w0 = b0 + (long long)warp * per_warp, w1 = min(b1, w0 + per_warp);
    uint32_t cur = (uint32_t)lane;
    for (long long c = w0; c < w1; ++c) cur = smem[(uint32_t)chunk_f[c] * 32 + cur];
    s_w[warp][lane] = (uint8_t)cur;
    __syncthreads();
    if (warp == 0) {
        uint32_t x = (uint32_t)lane;
        for (int w = 0; w < LF_WARPS; ++w) x = s_w[w][x];
        fn[(size_t)blockIdx.x * 32 + lane] = (uint8_t)x;
    }
}

// 32 warps: warp w composes a contiguous run of the block functions, then
// warp 0 composes the 32 runs in order.
__global__ void __launch_bounds__(1024) lex3_fn_final_kernel(const uint8_t* fn, int blocks, uint8_t* out) {
    __shared__ uint8_t s_w[32][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int per = (blocks + 31) / 32;
    const int b0 = warp * per, b1 = min(blocks, b0 + per);
    uint32_t x = (uint32_t)lane;
    for (int b = b0; b < b1; ++b) x = fn[(size_t)b * 32 + x];
    s_w[warp][lane] = (uint8_t)x;
    __syncthreads();
    if (warp == 0) {
        uint32_t y = (uint32_t)lane;
        for (int w = 0; w < 32; ++w) y = s_w[w][y];
        out[lane] = (uint8_t)y;
    }
}

// After the tile scan of a shard's counts: out[0] = tokens that end in the
// shard, out[1] = position (shard-relative) of its last token start, -1 if none.
__global__ void __launch_bounds__(LX_THREADS) lex3_shard_totals_kernel(Lex3Args a, long long* out) {
    __shared__ long long s_best[LX_THREADS / 32];
    __shared__ unsigned long long s_cnt[LX_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long C = a.n_chunks, T = a.num_tiles;
    long long best = -1;
    unsigned long long cnt = 0;
    for (long long c = (T - 1) * (LX_TILE / LX_CHUNK) + tid; c < C; c += LX_THREADS) {
        const uint32_t cc = a.chunk_c[c];
        cnt += cc & 0xffu;
        if ((cc >> 8) != LX_NOOFF) best = max(best, c * LX_CHUNK + (long long)(cc >> 8));
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
        best = max(best, (long long)__shfl_xor_sync(ALP_FULL_MASK, best, d));
        cnt += __shfl_xor_sync(ALP_FULL_MASK, cnt, d);
    }
    if (lane == 0) { s_best[warp] = best; s_cnt[warp] = cnt; }
    __syncthreads();
    if (tid == 0) {
        cnt = 0;
        for (int w = 0; w < LX_THREADS / 32; ++w) {
            best = max(best, s_best[w]);
            cnt += s_cnt[w];
        }
        const unsigned long long X = a.tile_cs[T - 1];  // exclusive: before the last tile
        if (best < 0 && (uint32_t)X != ALP_NONE32) best = (uint32_t)X;
        out[0] = (long long)(X >> 32) + (long long)cnt;
        out[1] = best;
    }
}

}  // namespace alp
