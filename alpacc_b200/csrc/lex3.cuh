// Three-kernel lexer for DFAs of at most 32 states (sm_100a).
//
// Same results as lex_seg_kernel (futhark/lexer.fut:73-172 per document),
// split so that no step waits on table lookups through L2:
//
//   lex3_fold_kernel  every 32-byte chunk -> its endomorphism id, folded with
//                     the step table in shared memory (constant E+s after a
//                     document head).  Streaming; no look-back.
//   lex3_scan_kernel  the composition scan over chunk endomorphisms.  With
//                     S <= 32 one warp holds a whole function, lane s the
//                     image of state s, so composing two functions is one
//                     shuffle and a tile's aggregate is 32 bytes.  Lanes walk
//                     the chunks of their warp through the apply table in
//                     shared memory; tiles chain through a decoupled look-back
//                     on these vectors.  Output: the state entering each chunk.
//   lex3_emit_kernel  the token pass (futhark/lexer.fut:103-133): each thread
//                     runs the DFA over its chunk from the known state with a
//                     256-column transition table whose entries carry the
//                     produce/ignore decisions, counts, takes its place
//                     through a (count, last start) look-back, and stages the
//                     tile's tokens in shared memory for coalesced stores.
#pragma once
#include "common.cuh"
#include "lexer.cuh"

namespace alp {

constexpr int LX_THREADS = 256;
constexpr int LX_ITEMS = 32;                    // bytes per thread = one chunk
constexpr int LX_TILE = LX_THREADS * LX_ITEMS;  // 8 KiB per tile
constexpr int LX_STAGE = 2560;                  // tokens one tile stages in shared memory
constexpr int LS_WARPS = 8;
constexpr int LS_G = 16;                        // chunks per lane in the state scan
constexpr int LS_TILE = LS_WARPS * 32 * LS_G;   // 4096 chunks per state-scan tile

// ent entries: next state | flags.  Rows are LX_ROW entries apart so that
// lanes reading the same byte in different states hit different banks.
constexpr int LX_ROW = 258;
constexpr uint32_t LX_NEXT = 0x1fu;
constexpr uint32_t LX_EMIT = 1u << 5;   // a kept token of term(st) ends before this byte
constexpr uint32_t LX_START = 1u << 6;  // a kept token starts at this byte

struct Lex3Tables {
    const uint8_t* cls;       // [256] byte -> class
    const uint16_t* cdelta;   // [S][C1] next | produce<<15
    const uint16_t* step;     // [E][C1] endo after one more byte of the class
    const uint8_t* app8;      // [E][32] state after endo e from state s (identity for s >= S)
    const uint16_t* ent;      // [S][LX_ROW] next | LX_EMIT | LX_START (columns 256.. unused)
    const uint32_t* tokinfo;  // [S] terminal | TOK_ACCEPT | TOK_IGNORE
    int S, C1, E;
};

struct Lex3Args {
    const uint8_t* in;
    long long n;
    int aligned16;
    Lex3Tables t;
    long long n_chunks;          // ceil(n / 32)
    uint16_t* chunk_f;           // [n_chunks] endomorphism of each chunk (E + s: constant s)
    uint8_t* chunk_s;            // [n_chunks] state entering each chunk
    uint32_t* lb_vec;            // [scan tiles][32] state-scan look-back words
    unsigned long long* lb_cs;   // [tiles] (count, start) look-back words
    unsigned int* tickets;       // [0] state scan, [1] emit
    const long long* tile_doc;   // [tiles] document holding each tile's first byte (n_docs > 1)
    void* out_term;
    void* out_start;
    void* out_end;
    long long cap;
    AlpResult* res;
    unsigned int num_tiles;      // 8 KiB tiles
    unsigned int num_scan_tiles; // LS_TILE-chunk tiles
};

__host__ __device__ inline size_t lex3_fold_smem(int S, int C1, int E) {
    size_t b = 256 + 2 * (size_t)S * C1;
    b = (b + 15) & ~(size_t)15;
    b += 2 * (size_t)E * C1;
    return (b + 15) & ~(size_t)15;
}
__host__ __device__ inline size_t lex3_scan_smem(int E) {
    return (32 * (size_t)E + 15) & ~(size_t)15;
}
__host__ __device__ inline size_t lex3_tok_off(int S) { return (2 * (size_t)S * LX_ROW + 15) & ~(size_t)15; }
__host__ __device__ inline size_t lex3_stage_off(int S) { return (lex3_tok_off(S) + 4 * (size_t)S + 15) & ~(size_t)15; }
__host__ __device__ inline size_t lex3_emit_smem(int S) { return lex3_stage_off(S) + (size_t)LX_STAGE * (2 + 4 + 4); }

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

// Document heads and last bytes of tile [t0, t1] as per-thread bit masks;
// *s_dmax = the last document with a byte at or before t1.
__device__ __forceinline__ void lx_mark_docs(const LexSeg& sg, long long n, long long d0, long long t0, long long t1,
                                             uint32_t* s_head, uint32_t* s_last, unsigned long long* s_dmax) {
    for (long long d = d0 + threadIdx.x; d <= sg.n_docs; d += LX_THREADS) {
        const long long h = sg.doc_off[d];
        if (h > t1 + 1) break;
        if (h >= t0 && h <= t1 && h < n) {
            const long long r = h - t0;
            atomicOr(&s_head[r >> 5], 1u << (r & 31));
        }
        if (h - 1 >= t0 && h - 1 <= t1 && s_last) {
            const long long r = h - 1 - t0;
            atomicOr(&s_last[r >> 5], 1u << (r & 31));
        }
        if (h <= t1 && d < sg.n_docs && s_dmax) atomicMax(s_dmax, (unsigned long long)d);
    }
}

// Load the (up to) 32 bytes of a thread starting at `my`.
__device__ __forceinline__ void lx_load(const Lex3Args& a, long long my, int lim, uint4 (&w)[2]) {
    if (a.aligned16 && lim == LX_ITEMS) {
        w[0] = __ldg(reinterpret_cast<const uint4*>(a.in + my));
        w[1] = __ldg(reinterpret_cast<const uint4*>(a.in + my) + 1);
    } else {
        uint32_t x[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            uint32_t y = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b)
                if (q * 4 + b < lim) y |= (uint32_t)a.in[my + q * 4 + b] << (8 * b);
            x[q] = y;
        }
        w[0] = make_uint4(x[0], x[1], x[2], x[3]);
        w[1] = make_uint4(x[4], x[5], x[6], x[7]);
    }
}

// ---- kernel 1: chunk endomorphisms ------------------------------------------
__global__ void __launch_bounds__(LX_THREADS, 4) lex3_fold_kernel(Lex3Args a, LexSeg sg) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int S = a.t.S, C1 = a.t.C1, E = a.t.E;
    uint8_t* s_cls = smem;
    uint16_t* s_cd = reinterpret_cast<uint16_t*>(smem + 256);
    const size_t off_step = (256 + 2 * (size_t)S * C1 + 15) & ~(size_t)15;
    uint16_t* s_step = reinterpret_cast<uint16_t*>(smem + off_step);
    __shared__ uint32_t s_head[LX_THREADS];

    const int tid = threadIdx.x;
    for (int i = tid; i < 256; i += LX_THREADS) s_cls[i] = a.t.cls[i];
    for (int i = tid; i < S * C1; i += LX_THREADS) s_cd[i] = a.t.cdelta[i];
    for (int i = tid; i < E * C1; i += LX_THREADS) s_step[i] = a.t.step[i];
    const long long n = a.n;
    const uint32_t INIT = 1u;
    for (unsigned tile = blockIdx.x; tile < a.num_tiles; tile += gridDim.x) {
        const long long t0 = (long long)tile * LX_TILE;
        const long long t1 = min(t0 + LX_TILE, n) - 1;
        s_head[tid] = 0;
        __syncthreads();
        lx_mark_docs(sg, n, sg.n_docs > 1 ? a.tile_doc[tile] : 0, t0, t1, s_head, nullptr, nullptr);
        __syncthreads();
        const long long my = t0 + (long long)tid * LX_ITEMS;
        const int lim = (int)max(0ll, min((long long)LX_ITEMS, n - my));
        if (lim > 0) {
            uint4 w[2];
            lx_load(a, my, lim, w);
            const uint32_t head = s_head[tid];
            uint32_t f = 0;
            if (head == 0 && lim == LX_ITEMS) {
#pragma unroll
                for (int j = 0; j < LX_ITEMS; ++j) f = s_step[f * C1 + s_cls[byte_of(w, j)]];
            } else {
#pragma unroll
                for (int j = 0; j < LX_ITEMS; ++j) {
                    if (j < lim) {
                        const uint32_t c = s_cls[byte_of(w, j)];
                        if ((head >> j) & 1u) f = E + (s_cd[INIT * C1 + c] & 0x7fffu);
                        else if (f >= (uint32_t)E) f = E + (s_cd[(f - E) * C1 + c] & 0x7fffu);
                        else f = s_step[f * C1 + c];
                    }
                }
            }
            a.chunk_f[my / LX_ITEMS] = (uint16_t)f;
        }
        __syncthreads();
    }
}

// ---- kernel 2: states entering the chunks -----------------------------------
__device__ __forceinline__ uint32_t lx_app(const uint8_t* s_app, uint32_t E, uint32_t f, uint32_t s) {
    return f >= E ? f - E : s_app[f * 32 + s];
}

__global__ void __launch_bounds__(LS_WARPS * 32) lex3_scan_kernel(Lex3Args a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t E = (uint32_t)a.t.E;
    uint8_t* s_app = smem;
    __shared__ uint8_t s_sv[LS_WARPS][32][32];  // [warp][lane segment][start state] -> state
    __shared__ uint8_t s_wagg[LS_WARPS][32];
    __shared__ uint8_t s_wpre[LS_WARPS][32];
    __shared__ uint32_t s_tile, s_sin;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.t.app8);
        uint4* dst = reinterpret_cast<uint4*>(s_app);
        for (uint32_t i = tid; i < E * 2; i += LS_WARPS * 32) dst[i] = src[i];
    }
    const uint32_t INIT = 1u;
    const long long M = a.n_chunks;
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(&a.tickets[0], 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= a.num_scan_tiles) break;
        const long long base = (long long)tile * LS_TILE + (long long)warp * (32 * LS_G) + (long long)lane * LS_G;

        // this lane's 16 chunk endomorphisms, two per word
        uint32_t fr[LS_G / 2];
        if (base + LS_G <= M) {
            const uint4* p = reinterpret_cast<const uint4*>(a.chunk_f + base);
            const uint4 v0 = p[0], v1 = p[1];
            fr[0] = v0.x; fr[1] = v0.y; fr[2] = v0.z; fr[3] = v0.w;
            fr[4] = v1.x; fr[5] = v1.y; fr[6] = v1.z; fr[7] = v1.w;
        } else {
#pragma unroll
            for (int q = 0; q < LS_G / 2; ++q) {
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
            for (int q = 0; q < LS_G / 2; ++q) {
                const uint32_t v = __shfl_sync(ALP_FULL_MASK, fr[q], l2);
                cur = lx_app(s_app, E, v & 0xffffu, cur);
                cur = lx_app(s_app, E, v >> 16, cur);
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
            uint32_t sin;
            if (tile == 0) {
                sin = INIT;
            } else {
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
        uint32_t ob[LS_G / 4] = {0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < LS_G / 2; ++q) {
            ob[q >> 1] |= st << (16 * (q & 1));
            st = lx_app(s_app, E, fr[q] & 0xffffu, st);
            ob[q >> 1] |= st << (16 * (q & 1) + 8);
            st = lx_app(s_app, E, fr[q] >> 16, st);
        }
        if (base + LS_G <= M) {
            *reinterpret_cast<uint4*>(a.chunk_s + base) = make_uint4(ob[0], ob[1], ob[2], ob[3]);
        } else {
#pragma unroll
            for (int g = 0; g < LS_G; ++g)
                if (base + g < M) a.chunk_s[base + g] = (uint8_t)(ob[g >> 2] >> (8 * (g & 3)));
        }
        __syncthreads();
    }
}

// ---- kernel 3: tokens ---------------------------------------------------------
template <typename TermT, typename PosT>
__global__ void __launch_bounds__(LX_THREADS, 4) lex3_emit_kernel(Lex3Args a, LexSeg sg) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int S = a.t.S;
    uint16_t* s_ent = reinterpret_cast<uint16_t*>(smem);
    uint32_t* s_tok = reinterpret_cast<uint32_t*>(smem + lex3_tok_off(S));
    uint32_t* s_start = reinterpret_cast<uint32_t*>(smem + lex3_stage_off(S));
    uint32_t* s_end = s_start + LX_STAGE;
    uint16_t* s_term = reinterpret_cast<uint16_t*>(s_end + LX_STAGE);

    __shared__ uint32_t s_tile;
    __shared__ long long s_d0;
    __shared__ unsigned long long s_dmax;
    __shared__ uint32_t s_head[LX_THREADS], s_last[LX_THREADS];
    __shared__ uint32_t s_wc[LX_THREADS / 32], s_wp[LX_THREADS / 32];
    __shared__ uint32_t s_xc, s_xp, s_bc;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.t.ent);
        uint4* dst = reinterpret_cast<uint4*>(s_ent);
        for (int i = tid; i < (S * LX_ROW * 2 + 15) / 16; i += LX_THREADS) dst[i] = src[i];
    }
    for (int i = tid; i < S; i += LX_THREADS) s_tok[i] = a.t.tokinfo[i];
    const long long n = a.n;
    const long long ND = sg.n_docs;
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
        if (tid == 0) {
            s_tile = atomicAdd(&a.tickets[1], 1u);
            if (s_tile < a.num_tiles) {
                s_d0 = ND > 1 ? a.tile_doc[s_tile] : 0;
                s_dmax = (unsigned long long)s_d0;
            }
        }
        s_head[tid] = 0;
        s_last[tid] = 0;
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= a.num_tiles) break;
        const long long t0 = (long long)tile * LX_TILE;
        const long long t1 = min(t0 + LX_TILE, n) - 1;
        const long long d0 = s_d0;
        lx_mark_docs(sg, n, d0, t0, t1, s_head, s_last, &s_dmax);
        __syncthreads();
        const long long dmax = (long long)s_dmax;
        const long long my = t0 + (long long)tid * LX_ITEMS;
        const int lim = (int)max(0ll, min((long long)LX_ITEMS, n - my));

        uint4 w[2];
        uint32_t s0 = INIT, head = 0, last = 0;
        long long mydoc = d0;
        if (lim > 0) {
            lx_load(a, my, lim, w);
            s0 = a.chunk_s[my / LX_ITEMS];
            head = s_head[tid];
            last = s_last[tid];
            if (dmax > d0) mydoc = doc_upper(sg.doc_off, d0, dmax, my);
        } else {
            w[0] = w[1] = make_uint4(0, 0, 0, 0);
        }
        const bool plain = (head | last) == 0 && lim == LX_ITEMS;

        // ---- pass 1: tokens ending here and the last start ----------------
        uint32_t cnt = 0, lastp = ALP_NONE32;
        {
            uint32_t st = s0;
            if (plain) {
#pragma unroll
                for (int j = 0; j < LX_ITEMS; ++j) {
                    const uint32_t e = s_ent[st * LX_ROW + byte_of(w, j)];
                    cnt += (e >> 5) & 1u;
                    if (e & LX_START) lastp = (uint32_t)(my + j);
                    st = e & LX_NEXT;
                }
            } else {
#pragma unroll
                for (int j = 0; j < LX_ITEMS; ++j) {
                    if (j < lim) {
                        if ((head >> j) & 1u) { st = INIT; lastp = (uint32_t)(my + j); }
                        const uint32_t e = s_ent[st * LX_ROW + byte_of(w, j)];
                        cnt += (e >> 5) & 1u;
                        if (e & LX_START) lastp = (uint32_t)(my + j);
                        st = e & LX_NEXT;
                        if (((last >> j) & 1u) && !(s_tok[st] & TOK_IGNORE)) ++cnt;
                    }
                }
            }
        }

        // ---- block scan and look-back of (count, last start) --------------
        uint32_t ic = cnt, ip = lastp;
        warp_scan_cs(ic, ip, lane);
        uint32_t ec = __shfl_up_sync(ALP_FULL_MASK, ic, 1), ep = __shfl_up_sync(ALP_FULL_MASK, ip, 1);
        if (lane == 0) { ec = 0; ep = ALP_NONE32; }
        if (lane == 31) { s_wc[warp] = ic; s_wp[warp] = ip; }
        __syncthreads();
        if (warp == 0) {
            uint32_t wc = lane < LX_THREADS / 32 ? s_wc[lane] : 0u;
            uint32_t wp = lane < LX_THREADS / 32 ? s_wp[lane] : ALP_NONE32;
            uint32_t bc = wc, bp = wp;
            warp_scan_cs(bc, bp, lane);
            uint32_t xc = __shfl_up_sync(ALP_FULL_MASK, bc, 1), xp = __shfl_up_sync(ALP_FULL_MASK, bp, 1);
            if (lane == 0) { xc = 0; xp = ALP_NONE32; }
            if (lane < LX_THREADS / 32) { s_wc[lane] = xc; s_wp[lane] = xp; }
            const uint32_t Bc = __shfl_sync(ALP_FULL_MASK, bc, LX_THREADS / 32 - 1);
            const uint32_t Bp = __shfl_sync(ALP_FULL_MASK, bp, LX_THREADS / 32 - 1);
            uint32_t Xc, Xp;
            if (tile == 0) {
                Xc = 0; Xp = 0;
                if (lane == 0) st_volatile64(&a.lb_cs[0], cs_pack(ST_P, Bc, Bp != ALP_NONE32 ? Bp : 0u));
            } else {
                if (lane == 0) st_volatile64(&a.lb_cs[tile], cs_pack(ST_A, Bc, Bp));
                uint32_t acc_c = 0, acc_p = ALP_NONE32;
                long long end = tile;
                while (true) {
                    const long long idx = end - 32 + lane;
                    const unsigned long long w2 = idx >= 0 ? wait64(&a.lb_cs[idx], &a.res->error) : cs_pack(ST_P, 0, 0);
                    const uint32_t flag = (uint32_t)(w2 >> 62);
                    const uint32_t pm = __ballot_sync(ALP_FULL_MASK, flag == ST_P);
                    const int p = pm ? 31 - __clz(pm) : -1;
                    uint32_t vc = lane >= p ? cs_count(w2) : 0u;
                    uint32_t vp = lane >= p ? cs_pos(w2) : ALP_NONE32;
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        const uint32_t oc = __shfl_down_sync(ALP_FULL_MASK, vc, d);
                        const uint32_t op = __shfl_down_sync(ALP_FULL_MASK, vp, d);
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
                if (lane == 0) st_volatile64(&a.lb_cs[tile], cs_pack(ST_P, Xc + Bc, Bp != ALP_NONE32 ? Bp : Xp));
            }
            if (lane == 0) { s_xc = Xc; s_xp = Xp; s_bc = Bc; }
        }
        __syncthreads();

        // ---- pass 2: emit ---------------------------------------------------
        const uint32_t Xc = s_xc;
        const bool staged = s_bc <= (uint32_t)LX_STAGE;
        uint32_t tcount = Xc + s_wc[warp] + ec;
        uint32_t cur = ep != ALP_NONE32 ? ep : (s_wp[warp] != ALP_NONE32 ? s_wp[warp] : s_xp);
        long long doc = mydoc;
        long long base = lim > 0 ? sg.doc_off[doc] : 0;
        auto tok = [&](uint32_t term, uint32_t st_abs, uint32_t en_abs) {
            if (staged) {
                const uint32_t k = tcount - Xc;
                s_term[k] = (uint16_t)term;
                s_start[k] = st_abs;
                s_end[k] = en_abs;
            } else {
                put((long long)tcount + sent * (2 * doc + 1), term, (long long)st_abs - base, (long long)en_abs - base);
            }
            ++tcount;
        };
        if (lim > 0) {
            uint32_t st = s0;
            if (plain) {
#pragma unroll
                for (int j = 0; j < LX_ITEMS; ++j) {
                    const uint32_t e = s_ent[st * LX_ROW + byte_of(w, j)];
                    if (e & LX_EMIT) tok(s_tok[st] & TOK_TERM_MASK, cur, (uint32_t)(my + j));
                    if (e & LX_START) cur = (uint32_t)(my + j);
                    st = e & LX_NEXT;
                }
            } else {
#pragma unroll
                for (int j = 0; j < LX_ITEMS; ++j) {
                    if (j < lim) {
                        const long long pos = my + j;
                        if ((head >> j) & 1u) {
                            // every document starting here (empty ones first, then the real one)
                            doc = doc_upper(sg.doc_off, d0, dmax, pos);
                            const long long dl = doc_lower(sg.doc_off, 0, doc, pos);
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
                        const uint32_t e = s_ent[st * LX_ROW + byte_of(w, j)];
                        if (e & LX_EMIT) tok(s_tok[st] & TOK_TERM_MASK, cur, (uint32_t)pos);
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
            }
        }
        if (my <= n - 1 && n - 1 < my + LX_ITEMS) {
            // documents that start at n (empty, at the end) and the closing offset
            for (long long e2 = doc + 1; e2 < ND; ++e2) {
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

        // ---- coalesced copy of the staged tokens -----------------------------
        if (staged) {
            const uint32_t Bc = s_bc;
            for (uint32_t k = tid; k < Bc; k += LX_THREADS) {
                const uint32_t en = s_end[k];
                const long long dk = dmax > d0 ? doc_upper(sg.doc_off, d0, dmax, (long long)en - 1) : d0;
                const long long bk = sg.doc_off[dk];
                put((long long)(Xc + k) + sent * (2 * dk + 1), s_term[k], (long long)s_start[k] - bk, (long long)en - bk);
            }
        }
        __syncthreads();
    }
}

}  // namespace alp
