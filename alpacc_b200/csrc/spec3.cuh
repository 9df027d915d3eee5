// Speculative front end of the multi-kernel lexer (sm_100a).
//
// The MLP predicts the DFA state at every block boundary (block = C bytes, a
// multiple of 256).  spec3_run_kernel runs each block from its predicted
// state (two blocks per thread) and writes exactly what lex3_fold/scan/count
// would: the state entering each 32-byte chunk and the chunk's token count and
// last token start, plus the block's end state.  The flag / fix kernels of
// spec.cuh list the blocks whose start differs from their predecessor's end,
// spec3_fixup_kernel re-runs them on the device until every start is exact
// (block 0 starts in the initial state), and spec3_tiles_kernel sums the chunk
// counts per 8 KiB tile for the tile scan and token pass of lex3.cuh.  At that fixpoint the
// chunk states are the composition scan's, so the tokens equal alp_lex's; the
// prediction only decides how much work is redone.  One document (the whole
// input); token semantics futhark/lexer.fut:103-172.
#pragma once
#include "common.cuh"
#include "lex3.cuh"
#include "spec.cuh"

namespace alp {

constexpr int SP3_GROUP = 8;  // chunks whose outputs a thread stores together
constexpr int SP3_FIX_CAP = 2048;  // blocks one fix-up round holds

// The DFA over one 32-byte chunk at p (lim bytes) from state st: token count
// and last start offset (LX_NOOFF: none); the document head at 0 starts a
// token, the last byte of the input ends one.
template <bool VEC>
__device__ __forceinline__ uint32_t sp3_chunk(const Lex3Args& a, const uint16_t* s_ent, const uint32_t* s_tok,
                                              long long p, int lim, const uint4 (&w)[2], uint32_t& st) {
    uint32_t cnt = 0, lo = p == 0 ? 0u : LX_NOOFF;
    if (VEC) {
#pragma unroll
        for (int k = 0; k < LX_CHUNK; ++k) {
            const uint32_t e = s_ent[st * LX_ROW + byte_of(w, k)];
            cnt += (e >> 6) & 1u;
            if (e & LX_START) lo = (uint32_t)k;
            st = e & LX_NEXT;
        }
    } else {
#pragma unroll 1
        for (int k = 0; k < lim; ++k) {
            const uint32_t e = s_ent[st * LX_ROW + __ldg(a.in + p + k)];
            cnt += (e >> 6) & 1u;
            if (e & LX_START) lo = (uint32_t)k;
            st = e & LX_NEXT;
        }
    }
    if (p + lim == a.n && !(s_tok[st] & TOK_IGNORE)) ++cnt;
    return cnt | (lo << 8);
}

__device__ __forceinline__ void sp3_tables(const Lex3Args& a, uint16_t* s_ent, uint32_t* s_tok) {
    const int S = a.t.S;
    const uint4* src = reinterpret_cast<const uint4*>(a.t.ent);
    uint4* dst = reinterpret_cast<uint4*>(s_ent);
    for (int i = threadIdx.x; i < (S * LX_ROW * 2 + 15) / 16; i += blockDim.x) dst[i] = src[i];
    for (int i = threadIdx.x; i < S; i += blockDim.x) s_tok[i] = a.t.tokinfo[i];
}

// One thread per pair of blocks (2i, 2i+1), two independent DFA chains with
// the next chunk's bytes loaded ahead: chunk states, chunk counts (stored
// eight chunks at a time), block end states.
__global__ void __launch_bounds__(256) spec3_run_kernel(SpecArgs sa, Lex3Args a) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint16_t* s_ent = reinterpret_cast<uint16_t*>(smem);
    uint32_t* s_tok = reinterpret_cast<uint32_t*>(smem + lex3_tok_off(a.t.S));
    sp3_tables(a, s_ent, s_tok);
    __syncthreads();
    const long long n = a.n;
    const long long pairs = (sa.K + 1) / 2;
    const bool vec_ok = a.aligned16 != 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < pairs;
         i += (long long)gridDim.x * blockDim.x) {
        long long b0[2], b1[2];
        uint32_t st[2];
        bool on[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const long long j = 2 * i + h;
            on[h] = j < sa.K;
            b0[h] = on[h] ? j * sa.C : n;
            b1[h] = on[h] ? min(b0[h] + sa.C, n) : n;
            st[h] = on[h] ? sa.st[j] : 1u;
        }
        // both blocks advance group by group (a group = SP3_GROUP chunks)
        const long long groups = (sa.C + SP3_GROUP * LX_CHUNK - 1) / (SP3_GROUP * LX_CHUNK);
        for (long long gi = 0; gi < groups; ++gi) {
            uint32_t gs[2][2] = {{0, 0}, {0, 0}};
            uint32_t gc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
            uint4 w[2][2], wn[2][2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const long long p = b0[h] + gi * SP3_GROUP * LX_CHUNK;
                if (vec_ok && p + LX_CHUNK <= b1[h]) {
                    w[h][0] = __ldg(reinterpret_cast<const uint4*>(a.in + p));
                    w[h][1] = __ldg(reinterpret_cast<const uint4*>(a.in + p) + 1);
                } else {
                    w[h][0] = w[h][1] = make_uint4(0, 0, 0, 0);
                }
            }
#pragma unroll 1
            for (int q = 0; q < SP3_GROUP; ++q) {
                // load the next chunk of each block while this one runs
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const long long pn = b0[h] + (gi * SP3_GROUP + q + 1) * LX_CHUNK;
                    if (q + 1 < SP3_GROUP && vec_ok && pn + LX_CHUNK <= b1[h]) {
                        wn[h][0] = __ldg(reinterpret_cast<const uint4*>(a.in + pn));
                        wn[h][1] = __ldg(reinterpret_cast<const uint4*>(a.in + pn) + 1);
                    } else {
                        wn[h][0] = wn[h][1] = make_uint4(0, 0, 0, 0);
                    }
                }
                const long long pa = b0[0] + (gi * SP3_GROUP + q) * LX_CHUNK;
                const long long pb = b0[1] + (gi * SP3_GROUP + q) * LX_CHUNK;
                const bool va = pa < b1[0], vb = pb < b1[1];
                const int la = va ? (int)min((long long)LX_CHUNK, b1[0] - pa) : 0;
                const int lb = vb ? (int)min((long long)LX_CHUNK, b1[1] - pb) : 0;
                if (va) gs[0][q >> 2] |= st[0] << (8 * (q & 3));
                if (vb) gs[1][q >> 2] |= st[1] << (8 * (q & 3));
                if (va && vb && vec_ok && la == LX_CHUNK && lb == LX_CHUNK && pa + la != n && pb + lb != n) {
                    // the common case: two full chunks, two interleaved chains
                    uint32_t ca = 0, cb = 0, oa = pa == 0 ? 0u : LX_NOOFF, ob = LX_NOOFF;
                    uint32_t sa0 = st[0], sb0 = st[1];
#pragma unroll
                    for (int k = 0; k < LX_CHUNK; ++k) {
                        const uint32_t ea = s_ent[sa0 * LX_ROW + byte_of(w[0], k)];
                        const uint32_t eb = s_ent[sb0 * LX_ROW + byte_of(w[1], k)];
                        ca += (ea >> 6) & 1u;
                        cb += (eb >> 6) & 1u;
                        if (ea & LX_START) oa = (uint32_t)k;
                        if (eb & LX_START) ob = (uint32_t)k;
                        sa0 = ea & LX_NEXT;
                        sb0 = eb & LX_NEXT;
                    }
                    st[0] = sa0;
                    st[1] = sb0;
                    gc[0][q >> 1] |= (ca | (oa << 8)) << (16 * (q & 1));
                    gc[1][q >> 1] |= (cb | (ob << 8)) << (16 * (q & 1));
                } else {
                    if (va) {
                        const uint32_t r = (vec_ok && la == LX_CHUNK) ? sp3_chunk<true>(a, s_ent, s_tok, pa, la, w[0], st[0])
                                                                   : sp3_chunk<false>(a, s_ent, s_tok, pa, la, w[0], st[0]);
                        gc[0][q >> 1] |= r << (16 * (q & 1));
                    }
                    if (vb) {
                        const uint32_t r = (vec_ok && lb == LX_CHUNK) ? sp3_chunk<true>(a, s_ent, s_tok, pb, lb, w[1], st[1])
                                                                   : sp3_chunk<false>(a, s_ent, s_tok, pb, lb, w[1], st[1]);
                        gc[1][q >> 1] |= r << (16 * (q & 1));
                    }
                }
#pragma unroll
                for (int h = 0; h < 2; ++h) { w[h][0] = wn[h][0]; w[h][1] = wn[h][1]; }
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const long long g0 = b0[h] + gi * SP3_GROUP * LX_CHUNK;
                if (g0 >= b1[h]) continue;
                const long long c0 = g0 / LX_CHUNK;
                if (g0 + SP3_GROUP * LX_CHUNK <= b1[h]) {
                    *reinterpret_cast<uint2*>(a.chunk_s + c0) = make_uint2(gs[h][0], gs[h][1]);
                    *reinterpret_cast<uint4*>(a.chunk_c + c0) = make_uint4(gc[h][0], gc[h][1], gc[h][2], gc[h][3]);
                } else {
                    for (int q = 0; q < SP3_GROUP && g0 + (long long)q * LX_CHUNK < b1[h]; ++q) {
                        a.chunk_s[c0 + q] = (uint8_t)(gs[h][q >> 2] >> (8 * (q & 3)));
                        a.chunk_c[c0 + q] = (uint16_t)(gc[h][q >> 1] >> (16 * (q & 1)));
                    }
                }
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
            if (on[h]) sa.en[2 * i + h] = (uint8_t)st[h];
    }
}

// Re-runs block j from its (corrected) start state, chunk by chunk, until its
// state at a chunk boundary equals the one the previous run stored there: from
// that chunk on the block's outputs and end state are unchanged.
__device__ __forceinline__ void sp3_rerun(const SpecArgs& sa, const Lex3Args& a, const uint16_t* s_ent,
                                          const uint32_t* s_tok, long long j) {
    const long long b0 = j * sa.C, b1 = min(b0 + sa.C, a.n);
    uint32_t st = sa.st[j];
    const bool vec_ok = a.aligned16 != 0;
    uint4 w[2], wn[2];
    w[0] = w[1] = make_uint4(0, 0, 0, 0);
    if (vec_ok && b0 + LX_CHUNK <= b1) {
        w[0] = __ldg(reinterpret_cast<const uint4*>(a.in + b0));
        w[1] = __ldg(reinterpret_cast<const uint4*>(a.in + b0) + 1);
    }
    for (long long p = b0; p < b1; p += LX_CHUNK) {
        const long long c = p / LX_CHUNK;
        const uint32_t old = a.chunk_s[c];
        // the next chunk's bytes while this one runs
        wn[0] = wn[1] = make_uint4(0, 0, 0, 0);
        if (vec_ok && p + 2 * LX_CHUNK <= b1) {
            wn[0] = __ldg(reinterpret_cast<const uint4*>(a.in + p + LX_CHUNK));
            wn[1] = __ldg(reinterpret_cast<const uint4*>(a.in + p + LX_CHUNK) + 1);
        }
        if (p > b0 && old == st) return;  // rejoined the stored trajectory
        a.chunk_s[c] = (uint8_t)st;
        const int lim = (int)min((long long)LX_CHUNK, b1 - p);
        a.chunk_c[c] = (uint16_t)((vec_ok && lim == LX_CHUNK) ? sp3_chunk<true>(a, s_ent, s_tok, p, lim, w, st)
                                                              : sp3_chunk<false>(a, s_ent, s_tok, p, lim, w, st));
        w[0] = wn[0];
        w[1] = wn[1];
    }
    sa.en[j] = (uint8_t)st;
}

// The fix-up loop on the device (one CTA): the listed blocks (flagged, with
// an unflagged predecessor) take their predecessor's end state and re-run;
// then the first block after each re-run block whose start differs from its
// predecessor's end is fixed the same way (blocks in between that were
// flagged at first and now agree are final), round after round, until none
// is left.
// res->aux[0] = rounds (-1: gave up), res->aux[1] = blocks re-run,
// res->aux[2] = blocks in the first list.
__global__ void __launch_bounds__(256) spec3_fixup_kernel(SpecArgs sa, Lex3Args a, const uint32_t* first,
                                                          const unsigned int* first_n, const uint8_t* flag0,
                                                          int max_rounds) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint16_t* s_ent = reinterpret_cast<uint16_t*>(smem);
    uint32_t* s_tok = reinterpret_cast<uint32_t*>(smem + lex3_tok_off(a.t.S));
    __shared__ uint32_t s_list[2][SP3_FIX_CAP];
    __shared__ unsigned int s_n[2];
    sp3_tables(a, s_ent, s_tok);
    if (threadIdx.x == 0) { s_n[0] = min(*first_n, (unsigned)SP3_FIX_CAP); s_n[1] = 0; }
    __syncthreads();
    const unsigned int n0 = s_n[0];
    if (*first_n > (unsigned)SP3_FIX_CAP) {
        if (threadIdx.x == 0) { a.res->aux[0] = -1; a.res->aux[1] = 0; a.res->aux[2] = *first_n; }
        return;
    }
    for (unsigned int i = threadIdx.x; i < n0; i += blockDim.x) s_list[0][i] = first[i];
    __syncthreads();
    long long rounds = 0, reruns = 0;
    int cur = 0;
    while (s_n[cur] > 0) {
        if (rounds >= max_rounds) { rounds = -1; break; }
        ++rounds;
        const unsigned int m = s_n[cur];
        reruns += m;
        for (unsigned int i = threadIdx.x; i < m; i += blockDim.x) sp3_rerun(sa, a, s_ent, s_tok, s_list[cur][i]);
        __syncthreads();
        if (threadIdx.x == 0) s_n[cur ^ 1] = 0;
        __syncthreads();
        bool overflow = false;
        for (unsigned int i = threadIdx.x; i < m; i += blockDim.x) {
            // Walk past successors that are consistent now: a block that was
            // inconsistent at first (its predecessor was too) and now agrees
            // with its predecessor ran from its exact start, so its end is
            // final and its own successor is checked next.
            for (long long j = (long long)s_list[cur][i] + 1; j < sa.K; ++j) {
                if (sa.st[j] != sa.en[j - 1]) {
                    sa.st[j] = sa.en[j - 1];
                    const unsigned int k = atomicAdd(&s_n[cur ^ 1], 1u);
                    if (k < (unsigned)SP3_FIX_CAP) s_list[cur ^ 1][k] = (uint32_t)j;
                    else overflow = true;
                    break;
                }
                if (!flag0[j]) break;  // consistent from the start: nothing waits behind it
            }
        }
        if (__syncthreads_or(overflow)) { rounds = -1; break; }
        cur ^= 1;
    }
    if (threadIdx.x == 0) { a.res->aux[0] = rounds; a.res->aux[1] = reruns; a.res->aux[2] = *first_n; }
}

// Per 8 KiB tile: (token count, last token start) from the chunk counts.
__global__ void __launch_bounds__(LX_THREADS) spec3_tiles_kernel(Lex3Args a) {
    __shared__ uint32_t s_c[LX_THREADS / 32], s_p[LX_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (unsigned tile = blockIdx.x; tile < a.num_tiles; tile += gridDim.x) {
        const long long c = (long long)tile * (LX_TILE / LX_CHUNK) + tid;
        uint32_t cnt = 0, p = ALP_NONE32;
        if (c < a.n_chunks) {
            const uint32_t cc = a.chunk_c[c];
            cnt = cc & 0xffu;
            if ((cc >> 8) != LX_NOOFF) p = (uint32_t)(c * LX_CHUNK + (cc >> 8));
        }
        cs_reduce_warp(cnt, p);
        if (lane == 0) { s_c[warp] = cnt; s_p[warp] = p; }
        __syncthreads();
        if (tid == 0) {
            uint32_t tc = 0, tp = ALP_NONE32;
            for (int w = 0; w < LX_THREADS / 32; ++w) {
                tc += s_c[w];
                if (s_p[w] != ALP_NONE32) tp = s_p[w];
            }
            a.tile_cs[tile] = ((unsigned long long)tc << 32) | tp;
        }
        __syncthreads();
    }
}

}  // namespace alp
