// Speculative front end of the multi-kernel lexer (sm_100a).
//
// The MLP predicts the DFA state at every block boundary (block = C bytes, a
// multiple of 256).  spec3_run_kernel runs one thread per block from its
// predicted state over the block's bytes and writes exactly what
// lex3_fold/scan/count would: the state entering each 32-byte chunk and the
// chunk's token count and last token start, plus the block's end state.  The
// flag / fix kernels of spec.cuh then repeat the blocks whose start differs
// from their predecessor's end until every start is exact (block 0 starts in
// the initial state), and spec3_tiles_kernel sums the chunk counts per 8 KiB
// tile for the tile scan and token pass of lex3.cuh.  At that fixpoint the
// chunk states are the composition scan's, so the tokens equal alp_lex's; the
// prediction only decides how much work is redone.  One document (the whole
// input); token semantics futhark/lexer.fut:103-172.
#pragma once
#include "common.cuh"
#include "lex3.cuh"
#include "spec.cuh"

namespace alp {

constexpr int SP3_GROUP = 8;  // chunks whose outputs a thread stores together

// One thread per block (or per listed block): chunk states, chunk counts,
// block end state.  Shared memory as lex3_count_kernel (transition table and
// token info).
__global__ void __launch_bounds__(256) spec3_run_kernel(SpecArgs sa, Lex3Args a) {
    extern __shared__ __align__(16) uint8_t smem[];
    const int S = a.t.S;
    uint16_t* s_ent = reinterpret_cast<uint16_t*>(smem);
    uint32_t* s_tok = reinterpret_cast<uint32_t*>(smem + lex3_tok_off(S));
    const int tid = threadIdx.x;
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.t.ent);
        uint4* dst = reinterpret_cast<uint4*>(s_ent);
        for (int i = tid; i < (S * LX_ROW * 2 + 15) / 16; i += blockDim.x) dst[i] = src[i];
    }
    for (int i = tid; i < S; i += blockDim.x) s_tok[i] = a.t.tokinfo[i];
    __syncthreads();
    const long long n = a.n;
    const long long total = sa.list ? sa.list_n : sa.K;
    for (long long idx = (long long)blockIdx.x * blockDim.x + tid; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long j = sa.list ? (long long)sa.list[idx] : idx;
        const long long b0 = j * sa.C, b1 = min(b0 + sa.C, n);
        uint32_t st = sa.st[j];
        for (long long g0 = b0; g0 < b1; g0 += SP3_GROUP * LX_CHUNK) {
            uint32_t gs[SP3_GROUP / 4] = {0, 0};    // chunk states, a byte each
            uint32_t gc[SP3_GROUP / 2] = {0, 0, 0, 0};  // chunk counts, 16 bits each
#pragma unroll 1
            for (int q = 0; q < SP3_GROUP; ++q) {
                const long long p = g0 + (long long)q * LX_CHUNK;
                if (p >= b1) break;
                const int lim = (int)min((long long)LX_CHUNK, b1 - p);
                gs[q >> 2] |= st << (8 * (q & 3));
                uint32_t cnt = 0, lo = p == 0 ? 0u : LX_NOOFF;  // the document head at 0 starts a token
                if (a.aligned16 && lim == LX_CHUNK) {
                    const uint4* src = reinterpret_cast<const uint4*>(a.in + p);
                    const uint4 w0 = __ldg(src), w1 = __ldg(src + 1);
                    const uint4 w[2] = {w0, w1};
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
                if (p + lim == n && !(s_tok[st] & TOK_IGNORE)) ++cnt;  // the last token of the document
                gc[q >> 1] |= (cnt | (lo << 8)) << (16 * (q & 1));
            }
            const long long c0 = g0 / LX_CHUNK;
            if (g0 + SP3_GROUP * LX_CHUNK <= b1) {
                *reinterpret_cast<uint2*>(a.chunk_s + c0) = make_uint2(gs[0], gs[1]);
                *reinterpret_cast<uint4*>(a.chunk_c + c0) = make_uint4(gc[0], gc[1], gc[2], gc[3]);
            } else {
                for (int q = 0; q < SP3_GROUP && g0 + (long long)q * LX_CHUNK < b1; ++q) {
                    a.chunk_s[c0 + q] = (uint8_t)(gs[q >> 2] >> (8 * (q & 3)));
                    a.chunk_c[c0 + q] = (uint16_t)(gc[q >> 1] >> (16 * (q & 1)));
                }
            }
        }
        sa.en[j] = (uint8_t)st;
    }
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
