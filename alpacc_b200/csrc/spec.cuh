// Speculative lexer (learned boundary states).
//
// The input is cut into chunks of C bytes.  Chunk 0 starts in the initial
// state; chunk j >= 1 starts in the state the MLP predicts from the 64 bytes
// before it.  Every chunk runs the DFA from its start state (spec_run_kernel),
// then verification compares each chunk's start with its predecessor's end:
// where they differ the start is replaced and the chunk re-runs
// (spec_fix_kernel, repeated until nothing changes).  At that fixpoint every
// start state is the exact state (chunk 0 is exact and each start equals the
// exact end of its predecessor), so the tokens written by spec_emit_kernel
// are exactly those of the composition scan -- the prediction only decides
// how much work is redone.  Token semantics are the single-pass lexer's
// (futhark/lexer.fut:103-172).
#pragma once
#include "common.cuh"
#include "lexer.cuh"

namespace alp {

struct SpecArgs {
    const uint8_t* in;
    long long n;
    long long C;               // chunk bytes (multiple of 16)
    long long K;               // chunks
    LexTables t;
    uint8_t* st;               // [K] start state per chunk
    uint8_t* en;               // [K] end state per chunk
    uint32_t* cnt;             // [K] tokens ending inside the chunk
    uint32_t* lastp;           // [K] last token start inside the chunk (NONE)
    const uint32_t* list;      // chunks to (re)run; null = all
    long long list_n;
    uint32_t* next_list;       // chunks whose start changed
    unsigned int* next_n;
    // emission
    const uint32_t* cnt_excl;  // [K] tokens before the chunk
    const uint32_t* pos_excl;  // [K] last token start before the chunk
    uint32_t* out_term;
    int64_t* out_start;
    int64_t* out_end;
    long long cap;
    AlpResult* res;
};

// Run the DFA over one chunk from its start state.
__device__ __forceinline__ void spec_chunk(const SpecArgs& a, long long j, const uint8_t* s_cls, const uint16_t* s_cd,
                                           const uint32_t* s_tok) {
    const int C1 = a.t.C1;
    const long long b0 = j * a.C, b1 = min(b0 + a.C, a.n);
    uint32_t s = a.st[j], cnt = 0, lp = ALP_NONE32;
    for (long long p = b0; p < b1; p += 16) {
        uint8_t bytes[16];
        if (p + 16 <= b1 && ((reinterpret_cast<uintptr_t>(a.in + p) & 15u) == 0)) {
            const uint4 w = __ldg(reinterpret_cast<const uint4*>(a.in + p));
            const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int q = 0; q < 16; ++q) bytes[q] = (uint8_t)(ws[q >> 2] >> (8 * (q & 3)));
        } else {
#pragma unroll
            for (int q = 0; q < 16; ++q) bytes[q] = p + q < b1 ? a.in[p + q] : 0;
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            if (p + q >= b1) break;
            const uint32_t e = s_cd[s * C1 + s_cls[bytes[q]]];
            const uint32_t s2 = e & 0x7fffu;
            if (e & 0x8000u) {
                if (!(s_tok[s] & TOK_IGNORE)) ++cnt;
                if (!(s_tok[s2] & TOK_IGNORE)) lp = (uint32_t)(p + q);
            }
            s = s2;
        }
    }
    a.en[j] = (uint8_t)s;
    a.cnt[j] = cnt;
    a.lastp[j] = lp;
}

__device__ __forceinline__ void spec_load_tables(const LexTables& t, uint8_t* s_cls, uint16_t* s_cd, uint32_t* s_tok) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) s_cls[i] = t.cls[i];
    for (int i = threadIdx.x; i < t.S * t.C1; i += blockDim.x) s_cd[i] = t.cdelta[i];
    for (int i = threadIdx.x; i < t.S; i += blockDim.x) s_tok[i] = t.tokinfo[i];
    __syncthreads();
}

constexpr size_t spec_smem_bytes(int S, int C1) { return 256 + 4 * (size_t)S + 2 * (size_t)S * C1 + 16; }

__global__ void spec_run_kernel(SpecArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint8_t* s_cls = smem;
    uint32_t* s_tok = reinterpret_cast<uint32_t*>(smem + 256);
    uint16_t* s_cd = reinterpret_cast<uint16_t*>(smem + 256 + 4 * a.t.S);
    spec_load_tables(a.t, s_cls, s_cd, s_tok);
    const long long total = a.list ? a.list_n : a.K;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
        spec_chunk(a, a.list ? (long long)a.list[i] : i, s_cls, s_cd, s_tok);
}

// Verification, step 1: flag every chunk whose start differs from its
// predecessor's end.
__global__ void spec_flag_kernel(SpecArgs a, uint8_t* flag) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < a.K; j += (long long)gridDim.x * blockDim.x)
        flag[j] = (j > 0 && a.st[j] != a.en[j - 1]) ? 1 : 0;
}

// Step 2: a flagged chunk whose predecessor is not flagged takes the
// predecessor's end as its start and is queued for a re-run.  A chunk behind
// another flagged chunk waits: that predecessor's end came from a start that is
// being replaced (often the dead state after a wrong guess), and copying it
// would carry the error forward one chunk per round.
__global__ void spec_fix_kernel(SpecArgs a, const uint8_t* flag) {
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x + 1; j < a.K; j += (long long)gridDim.x * blockDim.x) {
        if (flag[j] && !flag[j - 1]) {
            a.st[j] = a.en[j - 1];
            const unsigned int k = atomicAdd(a.next_n, 1u);
            a.next_list[k] = (uint32_t)j;
        }
    }
}

// Exclusive scan of (count, last start) over chunks: per-block pass, a pass
// over the block totals, then the fix-up pass.
constexpr int SPEC_SCAN_BLOCK = 1024;

__global__ void __launch_bounds__(SPEC_SCAN_BLOCK) spec_scan_local(const uint32_t* cnt, const uint32_t* lp, long long K,
                                                                   uint32_t* ex_c, uint32_t* ex_p, uint32_t* blk_c,
                                                                   uint32_t* blk_p) {
    __shared__ uint32_t s_c[32], s_p[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long j = (long long)blockIdx.x * SPEC_SCAN_BLOCK + tid;
    uint32_t c = j < K ? cnt[j] : 0u, p = j < K ? lp[j] : ALP_NONE32;
    const uint32_t c0 = c, p0 = p;
    warp_scan_cs(c, p, lane);
    if (lane == 31) { s_c[warp] = c; s_p[warp] = p; }
    __syncthreads();
    if (warp == 0) {
        uint32_t wc = s_c[lane], wp = s_p[lane];
        uint32_t ic = wc, ip = wp;
        warp_scan_cs(ic, ip, lane);
        uint32_t xc = __shfl_up_sync(ALP_FULL_MASK, ic, 1), xp = __shfl_up_sync(ALP_FULL_MASK, ip, 1);
        if (lane == 0) { xc = 0; xp = ALP_NONE32; }
        s_c[lane] = xc;
        s_p[lane] = xp;
        if (lane == 31) { blk_c[blockIdx.x] = ic; blk_p[blockIdx.x] = ip; }
    }
    __syncthreads();
    // exclusive within the block
    uint32_t ec = s_c[warp] + c - c0;
    uint32_t ep;
    {
        // exclusive take-right: the inclusive value of lanes before this one
        uint32_t ip2 = __shfl_up_sync(ALP_FULL_MASK, p, 1);
        if (lane == 0) ip2 = ALP_NONE32;
        ep = ip2 != ALP_NONE32 ? ip2 : s_p[warp];
    }
    (void)p0;
    if (j < K) { ex_c[j] = ec; ex_p[j] = ep; }
}

__global__ void __launch_bounds__(1024) spec_scan_blocks(uint32_t* blk_c, uint32_t* blk_p, long long nb) {
    // sequential over chunks of 1024 block totals (few thousand at most)
    __shared__ uint32_t s_c[32], s_p[32];
    __shared__ uint32_t carry_c, carry_p;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) { carry_c = 0; carry_p = 0; }  // the input starts a token at 0
    __syncthreads();
    for (long long b = 0; b < nb; b += 1024) {
        uint32_t c = b + tid < nb ? blk_c[b + tid] : 0u, p = b + tid < nb ? blk_p[b + tid] : ALP_NONE32;
        const uint32_t c0 = c;
        warp_scan_cs(c, p, lane);
        if (lane == 31) { s_c[warp] = c; s_p[warp] = p; }
        __syncthreads();
        if (warp == 0) {
            uint32_t ic = s_c[lane], ip = s_p[lane];
            warp_scan_cs(ic, ip, lane);
            uint32_t xc = __shfl_up_sync(ALP_FULL_MASK, ic, 1), xp = __shfl_up_sync(ALP_FULL_MASK, ip, 1);
            if (lane == 0) { xc = 0; xp = ALP_NONE32; }
            s_c[lane] = xc;
            s_p[lane] = xp;
        }
        __syncthreads();
        uint32_t ip2 = __shfl_up_sync(ALP_FULL_MASK, p, 1);
        if (lane == 0) ip2 = ALP_NONE32;
        uint32_t epw = ip2 != ALP_NONE32 ? ip2 : s_p[warp];
        const uint32_t ecw = s_c[warp] + c - c0;
        const uint32_t cc = carry_c, cp = carry_p;
        __syncthreads();
        if (b + tid < nb) {
            blk_c[b + tid] = cc + ecw;
            blk_p[b + tid] = epw != ALP_NONE32 ? epw : cp;
        }
        if (tid == 1023) {
            carry_c = cc + ecw + c0;
            const uint32_t lastp = p != ALP_NONE32 ? p : (epw != ALP_NONE32 ? epw : cp);
            carry_p = lastp;
        }
        __syncthreads();
    }
}

__global__ void spec_scan_add(uint32_t* ex_c, uint32_t* ex_p, long long K, const uint32_t* blk_c, const uint32_t* blk_p) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= K) return;
    const long long b = j / SPEC_SCAN_BLOCK;
    ex_c[j] += blk_c[b];
    if (ex_p[j] == ALP_NONE32) ex_p[j] = blk_p[b];
}

// Write every chunk's tokens (and, for the last chunk, the final token).
__global__ void spec_emit_kernel(SpecArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint8_t* s_cls = smem;
    uint32_t* s_tok = reinterpret_cast<uint32_t*>(smem + 256);
    uint16_t* s_cd = reinterpret_cast<uint16_t*>(smem + 256 + 4 * a.t.S);
    spec_load_tables(a.t, s_cls, s_cd, s_tok);
    const int C1 = a.t.C1;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < a.K; j += (long long)gridDim.x * blockDim.x) {
        const long long b0 = j * a.C, b1 = min(b0 + a.C, a.n);
        uint32_t s = a.st[j];
        uint32_t tc = a.cnt_excl[j];
        uint32_t cur = a.pos_excl[j];
        for (long long p = b0; p < b1; ++p) {
            const uint32_t e = s_cd[s * C1 + s_cls[a.in[p]]];
            const uint32_t s2 = e & 0x7fffu;
            if (e & 0x8000u) {
                const uint32_t ti = s_tok[s];
                if (!(ti & TOK_IGNORE)) {
                    if ((long long)tc < a.cap) {
                        a.out_term[tc] = ti & TOK_TERM_MASK;
                        a.out_start[tc] = cur;
                        a.out_end[tc] = p;
                    } else {
                        atomicOr(&a.res->error, ALP_DEV_ERR_CAPACITY);
                    }
                    ++tc;
                }
                if (!(s_tok[s2] & TOK_IGNORE)) cur = (uint32_t)p;
            }
            s = s2;
        }
        if (j == a.K - 1) {
            const uint32_t ti = s_tok[s];
            long long total = tc;
            if (!(ti & TOK_IGNORE)) {
                if (total < a.cap) {
                    a.out_term[total] = ti & TOK_TERM_MASK;
                    a.out_start[total] = cur;
                    a.out_end[total] = a.n;
                }
                ++total;
            }
            a.res->count = total;
            a.res->valid = (ti & TOK_ACCEPT) ? 1 : 0;
        }
    }
}

}  // namespace alp
