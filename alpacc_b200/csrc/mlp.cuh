// Boundary-state MLP (learned speculation): BF16 tensor-core kernels.
//
// The network predicts the DFA state at a chunk boundary from the 64 bytes
// before it: byte -> 16-d embedding (64 x 16 = 1024 inputs) -> 128 -> 128 ->
// logits over the lexer's states (padded to 32).  Weights and activations
// enter the tensor cores as BF16, every product accumulates in FP32: training
// GEMMs and the default inference kernel on tcgen05, the earlier inference
// kernel on mma.sync m16n8k16.  There is no reference counterpart: alpacc has no
// learned component; the speculative lexer that uses these predictions is
// verified against the exact composition scan, so its output is bit-exact
// whatever the network predicts.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"
#include "umma.cuh"

namespace alp {

constexpr int MLP_WIN = 64;     // window bytes
constexpr int MLP_EMB = 16;     // embedding width
constexpr int MLP_IN = MLP_WIN * MLP_EMB;  // 1024
constexpr int MLP_H = 128;      // hidden width
constexpr int MLP_OUT = 32;     // logits (states padded)

// Parameter block (FP32 masters, gradients and Adam moments share it).
constexpr int P_EMB = 0;
constexpr int P_W1 = P_EMB + 256 * MLP_EMB;
constexpr int P_B1 = P_W1 + MLP_IN * MLP_H;
constexpr int P_W2 = P_B1 + MLP_H;
constexpr int P_B2 = P_W2 + MLP_H * MLP_H;
constexpr int P_W3 = P_B2 + MLP_H;
constexpr int P_B3 = P_W3 + MLP_H * MLP_OUT;
constexpr int P_TOTAL = P_B3 + MLP_OUT;

struct MlpWeights {             // inference view: BF16 matrices, FP32 biases
    const __nv_bfloat16* emb;   // [256][16]
    const __nv_bfloat16* w1;    // [1024][128]  (k, n)
    const float* b1;
    const __nv_bfloat16* w2;    // [128][128]
    const float* b2;
    const __nv_bfloat16* w3;    // [128][32]
    const float* b3;
    int n_states;
};

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// ---------------------------------------------------------------------------
// Generic GEMM for training on the fifth-generation tensor cores:
// C[M][N] (FP32) (+)= A[M][K] . B[K][N], A and B BF16 addressed by strides (so
// transposes are free), M, N, K multiples of 16.  One CTA of 128 threads per
// 128 x UG_BN tile of C (N <= UG_BN: one tile of N columns).  Each K step of 64:
// the threads stage A (128 rows) and B^T (tile columns as rows) as K-major
// 128-byte-swizzled tiles, one thread issues four K = 16 MMAs into the tensor
// memory accumulator and commits them to an mbarrier (waits bounded), which
// hands the tiles back for the next step; the four warps then read their 32
// accumulator rows with tcgen05.ld.  Training moves about 0.3 MFLOP per
// window, so the kernel keeps one shared-memory stage and no warp roles; the
// next K step waits in registers (loads issued before the MMA wait).
// ---------------------------------------------------------------------------
struct GemmArgs {
    const __nv_bfloat16* A;
    long long sa_m, sa_k;
    const __nv_bfloat16* B;
    long long sb_k, sb_n;
    float* C;
    long long ldc;
    int M, N, K;
    int accumulate;             // C += instead of C =
    unsigned int* err;          // ALP_DEV_ERR_TIMEOUT when an MMA wait gives up
    int kper;                   // K per split (blockIdx.z); each split writes its own partial C
    long long part_stride;      // floats between splits' partials (0: one split, C itself)
};

constexpr int UG_BM = 128;
constexpr int UG_BN = 128;
constexpr int UG_BK = 64;
constexpr size_t UG_SMEM = (size_t)UG_BM * 128 + (size_t)UG_BN * 128 + 1024;  // A and B tiles, 1 KiB alignment slack

__global__ void __launch_bounds__(128) umma_gemm_kernel(GemmArgs g) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_abort;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t base = ((uint32_t)__cvta_generic_to_shared(smem_raw) + 1023u) & ~1023u;
    uint8_t* sp = smem_raw + (base - (uint32_t)__cvta_generic_to_shared(smem_raw));
    const uint32_t sa = base, sb = base + UG_BM * 128;
    const int m0 = blockIdx.y * UG_BM, n0 = blockIdx.x * UG_BN;
    const int bn = min(UG_BN, g.N - n0);               // columns of this tile: a multiple of 16
    const uint32_t ncols = bn <= 32 ? 32u : (bn <= 64 ? 64u : 128u);
    if (warp == 0) tmem_alloc(&s_tmem, ncols);
    if (tid == 0) {
        mbar_init(&s_bar, 1);
        mbar_fence_init();
        s_abort = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = umma_idesc_bf16_f32(UG_BM, bn);
    uint32_t phase = 0;
    const int kb = blockIdx.z * g.kper, ke = min(g.K, kb + g.kper);
    float* C = g.C + blockIdx.z * g.part_stride;
    // 16-byte loads where an operand's K run is contiguous and aligned
    const bool a_vec = g.sa_k == 1 && (g.sa_m & 7) == 0 && (reinterpret_cast<uintptr_t>(g.A) & 15) == 0;
    const bool b_vec = g.sb_k == 1 && (g.sb_n & 7) == 0 && (reinterpret_cast<uintptr_t>(g.B) & 15) == 0;
    // an operand whose rows are contiguous in memory (K strided: a transpose) is read with
    // consecutive threads on consecutive rows, so that every load is coalesced
    const bool a_rows = g.sa_m == 1 && g.sa_k != 1, b_rows = g.sb_n == 1 && g.sb_k != 1;
    // Each thread stages UG_CHUNKS 16-byte chunks of a K step: chunks 0 .. UG_BM/16 - 1
    // of A's rows m0.., the rest of B's columns n0.. (as rows), K-major.  All of a
    // step's loads are issued into registers before any is stored, and the next step's
    // loads are issued while the tensor cores work on this one, so a step costs about
    // one memory latency instead of one per chunk.
    constexpr int UG_CHUNKS = (UG_BM + UG_BN) * 8 / 128;
    constexpr int UG_ACH = UG_BM * 8 / 128;
    auto chunk_at = [&](int i, int& row, int& c) {
        const bool is_a = i < UG_ACH;
        const int ee = tid + (is_a ? i : i - UG_ACH) * 128, rows = is_a ? UG_BM : bn;
        const bool by_rows = is_a ? a_rows : b_rows;
        row = by_rows ? ee % rows : ee >> 3;
        c = by_rows ? ee / rows : ee & 7;
        return (is_a ? UG_BM : bn) * 8 > ee;  // B's chunks past bn columns stay unused
    };
    auto load_step = [&](int k0, uint4 (&r)[UG_CHUNKS]) {
#pragma unroll
        for (int i = 0; i < UG_CHUNKS; ++i) {
            const bool is_a = i < UG_ACH;
            int row, c;
            r[i] = make_uint4(0, 0, 0, 0);
            if (!chunk_at(i, row, c)) continue;
            const int kc = k0 + c * 8;
            if ((is_a ? a_vec : b_vec) && kc + 8 <= ke) {
                if (is_a) {
                    const int m = m0 + row;
                    if (m < g.M) r[i] = __ldg(reinterpret_cast<const uint4*>(g.A + (long long)m * g.sa_m + kc));
                } else {
                    r[i] = __ldg(reinterpret_cast<const uint4*>(g.B + (long long)(n0 + row) * g.sb_n + kc));
                }
            } else {
                uint32_t w[4];
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    uint32_t v = 0;
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const int k = kc + 2 * h + q;
                        unsigned short x = 0;
                        if (k < ke) {
                            if (is_a) {
                                const int m = m0 + row;
                                if (m < g.M)
                                    x = __ldg(reinterpret_cast<const unsigned short*>(g.A) + (long long)m * g.sa_m +
                                              (long long)k * g.sa_k);
                            } else {
                                x = __ldg(reinterpret_cast<const unsigned short*>(g.B) + (long long)k * g.sb_k +
                                          (long long)(n0 + row) * g.sb_n);
                            }
                        }
                        v |= (uint32_t)x << (16 * q);
                    }
                    w[h] = v;
                }
                r[i] = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
    };
    uint4 regs[UG_CHUNKS];
    if (kb < ke) load_step(kb, regs);
    for (int k0 = kb; k0 < ke; k0 += UG_BK) {
#pragma unroll
        for (int i = 0; i < UG_CHUNKS; ++i) {
            int row, c;
            if (chunk_at(i, row, c))
                *reinterpret_cast<uint4*>(sp + (i < UG_ACH ? 0 : UG_BM * 128) + sw128_offset((uint32_t)row, (uint32_t)c)) =
                    regs[i];
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
#pragma unroll
            for (int kk = 0; kk < UG_BK / 16; ++kk)
                if (k0 + kk * 16 < ke)
                    umma_bf16(tmem, umma_desc_sw128(sa) + 2 * kk, umma_desc_sw128(sb) + 2 * kk, idesc,
                              (k0 > kb || kk > 0) ? 1u : 0u);
            umma_commit(&s_bar);
        }
        if (k0 + UG_BK < ke) load_step(k0 + UG_BK, regs);  // in flight while the MMAs run
        // the tiles are free again once the MMAs that read them are done
        if (!mbar_wait(&s_bar, phase, g.err)) s_abort = 1;
        phase ^= 1u;
        tc_fence_after();
        __syncthreads();
        if (s_abort) break;
    }
    // epilogue: warp w holds accumulator rows 32w .. 32w + 31
    if (!s_abort) {
        const int m = m0 + warp * 32 + lane;
        // 16-byte stores when the rows of C allow them (columns come in multiples of 16)
        const bool c_vec = !(g.accumulate && !g.part_stride) && (g.ldc & 3) == 0 &&
                           (reinterpret_cast<uintptr_t>(C) & 15) == 0 && (n0 & 3) == 0;
        for (int c0 = 0; c0 < bn; c0 += 32) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            if (m < g.M && c_vec) {
                float4* row = reinterpret_cast<float4*>(&C[(long long)m * g.ldc + n0 + c0]);
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if (c0 + 4 * j < bn) row[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
            } else if (m < g.M) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int n = n0 + c0 + j;
                    if (c0 + j < bn) {
                        float* c = &C[(long long)m * g.ldc + n];
                        *c = (g.accumulate && !g.part_stride) ? *c + v[j] : v[j];
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, ncols);
}

// The split-K partials of umma_gemm_kernel summed in split order (the same
// order every run, so the gradients are deterministic).
__global__ void gemm_splits_kernel(const float* part, long long stride, int splits, float* C, long long ldc, int M,
                                   int N, int accumulate) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)M * N;
         e += (long long)gridDim.x * blockDim.x) {
        const long long m = e / N, n = e % N;
        float x = 0.f;
        for (int z = 0; z < splits; ++z) x += part[z * stride + m * N + n];
        float* c = &C[m * ldc + n];
        *c = accumulate ? *c + x : x;
    }
}

// ---------------------------------------------------------------------------
// Training helpers
// ---------------------------------------------------------------------------
// X[m][p*16+d] = emb[win[m][p]][d]
__global__ void gather_embed_kernel(const uint8_t* win, int M, const __nv_bfloat16* emb, __nv_bfloat16* X) {
    const long long total = (long long)M * MLP_IN;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const long long m = e / MLP_IN;
        const int p = (int)(e % MLP_IN) / MLP_EMB, d = (int)(e % MLP_EMB);
        X[e] = emb[win[m * MLP_WIN + p] * MLP_EMB + d];
    }
}

// H = relu(Z + b) as FP32 (kept for the mask) and BF16 (next GEMM input)
__global__ void bias_relu_kernel(const float* Z, const float* b, int M, int N, float* H, __nv_bfloat16* Hb) {
    const long long total = (long long)M * N;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const float v = fmaxf(Z[e] + b[e % N], 0.f);
        H[e] = v;
        Hb[e] = __float2bfloat16(v);
    }
}

// Softmax cross-entropy over the first S of 32 logits (one warp per row):
// dZ = (softmax - onehot) / M; loss summed into *loss; correct-count too.
__global__ void softmax_ce_kernel(const float* Z, const float* b3, const uint8_t* y, int M, int S, float* dZ,
                                  __nv_bfloat16* dZb, float* loss, unsigned int* correct) {
    const int warps = blockDim.x >> 5;
    const int lane = threadIdx.x & 31;
    for (long long m = (long long)blockIdx.x * warps + (threadIdx.x >> 5); m < M; m += (long long)gridDim.x * warps) {
        const float z = lane < S ? Z[m * MLP_OUT + lane] + b3[lane] : -INFINITY;
        float mx = z;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) mx = fmaxf(mx, __shfl_xor_sync(ALP_FULL_MASK, mx, d));
        const float ex = lane < S ? __expf(z - mx) : 0.f;
        float sum = ex;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) sum += __shfl_xor_sync(ALP_FULL_MASK, sum, d);
        const int t = y[m];
        const float p = ex / sum;
        const float g = (p - (lane == t ? 1.f : 0.f)) / (float)M;
        dZ[m * MLP_OUT + lane] = lane < S ? g : 0.f;
        dZb[m * MLP_OUT + lane] = __float2bfloat16(lane < S ? g : 0.f);
        // argmax (lowest index on ties)
        float bv = z;
        int bi = lane;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            const float ov = __shfl_xor_sync(ALP_FULL_MASK, bv, d);
            const int oi = __shfl_xor_sync(ALP_FULL_MASK, bi, d);
            if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        if (lane == t) atomicAdd(loss, -(z - mx - __logf(sum)));
        if (lane == 0 && bi == t) atomicAdd(correct, 1u);
    }
}

// dZ = dH * (H > 0), as BF16
__global__ void relu_back_kernel(const float* dH, const float* H, long long total, __nv_bfloat16* dZb, float* dZ) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const float v = H[e] > 0.f ? dH[e] : 0.f;
        dZ[e] = v;
        dZb[e] = __float2bfloat16(v);
    }
}

// out[n] (+)= sum over rows of Z[m][n]
__global__ void colsum_kernel(const float* Z, int M, int N, float* out) {
    const int n = blockIdx.x;
    float s = 0.f;
    for (int m = threadIdx.x; m < M; m += blockDim.x) s += Z[(long long)m * N + n];
    __shared__ float sh[256];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = sh[0];
}

// dEmb[win[m][p]][d] += dX[m][p*16+d]
__global__ void scatter_embed_kernel(const uint8_t* win, int M, const float* dX, float* dEmb) {
    const long long total = (long long)M * MLP_IN;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        const long long m = e / MLP_IN;
        const int p = (int)(e % MLP_IN) / MLP_EMB, d = (int)(e % MLP_EMB);
        atomicAdd(&dEmb[win[m * MLP_WIN + p] * MLP_EMB + d], dX[e]);
    }
}

// AdamW on the FP32 masters, then refresh the BF16 copies of the matrices.
// Weight decay applies to the matrices (embedding included), not to biases.
__global__ void adamw_kernel(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                             float eps, float wd, float bc1, float bc2, __nv_bfloat16* emb_b, __nv_bfloat16* w1_b,
                             __nv_bfloat16* w2_b, __nv_bfloat16* w3_b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bool is_bias = (i >= P_B1 && i < P_W2) || (i >= P_B2 && i < P_W3) || i >= P_B3;
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        float w = p[i];
        if (!is_bias) w -= lr * wd * w;
        w -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        p[i] = w;
        const __nv_bfloat16 wb = __float2bfloat16(w);
        if (i < P_W1) emb_b[i - P_EMB] = wb;
        else if (i < P_B1) w1_b[i - P_W1] = wb;
        else if (i >= P_W2 && i < P_B2) w2_b[i - P_W2] = wb;
        else if (i >= P_W3 && i < P_B3) w3_b[i - P_W3] = wb;
    }
}

// ---------------------------------------------------------------------------
// Fused inference: predicted state for each boundary position.
// Block = 128 boundaries, 8 warps x 16 rows.  Layer 1 walks the 64 window
// positions as 64 k-steps of 16 (one embedding per k-step), gathering the A
// fragment straight from the input bytes and the embedding table in shared
// memory; W1's 16-row slab for the step is staged in shared memory.  Layers 2
// and 3 run from shared-memory copies of H1, W2, W3.
// ---------------------------------------------------------------------------
constexpr int INF_ROWS = 128;
constexpr size_t INF_SMEM = 256 * MLP_EMB * 2          // embedding
                            + 2 * 16 * (MLP_H + 8) * 2  // W1 slab, double buffered
                            + INF_ROWS * (MLP_H + 8) * 2  // H (reused for H1, H2)
                            + MLP_H * (MLP_H + 8) * 2     // W2 transposed [n][k]
                            + MLP_OUT * (MLP_H + 8) * 2;  // W3 transposed [n][k]

__global__ void __launch_bounds__(256) mlp_infer_kernel(MlpWeights w, const uint8_t* in, long long n,
                                                        const long long* pos, long long count, uint8_t* pred) {
    extern __shared__ __align__(16) uint8_t smem[];
    __nv_bfloat16* s_emb = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* s_w1 = s_emb + 256 * MLP_EMB;                       // [2][16][136]
    __nv_bfloat16* s_h = s_w1 + 2 * 16 * (MLP_H + 8);                  // [128][136]
    __nv_bfloat16* s_w2t = s_h + INF_ROWS * (MLP_H + 8);               // [128][136]
    __nv_bfloat16* s_w3t = s_w2t + MLP_H * (MLP_H + 8);                // [32][136]
    __shared__ uint8_t s_win[INF_ROWS][MLP_WIN];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const long long r0 = (long long)blockIdx.x * INF_ROWS;
    for (int i = tid; i < 256 * MLP_EMB; i += 256) s_emb[i] = w.emb[i];
    for (int i = tid; i < MLP_H * MLP_H; i += 256) {
        const int k = i / MLP_H, c = i % MLP_H;
        s_w2t[c * (MLP_H + 8) + k] = w.w2[i];
    }
    for (int i = tid; i < MLP_H * MLP_OUT; i += 256) {
        const int k = i / MLP_OUT, c = i % MLP_OUT;
        s_w3t[c * (MLP_H + 8) + k] = w.w3[i];
    }
    for (int i = tid; i < INF_ROWS * MLP_WIN; i += 256) {
        const int r = i / MLP_WIN, p = i % MLP_WIN;
        uint8_t b = 0x20;  // before the input start: a space
        if (r0 + r < count) {
            const long long at = pos[r0 + r] - MLP_WIN + p;
            if (at >= 0 && at < n) b = in[at];
        }
        s_win[r][p] = b;
    }
    __syncthreads();
    // ---- layer 1 ----
    float acc[16][4];
#pragma unroll
    for (int j = 0; j < 16; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
    const int row = warp * 16 + gid;
    for (int p = 0; p < MLP_WIN; ++p) {
        __nv_bfloat16* slab = s_w1 + (p & 1) * 16 * (MLP_H + 8);
        for (int i = tid; i < 16 * MLP_H; i += 256) {
            const int k = i / MLP_H, c = i % MLP_H;
            slab[k * (MLP_H + 8) + c] = w.w1[(long long)(p * 16 + k) * MLP_H + c];
        }
        __syncthreads();
        const __nv_bfloat16* e0 = s_emb + s_win[row][p] * MLP_EMB;
        const __nv_bfloat16* e1 = s_emb + s_win[row + 8][p] * MLP_EMB;
        const uint32_t a0 = *reinterpret_cast<const uint32_t*>(e0 + tig * 2);
        const uint32_t a1 = *reinterpret_cast<const uint32_t*>(e1 + tig * 2);
        const uint32_t a2 = *reinterpret_cast<const uint32_t*>(e0 + tig * 2 + 8);
        const uint32_t a3 = *reinterpret_cast<const uint32_t*>(e1 + tig * 2 + 8);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int c = j * 8 + gid;
            const uint32_t b0 = pack2(slab[(tig * 2) * (MLP_H + 8) + c], slab[(tig * 2 + 1) * (MLP_H + 8) + c]);
            const uint32_t b1 = pack2(slab[(tig * 2 + 8) * (MLP_H + 8) + c], slab[(tig * 2 + 9) * (MLP_H + 8) + c]);
            mma_bf16(acc[j], a0, a1, a2, a3, b0, b1);
        }
    }
    // bias + relu -> H1 (BF16) in shared memory
#pragma unroll
    for (int j = 0; j < 16; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = warp * 16 + gid + (q >= 2 ? 8 : 0), c = j * 8 + tig * 2 + (q & 1);
            s_h[r * (MLP_H + 8) + c] = __float2bfloat16(fmaxf(acc[j][q] + w.b1[c], 0.f));
        }
    __syncwarp();
    // ---- layer 2 (rows of this warp only) ----
#pragma unroll
    for (int j = 0; j < 16; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
    for (int k0 = 0; k0 < MLP_H; k0 += 16) {
        const __nv_bfloat16* h0 = s_h + row * (MLP_H + 8) + k0;
        const __nv_bfloat16* h1 = s_h + (row + 8) * (MLP_H + 8) + k0;
        const uint32_t a0 = *reinterpret_cast<const uint32_t*>(h0 + tig * 2);
        const uint32_t a1 = *reinterpret_cast<const uint32_t*>(h1 + tig * 2);
        const uint32_t a2 = *reinterpret_cast<const uint32_t*>(h0 + tig * 2 + 8);
        const uint32_t a3 = *reinterpret_cast<const uint32_t*>(h1 + tig * 2 + 8);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const __nv_bfloat16* bt = s_w2t + (j * 8 + gid) * (MLP_H + 8) + k0;
            mma_bf16(acc[j], a0, a1, a2, a3, *reinterpret_cast<const uint32_t*>(bt + tig * 2),
                     *reinterpret_cast<const uint32_t*>(bt + tig * 2 + 8));
        }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 16; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int r = warp * 16 + gid + (q >= 2 ? 8 : 0), c = j * 8 + tig * 2 + (q & 1);
            s_h[r * (MLP_H + 8) + c] = __float2bfloat16(fmaxf(acc[j][q] + w.b2[c], 0.f));
        }
    __syncwarp();
    // ---- layer 3 ----
    float z[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) z[j][q] = 0.f;
    for (int k0 = 0; k0 < MLP_H; k0 += 16) {
        const __nv_bfloat16* h0 = s_h + row * (MLP_H + 8) + k0;
        const __nv_bfloat16* h1 = s_h + (row + 8) * (MLP_H + 8) + k0;
        const uint32_t a0 = *reinterpret_cast<const uint32_t*>(h0 + tig * 2);
        const uint32_t a1 = *reinterpret_cast<const uint32_t*>(h1 + tig * 2);
        const uint32_t a2 = *reinterpret_cast<const uint32_t*>(h0 + tig * 2 + 8);
        const uint32_t a3 = *reinterpret_cast<const uint32_t*>(h1 + tig * 2 + 8);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const __nv_bfloat16* bt = s_w3t + (j * 8 + gid) * (MLP_H + 8) + k0;
            mma_bf16(z[j], a0, a1, a2, a3, *reinterpret_cast<const uint32_t*>(bt + tig * 2),
                     *reinterpret_cast<const uint32_t*>(bt + tig * 2 + 8));
        }
    }
    // argmax over the S valid logits of rows (row) and (row + 8)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        float bv = -INFINITY;
        int bi = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int c = j * 8 + tig * 2 + q;
                const float v = c < w.n_states ? z[j][h * 2 + q] + w.b3[c] : -INFINITY;
                if (v > bv) { bv = v; bi = c; }
            }
#pragma unroll
        for (int d = 1; d < 4; d <<= 1) {
            const float ov = __shfl_xor_sync(ALP_FULL_MASK, bv, d);
            const int oi = __shfl_xor_sync(ALP_FULL_MASK, bi, d);
            if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        const long long r = r0 + warp * 16 + gid + h * 8;
        if (tig == 0 && r < count) pred[r] = (uint8_t)bi;
    }
}

// ---------------------------------------------------------------------------
// Inference, persistent: 128 windows per tile, one warp per 16 of them.
// W1 comes in pre-transposed ([n][k], mlp_w1t_kernel) and streams through
// shared memory in slabs of four window positions (k = 64) with cp.async
// double buffering; the other weights stay in shared memory for the CTA's
// lifetime.  Layers 2 and 3 take their A fragments straight from the previous
// layer's accumulators (bias, ReLU, BF16 rounding in registers): an m16n8
// accumulator pair is exactly an m16k16 A fragment.  Same arithmetic as
// mlp_infer_kernel (BF16 operands, FP32 accumulation, BF16 activations).
// ---------------------------------------------------------------------------
constexpr int I2_WARPS = 8;
constexpr int I2_ROWS = I2_WARPS * 16;          // windows per tile
constexpr int I2_KPOS = 4;                      // window positions per W1 slab
constexpr int I2_SLABS = MLP_WIN / I2_KPOS;
constexpr int I2_LDK = I2_KPOS * MLP_EMB + 8;   // 72: k stride of a slab row
constexpr int I2_LDH = MLP_H + 8;               // 136
constexpr int I2_LDW = 80;                      // window row stride (bytes): 20 words, conflict-free rows
constexpr size_t I2_SMEM = 256 * MLP_EMB * 2 + MLP_H * I2_LDH * 2 + MLP_OUT * I2_LDH * 2 +
                           (MLP_H + MLP_H + MLP_OUT) * 4 + 2 * MLP_H * I2_LDK * 2 + I2_ROWS * I2_LDW;

__global__ void mlp_w1t_kernel(const __nv_bfloat16* w1, __nv_bfloat16* w1t) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_IN * MLP_H; i += gridDim.x * blockDim.x) {
        const int k = i / MLP_H, c = i % MLP_H;
        w1t[c * MLP_IN + k] = w1[i];
    }
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ uint32_t relu_pack(float x, float y) {
    return pack2(__float2bfloat16(fmaxf(x, 0.f)), __float2bfloat16(fmaxf(y, 0.f)));
}

__global__ void __launch_bounds__(I2_WARPS * 32, 2) mlp_infer2_kernel(MlpWeights w, const __nv_bfloat16* w1t,
                                                                      const uint8_t* in, long long n,
                                                                      const long long* pos, long long count,
                                                                      uint8_t* pred) {
    extern __shared__ __align__(16) uint8_t smem[];
    __nv_bfloat16* s_emb = reinterpret_cast<__nv_bfloat16*>(smem);                 // [256][16]
    __nv_bfloat16* s_w2t = s_emb + 256 * MLP_EMB;                                   // [128][136]
    __nv_bfloat16* s_w3t = s_w2t + MLP_H * I2_LDH;                                  // [32][136]
    float* s_b1 = reinterpret_cast<float*>(s_w3t + MLP_OUT * I2_LDH);
    float* s_b2 = s_b1 + MLP_H;
    float* s_b3 = s_b2 + MLP_H;
    __nv_bfloat16* s_w1 = reinterpret_cast<__nv_bfloat16*>(s_b3 + MLP_OUT);         // [2][128][72]
    uint8_t* s_win = reinterpret_cast<uint8_t*>(s_w1 + 2 * MLP_H * I2_LDK);          // [128][80]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    for (int i = tid; i < 256 * MLP_EMB; i += I2_WARPS * 32) s_emb[i] = w.emb[i];
    for (int i = tid; i < MLP_H * MLP_H; i += I2_WARPS * 32) s_w2t[(i % MLP_H) * I2_LDH + i / MLP_H] = w.w2[i];
    for (int i = tid; i < MLP_H * MLP_OUT; i += I2_WARPS * 32) s_w3t[(i % MLP_OUT) * I2_LDH + i / MLP_OUT] = w.w3[i];
    for (int i = tid; i < MLP_H; i += I2_WARPS * 32) { s_b1[i] = w.b1[i]; s_b2[i] = w.b2[i]; }
    for (int i = tid; i < MLP_OUT; i += I2_WARPS * 32) s_b3[i] = w.b3[i];
    const bool in16 = (reinterpret_cast<uintptr_t>(in) & 15u) == 0;
    const long long tiles = (count + I2_ROWS - 1) / I2_ROWS;

    auto load_slab = [&](int s, int buf) {
        __nv_bfloat16* dst = s_w1 + buf * MLP_H * I2_LDK;
#pragma unroll
        for (int q = 0; q < (MLP_H * 8) / (I2_WARPS * 32); ++q) {
            const int idx = tid + q * I2_WARPS * 32;
            const int nn = idx >> 3, c = idx & 7;
            cp_async16(dst + nn * I2_LDK + c * 8, w1t + (size_t)nn * MLP_IN + s * (I2_KPOS * MLP_EMB) + c * 8);
        }
        cp_async_commit();
    };

    for (long long tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const long long r0 = tile * I2_ROWS;
        __syncthreads();  // the previous tile is done with s_win and the slabs
        load_slab(0, 0);
        // the tile's windows (spaces before the input's start and past its end)
        for (int i = tid; i < I2_ROWS * 4; i += I2_WARPS * 32) {
            const int r = i >> 2, q = i & 3;
            uint4 v = make_uint4(0x20202020u, 0x20202020u, 0x20202020u, 0x20202020u);
            if (r0 + r < count) {
                const long long p0 = pos[r0 + r] - MLP_WIN + 16 * q;
                if (in16 && p0 >= 0 && p0 + 16 <= n && (p0 & 15) == 0) {
                    v = __ldg(reinterpret_cast<const uint4*>(in + p0));
                } else {
                    uint32_t x[4];
#pragma unroll
                    for (int b = 0; b < 16; ++b) {
                        const long long at = p0 + b;
                        const uint32_t by = (at >= 0 && at < n) ? in[at] : 0x20u;
                        if ((b & 3) == 0) x[b >> 2] = 0;
                        x[b >> 2] |= by << (8 * (b & 3));
                    }
                    v = make_uint4(x[0], x[1], x[2], x[3]);
                }
            }
            *reinterpret_cast<uint4*>(s_win + r * I2_LDW + 16 * q) = v;
        }
        // ---- layer 1 ----
        float acc[16][4];
#pragma unroll
        for (int j = 0; j < 16; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
        const int row = warp * 16 + g;
        for (int s = 0; s < I2_SLABS; ++s) {
            if (s + 1 < I2_SLABS) {
                load_slab(s + 1, (s + 1) & 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            const __nv_bfloat16* slab = s_w1 + (s & 1) * MLP_H * I2_LDK;
#pragma unroll
            for (int kk = 0; kk < I2_KPOS; ++kk) {
                const int p = s * I2_KPOS + kk;
                const __nv_bfloat16* e0 = s_emb + s_win[row * I2_LDW + p] * MLP_EMB;
                const __nv_bfloat16* e1 = s_emb + s_win[(row + 8) * I2_LDW + p] * MLP_EMB;
                const uint32_t a0 = *reinterpret_cast<const uint32_t*>(e0 + 2 * t);
                const uint32_t a1 = *reinterpret_cast<const uint32_t*>(e1 + 2 * t);
                const uint32_t a2 = *reinterpret_cast<const uint32_t*>(e0 + 2 * t + 8);
                const uint32_t a3 = *reinterpret_cast<const uint32_t*>(e1 + 2 * t + 8);
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const __nv_bfloat16* bt = slab + (8 * j + g) * I2_LDK + kk * MLP_EMB + 2 * t;
                    mma_bf16(acc[j], a0, a1, a2, a3, *reinterpret_cast<const uint32_t*>(bt),
                             *reinterpret_cast<const uint32_t*>(bt + 8));
                }
            }
            __syncthreads();  // all warps are done with this slab before it is refilled
        }
        // ---- layer 2: A fragments from the layer-1 accumulators ----
        uint32_t ha[8][4];
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            const int c0 = 16 * s + 2 * t, c1 = c0 + 8;
            ha[s][0] = relu_pack(acc[2 * s][0] + s_b1[c0], acc[2 * s][1] + s_b1[c0 + 1]);
            ha[s][1] = relu_pack(acc[2 * s][2] + s_b1[c0], acc[2 * s][3] + s_b1[c0 + 1]);
            ha[s][2] = relu_pack(acc[2 * s + 1][0] + s_b1[c1], acc[2 * s + 1][1] + s_b1[c1 + 1]);
            ha[s][3] = relu_pack(acc[2 * s + 1][2] + s_b1[c1], acc[2 * s + 1][3] + s_b1[c1 + 1]);
        }
#pragma unroll
        for (int j = 0; j < 16; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
#pragma unroll
        for (int s = 0; s < 8; ++s)
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const __nv_bfloat16* bt = s_w2t + (8 * j + g) * I2_LDH + 16 * s + 2 * t;
                mma_bf16(acc[j], ha[s][0], ha[s][1], ha[s][2], ha[s][3], *reinterpret_cast<const uint32_t*>(bt),
                         *reinterpret_cast<const uint32_t*>(bt + 8));
            }
        // ---- layer 3 ----
#pragma unroll
        for (int s = 0; s < 8; ++s) {
            const int c0 = 16 * s + 2 * t, c1 = c0 + 8;
            ha[s][0] = relu_pack(acc[2 * s][0] + s_b2[c0], acc[2 * s][1] + s_b2[c0 + 1]);
            ha[s][1] = relu_pack(acc[2 * s][2] + s_b2[c0], acc[2 * s][3] + s_b2[c0 + 1]);
            ha[s][2] = relu_pack(acc[2 * s + 1][0] + s_b2[c1], acc[2 * s + 1][1] + s_b2[c1 + 1]);
            ha[s][3] = relu_pack(acc[2 * s + 1][2] + s_b2[c1], acc[2 * s + 1][3] + s_b2[c1 + 1]);
        }
        float z[4][4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) z[j][q] = 0.f;
#pragma unroll
        for (int s = 0; s < 8; ++s)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const __nv_bfloat16* bt = s_w3t + (8 * j + g) * I2_LDH + 16 * s + 2 * t;
                mma_bf16(z[j], ha[s][0], ha[s][1], ha[s][2], ha[s][3], *reinterpret_cast<const uint32_t*>(bt),
                         *reinterpret_cast<const uint32_t*>(bt + 8));
            }
        // argmax over the valid logits of rows g and g + 8 (lowest index on ties)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float bv = -INFINITY;
            int bi = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int c = j * 8 + t * 2 + q;
                    const float v = c < w.n_states ? z[j][h * 2 + q] + s_b3[c] : -INFINITY;
                    if (v > bv) { bv = v; bi = c; }
                }
#pragma unroll
            for (int d = 1; d < 4; d <<= 1) {
                const float ov = __shfl_xor_sync(ALP_FULL_MASK, bv, d);
                const int oi = __shfl_xor_sync(ALP_FULL_MASK, bi, d);
                if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
            }
            const long long r = r0 + warp * 16 + g + h * 8;
            if (t == 0 && r < count) pred[r] = (uint8_t)bi;
        }
    }
}


// ---------------------------------------------------------------------------
// Inference on the fifth-generation tensor cores (tcgen05), warp-specialised.
// A CTA takes 128 windows at a time (M = 128).  Layer 1 (K = 1024) runs as 8
// stages of K = 128 through a ring of I3_NS stages; a stage's A operand (the
// gathered embeddings, 128 rows x 128) lives in tensor memory and its B
// operand (W1 rows) in shared memory.  The K order is permuted so that K-slab
// s (0..15, 64 wide) holds window positions s, s + 16, s + 32, s + 48 (16
// embedding values each): a thread that owns 16 consecutive window bytes of a
// row (a quarter) supplies 16 K values of every slab from registers.  Roles:
//   * 16 builder warps: thread (row 32 (w % 4) + lane, quarter w / 4) keeps
//     its window bytes in registers (the next tile's are loaded while this
//     one is built), looks up the embeddings in shared memory and stores
//     them into its own tensor-memory lane (tcgen05.st: lane m = row m, two
//     BF16 K values per 32-bit column), then arrives on the stage's `full`
//     mbarrier (one arrival per warp);
//   * a producer warp: one bulk copy per stage of the W1 rows, already in the
//     128-byte swizzled K-major layout and permuted K order in a weight image
//     (mlp_wimg_kernel), onto the same `full` mbarrier (an arrival plus the
//     byte count), running ahead as stages come free;
//   * an MMA warp: one thread waits for a stage, issues eight 128x128x16 MMAs
//     (A from tensor memory, B from shared memory) and commits them to the
//     stage's `freed` mbarrier, which hands the stage back; during a tile's
//     layer 1 it also issues layers 2 and 3 of the previous tile;
//   * 8 epilogue warps (warp w owns rows 32 (w % 4) .. +31 and half of the
//     columns): bias + ReLU + BF16 of the layer-1 and layer-2 accumulators
//     into the next layer's A operand (s_h, two swizzled K-slabs in shared
//     memory), then the argmax of the layer-3 logits.
// Tensor memory (512 columns): the A ring in columns 0..255 (stage st at
// 64 st, K-slab h of it at + 32 h); two accumulator buffers of 128 columns
// at 256 + 128 b, each holding a tile's layer 1, then layer 2 (once the
// epilogue has read layer 1), then layer 3 (32 columns), so the epilogue of
// one tile overlaps layer 1 of the next.  Same rounding points as
// mlp_infer2_kernel (BF16 operands, FP32 accumulation, BF16 hidden
// activations).
//
// Every mbarrier wait is bounded: one that gives up records
// ALP_DEV_ERR_TIMEOUT and raises the CTA's abort flag, which every role
// checks before each wait; each role then leaves its loop, the CTA waits
// (bounded) for its copies and MMAs in flight and frees its tensor memory.
// ---------------------------------------------------------------------------
constexpr int I3_NS = 4;                          // stages of layer 1 in flight
constexpr int I3_BUILDERS = 16;                   // builder warps
constexpr int I3_EPI = 8;                         // epilogue warps
constexpr int I3_W_PROD = I3_BUILDERS + I3_EPI;   // producer warp index
constexpr int I3_W_MMA = I3_W_PROD + 1;           // MMA warp index
constexpr int I3_THREADS = (I3_W_MMA + 1) * 32;
constexpr int I3_ROWS = 128;                      // windows per tile (MMA M)
constexpr int I3_SLAB = 128 * 128;                // bytes of a 128-row x 64 BF16 swizzled K-slab
constexpr int I3_KSLABS = MLP_IN / 64;            // 16
constexpr int I3_STAGE = 2 * I3_SLAB;             // W1 bytes of a stage: two K-slabs (K = 128)
constexpr int I3_STAGES = I3_KSLABS / 2;          // 8 stages per tile
constexpr int I3_W3SLAB = MLP_OUT * 128;          // 32 rows x 64 BF16
constexpr uint32_t I3_TCOL_ACC = 256;             // first accumulator column
static_assert(I3_BUILDERS * 32 == I3_ROWS * 4, "one builder thread per (row, quarter)");
static_assert(I3_NS * 64 <= (int)I3_TCOL_ACC, "A ring in tensor memory");
// weight image (bytes): W1^T slabs (permuted K), W2^T slabs, W3^T slabs
constexpr int WIMG_W2 = I3_KSLABS * I3_SLAB;
constexpr int WIMG_W3 = WIMG_W2 + 2 * I3_SLAB;
constexpr int WIMG_BYTES = WIMG_W3 + 2 * I3_W3SLAB;
// shared memory (from a 1024-byte aligned base)
constexpr int I3_OFF_B = 0;
constexpr int I3_OFF_H = I3_NS * I3_STAGE;
constexpr int I3_OFF_W2 = I3_OFF_H + 2 * I3_SLAB;
constexpr int I3_OFF_W3 = I3_OFF_W2 + 2 * I3_SLAB;
constexpr int I3_OFF_EMB = I3_OFF_W3 + 2 * I3_W3SLAB;
constexpr int I3_OFF_BIAS = I3_OFF_EMB + 256 * MLP_EMB * 2;
constexpr int I3_OFF_BAR = I3_OFF_BIAS + (2 * MLP_H + MLP_OUT) * 4;
// full[NS], freed[NS], weights, acc[2], d_free[2], h_full, final
constexpr int I3_NBAR = 2 * I3_NS + 7;
constexpr int I3_OFF_TMEM = I3_OFF_BAR + I3_NBAR * 8;
constexpr size_t I3_SMEM = (size_t)I3_OFF_TMEM + 16 + 1024;  // + alignment slack
constexpr uint32_t I3_TMEM_COLS = 512;
static_assert(I3_OFF_BAR % 8 == 0 && I3_OFF_H % 1024 == 0 && I3_OFF_W2 % 1024 == 0 && I3_OFF_W3 % 1024 == 0,
              "layout");
static_assert(I3_SMEM + 1024 <= 227 * 1024, "shared memory");

// The weight image: element j (0..63) of row n of a K-slab sits at byte
// n * 128 + ((j / 8) ^ (n % 8)) * 16 + (j % 8) * 2 of the slab.  For W1, j of
// slab s is input k = 16 (s + 16 (j / 16)) + j % 16 (the permuted K order);
// for W2 and W3, k = 64 s + j.
__global__ void mlp_wimg_kernel(MlpWeights w, __nv_bfloat16* img) {
    constexpr int total = WIMG_BYTES / 2;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        const int b = 2 * e;
        int region_off, slab_bytes, N;
        const __nv_bfloat16* src;
        if (b < WIMG_W2) {
            region_off = 0; slab_bytes = I3_SLAB; N = MLP_H; src = w.w1;
        } else if (b < WIMG_W3) {
            region_off = WIMG_W2; slab_bytes = I3_SLAB; N = MLP_H; src = w.w2;
        } else {
            region_off = WIMG_W3; slab_bytes = I3_W3SLAB; N = MLP_OUT; src = w.w3;
        }
        const int slab = (b - region_off) / slab_bytes, o = (b - region_off) % slab_bytes;
        const int row = o >> 7, chunk = ((o >> 4) & 7) ^ (row & 7), j = chunk * 8 + ((o & 15) >> 1);
        const int k = region_off == 0 ? 16 * (slab + 16 * (j >> 4)) + (j & 15) : 64 * slab + j;
        img[e] = src[(size_t)k * N + row];  // the matrices are stored [k][n]
    }
}

__device__ __forceinline__ void mbar_arrive(uint64_t* mbar) {
    const uint32_t a = (uint32_t)__cvta_generic_to_shared(mbar);
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}

// The 16 window bytes [16 qq, 16 qq + 16) of the window ending before pos[row]
// (spaces before the input's start, past its end and for rows past count).
__device__ __forceinline__ uint4 window_quarter(const uint8_t* in, long long n, bool in16, long long p_end,
                                                bool live, int qq) {
    uint4 v = make_uint4(0x20202020u, 0x20202020u, 0x20202020u, 0x20202020u);
    if (!live) return v;
    const long long p0 = p_end - MLP_WIN + 16 * qq;
    if (in16 && p0 >= 0 && p0 + 16 <= n && (p0 & 15) == 0) return __ldg(reinterpret_cast<const uint4*>(in + p0));
    uint32_t x[4];
#pragma unroll
    for (int b = 0; b < 16; ++b) {
        const long long at = p0 + b;
        const uint32_t by = (at >= 0 && at < n) ? in[at] : 0x20u;
        if ((b & 3) == 0) x[b >> 2] = 0;
        x[b >> 2] |= by << (8 * (b & 3));
    }
    return make_uint4(x[0], x[1], x[2], x[3]);
}

__device__ __forceinline__ uint32_t quarter_byte(const uint4& v, int s) {
    const uint32_t wv = s < 4 ? v.x : s < 8 ? v.y : s < 12 ? v.z : v.w;
    return (wv >> (8 * (s & 3))) & 0xffu;
}

__global__ void __launch_bounds__(I3_THREADS, 1) mlp_infer3_kernel(MlpWeights w, const uint8_t* wimg,
                                                                    const uint8_t* in, long long n,
                                                                    const long long* pos, long long count,
                                                                    uint8_t* pred, unsigned int* err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    __shared__ int s_abort;
    uint8_t* sm = smem_raw + ((1024u - ((uint32_t)__cvta_generic_to_shared(smem_raw) & 1023u)) & 1023u);
    const uint32_t sb = (uint32_t)__cvta_generic_to_shared(sm);
    __nv_bfloat16* s_emb = reinterpret_cast<__nv_bfloat16*>(sm + I3_OFF_EMB);
    float* s_b1 = reinterpret_cast<float*>(sm + I3_OFF_BIAS);
    float* s_b2 = s_b1 + MLP_H;
    float* s_b3 = s_b2 + MLP_H;
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + I3_OFF_BAR);
    uint64_t* freed = full + I3_NS;
    uint64_t* wbar = freed + I3_NS;
    uint64_t* acc = wbar + 1;       // [2]: per accumulator buffer, layers 1, 2, 3 of its tile
    uint64_t* d_free = acc + 2;     // [2]: the epilogue is done with the buffer
    uint64_t* h_full = d_free + 2;  // the epilogue read the accumulator and wrote the next layer's A operand
    uint64_t* fin = h_full + 1;
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(sm + I3_OFF_TMEM);
    volatile int* abort_flag = &s_abort;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long tiles = (count + I3_ROWS - 1) / I3_ROWS;

    if (tid == 0) {
        for (int i = 0; i < I3_NS; ++i) {
            mbar_init(full + i, I3_BUILDERS + 1);  // builder warps + the producer's copy
            mbar_init(freed + i, 1);
        }
        mbar_init(wbar, 1);
        for (int i = 0; i < 2; ++i) {
            mbar_init(acc + i, 1);
            mbar_init(d_free + i, I3_EPI);
        }
        mbar_init(h_full, I3_EPI);
        mbar_init(fin, 1);
        mbar_fence_init();
        s_abort = 0;
    }
    __syncwarp();
    if (warp == 0) tmem_alloc(s_tmem, I3_TMEM_COLS);
    // embedding row b as two 16-byte halves, swapped when bit 2 of b is set, so
    // that eight gathers of random rows spread over all eight 16-byte bank groups
    for (int i = tid; i < 256 * MLP_EMB; i += I3_THREADS) {
        const int eb = i >> 4, d = i & 15;
        s_emb[(2 * eb + ((d >> 3) ^ ((eb >> 2) & 1))) * 8 + (d & 7)] = w.emb[i];
    }
    for (int i = tid; i < MLP_H; i += I3_THREADS) { s_b1[i] = w.b1[i]; s_b2[i] = w.b2[i]; }
    for (int i = tid; i < MLP_OUT; i += I3_THREADS) s_b3[i] = w.b3[i];
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *s_tmem;
    // a wait that gives up raises the abort flag; after it no role waits again
    auto wait_ok = [&](uint64_t* bar, uint32_t parity) -> bool {
        if (*abort_flag) return false;
        if (mbar_wait(bar, parity, err)) return true;
        *abort_flag = 1;
        return false;
    };
    // the same for a whole warp: lane 0 waits (few threads polling the
    // mbarrier unit), the warp goes on or leaves together
    auto warp_wait_ok = [&](uint64_t* bar, uint32_t parity) -> bool {
        bool ok = true;
        if (lane == 0) ok = wait_ok(bar, parity);
        __syncwarp();
        return __shfl_sync(ALP_FULL_MASK, ok ? 1 : 0, 0) != 0;
    };
    // this thread's tensor-memory lane (row): warps access lanes 32 (w % 4) .. +31
    const uint32_t t_lane = tbase + ((uint32_t)(32 * (warp & 3)) << 16);

    if (warp < I3_BUILDERS) {
        // ---------------- builders: layer-1 A operands into tensor memory ----------------
        const bool in16 = (reinterpret_cast<uintptr_t>(in) & 15u) == 0;
        const int qq = warp >> 2, rr = 32 * (warp & 3) + lane;
        long long tile = blockIdx.x;
        uint4 cur, nxt = make_uint4(0, 0, 0, 0);
        {
            const long long r = tile * I3_ROWS + rr;
            const bool live = tile < tiles && r < count;
            cur = window_quarter(in, n, in16, live ? pos[r] : 0, live, qq);
        }
        for (uint32_t t = 0; tile < tiles; tile += gridDim.x, ++t) {
            const long long nt = tile + gridDim.x, nr = nt * I3_ROWS + rr;
            const bool nlive = nt < tiles && nr < count;
            long long np = 0;
            bool ok = true;
#pragma unroll
            for (int S = 0; S < I3_STAGES; ++S) {
                if (S == 0 && nlive) np = pos[nr];  // the next tile's window position ...
                if (S == I3_STAGES / 2) nxt = window_quarter(in, n, in16, np, nlive, qq);  // ... and bytes
                const uint32_t g = t * I3_STAGES + S, st = g % I3_NS, u = g / I3_NS;
                if (u > 0 && !warp_wait_ok(freed + st, (u - 1) & 1u)) { ok = false; break; }
                tc_fence_after();
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    // K values 16 qq .. 16 qq + 15 of K-slab 2 S + h: columns 8 qq .. 8 qq + 7
                    const uint32_t eb = quarter_byte(cur, 2 * S + h), sw = (eb >> 2) & 1u;
                    const uint4* e = reinterpret_cast<const uint4*>(s_emb + eb * MLP_EMB);
                    const uint4 lo = e[sw], hi = e[sw ^ 1u];
                    const uint32_t v[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
                    tmem_st8(t_lane + 64 * st + 32 * h + 8 * qq, v);
                }
                tmem_wait_st();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(full + st);
            }
            if (!ok) break;
            cur = nxt;
        }
    } else if (warp < I3_W_PROD) {
        // ---------------- epilogue: rows 32 (w % 4) + lane, columns half hc ----------------
        const int hc = (warp - I3_BUILDERS) >> 2;
        const int r = 32 * (warp & 3) + lane;
        // bias + ReLU + BF16 of accumulator columns [64 hc, +64): K-slab hc of the next layer's A
        auto hidden_out = [&](uint32_t col0, const float* bias) {
            uint8_t* H = sm + I3_OFF_H + hc * I3_SLAB;
#pragma unroll 1
            for (int j = 0; j < 2; ++j) {  // 32 columns at a time: chunks 4 j .. 4 j + 3
                float v[32];
                tmem_ld32(t_lane + col0 + 64 * hc + 32 * j, v);
                const float4* b4 = reinterpret_cast<const float4*>(bias + 64 * hc + 32 * j);
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float4 p = b4[2 * c], q4 = b4[2 * c + 1];
                    const float bb[8] = {p.x, p.y, p.z, p.w, q4.x, q4.y, q4.z, q4.w};
                    uint32_t pk[4];
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        pk[e] = relu_pack(v[8 * c + 2 * e] + bb[2 * e], v[8 * c + 2 * e + 1] + bb[2 * e + 1]);
                    *reinterpret_cast<uint4*>(H + sw128_offset(r, 4 * j + c)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                }
            }
        };
        auto publish = [&](uint64_t* bar) {
            fence_async_smem();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(bar);
        };
        for (uint32_t t = 0; (long long)blockIdx.x + (long long)t * gridDim.x < tiles; ++t) {
            const uint32_t b = t & 1u, k3 = 3u * (t >> 1);
            const uint32_t col = I3_TCOL_ACC + 128u * b;
            if (!warp_wait_ok(acc + b, k3 & 1u)) break;
            tc_fence_after();
            hidden_out(col, s_b1);
            publish(h_full);
            if (!warp_wait_ok(acc + b, (k3 + 1) & 1u)) break;
            tc_fence_after();
            hidden_out(col, s_b2);
            publish(h_full);
            if (!warp_wait_ok(acc + b, (k3 + 2) & 1u)) break;
            tc_fence_after();
            if (hc == 0) {
                float z[32];
                tmem_ld32(t_lane + col, z);
                float bv = -INFINITY;
                int bi = 0;
#pragma unroll
                for (int c = 0; c < MLP_OUT; ++c) {
                    const float v = c < w.n_states ? z[c] + s_b3[c] : -INFINITY;
                    if (v > bv) { bv = v; bi = c; }
                }
                const long long row = ((long long)blockIdx.x + (long long)t * gridDim.x) * I3_ROWS + r;
                if (row < count) pred[row] = (uint8_t)bi;
            }
            publish(d_free + b);
        }
    } else if (warp == I3_W_PROD) {
        // ---------------- producer: W2 / W3 once, then W1 stages ahead of the MMAs ----------------
        if (lane == 0) {
            mbar_expect_tx(wbar, 2 * I3_SLAB + 2 * I3_W3SLAB);
            bulk_g2s(sb + I3_OFF_W2, wimg + WIMG_W2, 2 * I3_SLAB, wbar);
            bulk_g2s(sb + I3_OFF_W3, wimg + WIMG_W3, 2 * I3_W3SLAB, wbar);
            uint32_t issued = 0, ppar = 0;  // stages with a copy issued, and its phase parity
            uint32_t g = 0;
            bool ok = true;
            for (long long tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
                for (int S = 0; S < I3_STAGES; ++S, ++g) {
                    const uint32_t st = g % I3_NS, u = g / I3_NS;
                    if (u > 0 && !wait_ok(freed + st, (u - 1) & 1u)) { ok = false; break; }
                    mbar_expect_tx(full + st, I3_STAGE);
                    bulk_g2s(sb + I3_OFF_B + st * I3_STAGE, wimg + (size_t)S * I3_STAGE, I3_STAGE, full + st);
                    issued |= 1u << st;
                    ppar = (ppar & ~(1u << st)) | ((u & 1u) << st);
                }
            }
            // every copy has landed before the CTA's shared memory goes away (the
            // phase completes once the copy and this stage's builders are done;
            // on an abort the wait may give up, bounded)
            mbar_wait(wbar, 0, err);
            for (uint32_t st = 0; st < (uint32_t)I3_NS; ++st)
                if (issued & (1u << st)) mbar_wait(full + st, (ppar >> st) & 1u, err);
        }
        __syncwarp();
    } else {
        // ---------------- MMA issue: one thread ----------------
        if (lane == 0) {
            constexpr uint32_t ID_H = umma_idesc_bf16_f32(I3_ROWS, MLP_H);
            constexpr uint32_t ID_O = umma_idesc_bf16_f32(I3_ROWS, MLP_OUT);
            uint32_t g = 0, nh = 0;
            bool wready = false, ok = true, ready = false;
            // layer 2 / layer 3 of the tile in accumulator buffer pb, into the same
            // columns, once the epilogue has read them and written the A operand
            auto layer2 = [&](uint32_t pb) -> bool {
                if (!wait_ok(h_full, nh & 1u)) return false;
                ++nh;
                if (!wready) {
                    if (!wait_ok(wbar, 0)) return false;
                    wready = true;
                }
                tc_fence_after();
#pragma unroll
                for (int kk = 0; kk < 8; ++kk) {
                    const uint32_t off = (kk >> 2) * I3_SLAB;
                    umma_bf16(tbase + I3_TCOL_ACC + 128 * pb, umma_desc_sw128(sb + I3_OFF_H + off) + 2 * (kk & 3),
                              umma_desc_sw128(sb + I3_OFF_W2 + off) + 2 * (kk & 3), ID_H, kk != 0);
                }
                umma_commit(acc + pb);
                return true;
            };
            auto layer3 = [&](uint32_t pb) -> bool {
                if (!wait_ok(h_full, nh & 1u)) return false;
                ++nh;
                tc_fence_after();
#pragma unroll
                for (int kk = 0; kk < 8; ++kk)
                    umma_bf16(tbase + I3_TCOL_ACC + 128 * pb,
                              umma_desc_sw128(sb + I3_OFF_H + (kk >> 2) * I3_SLAB) + 2 * (kk & 3),
                              umma_desc_sw128(sb + I3_OFF_W3 + (kk >> 2) * I3_W3SLAB) + 2 * (kk & 3), ID_O,
                              kk != 0);
                umma_commit(acc + pb);
                return true;
            };
            uint32_t t = 0;
            for (long long tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, ++t) {
                const uint32_t b = t & 1u;
                // the epilogue is done with this buffer's previous tile
                if (t >= 2 && !wait_ok(d_free + b, ((t >> 1) - 1) & 1u)) { ok = false; break; }
                for (int S = 0; S < I3_STAGES; ++S, ++g) {
                    const uint32_t st = g % I3_NS, par = (g / I3_NS) & 1u;
                    if (!ready && !wait_ok(full + st, par)) { ok = false; break; }
                    // test the next stage now: the query's latency hides behind this stage's issue
                    ready = mbar_test(full + (g + 1) % I3_NS, ((g + 1) / I3_NS) & 1u);
                    tc_fence_after();
#pragma unroll
                    for (int kk = 0; kk < 8; ++kk)
                        umma_bf16_ts(tbase + I3_TCOL_ACC + 128 * b, tbase + 64 * st + 8 * kk,
                                     umma_desc_sw128(sb + I3_OFF_B + st * I3_STAGE + (kk >> 2) * I3_SLAB) +
                                         2 * (kk & 3),
                                     ID_H, (S | kk) != 0);
                    umma_commit(freed + st);
                    // the previous tile's layers 2 and 3, once its epilogue has had time for each
                    if (S == 2 && t > 0 && !layer2(b ^ 1u)) { ok = false; break; }
                    if (S == 5 && t > 0 && !layer3(b ^ 1u)) { ok = false; break; }
                }
                if (!ok) break;
                umma_commit(acc + b);  // layer 1 of this tile
            }
            if (ok && t > 0) {  // the last tile's layers 2 and 3
                const uint32_t pb = (t - 1) & 1u;
                if (layer2(pb)) layer3(pb);
            }
            // every MMA has completed before the tensor memory is freed
            umma_commit(fin);
            mbar_wait(fin, 0, err);
        }
        __syncwarp();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_free(tbase, I3_TMEM_COLS);
}

}  // namespace alp
