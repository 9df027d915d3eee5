// Boundary-state MLP (learned speculation): BF16 tensor-core kernels.
//
// The network predicts the DFA state at a chunk boundary from the 64 bytes
// before it: byte -> 16-d embedding (64 x 16 = 1024 inputs) -> 128 -> 128 ->
// logits over the lexer's states (padded to 32).  Weights and activations
// enter the tensor cores as BF16, every product accumulates in FP32
// (mma.sync m16n8k16).  There is no reference counterpart: alpacc has no
// learned component; the speculative lexer that uses these predictions is
// verified against the exact composition scan, so its output is bit-exact
// whatever the network predicts.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

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
// Generic GEMM for training: C[M][N] (FP32) = A[M][K] . B[K][N], A and B BF16
// addressed by strides (so transposes are free).  M, N, K multiples of 16.
// 64 x 64 tile per block, 4 warps of 32 x 32.
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
};

__global__ void __launch_bounds__(128) gemm_bf16_kernel(GemmArgs g) {
    __shared__ __align__(16) __nv_bfloat16 sA[64][16 + 8];
    __shared__ __align__(16) __nv_bfloat16 sB[64][16 + 8];  // transposed: [n][k]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int gid = lane >> 2, tig = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
    for (int k0 = 0; k0 < g.K; k0 += 16) {
        for (int e = tid; e < 64 * 16; e += 128) {
            const int r = e >> 4, c = e & 15;
            const int m = m0 + r, n = n0 + r, k = k0 + c;
            sA[r][c] = (m < g.M) ? g.A[m * g.sa_m + (long long)k * g.sa_k] : __float2bfloat16(0.f);
            sB[r][c] = (n < g.N) ? g.B[(long long)k * g.sb_k + n * g.sb_n] : __float2bfloat16(0.f);
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = wm + i * 16 + gid;
            const uint32_t a0 = *reinterpret_cast<const uint32_t*>(&sA[r][tig * 2]);
            const uint32_t a1 = *reinterpret_cast<const uint32_t*>(&sA[r + 8][tig * 2]);
            const uint32_t a2 = *reinterpret_cast<const uint32_t*>(&sA[r][tig * 2 + 8]);
            const uint32_t a3 = *reinterpret_cast<const uint32_t*>(&sA[r + 8][tig * 2 + 8]);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int n = wn + j * 8 + gid;
                const uint32_t b0 = *reinterpret_cast<const uint32_t*>(&sB[n][tig * 2]);
                const uint32_t b1 = *reinterpret_cast<const uint32_t*>(&sB[n][tig * 2 + 8]);
                mma_bf16(acc[i][j], a0, a1, a2, a3, b0, b1);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int m = m0 + wm + i * 16 + gid + (r >= 2 ? 8 : 0);
                const int n = n0 + wn + j * 8 + tig * 2 + (r & 1);
                if (m < g.M && n < g.N) {
                    float* c = &g.C[(long long)m * g.ldc + n];
                    *c = g.accumulate ? *c + acc[i][j][r] : acc[i][j][r];
                }
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

}  // namespace alp
