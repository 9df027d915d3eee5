// C ABI of alpacc_b200 (include/alpacc_b200.h): context, table upload, and
// the host side of every entry point.  Kernels live in the .cuh files.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/alpacc_b200.h"
#include "common.cuh"
#include "host_pool.h"
#include "lexer.cuh"
#include "lex3.cuh"
#include "parser.cuh"
#include "mlp.cuh"
#include "spec.cuh"
#include "spec3.cuh"

using namespace alp;

namespace {

constexpr uint32_t BLOB_MAGIC = 0x42504C41u;
constexpr int LEX_ITEMS = 16;
constexpr int LEX_TILE = LEX_THREADS * LEX_ITEMS;

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// ---------------------------------------------------------------------------
// Host widening.  alp_parse_host brings node fields whose values all lie in
// [-1, 2^31) across PCIe as 32-bit values and sign-extends them into the
// caller's 64-bit arrays on the host while later chunks are still in flight:
// 17 bytes a node cross the bus instead of 29.  The chunks land in a ring of
// RING_SLOTS pinned slots of RING_CHUNK values (64 MiB in all: the copies and
// the widening's reads stay within a small working set instead of streaming a
// landing buffer the size of the tree through DRAM); a slot takes the next
// chunk once its widening is done.  The widening runs on a pool of at most
// alp_host::HOST_WORKERS threads (the calling thread joins in; more threads
// than that took memory bandwidth from the copies) in slices of WIDEN_SLICE
// values, with streaming stores (no read of the destination): host_pool.h.
// ---------------------------------------------------------------------------
constexpr int RING_SLOTS = 16;
constexpr long long RING_CHUNK = 1LL << 20;

using alp_host::HostPool;
using alp_host::WIDEN_SLICE;
using alp_host::host_workers;

}  // namespace

// Launch shapes the autotuner picks (alp_tune_parse); zeros are the defaults.
struct Tuning {
    int ple = 0;          // index into ple_shapes
    int pairs_ctas = 0;   // CTAs per SM of the persistent pair kernel (0: as many as fit)
    int expand_ctas = 0;  // same for the expand kernel
    int mlp = 0;          // boundary-MLP inference: 0 tcgen05 kernel, 1 mma.sync kernel
    int lex_split = 1;    // lexer token pass: 0 fused (counts, look-back, tokens), 1 count pass + tile scan + token pass
    int parse_split = 1;  // parser position pass: 0 fused (pairs, look-back, expand), 1 pair pass + scan + expand
    int scan_g = 0;       // lexer state scan: chunks per lane, 8, 16 or 32 (0: LS_G)
};

struct alp_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    // ---- lexer tables ----
    bool has_lexer = false;
    int S = 0, C = 0, E = 0;
    uint32_t ignore_term = 0xffffffffu, dead_term = 0, n_terms = 0;
    std::vector<uint32_t> h_tokinfo;
    LexTables lt{};
    size_t lex_smem = 0;
    bool lex3 = false;                    // DFA small enough for the multi-kernel lexer (lex3.cuh)
    Lex3Tables l3{};
    size_t l3_fold_smem = 0, l3_scan_smem = 0, l3_count_smem = 0, l3_emit_smem = 0;
    // ---- parser tables ----
    bool has_parser = false;
    ParseTables pt{};
    ParseHost ph{};
    // ---- memory ----
    std::vector<void*> owned;             // table allocations
    DevBuf scratch;                       // look-back status words, results
    DevBuf out[8];                        // context-owned outputs
    DevBuf tmp[32];                       // intermediates
    long long* h_stage = nullptr;         // pinned staging for small host->device values
    // alp_parse_host's host buffers: the node fields the searches leave alone start to
    // the host as soon as the expansion has written them
    struct HostTree {
        uint32_t* tag;
        uint8_t* kind;
        int64_t* start;
        int64_t* end;
        long long cap;
        bool started;
        bool wide;   // spans sent as 32-bit values, widened on the host
    }* host_tree = nullptr;
    cudaEvent_t ev_nodes = nullptr;
    // node fields on their way to the host (alp_parse_host): the copies in the order to
    // issue them, the pinned ring their 32-bit values land in, and the widening threads
    struct HostCopy {
        const void* src;  // device
        void* dst;        // host: the caller's 64-bit array (widened) or its array (direct)
        size_t n;         // widened: 32-bit values; direct: bytes
        bool widen;
    };
    std::vector<HostCopy> copies;
    int32_t* h_ring = nullptr;
    cudaEvent_t ev_ring[RING_SLOTS] = {};
    HostPool* pool = nullptr;
    long long last_h2d = 0, last_d2h = 0;  // data bytes the last host-buffer call moved
    // when set (pinned, in h_stage): the lexer copies the validity of document 0
    // here in the same wait as its token count, which saves the caller a wait of its own
    uint8_t* lex_valid0 = nullptr;
    AlpResult* h_res = nullptr;           // pinned
    // optional per-kernel timing (alp_ctx_profile)
    int prof = 0;
    std::vector<std::pair<const char*, cudaEvent_t>> marks;
    uint8_t* state_out = nullptr;         // set only inside alp_lex_states
    long long last_tokens = 0;            // counts of the last call, for alp_ctx_info
    long long last_positions = 0;
    long long last_brackets = 0;
    long long last_kept = 0;              // brackets left for the search after closing adjacent pairs
    long long dev_allocs = 0;             // cudaMalloc calls made for this context's buffers
    double est_nodes = 0, est_kept = 0;   // nodes and kept brackets per position of the last parse (sizes)
    DevBuf mlp[16];                       // MLP training activations
    DevBuf spec[16];                      // speculative lexer chunk arrays
    // host-input token streams (alp_lex_host_stream): copy streams, events,
    // two slots of piece and token buffers, the carry and its pinned mirrors
    cudaStream_t cp_in = nullptr, cp_out = nullptr;
    // the bracket search runs beside the node search on this stream (fork / join events)
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_in[2] = {}, ev_done[2] = {}, ev_out[2] = {};
    DevBuf pipe;
    DevBuf carry;
    LexCarry* h_carry = nullptr;          // pinned, [2]
    Tuning tune;
};

struct alp_lex_stream {
    alp_ctx* ctx = nullptr;
    LexCarry* d_carry = nullptr;
    LexCarry* h_carry = nullptr;          // pinned
    uint32_t* term = nullptr;
    int64_t* start = nullptr;
    int64_t* end = nullptr;
    long long cap = 0;
    long long pos = 0;                    // bytes pushed so far
    long long first = 0;                  // stream token stored at element 0 of the outputs
    int ended = 0;
};

namespace {

// Record a named event on the context stream when profiling is on; the time
// between consecutive marks is attributed to the later mark's name.
void mark(alp_ctx* ctx, const char* name) {
    if (!ctx->prof) return;
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    cudaEventRecord(e, ctx->stream);
    ctx->marks.emplace_back(name, e);
}

int fail(alp_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return fail(ctx, ALP_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// 64-bit fields as 32-bit values (each in [-1, 2^31)) for the copy to the host;
// b and ob may be null; when dn is set, the count is min(n, *dn).  Grid-stride,
// four elements per thread per step.
constexpr int NARROW_GRID = 148 * 8;
__global__ void narrow_i64_kernel(const int64_t* __restrict__ a, const int64_t* __restrict__ b, long long n,
                                  int32_t* __restrict__ oa, int32_t* __restrict__ ob,
                                  const long long* dn = nullptr) {
    if (dn) n = min(n, *dn);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += 4 * stride) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const long long i = i0 + u * stride;
            if (i < n) {
                oa[i] = (int32_t)__ldg(a + i);
                if (b) ob[i] = (int32_t)__ldg(b + i);
            }
        }
    }
}

// Issue ctx->copies on stream s in order: a direct copy at once, a widened one
// when a ring slot is free.  The calling thread hands each landed slot (its
// event passed, in issue order) to the widening threads and widens slices
// itself meanwhile.  Returns when every copy has landed and been widened.
int send_to_host(alp_ctx* ctx, cudaStream_t s) {
    if (!ctx->pool) ctx->pool = new HostPool(host_workers());
    if (!ctx->h_ring) {
        CK(cudaHostAlloc((void**)&ctx->h_ring, (size_t)RING_SLOTS * RING_CHUNK * 4, cudaHostAllocDefault));
        for (auto& e : ctx->ev_ring) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    HostPool& pool = *ctx->pool;
    int state[RING_SLOTS] = {};  // 0 free, 1 copy in flight, 2 widening
    std::atomic<int> left[RING_SLOTS];
    const alp_ctx::HostCopy* job[RING_SLOTS] = {};
    for (auto& l : left) l.store(0);
    std::deque<int> flying;  // slots with a copy in flight, in issue order
    size_t next = 0;
    int rc = ALP_OK;
    auto free_slot = [&]() -> int {
        for (int k = 0; k < RING_SLOTS; ++k) {
            if (state[k] == 2 && left[k].load(std::memory_order_acquire) == 0) state[k] = 0;
            if (state[k] == 0) return k;
        }
        return -1;
    };
    while (!rc) {
        for (; next < ctx->copies.size(); ++next) {
            const alp_ctx::HostCopy& c = ctx->copies[next];
            cudaError_t e;
            if (!c.widen) {
                e = cudaMemcpyAsync(c.dst, c.src, c.n, cudaMemcpyDeviceToHost, s);
            } else {
                const int k = free_slot();
                if (k < 0) break;
                e = cudaMemcpyAsync(ctx->h_ring + (size_t)k * RING_CHUNK, c.src, c.n * 4, cudaMemcpyDeviceToHost, s);
                if (e == cudaSuccess) e = cudaEventRecord(ctx->ev_ring[k], s);
                state[k] = 1;
                job[k] = &c;
                flying.push_back(k);
            }
            if (e != cudaSuccess) {
                rc = fail(ctx, ALP_ERR_CUDA, "copy to the host: %s", cudaGetErrorString(e));
                break;
            }
        }
        if (rc) break;
        if (!flying.empty()) {
            const int k = flying.front();
            const cudaError_t e = cudaEventQuery(ctx->ev_ring[k]);
            if (e == cudaSuccess) {
                flying.pop_front();
                state[k] = 2;
                left[k].store(HostPool::slices(job[k]->n), std::memory_order_relaxed);
                pool.push(ctx->h_ring + (size_t)k * RING_CHUNK, (int64_t*)job[k]->dst, job[k]->n, &left[k]);
                continue;
            }
            if (e != cudaErrorNotReady) {
                rc = fail(ctx, ALP_ERR_CUDA, "copy to the host: %s", cudaGetErrorString(e));
                break;
            }
        } else if (next == ctx->copies.size()) {
            break;
        }
        if (!pool.help()) std::this_thread::yield();
    }
    // on an error too: no slice may outlive the call, nor a copy into the ring
    pool.wait();
    ctx->copies.clear();
    const cudaError_t e = cudaStreamSynchronize(s);
    if (!rc && e != cudaSuccess) rc = fail(ctx, ALP_ERR_CUDA, "copy to the host: %s", cudaGetErrorString(e));
    return rc;
}

int grow(alp_ctx* ctx, DevBuf& b, size_t bytes) {
    if (b.bytes >= bytes && b.p) return ALP_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    size_t want = bytes < 256 ? 256 : bytes;
    CK(cudaMalloc(&b.p, want));
    ++ctx->dev_allocs;
    b.bytes = want;
    return ALP_OK;
}

template <typename T>
int upload(alp_ctx* ctx, const T* h, size_t count, const T** d) {
    void* p = nullptr;
    size_t bytes = count * sizeof(T);
    CK(cudaMalloc(&p, bytes < 16 ? 16 : bytes));
    ++ctx->dev_allocs;
    if (bytes) CK(cudaMemcpy(p, h, bytes, cudaMemcpyHostToDevice));
    ctx->owned.push_back(p);
    *d = reinterpret_cast<const T*>(p);
    return ALP_OK;
}

struct Reader {
    const uint8_t* p;
    const uint8_t* e;
    bool ok = true;
    uint32_t u32() {
        if (p + 4 > e) { ok = false; return 0; }
        uint32_t v;
        memcpy(&v, p, 4);
        p += 4;
        return v;
    }
    const uint8_t* take(size_t n) {
        size_t padded = (n + 3) & ~(size_t)3;
        if (p + n > e) { ok = false; return nullptr; }
        const uint8_t* r = p;
        p = (p + padded <= e) ? p + padded : e;
        return r;
    }
};

int load_lexer(alp_ctx* ctx, Reader& r) {
    ctx->S = (int)r.u32();
    ctx->C = (int)r.u32();
    ctx->E = (int)r.u32();
    ctx->ignore_term = r.u32();
    ctx->dead_term = r.u32();
    ctx->n_terms = r.u32();
    const int S = ctx->S, C1 = ctx->C + 1, E = ctx->E;
    if (!r.ok || S < 2 || S > 32767 || C1 < 2 || C1 > 256 || E < 1 || E > 65535)
        return fail(ctx, ALP_ERR_TABLE, "bad lexer table sizes");
    const uint8_t* cls = r.take(256);
    r.take((size_t)S * 256 * 2);  // oracle form
    const uint16_t* cd = reinterpret_cast<const uint16_t*>(r.take((size_t)S * C1 * 2));
    const uint32_t* tok = reinterpret_cast<const uint32_t*>(r.take((size_t)S * 4));
    const uint8_t* acc = r.take(S);
    const uint16_t* step = reinterpret_cast<const uint16_t*>(r.take((size_t)E * C1 * 2));
    const uint16_t* comp = reinterpret_cast<const uint16_t*>(r.take((size_t)E * E * 2));
    const uint16_t* app = reinterpret_cast<const uint16_t*>(r.take((size_t)E * S * 2));
    if (!r.ok) return fail(ctx, ALP_ERR_TABLE, "truncated lexer tables");
    std::vector<uint8_t> vcls(cls, cls + 256);
    std::vector<uint16_t> vcd((size_t)S * C1), vstep((size_t)E * C1), vcomp((size_t)E * E), vapp((size_t)E * S);
    memcpy(vcd.data(), cd, vcd.size() * 2);
    memcpy(vstep.data(), step, vstep.size() * 2);
    memcpy(vcomp.data(), comp, vcomp.size() * 2);
    memcpy(vapp.data(), app, vapp.size() * 2);
    ctx->h_tokinfo.resize(S);
    for (int s = 0; s < S; ++s) {
        uint32_t t;
        memcpy(&t, tok + s, 4);
        if (t > TOK_TERM_MASK) return fail(ctx, ALP_ERR_TABLE, "terminal id too large");
        uint32_t v = t;
        if (acc[s]) v |= TOK_ACCEPT;
        if (ctx->ignore_term != 0xffffffffu && t == ctx->ignore_term) v |= TOK_IGNORE;
        ctx->h_tokinfo[s] = v;
    }
    for (uint8_t b : vcls)
        if (b >= C1 - 1) return fail(ctx, ALP_ERR_TABLE, "byte class out of range");
    // every table entry that a kernel uses as an index must be in range
    for (uint16_t v : vcd)
        if ((v & 0x7fffu) >= (uint32_t)S) return fail(ctx, ALP_ERR_TABLE, "lexer transition out of range");
    for (uint16_t v : vstep)
        if (v >= (uint32_t)E) return fail(ctx, ALP_ERR_TABLE, "endomorphism step out of range");
    for (uint16_t v : vcomp)
        if (v >= (uint32_t)E) return fail(ctx, ALP_ERR_TABLE, "endomorphism composition out of range");
    for (uint16_t v : vapp)
        if (v >= (uint32_t)S) return fail(ctx, ALP_ERR_TABLE, "endomorphism application out of range");
    int rc;
    if ((rc = upload(ctx, vcls.data(), vcls.size(), &ctx->lt.cls))) return rc;
    if ((rc = upload(ctx, vcd.data(), vcd.size(), &ctx->lt.cdelta))) return rc;
    if ((rc = upload(ctx, ctx->h_tokinfo.data(), ctx->h_tokinfo.size(), &ctx->lt.tokinfo))) return rc;
    if ((rc = upload(ctx, vstep.data(), vstep.size(), &ctx->lt.step))) return rc;
    if ((rc = upload(ctx, vcomp.data(), vcomp.size(), &ctx->lt.comp))) return rc;
    if ((rc = upload(ctx, vapp.data(), vapp.size(), &ctx->lt.apply))) return rc;
    ctx->lt.S = S;
    ctx->lt.C1 = C1;
    ctx->lt.E = E;
    ctx->lex_smem = lex_smem_bytes(S, C1, E);
    if (ctx->lex_smem > 200 * 1024) return fail(ctx, ALP_ERR_TABLE, "lexer tables exceed shared memory");
    ctx->has_lexer = true;

    // Multi-kernel lexer tables: apply as [E+S][32] bytes and a 256-column
    // transition table whose entries carry the emit / start decisions.
    bool small = S <= 32 && E + S <= 65535 && lex3_fold_smem(S, C1, E) <= 200 * 1024 &&
                 lex3_scan_smem(S, E) <= 160 * 1024 && lex3_emit_smem(S) <= 200 * 1024;
    for (int s = 0; s < S && small; ++s)
        if ((ctx->h_tokinfo[s] & TOK_TERM_MASK) >= (1u << (16 - LX_TERM_SHIFT))) small = false;
    if (small) {
        std::vector<uint8_t> app8(((size_t)E + S) * 32);
        for (int e = 0; e < E; ++e)
            for (int s = 0; s < 32; ++s) app8[(size_t)e * 32 + s] = (uint8_t)(s < S ? vapp[(size_t)e * S + s] : s);
        for (int c = 0; c < S; ++c)  // constant functions E + c (the state after a document head)
            for (int s = 0; s < 32; ++s) app8[((size_t)E + c) * 32 + s] = (uint8_t)c;
        std::vector<uint16_t> ent((size_t)S * LX_ROW + 8, 0);
        for (int s = 0; s < S; ++s)
            for (int b = 0; b < 256; ++b) {
                const uint16_t e = vcd[(size_t)s * C1 + vcls[b]];
                const uint32_t nx = e & 0x7fffu;
                uint32_t v = nx;
                if (e & 0x8000u) {
                    if (!(ctx->h_tokinfo[s] & TOK_IGNORE))
                        v |= LX_EMIT | ((ctx->h_tokinfo[s] & TOK_TERM_MASK) << LX_TERM_SHIFT);
                    if (!(ctx->h_tokinfo[nx] & TOK_IGNORE)) v |= LX_START;
                }
                ent[(size_t)s * LX_ROW + b] = (uint16_t)v;
            }
        ctx->l3.cls = ctx->lt.cls;
        ctx->l3.cdelta = ctx->lt.cdelta;
        ctx->l3.step = ctx->lt.step;
        ctx->l3.tokinfo = ctx->lt.tokinfo;
        if ((rc = upload(ctx, app8.data(), app8.size(), &ctx->l3.app8))) return rc;
        if ((rc = upload(ctx, ent.data(), ent.size(), &ctx->l3.ent))) return rc;
        ctx->l3.S = S;
        ctx->l3.C1 = C1;
        ctx->l3.E = E;
        ctx->l3_fold_smem = lex3_fold_smem(S, C1, E);
        ctx->l3_scan_smem = lex3_scan_smem(S, E);
        ctx->l3_count_smem = lex3_count_smem(S);
        ctx->l3_emit_smem = lex3_emit_smem(S);
        ctx->lex3 = true;
    }
    return ALP_OK;
}

template <int ITEMS, typename TermT, typename PosT>
int launch_lex(alp_ctx* ctx, const uint8_t* d_in, long long n, void* term, void* start, void* end,
               long long cap) {
    const long long tiles = (n + LEX_TILE - 1) / LEX_TILE;
    size_t sbytes = 256 + 8 * (size_t)tiles + 4 * (size_t)tiles;
    int rc = grow(ctx, ctx->scratch, sbytes);
    if (rc) return rc;
    uint8_t* base = reinterpret_cast<uint8_t*>(ctx->scratch.p);
    CK(cudaMemsetAsync(base, 0, sbytes, ctx->stream));
    LexArgs a;
    a.in = d_in;
    a.n = n;
    a.aligned16 = ((reinterpret_cast<uintptr_t>(d_in) & 15u) == 0) ? 1 : 0;
    a.t = ctx->lt;
    a.res = reinterpret_cast<AlpResult*>(base);
    a.ticket = reinterpret_cast<unsigned int*>(base + 128);
    a.stB = reinterpret_cast<unsigned long long*>(base + 256);
    a.stA = reinterpret_cast<uint32_t*>(base + 256 + 8 * (size_t)tiles);
    a.out_term = term;
    a.out_start = start;
    a.out_end = end;
    a.cap = cap;
    a.num_tiles = (unsigned)tiles;
    a.state_out = ctx->state_out;
    auto k = lex_kernel<ITEMS, TermT, PosT>;
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->lex_smem));
    // persistent: as many CTAs as fit at once, each loops over tile tickets
    int per_sm = 0, sms = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, LEX_THREADS, ctx->lex_smem));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    long long grid = (long long)(per_sm > 0 ? per_sm : 1) * sms;
    if (grid > tiles) grid = tiles;
    mark(ctx, "start");
    k<<<(unsigned)grid, LEX_THREADS, ctx->lex_smem, ctx->stream>>>(a);
    CK(cudaGetLastError());
    mark(ctx, "lex_kernel");
    CK(cudaMemcpyAsync(ctx->h_res, a.res, sizeof(AlpResult), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->h_res->error & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "lexer look-back timed out");
    return ALP_OK;
}

// Input size limit: 2^30 - 1 bytes for paths that can reach the single-pass
// lexer kernels (30-bit token counts in their look-back words); just under
// 2^31 where the multi-kernel lexer handles the input (32-bit counts and
// positions, int32 parser positions).
int check_in(alp_ctx* ctx, const void* p, int64_t n, bool allow_wide = false) {
    if (!ctx) return ALP_ERR_ARG;
    const int64_t lim = (allow_wide && ctx->lex3) ? (int64_t)0x7ff00000LL : (int64_t)0x3fffffffLL;
    if (n < 0 || n > lim) return fail(ctx, ALP_ERR_ARG, "input size %lld out of range", (long long)n);
    if (n > 0 && !p) return fail(ctx, ALP_ERR_ARG, "null input");
    return ALP_OK;
}

// Buffers of one parse (indices into ctx->tmp).
enum {
    T_HIN = 0, T_TTERM, T_TSTART, T_TEND, T_PID, T_TSUMS, T_VBUF, T_BRBUF, T_DSBUF,
    T_N_TMIN, T_N_M32, T_N_M1024, T_N_SVAL, T_N_SIDX, T_N_SLEN, T_N_ESC,
    T_B_TMIN, T_B_M32, T_B_M1024, T_B_SVAL, T_B_SIDX, T_B_SLEN, T_B_ESC,
    T_DOCOFF, T_TOKOFF, T_NODEOFF, T_BROFF, T_DVALID, T_NARROW, T_HOFF, T_CNT
};

struct ParseOut {
    int64_t* parent;
    uint32_t* tag;
    uint8_t* kind;
    int64_t* start;
    int64_t* end;
};

int set_result(alp_ctx* ctx, AlpResult* d_res, int valid) {
    memset(ctx->h_res, 0, sizeof(AlpResult));
    ctx->h_res->valid = valid;
    CK(cudaMemcpyAsync(d_res, ctx->h_res, sizeof(AlpResult), cudaMemcpyHostToDevice, ctx->stream));
    return ALP_OK;
}

int read_result(alp_ctx* ctx, AlpResult* d_res) {
    CK(cudaMemcpyAsync(ctx->h_res, d_res, sizeof(AlpResult), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(cudaGetLastError());
    if (ctx->h_res->error & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "kernel wait timed out");
    if (ctx->h_res->error & ALP_DEV_ERR_CAPACITY) return fail(ctx, ALP_ERR_CAPACITY, "internal buffer too small");
    return ALP_OK;
}

// Previous-smaller-or-equal over `n` values (nodes: writes parent; brackets:
// checks each right bracket against its match and clears res->valid).
// Tile shapes of the previous-smaller-or-equal kernel (threads x elements per thread).
struct PleShape {
    int threads, items;
    const void* fn;
    size_t smem;
};
const PleShape ple_shapes[] = {
    {256, 16, (const void*)ple_tile_kernel<256, 16>, ple_smem(256, 16)},
    {256, 8, (const void*)ple_tile_kernel<256, 8>, ple_smem(256, 8)},
    {128, 16, (const void*)ple_tile_kernel<128, 16>, ple_smem(128, 16)},
    {512, 8, (const void*)ple_tile_kernel<512, 8>, ple_smem(512, 8)},
};
constexpr int N_PLE_SHAPES = (int)(sizeof(ple_shapes) / sizeof(ple_shapes[0]));

// CTAs per SM of a persistent kernel: the tuned count, at most what fits
int persistent_ctas(int fit, int tuned) {
    if (fit < 1) fit = 1;
    return (tuned > 0 && tuned < fit) ? tuned : fit;
}

// With dn, n is a capacity and the element count is read from device memory
// (no host round trip; grids cover the capacity).
// A shard of a document (xq set): elements with no answer inside the shard are
// appended to xq for the shards before it, and parents are shifted by out_off.
int run_ple(alp_ctx* ctx, const int32_t* val, long long n, const uint32_t* sym, int64_t* parent, int first,
            const long long* seg_off, long long n_seg, uint8_t* seg_valid, AlpResult* d_res,
            const long long* dn = nullptr, long long out_off = 0, unsigned long long* xq = nullptr,
            unsigned int* xq_count = nullptr, long long xq_cap = 0, cudaStream_t stream = nullptr) {
    if (n == 0) return ALP_OK;
    cudaStream_t st = stream ? stream : ctx->stream;
    const PleShape& sh = ple_shapes[ctx->tune.ple];
    const int tile = sh.threads * sh.items;
    const long long tiles = (n + tile - 1) / tile;
    const long long n32 = (tiles + 31) / 32, n1024 = (tiles + 1023) / 1024;
    int rc;
    if ((rc = grow(ctx, ctx->tmp[first + 0], tiles * 4)) || (rc = grow(ctx, ctx->tmp[first + 1], n32 * 4)) ||
        (rc = grow(ctx, ctx->tmp[first + 2], n1024 * 4)) ||
        (rc = grow(ctx, ctx->tmp[first + 3], (size_t)tiles * tile * 4)) ||
        (rc = grow(ctx, ctx->tmp[first + 4], (size_t)tiles * tile * 4)) ||
        (rc = grow(ctx, ctx->tmp[first + 5], tiles * 4)) ||
        (rc = grow(ctx, ctx->tmp[first + 6], (size_t)n * 8 + 64)))
        return rc;
    unsigned int* esc_count = reinterpret_cast<unsigned int*>(reinterpret_cast<uint8_t*>(ctx->tmp[first + 6].p) +
                                                              (size_t)n * 8);
    CK(cudaMemsetAsync(esc_count, 0, 16, st));
    PleArgs a;
    a.val = val;
    a.n = n;
    a.sym = sym;
    a.out_parent = reinterpret_cast<long long*>(parent);
    a.seg_off = seg_off;
    a.n_seg = n_seg;
    a.seg_valid = seg_valid;
    a.tile_min = (int32_t*)ctx->tmp[first + 0].p;
    a.stair_val = (int32_t*)ctx->tmp[first + 3].p;
    a.stair_idx = (uint32_t*)ctx->tmp[first + 4].p;
    a.stair_len = (int32_t*)ctx->tmp[first + 5].p;
    a.esc = (unsigned long long*)ctx->tmp[first + 6].p;
    a.esc_count = esc_count;
    a.esc_cap = n;
    a.res = d_res;
    a.dn = dn;
    a.out_off = out_off;
    a.xq = xq;
    a.xq_count = xq_count;
    a.xq_cap = xq_cap;
    CK(cudaFuncSetAttribute(sh.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem));
    mark(ctx, "start");
    {
        void* args[] = {&a};
        CK(cudaLaunchKernel(sh.fn, dim3((unsigned)tiles), dim3(sh.threads), args, sh.smem, st));
    }
    mark(ctx, sym ? "ple_tile_kernel(brackets)" : "ple_tile_kernel(nodes)");
    tile_min_levels_kernel<<<(unsigned)((n32 + 255) / 256), 256, 0, st>>>(
        a.tile_min, tiles, (int32_t*)ctx->tmp[first + 1].p, (int32_t*)ctx->tmp[first + 2].p, dn, tile);
    CK(cudaGetLastError());
    EscArgs e;
    e.esc = a.esc;
    e.esc_count = esc_count;
    e.esc_cap = n;
    e.tile_min = a.tile_min;
    e.m32 = (const int32_t*)ctx->tmp[first + 1].p;
    e.m1024 = (const int32_t*)ctx->tmp[first + 2].p;
    e.stair_val = a.stair_val;
    e.stair_idx = a.stair_idx;
    e.stair_len = a.stair_len;
    e.sym = sym;
    e.out_parent = a.out_parent;
    e.seg_off = seg_off;
    e.n_seg = n_seg;
    e.seg_valid = seg_valid;
    e.res = d_res;
    e.tile = tile;
    e.out_off = out_off;
    e.xq = xq;
    e.xq_count = xq_count;
    e.xq_cap = xq_cap;
    ple_escape_kernel<<<148 * 4, 256, 0, st>>>(e);
    CK(cudaGetLastError());
    mark(ctx, sym ? "tile_min+ple_escape(brackets)" : "tile_min+ple_escape(nodes)");
    return ALP_OK;
}

// Multi-kernel lexer (DFAs of at most 32 states): chunk endomorphisms, the
// state scan over them, token counts, the tile scan of the counts, and the
// token pass.  Same contract as lex_seg.  Split in stages so that the
// speculative lexer can replace the front (states and counts per chunk).
struct Lex3Run {
    Lex3Args a;
    LexSeg sg;
    uint8_t* base;
    size_t o_td, o_ccs;
    long long tiles, wide, chunks, stiles, nd;
    int sms;
};

int scan_g(const alp_ctx* ctx) { return ctx->tune.scan_g ? ctx->tune.scan_g : LS_G; }

inline const void* scan_kernel_for(int g) {
    if (g == 8) return (const void*)lex3_scan_kernel<8>;
    if (g == 32) return (const void*)lex3_scan_kernel<32>;
    return (const void*)lex3_scan_kernel<16>;
}

// the state scan over the chunk endomorphisms, chunks per lane as tuned
int lex3_scan(alp_ctx* ctx, Lex3Run& r);

int lex3_grid(alp_ctx* ctx, const Lex3Run& r, const void* k, int threads, size_t smem, long long work, unsigned* g) {
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem));
    long long x = (long long)(per_sm > 0 ? per_sm : 1) * r.sms;
    *g = (unsigned)(x < work ? x : work);
    return ALP_OK;
}

int lex3_prepare(alp_ctx* ctx, const uint8_t* d_in, long long n, const long long* d_off, long long nd, int sentinels,
                 void* term, void* start, void* end, long long cap, uint8_t* valid, Lex3Run& r) {
    r.tiles = (n + LX_TILE - 1) / LX_TILE;
    r.wide = (n + LX_WIDE - 1) / LX_WIDE;
    r.chunks = (n + LX_CHUNK - 1) / LX_CHUNK;
    r.stiles = (r.chunks + ls_tile(scan_g(ctx)) - 1) / ls_tile(scan_g(ctx));
    r.nd = nd;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t o_vec = 256, o_cs = o_vec + al(128 * (size_t)r.stiles), o_f = o_cs + al(8 * (size_t)r.tiles);
    const size_t o_s = o_f + al(2 * (size_t)r.chunks + 64), o_c = o_s + al((size_t)r.chunks + 64);
    r.o_td = o_c + al(2 * (size_t)r.chunks + 64);
    r.o_ccs = r.o_td + al(8 * (size_t)r.tiles);
    const size_t sbytes = r.o_ccs + al(8 * ((size_t)r.tiles / LT_CHUNK + 2));
    int rc;
    if ((rc = grow(ctx, ctx->scratch, sbytes))) return rc;
    uint8_t* base = reinterpret_cast<uint8_t*>(ctx->scratch.p);
    r.base = base;
    CK(cudaMemsetAsync(base, 0, o_cs, ctx->stream));  // result, tickets, look-back words
    Lex3Args& a = r.a;
    a.in = d_in;
    a.n = n;
    a.aligned16 = ((reinterpret_cast<uintptr_t>(d_in) & 15u) == 0) ? 1 : 0;
    a.t = ctx->l3;
    a.n_chunks = r.chunks;
    a.chunk_f = reinterpret_cast<uint16_t*>(base + o_f);
    a.chunk_s = base + o_s;
    a.chunk_c = reinterpret_cast<uint16_t*>(base + o_c);
    a.tile_cs = reinterpret_cast<unsigned long long*>(base + o_cs);
    a.lb_vec = reinterpret_cast<uint32_t*>(base + o_vec);
    a.res = reinterpret_cast<AlpResult*>(base);
    a.tickets = reinterpret_cast<unsigned int*>(base + 128);
    a.tile_doc = reinterpret_cast<const long long*>(base + r.o_td);
    a.out_term = term;
    a.out_start = start;
    a.out_end = end;
    a.cap = cap;
    a.num_tiles = (unsigned)r.tiles;
    a.num_wide = (unsigned)r.wide;
    a.num_scan_tiles = (unsigned)r.stiles;
    a.carry = nullptr;
    a.pos_base = 0;
    a.carry_tokens = 0;
    a.tok_first = 0;
    LexSeg& sg = r.sg;
    sg.cont = 0;
    sg.end1 = 0;
    sg.doc_off = d_off;
    sg.n_docs = nd;
    sg.tok_off = (long long*)ctx->tmp[T_TOKOFF].p;
    sg.valid = valid;
    sg.sentinels = sentinels;
    sg.sent_l = ctx->has_parser ? ctx->pt.start : 0;
    sg.sent_r = ctx->has_parser ? ctx->pt.end : 0;
    CK(cudaDeviceGetAttribute(&r.sms, cudaDevAttrMultiProcessorCount, ctx->device));
    if (nd > 1) {
        const long long gb = (nd + 255) / 256;
        CK(cudaMemsetAsync(base + r.o_td, 0, 8 * (size_t)r.tiles, ctx->stream));
        mark(ctx, "start");
        lex3_tile_doc_kernel<<<(unsigned)(gb < 4096 ? gb : 4096), 256, 0, ctx->stream>>>(
            d_off, nd, reinterpret_cast<long long*>(base + r.o_td), r.tiles);
        CK(cudaGetLastError());
        mark(ctx, "lex3_tile_doc_kernel");
    }
    return ALP_OK;
}

// chunk endomorphisms
int lex3_fold(alp_ctx* ctx, Lex3Run& r) {
    unsigned g1;
    int rc;
    CK(cudaFuncSetAttribute(lex3_fold_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->l3_fold_smem));
    CK(cudaFuncSetAttribute(lex3_fold_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    if ((rc = lex3_grid(ctx, r, (const void*)lex3_fold_kernel, LX_THREADS, ctx->l3_fold_smem, r.wide, &g1))) return rc;
    mark(ctx, "start");
    lex3_fold_kernel<<<g1, LX_THREADS, ctx->l3_fold_smem, ctx->stream>>>(r.a, r.sg);
    CK(cudaGetLastError());
    mark(ctx, "lex3_fold_kernel");
    return ALP_OK;
}

// chunk endomorphisms -> chunk states -> chunk counts and tile counts
int lex3_front(alp_ctx* ctx, Lex3Run& r, bool folded = false) {
    unsigned g3;
    int rc;
    if (!folded && (rc = lex3_fold(ctx, r))) return rc;
    CK(cudaFuncSetAttribute(lex3_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->l3_count_smem));
    if ((rc = lex3_grid(ctx, r, (const void*)lex3_count_kernel, LX_THREADS, ctx->l3_count_smem, r.wide, &g3)))
        return rc;
    if ((rc = lex3_scan(ctx, r))) return rc;
    lex3_count_kernel<<<g3, LX_THREADS, ctx->l3_count_smem, ctx->stream>>>(r.a, r.sg);
    CK(cudaGetLastError());
    mark(ctx, "lex3_count_kernel");
    return ALP_OK;
}

// tile scan of the counts -> token pass (stream-ordered, no wait)
// exclusive (count, last start) over the tiles
int lex3_tiles(alp_ctx* ctx, Lex3Run& r) {
    const long long lchunks = (r.tiles + LT_CHUNK - 1) / LT_CHUNK;
    unsigned long long* ccs = reinterpret_cast<unsigned long long*>(r.base + r.o_ccs);
    lex3_tile_reduce_kernel<<<(unsigned)lchunks, LT_CHUNK, 0, ctx->stream>>>(r.a.tile_cs, r.tiles, ccs);
    CK(cudaGetLastError());
    lex3_tile_scan_kernel<<<(unsigned)lchunks, LT_CHUNK, 0, ctx->stream>>>(r.a.tile_cs, r.tiles, ccs);
    CK(cudaGetLastError());
    return ALP_OK;
}

template <typename TermT, typename PosT>
int lex3_emit(alp_ctx* ctx, Lex3Run& r, bool tiles_done = false) {
    auto k5 = lex3_emit_kernel<TermT, PosT>;
    unsigned g5;
    int rc;
    CK(cudaFuncSetAttribute(k5, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->l3_emit_smem));
    CK(cudaFuncSetAttribute(k5, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    if ((rc = lex3_grid(ctx, r, (const void*)k5, LX_THREADS, ctx->l3_emit_smem, r.tiles, &g5))) return rc;
    mark(ctx, "start");
    if (!tiles_done && (rc = lex3_tiles(ctx, r))) return rc;
    mark(ctx, "lex3_tile_reduce+lex3_tile_scan");
    k5<<<g5, LX_THREADS, ctx->l3_emit_smem, ctx->stream>>>(r.a, r.sg);
    CK(cudaGetLastError());
    mark(ctx, "lex3_emit_kernel");
    return ALP_OK;
}

// tile scan of the counts -> token pass -> result
template <typename TermT, typename PosT>
int lex3_back(alp_ctx* ctx, Lex3Run& r, long long* total) {
    int rc;
    if ((rc = lex3_emit<TermT, PosT>(ctx, r))) return rc;
    CK(cudaMemcpyAsync(ctx->h_res, r.a.res, sizeof(AlpResult), cudaMemcpyDeviceToHost, ctx->stream));
    if (ctx->lex_valid0) CK(cudaMemcpyAsync(ctx->lex_valid0, r.sg.valid, 1, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->h_res->error & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "lexer look-back timed out");
    *total = ctx->h_res->count;
    ctx->last_tokens = *total;
    if (ctx->h_res->error & ALP_DEV_ERR_CAPACITY) return fail(ctx, ALP_ERR_CAPACITY, "token buffer too small");
    return ALP_OK;
}

// The fused token pass (counts, look-back over tiles, tokens) after the
// state scan: one input pass fewer than lex3_front + lex3_back.
template <typename TermT, typename PosT>
int lex3_tok(alp_ctx* ctx, Lex3Run& r, long long* total) {
    auto k = lex3_tok_kernel<TermT, PosT>;
    unsigned g;
    int rc;
    const size_t sm = lex3_tok_smem(ctx->S);
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    CK(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    if ((rc = lex3_grid(ctx, r, (const void*)k, LX_THREADS, sm, r.tiles, &g))) return rc;
    CK(cudaMemsetAsync(r.a.tile_cs, 0, 8 * (size_t)r.tiles, ctx->stream));  // look-back words
    mark(ctx, "start");
    k<<<g, LX_THREADS, sm, ctx->stream>>>(r.a, r.sg);
    CK(cudaGetLastError());
    mark(ctx, "lex3_tok_kernel");
    CK(cudaMemcpyAsync(ctx->h_res, r.a.res, sizeof(AlpResult), cudaMemcpyDeviceToHost, ctx->stream));
    if (ctx->lex_valid0) CK(cudaMemcpyAsync(ctx->lex_valid0, r.sg.valid, 1, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->h_res->error & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "lexer look-back timed out");
    *total = ctx->h_res->count;
    ctx->last_tokens = *total;
    if (ctx->h_res->error & ALP_DEV_ERR_CAPACITY) return fail(ctx, ALP_ERR_CAPACITY, "token buffer too small");
    return ALP_OK;
}

// chunk endomorphisms -> chunk states (no count pass)
int lex3_states(alp_ctx* ctx, Lex3Run& r) {
    int rc;
    if ((rc = lex3_fold(ctx, r))) return rc;
    return lex3_scan(ctx, r);
}

int lex3_scan(alp_ctx* ctx, Lex3Run& r) {
    const void* k = scan_kernel_for(scan_g(ctx));
    unsigned g2;
    int rc;
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->l3_scan_smem));
    if ((rc = lex3_grid(ctx, r, k, LS_WARPS * 32, ctx->l3_scan_smem, r.stiles, &g2))) return rc;
    mark(ctx, "start");
    {
        void* args[] = {&r.a};
        CK(cudaLaunchKernel(k, dim3(g2), dim3(LS_WARPS * 32), args, ctx->l3_scan_smem, ctx->stream));
    }
    mark(ctx, "lex3_scan_kernel");
    return ALP_OK;
}

template <typename TermT, typename PosT>
int lex3_run(alp_ctx* ctx, const uint8_t* d_in, long long n, const long long* d_off, long long nd, int sentinels,
             TermT* term, PosT* start, PosT* end, long long cap, uint8_t* valid, long long* total) {
    Lex3Run r;
    int rc;
    if ((rc = lex3_prepare(ctx, d_in, n, d_off, nd, sentinels, term, start, end, cap, valid, r))) return rc;
    if (ctx->tune.lex_split) {
        if ((rc = lex3_front(ctx, r))) return rc;
        return lex3_back<TermT, PosT>(ctx, r, total);
    }
    if ((rc = lex3_states(ctx, r))) return rc;
    return lex3_tok<TermT, PosT>(ctx, r, total);
}

// Segmented lexer over documents at d_off[0..nd] (device).  sentinels: the
// parser layout (⊢ tokens ⊣ per document) into tmp[T_TTERM..T_TEND] with
// u16/u32 types; otherwise the lexer API layout into the given buffers.
// Per-document token offsets land in tmp[T_TOKOFF], validity in `valid`.
template <typename TermT, typename PosT>
int lex_seg(alp_ctx* ctx, const uint8_t* d_in, long long n, const long long* d_off, long long nd, int sentinels,
            TermT* term, PosT* start, PosT* end, long long cap, uint8_t* valid, long long* total) {
    *total = 0;
    int rc;
    if ((rc = grow(ctx, ctx->tmp[T_TOKOFF], (size_t)(nd + 1) * 8))) return rc;
    if (n == 0) {
        // every document is empty: rejected, no tokens
        CK(cudaMemsetAsync(ctx->tmp[T_TOKOFF].p, 0, (size_t)(nd + 1) * 8, ctx->stream));
        CK(cudaMemsetAsync(valid, 0, (size_t)nd, ctx->stream));
        if (sentinels) {
            // ⊢ ⊣ for each document
            std::vector<uint16_t> h(2 * nd);
            for (long long i = 0; i < nd; ++i) { h[2 * i] = (uint16_t)ctx->pt.start; h[2 * i + 1] = (uint16_t)ctx->pt.end; }
            if (2 * nd > cap) return fail(ctx, ALP_ERR_CAPACITY, "token buffer too small");
            CK(cudaMemcpy(term, h.data(), 2 * nd * sizeof(uint16_t), cudaMemcpyHostToDevice));
        }
        return ALP_OK;
    }
    if (ctx->lex3) return lex3_run<TermT, PosT>(ctx, d_in, n, d_off, nd, sentinels, term, start, end, cap, valid, total);
    const long long tiles = (n + SEG_TILE - 1) / SEG_TILE;
    size_t sbytes = 256 + 8 * (size_t)tiles + 4 * (size_t)tiles;
    if ((rc = grow(ctx, ctx->scratch, sbytes))) return rc;
    uint8_t* base = reinterpret_cast<uint8_t*>(ctx->scratch.p);
    CK(cudaMemsetAsync(base, 0, sbytes, ctx->stream));
    LexArgs a;
    a.in = d_in;
    a.n = n;
    a.aligned16 = ((reinterpret_cast<uintptr_t>(d_in) & 15u) == 0) ? 1 : 0;
    a.t = ctx->lt;
    a.res = reinterpret_cast<AlpResult*>(base);
    a.ticket = reinterpret_cast<unsigned int*>(base + 128);
    a.stB = reinterpret_cast<unsigned long long*>(base + 256);
    a.stA = reinterpret_cast<uint32_t*>(base + 256 + 8 * (size_t)tiles);
    a.out_term = term;
    a.out_start = start;
    a.out_end = end;
    a.cap = cap;
    a.num_tiles = (unsigned)tiles;
    a.state_out = nullptr;
    LexSeg sg{};
    sg.doc_off = d_off;
    sg.n_docs = nd;
    sg.tok_off = (long long*)ctx->tmp[T_TOKOFF].p;
    sg.valid = valid;
    sg.sentinels = sentinels;
    sg.sent_l = ctx->has_parser ? ctx->pt.start : 0;
    sg.sent_r = ctx->has_parser ? ctx->pt.end : 0;
    auto k = lex_seg_kernel<TermT, PosT>;
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->lex_smem));
    CK(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    int per_sm = 0, sms = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, LEX_THREADS, ctx->lex_smem));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    long long grid = (long long)(per_sm > 0 ? per_sm : 1) * sms;
    if (grid > tiles) grid = tiles;
    mark(ctx, "start");
    k<<<(unsigned)grid, LEX_THREADS, ctx->lex_smem, ctx->stream>>>(a, sg);
    CK(cudaGetLastError());
    mark(ctx, "lex_seg_kernel");
    CK(cudaMemcpyAsync(ctx->h_res, a.res, sizeof(AlpResult), cudaMemcpyDeviceToHost, ctx->stream));
    if (ctx->lex_valid0) CK(cudaMemcpyAsync(ctx->lex_valid0, valid, 1, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->h_res->error & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "lexer look-back timed out");
    *total = ctx->h_res->count;
    ctx->last_tokens = *total;
    if (ctx->h_res->error & ALP_DEV_ERR_CAPACITY) return fail(ctx, ALP_ERR_CAPACITY, "token buffer too small");
    return ALP_OK;
}

int put_doc_off(alp_ctx* ctx, long long n) {
    int rc = grow(ctx, ctx->tmp[T_DOCOFF], 16);
    if (rc) return rc;
    ctx->h_stage[0] = 0;
    ctx->h_stage[1] = n;
    CK(cudaMemcpyAsync(ctx->tmp[T_DOCOFF].p, ctx->h_stage, 16, cudaMemcpyHostToDevice, ctx->stream));
    return ALP_OK;
}

// Positions (⊢ tokens ⊣ per document, L of them) already in
// tmp[T_TTERM..T_TEND] and per-document validity in `dvalid` -> tree.
// `want_tree` 0 gives the production sequence only.  Node offsets of the
// documents land in tmp[T_NODEOFF].
// Output buffers for N nodes (context-owned when ctx_out) and the node and
// bracket intermediates for N nodes and K kept brackets.
int parse_buffers(alp_ctx* ctx, ParseOut* o, int ctx_out, long long N, long long K, ParseArgs& a) {
    int rc;
    if (ctx_out) {
        if ((rc = grow(ctx, ctx->out[3], N * 8 + 8)) || (rc = grow(ctx, ctx->out[4], N * 4 + 8)) ||
            (rc = grow(ctx, ctx->out[5], N + 8)) || (rc = grow(ctx, ctx->out[6], N * 8 + 8)) ||
            (rc = grow(ctx, ctx->out[7], N * 8 + 8)))
            return rc;
        o->parent = (int64_t*)ctx->out[3].p;
        o->tag = (uint32_t*)ctx->out[4].p;
        o->kind = (uint8_t*)ctx->out[5].p;
        o->start = (int64_t*)ctx->out[6].p;
        o->end = (int64_t*)ctx->out[7].p;
    }
    if ((rc = grow(ctx, ctx->tmp[T_VBUF], N * 4 + 8)) || (rc = grow(ctx, ctx->tmp[T_BRBUF], K * 4 + 8)) ||
        (rc = grow(ctx, ctx->tmp[T_DSBUF], K * 4 + 8)))
        return rc;
    a.tag = o->tag;
    a.kind = o->kind;
    a.nstart = o->start;
    a.nend = o->end;
    a.vbuf = (int32_t*)ctx->tmp[T_VBUF].p;
    a.brbuf = (uint32_t*)ctx->tmp[T_BRBUF].p;
    a.dsbuf = (int32_t*)ctx->tmp[T_DSBUF].p;
    a.cap_nodes = N;
    a.cap_brs = K;
    return ALP_OK;
}

// The expand kernel with the pair lookup and a look-back over tiles in it,
// for a grammar's (q, k) (see parse_pairs_kernel).
inline const void* fused_expand_for(int q, int k) {
    if (q == 1 && k == 1) return (const void*)parse_expand_kernel<1, 1, true>;
    if (q == 1 && k == 2) return (const void*)parse_expand_kernel<1, 2, true>;
    if (q == 1 && k == 3) return (const void*)parse_expand_kernel<1, 3, true>;
    if (q == 2 && k == 1) return (const void*)parse_expand_kernel<2, 1, true>;
    if (q == 2 && k == 2) return (const void*)parse_expand_kernel<2, 2, true>;
    return (const void*)parse_expand_kernel<0, 0, true>;
}

// Dynamic shared memory of an expand launch (*sm): its tables, position records and
// node owners, and past them up to EX_SPAN_BYTES more for the tile's token spans, as
// many as leave room for the CTAs per SM that run without them (or the tuned count).
int expand_smem(alp_ctx* ctx, const void* fn, ParseArgs& a, size_t* sm) {
    const size_t base = expand_smem_bytes(ctx->pt.n_pairs, ctx->pt.n_pseq, ctx->pt.n_stack);
    *sm = base;
    a.span_cap = 0;
    int fit = 0, per_sm = 0, reserved = 0, optin = 0;
    cudaFuncAttributes fa;
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)base));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, fn, PP_THREADS, base));
    CK(cudaFuncGetAttributes(&fa, fn));
    CK(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device));
    CK(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, ctx->device));
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    const int ctas = persistent_ctas(fit, ctx->tune.expand_ctas);
    long long room = (long long)per_sm / ctas - reserved - (long long)fa.sharedSizeBytes - (long long)base;
    room = std::min(room, (long long)optin - (long long)fa.sharedSizeBytes - (long long)base);
    room = std::min(room, (long long)EX_SPAN_BYTES) & ~31LL;
    if (room < 1024) return ALP_OK;
    int fit2 = 0;
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(base + room)));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit2, fn, PP_THREADS, base + room));
    if (fit2 < ctas) return ALP_OK;  // token spans through L1, as without the stage
    a.span_cap = (int)(room / 8);     // a multiple of 4
    *sm = base + (size_t)room;
    return ALP_OK;
}

int expand_grid(alp_ctx* ctx, const void* fn, size_t sm2, long long tiles, unsigned* g) {
    int sms = 0, per2 = 0;
    CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, fn, PP_THREADS, sm2));
    const long long x = (long long)persistent_ctas(per2, ctx->tune.expand_ctas) * sms;
    *g = (unsigned)(x < tiles ? x : tiles);
    return ALP_OK;
}

// Positions (⊢ tokens ⊣ per document, L of them) already in
// tmp[T_TTERM..T_TEND] and per-document validity in `dvalid` -> tree.
// `want_tree` 0 gives the production sequence only.  Node offsets of the
// documents land in tmp[T_NODEOFF].
//
// Two forms of the position pass.  The fused one (one kernel: keys, pair
// lookup, look-back over tiles, expansion) needs its output capacities before
// it runs; they come from the nodes and kept brackets per position of the
// last parse on this context, and when the document needs more, the pass runs
// again at the exact sizes it reported.  The first parse on a context, and
// grammars whose counts could pass 32 bits, take the two-pass form: the pair
// kernel and a scan of its tile sums give the exact sizes first.
// h_valid0 (pinned, optional): document 0's validity, read in the same final wait.
int parse_positions(alp_ctx* ctx, long long L, long long nd, uint8_t* dvalid, ParseOut* o, int64_t cap, int ctx_out,
                    int64_t* n_node, int want_tree, uint8_t* h_valid0 = nullptr) {
    *n_node = 0;
    if (L >= 0x7fffffffLL) return fail(ctx, ALP_ERR_ARG, "too many positions (%lld)", L);
    const long long tiles = (L + PP_TILE - 1) / PP_TILE;
    int rc;
    if ((rc = grow(ctx, ctx->tmp[T_NODEOFF], (size_t)(nd + 1) * 8)) || (rc = grow(ctx, ctx->tmp[T_BROFF], (size_t)(nd + 1) * 8)) ||
        (rc = grow(ctx, ctx->scratch, 256)))
        return rc;
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    if ((rc = set_result(ctx, d_res, 1))) return rc;
    ParseArgs a;
    memset(&a, 0, sizeof a);
    a.t = ctx->pt;
    a.P = (const uint16_t*)ctx->tmp[T_TTERM].p;
    a.pstart = (const uint32_t*)ctx->tmp[T_TSTART].p;
    a.pend = (const uint32_t*)ctx->tmp[T_TEND].p;
    a.L = L;
    a.n_docs = nd;
    a.res = d_res;
    a.node_off = (long long*)ctx->tmp[T_NODEOFF].p;
    a.br_off = (long long*)ctx->tmp[T_BROFF].p;
    a.doc_valid = dvalid;
    a.subst_terminals = want_tree;
    if (expand_smem_bytes(ctx->pt.n_pairs, ctx->pt.n_pseq, ctx->pt.n_stack) > 220 * 1024)
        return fail(ctx, ALP_ERR_TABLE, "parser tables too large for shared memory");
    size_t sm2 = expand_smem_bytes(ctx->pt.n_pairs, ctx->pt.n_pseq, ctx->pt.n_stack);
    long long N = 0, B = 0, K = 0;
    const bool fits32 = (unsigned long long)L * (unsigned long long)(ctx->ph.max_prods + 1) < (1ull << 32) &&
                        (unsigned long long)L * (unsigned long long)(ctx->ph.max_brackets + 1) < (1ull << 32);
    if (!ctx->tune.parse_split && fits32 && ctx->est_nodes > 0) {
        // ---- fused: capacities from the last parse, exact sizes on a second run if short
        const void* fn = fused_expand_for(ctx->pt.q, ctx->pt.k);
        unsigned g = 1;
        if ((rc = expand_grid(ctx, fn, sm2, tiles, &g))) return rc;
        if ((rc = grow(ctx, ctx->tmp[T_TSUMS], (size_t)tiles * (4 + 2 * sizeof(PosSums)) + 256))) return rc;
        uint8_t* lb = reinterpret_cast<uint8_t*>(ctx->tmp[T_TSUMS].p);
        a.ticket = reinterpret_cast<unsigned int*>(lb);
        a.lb_flag = reinterpret_cast<uint32_t*>(lb + 16);
        const size_t o_agg = (16 + 4 * (size_t)tiles + 31) & ~(size_t)31;
        a.lb_agg = reinterpret_cast<PosSums*>(lb + o_agg);
        a.lb_inc = a.lb_agg + tiles;
        long long capN = ctx_out ? (long long)(ctx->est_nodes * (double)L * 1.01) + 4096 : cap;
        long long capK = (long long)(ctx->est_kept * (double)L * 1.01) + 4096;
        for (int attempt = 0; attempt < 2; ++attempt) {
            if ((rc = parse_buffers(ctx, o, ctx_out, capN, capK, a))) return rc;
            CK(cudaMemsetAsync(lb, 0, 16 + 4 * (size_t)tiles, ctx->stream));  // ticket, look-back flags
            mark(ctx, "start");
            {
                void* args[] = {&a};
                CK(cudaLaunchKernel(fn, dim3(g), dim3(PP_THREADS), args, sm2, ctx->stream));
            }
            mark(ctx, "parse_expand_kernel(fused)");
            if ((rc = read_result(ctx, d_res))) return rc;
            N = ctx->h_res->aux[0];
            B = ctx->h_res->aux[1];
            K = ctx->h_res->aux[6];
            if (N <= capN && K <= capK) break;
            if (!ctx_out && N > cap) {
                *n_node = N;
                return fail(ctx, ALP_ERR_CAPACITY, "node buffer too small (%lld needed)", (long long)N);
            }
            if (attempt == 1) return fail(ctx, ALP_ERR_CUDA, "fused parse pass reported inconsistent sizes");
            capN = ctx_out ? N : cap;  // run again at the exact sizes
            capK = K;
        }
        a.cap_nodes = N;
        a.cap_brs = K;
    } else {
        // ---- two passes: pair ids and tile sums, their scan, the sizes, then expand
        if ((rc = grow(ctx, ctx->tmp[T_PID], (size_t)L * 2 + 64)) ||
            (rc = grow(ctx, ctx->tmp[T_TSUMS], (tiles + tiles / ST_CHUNK + 2) * sizeof(PosSums))))
            return rc;
        a.pid = (uint16_t*)ctx->tmp[T_PID].p;
        a.tile_sums = (PosSums*)ctx->tmp[T_TSUMS].p;
        const size_t sm1 = pairs_smem_bytes(ctx->pt.n_pairs, ctx->pt.q + ctx->pt.k);
        CK(cudaFuncSetAttribute(pairs_kernel_for(ctx->pt.q, ctx->pt.k), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
        mark(ctx, "start");
        unsigned g_pairs = 1, g_expand = 1;
        {
            int sms = 0, per1 = 0;
            CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per1, pairs_kernel_for(ctx->pt.q, ctx->pt.k), PP_THREADS, sm1));
            const long long x = (long long)persistent_ctas(per1, ctx->tune.pairs_ctas) * sms;
            g_pairs = (unsigned)(x < tiles ? x : tiles);
        }
        {
            void* args[] = {&a};
            CK(cudaLaunchKernel(pairs_kernel_for(ctx->pt.q, ctx->pt.k), dim3(g_pairs), dim3(PP_THREADS), args, sm1,
                                ctx->stream));
        }
        mark(ctx, "parse_pairs_kernel");
        {
            const long long chunks = (tiles + ST_CHUNK - 1) / ST_CHUNK;
            PosSums* csum = a.tile_sums + tiles;  // chunk sums after the tile sums
            scan_tiles_reduce_kernel<<<(unsigned)chunks, ST_CHUNK, 0, ctx->stream>>>(a.tile_sums, tiles, csum, nullptr);
            CK(cudaGetLastError());
            scan_tiles_kernel<<<(unsigned)chunks, ST_CHUNK, 0, ctx->stream>>>(a.tile_sums, tiles, csum, d_res, a.node_off,
                                                                             a.br_off, nd, nullptr);
            CK(cudaGetLastError());
        }
        mark(ctx, "scan_tiles_reduce+scan_tiles");
        if ((rc = read_result(ctx, d_res))) return rc;
        // nodes, brackets, and brackets left after closing adjacent pairs
        N = ctx->h_res->aux[0];
        B = ctx->h_res->aux[1];
        K = ctx->h_res->aux[6];
        if (N > 0xffffffffLL || B > 0xffffffffLL) return fail(ctx, ALP_ERR_ARG, "tree too large");
        if (!ctx_out && N > cap) {
            *n_node = N;
            return fail(ctx, ALP_ERR_CAPACITY, "node buffer too small (%lld needed)", (long long)N);
        }
        if ((rc = parse_buffers(ctx, o, ctx_out, N, K, a))) return rc;
        // one document: the expansion's thread-level sums need no restarts
        const void* ex = nd == 1 ? (const void*)parse_expand_kernel<0, 0, false, true>
                                 : (const void*)parse_expand_kernel<0, 0, false, false>;
        if ((rc = expand_smem(ctx, ex, a, &sm2)) || (rc = expand_grid(ctx, ex, sm2, tiles, &g_expand))) return rc;
        mark(ctx, "start");
        {
            void* args[] = {&a};
            CK(cudaLaunchKernel(ex, dim3(g_expand), dim3(PP_THREADS), args, sm2, ctx->stream));
        }
        mark(ctx, "parse_expand_kernel");
    }
    ctx->last_positions = L;
    ctx->last_brackets = B;
    ctx->last_kept = K;
    ctx->est_nodes = (double)N / (double)L;
    ctx->est_kept = (double)K / (double)L;
    if (ctx->host_tree && want_tree && N > 0 && N <= ctx->host_tree->cap) {
        // tags, kinds and spans are final: their copy to the host overlaps the searches
        alp_ctx::HostTree& h = *ctx->host_tree;
        if (!ctx->cp_out) CK(cudaStreamCreateWithFlags(&ctx->cp_out, cudaStreamNonBlocking));
        if (!ctx->ev_nodes) CK(cudaEventCreateWithFlags(&ctx->ev_nodes, cudaEventDisableTiming));
        CK(cudaEventRecord(ctx->ev_nodes, ctx->stream));
        CK(cudaStreamWaitEvent(ctx->cp_out, ctx->ev_nodes, 0));
        h.started = true;
        if (N <= 0x7fffffffLL) {
            // spans (in [0, 2^31): inputs are shorter) to 32-bit values during the searches;
            // alp_parse_host sends them with the parents, tags and kinds
            if ((rc = grow(ctx, ctx->tmp[T_NARROW], (size_t)N * 12))) return rc;
            int32_t* d32 = (int32_t*)ctx->tmp[T_NARROW].p;
            narrow_i64_kernel<<<NARROW_GRID, 256, 0, ctx->cp_out>>>(o->start, o->end, N, d32, d32 + N);
            CK(cudaGetLastError());
            h.wide = true;
        } else {
            CK(cudaMemcpyAsync(h.tag, o->tag, (size_t)N * 4, cudaMemcpyDeviceToHost, ctx->cp_out));
            CK(cudaMemcpyAsync(h.kind, o->kind, (size_t)N, cudaMemcpyDeviceToHost, ctx->cp_out));
            CK(cudaMemcpyAsync(h.start, o->start, (size_t)N * 8, cudaMemcpyDeviceToHost, ctx->cp_out));
            CK(cudaMemcpyAsync(h.end, o->end, (size_t)N * 8, cudaMemcpyDeviceToHost, ctx->cp_out));
        }
    }
    if (want_tree && !ctx->prof) {
        // the node and bracket searches share nothing but the result block (atomic
        // error bits) and document validity (cleared only): the bracket search runs on a
        // second stream beside the node search, each half-filling the SMs alone
        if (!ctx->aux) {
            CK(cudaStreamCreateWithFlags(&ctx->aux, cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
        }
        CK(cudaEventRecord(ctx->ev_fork, ctx->stream));
        CK(cudaStreamWaitEvent(ctx->aux, ctx->ev_fork, 0));
        rc = run_ple(ctx, a.dsbuf, K, a.brbuf, nullptr, T_B_TMIN, a.br_off, nd, dvalid, d_res, nullptr, 0, nullptr,
                     nullptr, 0, ctx->aux);
        if (!rc) rc = run_ple(ctx, a.vbuf, N, nullptr, o->parent, T_N_TMIN, a.node_off, nd, dvalid, d_res);
        // joined on an error too: no later call on this context may reuse buffers that
        // the bracket search could still be reading
        CK(cudaEventRecord(ctx->ev_join, ctx->aux));
        CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
        if (rc) return rc;
    } else {
        // profiled calls keep one stream, so that every kernel's time is its own
        if (want_tree) {
            if ((rc = run_ple(ctx, a.vbuf, N, nullptr, o->parent, T_N_TMIN, a.node_off, nd, dvalid, d_res))) return rc;
        }
        if ((rc = run_ple(ctx, a.dsbuf, K, a.brbuf, nullptr, T_B_TMIN, a.br_off, nd, dvalid, d_res))) return rc;
    }
    if (h_valid0) CK(cudaMemcpyAsync(h_valid0, dvalid, 1, cudaMemcpyDeviceToHost, ctx->stream));
    if ((rc = read_result(ctx, d_res))) return rc;
    *n_node = N;
    return ALP_OK;
}

int read_valid0(alp_ctx* ctx, const uint8_t* dvalid, int* valid) {
    uint8_t v = 0;
    CK(cudaMemcpyAsync(ctx->h_stage, dvalid, 1, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    memcpy(&v, ctx->h_stage, 1);
    *valid = v ? 1 : 0;
    return ALP_OK;
}

// Lex into typed buffers; sets *count (needed count even when over capacity)
// and *valid.  Returns ALP_ERR_CAPACITY when cap was too small.
template <typename TermT, typename PosT>
int lex_core(alp_ctx* ctx, const uint8_t* d_in, int64_t n, TermT* term, PosT* start, PosT* end, int64_t cap,
             int64_t* count, int* valid) {
    *count = 0;
    *valid = 0;
    if (!ctx->has_lexer) return fail(ctx, ALP_ERR_MODE, "these tables have no lexer");
    if (n == 0) {
        *valid = (ctx->h_tokinfo[1] & TOK_ACCEPT) ? 1 : 0;
        return ALP_OK;
    }
    if (ctx->lex3 && !ctx->state_out) {
        int rc;
        if ((rc = grow(ctx, ctx->tmp[T_DVALID], 16)) || (rc = put_doc_off(ctx, n))) return rc;
        uint8_t* dvalid = (uint8_t*)ctx->tmp[T_DVALID].p;
        long long total = 0;
        rc = lex_seg<TermT, PosT>(ctx, d_in, n, (const long long*)ctx->tmp[T_DOCOFF].p, 1, 0, term, start, end, cap,
                                  dvalid, &total);
        *count = total;
        if (rc) return rc;
        int v = 0;
        if ((rc = read_valid0(ctx, dvalid, &v))) return rc;
        *valid = v;
        if (!v) *count = 0;
        return ALP_OK;
    }
    int rc = launch_lex<LEX_ITEMS, TermT, PosT>(ctx, d_in, n, term, start, end, cap);
    if (rc) return rc;
    *valid = ctx->h_res->valid;
    *count = ctx->h_res->count;
    if (ctx->h_res->error & ALP_DEV_ERR_CAPACITY) return fail(ctx, ALP_ERR_CAPACITY, "token buffer too small");
    if (!*valid) *count = 0;
    return ALP_OK;
}


int parse_core(alp_ctx* ctx, const uint8_t* d_in, int64_t n, ParseOut* o, int64_t cap, int ctx_out,
               int64_t* n_node, int* valid) {
    *n_node = 0;
    *valid = 0;
    if (!ctx->has_lexer || !ctx->has_parser) return fail(ctx, ALP_ERR_MODE, "these tables are not lexer+parser tables");
    int rc;
    const size_t tcap = (size_t)n + 2 + 16;
    if ((rc = grow(ctx, ctx->tmp[T_TTERM], tcap * 2)) || (rc = grow(ctx, ctx->tmp[T_TSTART], tcap * 4)) ||
        (rc = grow(ctx, ctx->tmp[T_TEND], tcap * 4)) || (rc = grow(ctx, ctx->tmp[T_DVALID], 16)) ||
        (rc = put_doc_off(ctx, n)))
        return rc;
    uint8_t* dvalid = (uint8_t*)ctx->tmp[T_DVALID].p;
    long long m = 0;
    // the document's validity comes back with the lexer's token count and with the
    // parser's final counts (pinned bytes in h_stage), not in waits of their own
    uint8_t* hv = reinterpret_cast<uint8_t*>(ctx->h_stage) + 200;
    hv[0] = 0;  // stays 0 for an empty input (the lexer then launches nothing)
    hv[1] = 0;
    ctx->lex_valid0 = hv;
    rc = lex_seg<uint16_t, uint32_t>(ctx, d_in, n, (const long long*)ctx->tmp[T_DOCOFF].p, 1, 1,
                                     (uint16_t*)ctx->tmp[T_TTERM].p, (uint32_t*)ctx->tmp[T_TSTART].p,
                                     (uint32_t*)ctx->tmp[T_TEND].p, (long long)tcap, dvalid, &m);
    ctx->lex_valid0 = nullptr;
    if (rc) return rc;
    if (!hv[0]) return ALP_OK;
    int64_t N = 0;
    rc = parse_positions(ctx, m + 2, 1, dvalid, o, cap, ctx_out, &N, 1, hv + 1);
    if (rc) { *n_node = N; return rc; }
    *valid = hv[1] ? 1 : 0;
    *n_node = *valid ? N : 0;
    return ALP_OK;
}

// Token arrays from the caller (uint32 ids, int64 spans) -> positions ⊢ tokens ⊣.
__global__ void tokens_in_kernel(const uint32_t* term, const int64_t* ts, const int64_t* te, long long m, uint16_t* P,
                                 uint32_t* s32, uint32_t* e32, uint32_t sl, uint32_t sr, AlpResult* res) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m + 2; i += (long long)gridDim.x * blockDim.x) {
        if (i == 0 || i == m + 1) {
            P[i] = (uint16_t)(i == 0 ? sl : sr);
            s32[i] = 0;
            e32[i] = 0;
            continue;
        }
        const uint32_t t = term[i - 1];
        if (t > 0xffffu || t == sl || t == sr) res->valid = 0;
        P[i] = (uint16_t)t;
        s32[i] = ts ? (uint32_t)ts[i - 1] : 0u;
        e32[i] = te ? (uint32_t)te[i - 1] : 0u;
    }
}

int tokens_in(alp_ctx* ctx, const uint32_t* term, const int64_t* ts, const int64_t* te, int64_t m) {
    int rc;
    if ((rc = grow(ctx, ctx->tmp[T_TTERM], (size_t)(m + 2) * 2 + 16)) || (rc = grow(ctx, ctx->tmp[T_TSTART], (size_t)(m + 2) * 4 + 16)) ||
        (rc = grow(ctx, ctx->tmp[T_TEND], (size_t)(m + 2) * 4 + 16)) || (rc = grow(ctx, ctx->scratch, 256)) ||
        (rc = grow(ctx, ctx->tmp[T_DVALID], 16)))
        return rc;
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    if ((rc = set_result(ctx, d_res, 1))) return rc;
    tokens_in_kernel<<<148 * 4, 256, 0, ctx->stream>>>(term, ts, te, m, (uint16_t*)ctx->tmp[T_TTERM].p,
                                                      (uint32_t*)ctx->tmp[T_TSTART].p, (uint32_t*)ctx->tmp[T_TEND].p,
                                                      ctx->pt.start, ctx->pt.end, d_res);
    CK(cudaGetLastError());
    if ((rc = read_result(ctx, d_res))) return rc;
    if (!ctx->h_res->valid) return fail(ctx, ALP_ERR_ARG, "terminal id out of range");
    CK(cudaMemsetAsync(ctx->tmp[T_DVALID].p, 1, 1, ctx->stream));
    return ALP_OK;
}


// ---- learned speculation: MLP training and inference, speculative lexer ----
enum { M_X = 0, M_Z1, M_H1, M_H1B, M_Z2, M_H2, M_H2B, M_Z3, M_DZ3, M_DZ3B, M_DH, M_DZ, M_DZB, M_DX, M_SCAL, M_PART,
       M_CNT };

__global__ void positions_kernel(long long* pos, long long count, long long C) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (long long)gridDim.x * blockDim.x)
        pos[i] = (i + 1) * C;
}

inline unsigned grid_for(long long n);

int gemm(alp_ctx* ctx, const __nv_bfloat16* A, long long sa_m, long long sa_k, const __nv_bfloat16* B, long long sb_k,
         long long sb_n, float* C, long long ldc, int M, int N, int K) {
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    const long long tiles = (long long)((N + UG_BN - 1) / UG_BN) * ((M + UG_BM - 1) / UG_BM);
    // split K while the tiles alone leave most SMs idle and each split keeps >= 4 K steps
    int splits = 1;
    while (tiles * splits < 128 && K / (splits * 2) >= 4 * UG_BK) splits *= 2;
    const int kper = ((K + splits * UG_BK - 1) / (splits * UG_BK)) * UG_BK;
    splits = (K + kper - 1) / kper;
    GemmArgs g{A, sa_m, sa_k, B, sb_k, sb_n, C, ldc, M, N, K, 0, &d_res->error, kper, 0};
    const long long stride = (long long)M * N;
    if (splits > 1) {
        int rc;
        if ((rc = grow(ctx, ctx->mlp[M_PART], (size_t)splits * stride * 4))) return rc;
        g.C = reinterpret_cast<float*>(ctx->mlp[M_PART].p);
        g.ldc = N;
        g.part_stride = stride;
    }
    dim3 grid((N + UG_BN - 1) / UG_BN, (M + UG_BM - 1) / UG_BM, splits);
    CK(cudaFuncSetAttribute(umma_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UG_SMEM));
    umma_gemm_kernel<<<grid, 128, UG_SMEM, ctx->stream>>>(g);
    CK(cudaGetLastError());
    if (splits > 1) {
        gemm_splits_kernel<<<grid_for(stride), 256, 0, ctx->stream>>>(g.C, stride, splits, C, ldc, M, N, 0);
        CK(cudaGetLastError());
    }
    return ALP_OK;
}

inline unsigned grid_for(long long n) {
    long long g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    return (unsigned)(g < 1 ? 1 : g);
}

// The tail of alp_parse_host and alp_parse_batch_host: after the parse (rc) the
// tree's N nodes to the caller's host arrays (capacity cap), with parents and
// spans as 32-bit values widened on the host when parse_positions narrowed the
// spans (ht.wide), else as plain copies.  Waits for every copy in either case.
int tree_to_host(alp_ctx* ctx, int rc, const ParseOut& o, int64_t n_node, int64_t cap, alp_ctx::HostTree& ht,
                 int64_t* h_parent) {
    auto join = [&]() -> int {
        if (ht.started) CK(cudaStreamSynchronize(ctx->cp_out));
        ctx->copies.clear();
        return ALP_OK;
    };
    if (rc) {
        join();
        return rc;
    }
    if (n_node > cap) {
        join();
        return fail(ctx, ALP_ERR_CAPACITY, "host node buffer too small");
    }
    const size_t N = (size_t)n_node;
    if (N && ht.wide) {
        // parents (in [0, N)) to 32-bit values after the searches; then every field goes
        // out chunk by chunk, the widened ones interleaved with the direct copies of tags
        // and kinds so that the widening has the whole transfer to keep up
        int32_t* d32 = (int32_t*)ctx->tmp[T_NARROW].p;
        narrow_i64_kernel<<<NARROW_GRID, 256, 0, ctx->stream>>>(o.parent, nullptr, (long long)N, d32 + 2 * N,
                                                                 nullptr);
        auto issue = [&]() -> int {
            CK(cudaGetLastError());
            CK(cudaEventRecord(ctx->ev_nodes, ctx->stream));
            CK(cudaStreamWaitEvent(ctx->cp_out, ctx->ev_nodes, 0));
            for (size_t c = 0; c < N; c += (size_t)RING_CHUNK) {
                const size_t len = std::min((size_t)RING_CHUNK, N - c);
                ctx->copies.push_back({d32 + c, ht.start + c, len, true});
                ctx->copies.push_back({d32 + N + c, ht.end + c, len, true});
                ctx->copies.push_back({d32 + 2 * N + c, h_parent + c, len, true});
                ctx->copies.push_back({o.tag + c, ht.tag + c, len * 4, false});
                ctx->copies.push_back({o.kind + c, ht.kind + c, len, false});
            }
            return send_to_host(ctx, ctx->cp_out);
        };
        if ((rc = issue())) {
            join();
            return rc;
        }
        ctx->last_d2h += (long long)N * 17;
    } else if (N) {
        CK(cudaMemcpyAsync(h_parent, o.parent, N * 8, cudaMemcpyDeviceToHost, ctx->stream));
        if (!ht.started) {
            CK(cudaMemcpyAsync(ht.tag, o.tag, N * 4, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaMemcpyAsync(ht.kind, o.kind, N, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaMemcpyAsync(ht.start, o.start, N * 8, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaMemcpyAsync(ht.end, o.end, N * 8, cudaMemcpyDeviceToHost, ctx->stream));
        }
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->last_d2h += (long long)N * 29;
    }
    return join();
}

// alp_parse_batch after its argument checks: n bytes of documents at d_in with
// offsets d_off[0..n_docs] (both on the device); the tree in o, N nodes.
int parse_batch_core(alp_ctx* ctx, const uint8_t* d_in, const int64_t* d_off, int64_t n_docs, int64_t n, ParseOut* o,
                     int64_t* N) {
    int rc;
    const size_t tcap = (size_t)n + 2 * (size_t)n_docs + 16;
    if ((rc = grow(ctx, ctx->tmp[T_TTERM], tcap * 2)) || (rc = grow(ctx, ctx->tmp[T_TSTART], tcap * 4)) ||
        (rc = grow(ctx, ctx->tmp[T_TEND], tcap * 4)) || (rc = grow(ctx, ctx->tmp[T_DVALID], (size_t)n_docs + 16)))
        return rc;
    uint8_t* dvalid = (uint8_t*)ctx->tmp[T_DVALID].p;
    long long m = 0;
    rc = lex_seg<uint16_t, uint32_t>(ctx, d_in, n, (const long long*)d_off, n_docs, 1, (uint16_t*)ctx->tmp[T_TTERM].p,
                                     (uint32_t*)ctx->tmp[T_TSTART].p, (uint32_t*)ctx->tmp[T_TEND].p, (long long)tcap,
                                     dvalid, &m);
    if (rc) return rc;
    return parse_positions(ctx, m + 2 * n_docs, n_docs, dvalid, o, 0, 1, N, 1);
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

int alp_ctx_create(const void* blob, size_t len, int device, alp_ctx** out) {
    if (!blob || !out) return ALP_ERR_ARG;
    *out = nullptr;
    alp_ctx* ctx = new alp_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete ctx;
        return ALP_ERR_CUDA;
    }
    Reader r{reinterpret_cast<const uint8_t*>(blob), reinterpret_cast<const uint8_t*>(blob) + len};
    uint32_t magic = r.u32(), ver = r.u32(), hl = r.u32(), hp = r.u32();
    int rc = ALP_OK;
    if (!r.ok || magic != BLOB_MAGIC || ver != 1) rc = fail(ctx, ALP_ERR_TABLE, "not an alpacc_b200 table blob");
    if (!rc && hl) rc = load_lexer(ctx, r);
    if (!rc && hp) rc = load_parser(ctx->pt, ctx->ph, r.p, r.e, ctx->owned, ctx->err);
    if (!rc && hp) ctx->has_parser = true;
    if (!rc && hl && hp) {
        // the parser indexes its key table with the lexer's terminal ids
        const uint32_t T = (uint32_t)ctx->pt.T;
        for (uint32_t v : ctx->h_tokinfo)
            if ((v & TOK_TERM_MASK) >= T) { rc = fail(ctx, ALP_ERR_TABLE, "lexer terminal id outside the parser's"); break; }
        if (!rc && (ctx->pt.start >= T || ctx->pt.end >= T || ctx->pt.empty >= T))
            rc = fail(ctx, ALP_ERR_TABLE, "parser sentinel ids out of range");
    }
    if (!rc && cudaMallocHost(&ctx->h_res, sizeof(AlpResult)) != cudaSuccess)
        rc = fail(ctx, ALP_ERR_CUDA, "cudaMallocHost failed");
    if (!rc && cudaMallocHost(&ctx->h_stage, 256) != cudaSuccess) rc = fail(ctx, ALP_ERR_CUDA, "cudaMallocHost failed");
    if (rc) {
        alp_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return ALP_OK;
}

void alp_ctx_destroy(alp_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    for (void* p : ctx->owned) cudaFree(p);
    if (ctx->scratch.p) cudaFree(ctx->scratch.p);
    for (auto& b : ctx->out)
        if (b.p) cudaFree(b.p);
    for (auto& b : ctx->tmp)
        if (b.p) cudaFree(b.p);
    for (auto& b : ctx->mlp)
        if (b.p) cudaFree(b.p);
    for (auto& b : ctx->spec)
        if (b.p) cudaFree(b.p);
    if (ctx->h_res) cudaFreeHost(ctx->h_res);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    for (auto& m : ctx->marks) cudaEventDestroy(m.second);
    if (ctx->pipe.p) cudaFree(ctx->pipe.p);
    if (ctx->carry.p) cudaFree(ctx->carry.p);
    if (ctx->h_carry) cudaFreeHost(ctx->h_carry);
    for (int i = 0; i < 2; ++i) {
        if (ctx->ev_in[i]) cudaEventDestroy(ctx->ev_in[i]);
        if (ctx->ev_done[i]) cudaEventDestroy(ctx->ev_done[i]);
        if (ctx->ev_out[i]) cudaEventDestroy(ctx->ev_out[i]);
    }
    if (ctx->cp_in) cudaStreamDestroy(ctx->cp_in);
    if (ctx->cp_out) cudaStreamDestroy(ctx->cp_out);
    if (ctx->aux) cudaStreamDestroy(ctx->aux);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    if (ctx->ev_nodes) cudaEventDestroy(ctx->ev_nodes);
    for (cudaEvent_t e : ctx->ev_ring)
        if (e) cudaEventDestroy(e);
    if (ctx->h_ring) cudaFreeHost(ctx->h_ring);
    delete ctx->pool;
    delete ctx;
}

const char* alp_last_error(const alp_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int alp_set_stream(alp_ctx* ctx, void* stream) {
    if (!ctx) return ALP_ERR_ARG;
    ctx->stream = reinterpret_cast<cudaStream_t>(stream);
    return ALP_OK;
}

int alp_ctx_info(const alp_ctx* ctx, int64_t* out, int n_out) {
    if (!ctx || !out) return ALP_ERR_ARG;
    int64_t v[15] = {ctx->has_lexer, ctx->has_parser, ctx->has_parser ? ctx->ph.n_terms : ctx->n_terms,
                     ctx->ph.n_prods, ctx->ph.q, ctx->ph.k, ctx->ph.max_prods, ctx->ph.max_brackets,
                     ctx->last_tokens, ctx->last_positions, ctx->last_brackets, ctx->last_kept, ctx->dev_allocs,
                     ctx->last_h2d, ctx->last_d2h};
    for (int i = 0; i < n_out && i < 15; ++i) out[i] = v[i];
    return ALP_OK;
}

int alp_ctx_profile(alp_ctx* ctx, int on) {
    if (!ctx) return ALP_ERR_ARG;
    for (auto& m : ctx->marks) cudaEventDestroy(m.second);
    ctx->marks.clear();
    ctx->prof = on ? 1 : 0;
    return ALP_OK;
}

int alp_ctx_timings(alp_ctx* ctx, char* buf, size_t len) {
    if (!ctx || !buf || !len) return ALP_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    std::string out;
    for (size_t i = 1; i < ctx->marks.size(); ++i) {
        if (strcmp(ctx->marks[i].first, "start") == 0) continue;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->marks[i - 1].second, ctx->marks[i].second);
        char line[160];
        snprintf(line, sizeof line, "%s %.6f\n", ctx->marks[i].first, ms);
        out += line;
    }
    for (auto& m : ctx->marks) cudaEventDestroy(m.second);
    ctx->marks.clear();
    snprintf(buf, len, "%s", out.c_str());
    return out.size() < len ? ALP_OK : ALP_ERR_CAPACITY;
}

// One thread waits, with the kernels' own bounded waits, on a 32-bit and a
// 64-bit status word that nothing ever sets: each wait gives up after its
// poll limit and records the timeout, as a look-back wait does when a tile
// never publishes.
__global__ void wait_check_kernel(const uint32_t* w32, const unsigned long long* w64, AlpResult* res) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t a = wait32(w32, &res->error);
    const unsigned long long b = wait64(w64, &res->error);
    res->aux[0] = (long long)(a >> 30);
    res->aux[1] = (long long)(b >> 62);
}

int alp_check_bounded_wait(alp_ctx* ctx) {
    if (!ctx) return ALP_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    int rc;
    if ((rc = grow(ctx, ctx->scratch, 256))) return rc;
    uint8_t* base = reinterpret_cast<uint8_t*>(ctx->scratch.p);
    AlpResult* res = reinterpret_cast<AlpResult*>(base);
    CK(cudaMemsetAsync(base, 0, 256, ctx->stream));  // result and two status words in state X
    wait_check_kernel<<<1, 32, 0, ctx->stream>>>(reinterpret_cast<const uint32_t*>(base + 128),
                                                  reinterpret_cast<const unsigned long long*>(base + 136), res);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->h_res, res, sizeof(AlpResult), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->h_res->error & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "bounded wait gave up");
    return fail(ctx, ALP_ERR_CUDA, "bounded wait returned without giving up");
}

int alp_tune_get(const alp_ctx* ctx, int32_t* cfg, int n) {
    if (!ctx || !cfg || n < 3) return ALP_ERR_ARG;
    cfg[0] = ctx->tune.ple;
    cfg[1] = ctx->tune.pairs_ctas;
    cfg[2] = ctx->tune.expand_ctas;
    if (n > 3) cfg[3] = ctx->tune.mlp;
    if (n > 4) cfg[4] = ctx->tune.lex_split;
    if (n > 5) cfg[5] = ctx->tune.parse_split;
    if (n > 6) cfg[6] = scan_g(ctx);
    return ALP_OK;
}

int alp_tune_set(alp_ctx* ctx, const int32_t* cfg, int n) {
    if (!ctx || !cfg || n < 3) return ALP_ERR_ARG;
    if (cfg[0] < 0 || cfg[0] >= N_PLE_SHAPES || cfg[1] < 0 || cfg[1] > 32 || cfg[2] < 0 || cfg[2] > 32)
        return fail(ctx, ALP_ERR_ARG, "tuning values out of range");
    if (n > 3 && (cfg[3] < 0 || cfg[3] > 1)) return fail(ctx, ALP_ERR_ARG, "MLP kernel choice out of range");
    if (n > 4 && (cfg[4] < 0 || cfg[4] > 1)) return fail(ctx, ALP_ERR_ARG, "lexer token pass choice out of range");
    if (n > 5 && (cfg[5] < 0 || cfg[5] > 1)) return fail(ctx, ALP_ERR_ARG, "parser position pass choice out of range");
    if (n > 6 && cfg[6] != 0 && cfg[6] != 8 && cfg[6] != 16 && cfg[6] != 32)
        return fail(ctx, ALP_ERR_ARG, "state-scan chunks per lane must be 8, 16 or 32");
    ctx->tune.ple = cfg[0];
    ctx->tune.pairs_ctas = cfg[1];
    ctx->tune.expand_ctas = cfg[2];
    if (n > 3) ctx->tune.mlp = cfg[3];
    if (n > 4) ctx->tune.lex_split = cfg[4];
    if (n > 5) ctx->tune.parse_split = cfg[5];
    if (n > 6) ctx->tune.scan_g = cfg[6];
    return ALP_OK;
}

int alp_tune_shapes(int32_t* out, int n) {
    if (!out) return N_PLE_SHAPES;
    for (int i = 0; i < N_PLE_SHAPES && 2 * i + 1 < n; ++i) {
        out[2 * i] = ple_shapes[i].threads;
        out[2 * i + 1] = ple_shapes[i].items;
    }
    return N_PLE_SHAPES;
}

int alp_tune_parse(alp_ctx* ctx, const uint8_t* d_in, int64_t n, int reps, char* report, size_t report_len) {
    if (!ctx) return ALP_ERR_ARG;
    if (!ctx->has_lexer || !ctx->has_parser) return fail(ctx, ALP_ERR_MODE, "these tables are not lexer+parser tables");
    if (reps < 1 || reps > 100) return fail(ctx, ALP_ERR_ARG, "reps out of range");
    int rc = check_in(ctx, d_in, n, true);
    if (rc) return rc;
    CK(cudaSetDevice(ctx->device));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    std::string rep;
    long long nodes0 = -1;
    // median ms of `reps` calls with the context's current tuning
    auto measure = [&](double* ms) -> int {
        int64_t *pp, *ps, *pe;
        uint32_t* pt;
        uint8_t* pk;
        int64_t nn = 0;
        int valid = 0;
        int r = alp_parse(ctx, d_in, n, &pp, &pt, &pk, &ps, &pe, &nn, &valid);  // warm-up
        if (r) return r;
        if (nodes0 < 0) nodes0 = nn;
        if (nn != nodes0) return fail(ctx, ALP_ERR_CUDA, "tuning variants disagree on the node count");
        std::vector<float> t;
        for (int i = 0; i < reps; ++i) {
            if (cudaEventRecord(e0, ctx->stream) != cudaSuccess) return fail(ctx, ALP_ERR_CUDA, "event record failed");
            if ((r = alp_parse(ctx, d_in, n, &pp, &pt, &pk, &ps, &pe, &nn, &valid))) return r;
            if (cudaEventRecord(e1, ctx->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
                return fail(ctx, ALP_ERR_CUDA, "event record failed");
            float x = 0;
            cudaEventElapsedTime(&x, e0, e1);
            t.push_back(x);
        }
        std::sort(t.begin(), t.end());
        *ms = t[t.size() / 2];
        return ALP_OK;
    };
    auto line = [&](const char* what, int v, double ms) {
        char b[96];
        snprintf(b, sizeof b, "%s %d %.4f\n", what, v, ms);
        rep += b;
    };
    const Tuning saved = ctx->tune;
    auto done = [&](int r) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (r) ctx->tune = saved;
        if (report && report_len) {
            const size_t k = rep.size() < report_len - 1 ? rep.size() : report_len - 1;
            memcpy(report, rep.data(), k);
            report[k] = 0;
        }
        return r;
    };
    // one knob at a time, the others held at their best so far
    double best = 1e30, ms = 0;
    int arg = 0;
    auto knob = [&](const char* what, int* field, const int* values, int count) -> int {
        best = 1e30;
        arg = values[0];
        for (int i = 0; i < count; ++i) {
            *field = values[i];
            int r = measure(&ms);
            if (r) return r;
            line(what, values[i], ms);
            if (ms < best) { best = ms; arg = values[i]; }
        }
        *field = arg;
        return ALP_OK;
    };
    // lexer: the token pass's form, the state scan's chunks per lane
    {
        const int forms[] = {0, 1}, gs[] = {8, 16, 32};
        if ((rc = knob("lex_token_pass_split", &ctx->tune.lex_split, forms, 2)) ||
            (rc = knob("lex_scan_chunks_per_lane", &ctx->tune.scan_g, gs, 3)) ||
            (rc = knob("parse_position_pass_split", &ctx->tune.parse_split, forms, 2)))
            return done(rc);
    }
    int fit_pairs = 1, fit_expand = 1;
    {
        const size_t sm1 = pairs_smem_bytes(ctx->pt.n_pairs, ctx->pt.q + ctx->pt.k);
        const size_t sm2 = expand_smem_bytes(ctx->pt.n_pairs, ctx->pt.n_pseq, ctx->pt.n_stack);
        const void* ex = ctx->tune.parse_split ? (const void*)parse_expand_kernel<0, 0, false>
                                               : fused_expand_for(ctx->pt.q, ctx->pt.k);
        CK(cudaFuncSetAttribute(pairs_kernel_for(ctx->pt.q, ctx->pt.k), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
        CK(cudaFuncSetAttribute(ex, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit_pairs, pairs_kernel_for(ctx->pt.q, ctx->pt.k), PP_THREADS, sm1));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit_expand, ex, PP_THREADS, sm2));
    }
    best = 1e30;
    arg = 0;
    for (int i = 0; i < N_PLE_SHAPES; ++i) {
        ctx->tune.ple = i;
        if ((rc = measure(&ms))) return done(rc);
        char what[48];
        snprintf(what, sizeof what, "ple_shape_%dx%d", ple_shapes[i].threads, ple_shapes[i].items);
        line(what, i, ms);
        if (ms < best) { best = ms; arg = i; }
    }
    ctx->tune.ple = arg;
    best = 1e30;
    arg = 0;
    for (int c = 1; c <= fit_expand; ++c) {
        ctx->tune.expand_ctas = c;
        if ((rc = measure(&ms))) return done(rc);
        line("expand_ctas_per_sm", c, ms);
        if (ms < best) { best = ms; arg = c; }
    }
    ctx->tune.expand_ctas = arg;
    if (ctx->tune.parse_split) {  // the pair kernel runs only in the two-pass form
        best = 1e30;
        arg = 0;
        for (int c = 1; c <= fit_pairs; ++c) {
            ctx->tune.pairs_ctas = c;
            if ((rc = measure(&ms))) return done(rc);
            line("pairs_ctas_per_sm", c, ms);
            if (ms < best) { best = ms; arg = c; }
        }
        ctx->tune.pairs_ctas = arg;
    }
    line("best_ms", 0, best);
    return done(ALP_OK);
}

int alp_write_reference_format(int mode, int64_t n_docs, const uint8_t* valid, const int64_t* off,
                               const uint32_t* id, const int64_t* parent, const uint8_t* kind,
                               const int64_t* start, const int64_t* end, uint8_t* out, size_t cap,
                               size_t* len) {
    if (!len || n_docs < 0 || (n_docs > 0 && (!valid || !off))) return ALP_ERR_ARG;
    *len = 0;
    size_t rec;
    switch (mode) {
        case ALP_WIRE_LEXER: rec = 24; if (!id || !start || !end) return ALP_ERR_ARG; break;
        case ALP_WIRE_LEXPARSE: rec = 33; if (!id || !parent || !kind || !start || !end) return ALP_ERR_ARG; break;
        case ALP_WIRE_PARSER: rec = 8; if (!id) return ALP_ERR_ARG; break;
        default: return ALP_ERR_ARG;
    }
    // the size first: a boolean per input, a count and the records per accepted one
    size_t total = 8;
    for (int64_t d = 0; d < n_docs; ++d) {
        if (off[d] < 0 || off[d + 1] < off[d]) return ALP_ERR_ARG;
        total += 1;
        if (valid[d]) total += 8 + rec * (size_t)(off[d + 1] - off[d]);
    }
    *len = total;
    if (!out) return ALP_OK;
    if (cap < total) return ALP_ERR_CAPACITY;
    if (mode == ALP_WIRE_LEXPARSE)
        for (int64_t d = 0; d < n_docs; ++d)
            if (valid[d])
                for (int64_t e = off[d]; e < off[d + 1]; ++e)
                    if (kind[e] > 1) return ALP_ERR_ARG;
    uint8_t* p = out;
    auto u64 = [&p](uint64_t v) {
        for (int b = 7; b >= 0; --b) *p++ = (uint8_t)(v >> (8 * b));
    };
    u64((uint64_t)n_docs);
    for (int64_t d = 0; d < n_docs; ++d) {
        *p++ = valid[d] ? 1 : 0;
        if (!valid[d]) continue;
        u64((uint64_t)(off[d + 1] - off[d]));
        for (int64_t e = off[d]; e < off[d + 1]; ++e) {
            if (mode == ALP_WIRE_LEXER) {
                u64(id[e]);
                u64((uint64_t)start[e]);
                u64((uint64_t)end[e]);
            } else if (mode == ALP_WIRE_LEXPARSE) {
                *p++ = kind[e];
                u64((uint64_t)parent[e]);
                u64(id[e]);
                u64(kind[e] ? (uint64_t)start[e] : 0);
                u64(kind[e] ? (uint64_t)end[e] : 0);
            } else {
                u64(id[e]);
            }
        }
    }
    return ALP_OK;
}

// The check of lexerTestsCompare / lexerParserTestsCompare / parserTestsCompare
// (src/Alpacc/Test/Lexer.hs:181-231, LexerParser.hs:342-392, Parser.hs:140-167):
// equal numbers of results, then the results equal input by input.
int alp_compare_reference_format(int mode, const uint8_t* a, size_t a_len, const uint8_t* b, size_t b_len,
                                 int64_t* first_diff, int* field) {
    if (!first_diff || !field || (a_len && !a) || (b_len && !b)) return ALP_ERR_ARG;
    *first_diff = -1;
    *field = -1;
    int nf;
    switch (mode) {
        case ALP_WIRE_LEXER: nf = 3; break;
        case ALP_WIRE_LEXPARSE: nf = 5; break;
        case ALP_WIRE_PARSER: nf = 1; break;
        default: return ALP_ERR_ARG;
    }
    const size_t rec = mode == ALP_WIRE_LEXER ? 24 : (mode == ALP_WIRE_LEXPARSE ? 33 : 8);
    // one file's inputs: (accepted, element count, first record); false when malformed
    // (truncated, a boolean or kind byte out of range, bytes after the last input)
    struct Item {
        bool ok;
        uint64_t n;
        const uint8_t* r;
    };
    auto u64 = [](const uint8_t* q) {
        uint64_t v = 0;
        for (int k = 0; k < 8; ++k) v = v << 8 | q[k];
        return v;
    };
    auto scan = [&](const uint8_t* f, size_t len, std::vector<Item>& items) -> bool {
        if (len < 8) return false;
        const uint64_t count = u64(f);
        size_t p = 8;
        if (count > len) return false;  // at least one byte per input
        items.reserve((size_t)count);
        for (uint64_t i = 0; i < count; ++i) {
            if (p >= len || f[p] > 1) return false;
            if (!f[p++]) {
                items.push_back({false, 0, nullptr});
                continue;
            }
            if (len - p < 8) return false;
            const uint64_t n = u64(f + p);
            p += 8;
            if (n > (len - p) / rec) return false;
            if (mode == ALP_WIRE_LEXPARSE)
                for (uint64_t e = 0; e < n; ++e)
                    if (f[p + e * rec] > 1) return false;
            items.push_back({true, n, f + p});
            p += (size_t)n * rec;
        }
        return p == len;
    };
    std::vector<Item> x, y;
    if (!scan(a, a_len, x) || !scan(b, b_len, y)) return ALP_ERR_ARG;
    // different numbers of results fail before any result is compared
    const size_t m = std::min(x.size(), y.size());
    if (x.size() != y.size()) {
        *first_diff = (int64_t)m;
        return ALP_OK;
    }
    for (size_t i = 0; i < m; ++i) {
        if (x[i].ok != y[i].ok || x[i].n != y[i].n) {
            *first_diff = (int64_t)i;
            return ALP_OK;
        }
        if (!x[i].ok) continue;
        // the first differing field of the first differing record, in record order
        // (lexer: term, start, end; lexer+parser: kind, parent, id, start, end)
        for (uint64_t e = 0; e < x[i].n; ++e) {
            const uint8_t *u = x[i].r + e * rec, *v = y[i].r + e * rec;
            if (memcmp(u, v, rec) == 0) continue;
            *first_diff = (int64_t)i;
            int k = 0, o = 0;
            if (mode == ALP_WIRE_LEXPARSE) {
                if (u[0] != v[0]) {
                    *field = 0;
                    return ALP_OK;
                }
                k = 1;
                o = 1;
            }
            for (; k < nf; ++k, o += 8)
                if (memcmp(u + o, v + o, 8) != 0) break;
            *field = k;
            return ALP_OK;
        }
    }
    return ALP_OK;
}

int alp_memcpy(alp_ctx* ctx, void* dst, const void* src, size_t bytes) {
    if (!ctx || (bytes && (!dst || !src))) return ALP_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    if (bytes) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return ALP_OK;
}

int alp_lex_into(alp_ctx* ctx, const uint8_t* d_in, int64_t n, uint32_t* d_term, int64_t* d_start,
                 int64_t* d_end, int64_t cap, int64_t* n_tok, int* valid) {
    int rc = check_in(ctx, d_in, n, true);
    if (rc) return rc;
    if (!n_tok || !valid || (cap > 0 && (!d_term || !d_start || !d_end)))
        return fail(ctx, ALP_ERR_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    return lex_core<uint32_t, int64_t>(ctx, d_in, n, d_term, d_start, d_end, cap, n_tok, valid);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Scratch-free lexing: alp_lex_noalloc
//
// Some callers cannot allocate device memory at the moment they lex: code that
// owns every byte of the device through its own pool (a serving framework that
// reserved the GPU up front), or a path where cudaMalloc/cudaFree would
// synchronise the device and stall other streams.  alp_lex_noalloc serves them:
// the look-back status words and the result block live in the fixed array
// below, compiled into the library, instead of in context scratch that grows
// with cudaMalloc.  The caller still passes the input and the output buffers.
// The call blocks on the context stream until the token count is read back.
// ---------------------------------------------------------------------------
namespace {

constexpr long long NOALLOC_MAX_BYTES = 128ll << 20;                    // largest input
constexpr long long NOALLOC_MAX_TILES = NOALLOC_MAX_BYTES / LEX_TILE;  // 32768 tiles
constexpr size_t NOALLOC_SCRATCH_BYTES = 256 + 12 * (size_t)NOALLOC_MAX_TILES;  // 393,472 bytes

// Every GPU that loads this library holds one copy until the process exits.
// Host code must not pass `g_noalloc_scratch` itself to a kernel: on the host
// the name is only a stand-in, so its device address comes from
// cudaGetSymbolAddress, asked again on every call.  The lookup allocates
// nothing, and asking each time keeps the address right when the device's
// primary context was reset and the module reloaded at another address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

}  // namespace

extern "C" {

int alp_lex_noalloc(alp_ctx* ctx, const uint8_t* d_in, int64_t n, uint32_t* d_term, int64_t* d_start,
                    int64_t* d_end, int64_t cap, int64_t* n_tok, int* valid) {
    if (!ctx) return ALP_ERR_ARG;
    if (n < 0 || (n > 0 && !d_in)) return fail(ctx, ALP_ERR_ARG, "alp_lex_noalloc: bad input");
    if (n > NOALLOC_MAX_BYTES)
        return fail(ctx, ALP_ERR_ARG, "alp_lex_noalloc: input of %lld bytes exceeds the %lld-byte limit",
                    (long long)n, NOALLOC_MAX_BYTES);
    if (!n_tok || !valid || (cap > 0 && (!d_term || !d_start || !d_end)))
        return fail(ctx, ALP_ERR_ARG, "alp_lex_noalloc: null output");
    if (!ctx->has_lexer) return fail(ctx, ALP_ERR_MODE, "these tables have no lexer");
    *n_tok = 0;
    *valid = 0;
    CK(cudaSetDevice(ctx->device));
    if (n == 0) {
        *valid = (ctx->h_tokinfo[1] & TOK_ACCEPT) ? 1 : 0;
        return ALP_OK;
    }
    void* sym = nullptr;
    const cudaError_t se = cudaGetSymbolAddress(&sym, g_noalloc_scratch);
    if (se != cudaSuccess || !sym) return fail(ctx, ALP_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(se));
    uint8_t* base = reinterpret_cast<uint8_t*>(sym);
    const long long tiles = (n + LEX_TILE - 1) / LEX_TILE;
    const size_t used = 256 + 12 * (size_t)tiles;
    // the array keeps the previous call's words: clear the part this call uses
    CK(cudaMemsetAsync(base, 0, used, ctx->stream));
    LexArgs a;
    a.in = d_in;
    a.n = n;
    a.aligned16 = ((reinterpret_cast<uintptr_t>(d_in) & 15u) == 0) ? 1 : 0;
    a.t = ctx->lt;
    a.res = reinterpret_cast<AlpResult*>(base);
    a.ticket = reinterpret_cast<unsigned int*>(base + 128);
    a.stB = reinterpret_cast<unsigned long long*>(base + 256);
    a.stA = reinterpret_cast<uint32_t*>(base + 256 + 8 * (size_t)tiles);
    a.out_term = d_term;
    a.out_start = d_start;
    a.out_end = d_end;
    a.cap = cap;
    a.num_tiles = (unsigned)tiles;
    a.state_out = nullptr;
    auto k = lex_kernel<LEX_ITEMS, uint32_t, int64_t>;
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->lex_smem));
    // persistent like launch_lex: as many CTAs as fit at once, each taking tile tickets
    int per_sm = 0, sms = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, LEX_THREADS, ctx->lex_smem));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    long long grid = (long long)(per_sm > 0 ? per_sm : 1) * sms;
    if (grid > tiles) grid = tiles;
    k<<<(unsigned)grid, LEX_THREADS, ctx->lex_smem, ctx->stream>>>(a);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(ctx->h_res, a.res, sizeof(AlpResult), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->h_res->error & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "lexer look-back timed out");
    *valid = ctx->h_res->valid;
    *n_tok = ctx->h_res->count;
    if (ctx->h_res->error & ALP_DEV_ERR_CAPACITY) return fail(ctx, ALP_ERR_CAPACITY, "token buffer too small");
    if (!*valid) *n_tok = 0;
    return ALP_OK;
}

int alp_lex(alp_ctx* ctx, const uint8_t* d_in, int64_t n, uint32_t** d_term, int64_t** d_start,
            int64_t** d_end, int64_t* n_tok, int* valid) {
    int rc = check_in(ctx, d_in, n, true);
    if (rc) return rc;
    if (!d_term || !d_start || !d_end || !n_tok || !valid) return fail(ctx, ALP_ERR_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    int64_t cap = n / 2 + 1024;
    for (int attempt = 0; attempt < 2; ++attempt) {
        if ((rc = grow(ctx, ctx->out[0], cap * 4)) || (rc = grow(ctx, ctx->out[1], cap * 8)) ||
            (rc = grow(ctx, ctx->out[2], cap * 8)))
            return rc;
        cap = (int64_t)(ctx->out[1].bytes / 8);
        rc = lex_core<uint32_t, int64_t>(ctx, d_in, n, (uint32_t*)ctx->out[0].p, (int64_t*)ctx->out[1].p,
                                         (int64_t*)ctx->out[2].p, cap, n_tok, valid);
        if (rc != ALP_ERR_CAPACITY) break;
        cap = *n_tok + 1;
    }
    if (rc) return rc;
    *d_term = (uint32_t*)ctx->out[0].p;
    *d_start = (int64_t*)ctx->out[1].p;
    *d_end = (int64_t*)ctx->out[2].p;
    return ALP_OK;
}

int alp_lex_host(alp_ctx* ctx, const uint8_t* h_in, int64_t n, uint32_t* h_term, int64_t* h_start,
                 int64_t* h_end, int64_t cap, int64_t* n_tok, int* valid) {
    int rc = check_in(ctx, h_in, n, true);
    if (rc) return rc;
    if (!n_tok || !valid || cap < 0 || (cap > 0 && (!h_term || !h_start || !h_end)))
        return fail(ctx, ALP_ERR_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    if ((rc = grow(ctx, ctx->tmp[0], (size_t)n + 16))) return rc;
    if (n) CK(cudaMemcpyAsync(ctx->tmp[0].p, h_in, (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    uint32_t* dt;
    int64_t *ds, *de;
    ctx->last_h2d = n;
    ctx->last_d2h = 0;
    rc = alp_lex(ctx, (const uint8_t*)ctx->tmp[0].p, n, &dt, &ds, &de, n_tok, valid);
    if (rc) return rc;
    if (*n_tok > cap) return fail(ctx, ALP_ERR_CAPACITY, "host token buffer too small");
    const size_t M = (size_t)*n_tok;
    if (M && M <= 0x7fffffffu) {
        // spans (positions below 2^31) cross as 32-bit values, widened on the host
        if ((rc = grow(ctx, ctx->tmp[T_NARROW], M * 8))) return rc;
        int32_t* d32 = (int32_t*)ctx->tmp[T_NARROW].p;
        narrow_i64_kernel<<<NARROW_GRID, 256, 0, ctx->stream>>>(ds, de, (long long)M, d32, d32 + M);
        CK(cudaGetLastError());
        ctx->copies.clear();
        for (size_t c = 0; c < M; c += (size_t)RING_CHUNK) {
            const size_t len = std::min((size_t)RING_CHUNK, M - c);
            ctx->copies.push_back({d32 + c, h_start + c, len, true});
            ctx->copies.push_back({d32 + M + c, h_end + c, len, true});
            ctx->copies.push_back({dt + c, h_term + c, len * 4, false});
        }
        if ((rc = send_to_host(ctx, ctx->stream))) return rc;
        ctx->last_d2h = (long long)M * 12;
    } else if (M) {
        CK(cudaMemcpyAsync(h_term, dt, M * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(h_start, ds, M * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(h_end, de, M * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->last_d2h = (long long)M * 20;
    }
    return ALP_OK;
}


// ---- token streams ----------------------------------------------------------
// Input that arrives in pieces, lexed piece by piece with the DFA state and the
// start of the token in progress carried on the device, so that the tokens are
// those of alp_lex on the concatenation (the reference's chunk loop:
// futhark/lexer.fut:148-160, cuda/lexer.cu:452-543).  A piece writes the tokens
// that end inside it; the last token follows when the stream ends.

// One piece [d_in, d_in + n) at stream position pos: the five lexer kernels
// with the carry as entry state and no end of input, then the carry update.
// global: tokens go after carry->tokens, else from index 0.  Stream-ordered.
static int stream_piece(alp_ctx* ctx, LexCarry* carry, const uint8_t* d_in, long long n, long long pos, int global,
                        long long first, uint32_t* term, int64_t* start, int64_t* end, long long cap) {
    int rc;
    if ((rc = grow(ctx, ctx->tmp[T_TOKOFF], 64))) return rc;
    Lex3Run r;
    if ((rc = lex3_prepare(ctx, d_in, n, nullptr, 1, 0, term, start, end, cap,
                           reinterpret_cast<uint8_t*>(ctx->tmp[T_TOKOFF].p) + 32, r)))
        return rc;
    r.sg.cont = 1;
    r.sg.end1 = n + 1;  // the input does not end in this piece
    r.a.carry = carry;
    r.a.pos_base = pos;
    r.a.carry_tokens = global;
    r.a.tok_first = first;
    if ((rc = lex3_front(ctx, r)) || (rc = lex3_emit<uint32_t, int64_t>(ctx, r))) return rc;
    lex3_stream_tail_kernel<<<1, LX_THREADS, 0, ctx->stream>>>(r.a);
    CK(cudaGetLastError());
    mark(ctx, "lex3_stream_tail_kernel");
    return ALP_OK;
}

static int stream_end(alp_ctx* ctx, LexCarry* carry, long long total, int global, long long first, uint32_t* term,
                      int64_t* start, int64_t* end, long long cap) {
    lex3_stream_end_kernel<<<1, 32, 0, ctx->stream>>>(carry, ctx->l3.tokinfo, total, global, first, term,
                                                      reinterpret_cast<long long*>(start),
                                                      reinterpret_cast<long long*>(end), cap);
    CK(cudaGetLastError());
    return ALP_OK;
}

static int stream_ok(alp_ctx* ctx) {
    if (!ctx) return ALP_ERR_ARG;
    if (!ctx->has_lexer) return fail(ctx, ALP_ERR_MODE, "tables have no lexer");
    if (!ctx->lex3) return fail(ctx, ALP_ERR_TABLE, "token streams need a DFA of at most 32 states");
    return ALP_OK;
}

static LexCarry carry_init() {
    LexCarry c{};
    c.state = 1u;  // the DFA's initial state
    return c;
}

int alp_lex_stream_begin(alp_ctx* ctx, uint32_t* d_term, int64_t* d_start, int64_t* d_end, int64_t cap,
                         alp_lex_stream** out) {
    int rc;
    if ((rc = stream_ok(ctx))) return rc;
    if (!out || cap < 0 || (cap > 0 && (!d_term || !d_start || !d_end))) return fail(ctx, ALP_ERR_ARG, "bad argument");
    *out = nullptr;
    CK(cudaSetDevice(ctx->device));
    alp_lex_stream* s = new alp_lex_stream();
    s->ctx = ctx;
    s->term = d_term;
    s->start = d_start;
    s->end = d_end;
    s->cap = cap;
    const LexCarry c0 = carry_init();
    cudaError_t e = cudaMalloc(&s->d_carry, sizeof(LexCarry));
    if (e == cudaSuccess) e = cudaHostAlloc(&s->h_carry, sizeof(LexCarry), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->d_carry, &c0, sizeof c0, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        alp_lex_stream_free(s);
        return fail(ctx, ALP_ERR_CUDA, "stream setup: %s", cudaGetErrorString(e));
    }
    *out = s;
    return ALP_OK;
}

int alp_lex_stream_push(alp_lex_stream* s, const uint8_t* d_piece, int64_t n) {
    if (!s) return ALP_ERR_ARG;
    alp_ctx* ctx = s->ctx;
    int rc = check_in(ctx, d_piece, n, true);
    if (rc) return rc;
    if (s->ended) return fail(ctx, ALP_ERR_ARG, "stream already ended");
    if (n == 0) return ALP_OK;
    CK(cudaSetDevice(ctx->device));
    if ((rc = stream_piece(ctx, s->d_carry, d_piece, n, s->pos, 1, s->first, s->term, s->start, s->end, s->cap)))
        return rc;
    s->pos += n;
    return ALP_OK;
}

// Waits for the pushed pieces; *n_tok = tokens written so far.
static int stream_read(alp_lex_stream* s, int64_t* n_tok) {
    alp_ctx* ctx = s->ctx;
    CK(cudaMemcpyAsync(s->h_carry, s->d_carry, sizeof(LexCarry), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (s->h_carry->error & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "lexer look-back timed out");
    *n_tok = s->h_carry->tokens;
    if (s->h_carry->error & ALP_DEV_ERR_CAPACITY) return fail(ctx, ALP_ERR_CAPACITY, "token buffer too small");
    return ALP_OK;
}

int alp_lex_stream_tokens(alp_lex_stream* s, int64_t* n_tok) {
    if (!s || !n_tok) return s ? fail(s->ctx, ALP_ERR_ARG, "null output") : ALP_ERR_ARG;
    alp_ctx* ctx = s->ctx;
    CK(cudaSetDevice(ctx->device));
    return stream_read(s, n_tok);
}

int alp_lex_stream_end(alp_lex_stream* s, int64_t* n_tok, int* valid) {
    if (!s) return ALP_ERR_ARG;
    alp_ctx* ctx = s->ctx;
    if (!n_tok || !valid) return fail(ctx, ALP_ERR_ARG, "null output");
    if (s->ended) return fail(ctx, ALP_ERR_ARG, "stream already ended");
    CK(cudaSetDevice(ctx->device));
    int rc;
    if ((rc = stream_end(ctx, s->d_carry, s->pos, 1, s->first, s->term, s->start, s->end, s->cap))) return rc;
    s->ended = 1;
    rc = stream_read(s, n_tok);
    *valid = s->h_carry->valid;
    if (!rc && !*valid) *n_tok = 0;  // a rejected input has no tokens
    ctx->last_tokens = *n_tok;
    return rc;
}

int alp_lex_stream_window(alp_lex_stream* s, uint32_t* d_term, int64_t* d_start, int64_t* d_end, int64_t cap,
                          int64_t first) {
    if (!s) return ALP_ERR_ARG;
    alp_ctx* ctx = s->ctx;
    if (cap < 0 || first < 0 || (cap > 0 && (!d_term || !d_start || !d_end)))
        return fail(ctx, ALP_ERR_ARG, "bad argument");
    s->term = d_term;
    s->start = d_start;
    s->end = d_end;
    s->cap = cap;
    s->first = first;
    return ALP_OK;
}

void alp_lex_stream_free(alp_lex_stream* s) {
    if (!s) return;
    if (s->ctx) cudaSetDevice(s->ctx->device);
    if (s->d_carry) cudaFree(s->d_carry);
    if (s->h_carry) cudaFreeHost(s->h_carry);
    delete s;
}

// Host input in pieces of `piece` bytes through two slots: the copy of piece
// i+1 in, the lexing of piece i and the copy of piece i-1's tokens out run at
// once on three streams.  Host buffers should be pinned for the copies to
// overlap.
int alp_lex_host_stream(alp_ctx* ctx, const uint8_t* h_in, int64_t n, int64_t piece, uint32_t* h_term,
                        int64_t* h_start, int64_t* h_end, int64_t cap, int64_t* n_tok, int* valid) {
    int rc;
    if ((rc = stream_ok(ctx))) return rc;
    if (n < 0 || (n > 0 && !h_in)) return fail(ctx, ALP_ERR_ARG, "bad input");
    if (!n_tok || !valid || cap < 0 || (cap > 0 && (!h_term || !h_start || !h_end)))
        return fail(ctx, ALP_ERR_ARG, "bad argument");
    if (piece <= 0) piece = 16ll << 20;
    piece = (piece + 255) & ~255ll;
    if (piece > 0x40000000ll) return fail(ctx, ALP_ERR_ARG, "piece size %lld out of range", (long long)piece);
    *n_tok = 0;
    *valid = 0;
    if (n == 0) {  // the empty input: accepted iff the initial state accepts, no token
        *valid = (ctx->h_tokinfo[1] & TOK_ACCEPT) ? 1 : 0;
        return ALP_OK;
    }
    CK(cudaSetDevice(ctx->device));
    const long long P = piece < n ? piece : ((n + 255) & ~255ll);
    const long long tcap = P + 1;  // tokens of one piece: one per byte at most, plus the last token
    // positions below 2^31: spans cross as 32-bit values, widened on the host
    const bool narrow = n <= 0x7fffffffLL;
    const size_t b_in = (size_t)P + 256, b_term = ((size_t)tcap * 4 + 255) & ~(size_t)255,
                 b_pos = ((size_t)tcap * 8 + 255) & ~(size_t)255;
    const size_t b_slot = b_in + b_term + 2 * b_pos + (narrow ? 2 * b_term : 0);
    if ((rc = grow(ctx, ctx->pipe, 2 * b_slot)) || (rc = grow(ctx, ctx->carry, sizeof(LexCarry)))) return rc;
    if (!ctx->cp_in) {
        CK(cudaStreamCreateWithFlags(&ctx->cp_in, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&ctx->cp_out, cudaStreamNonBlocking));
        for (int i = 0; i < 2; ++i) {
            CK(cudaEventCreateWithFlags(&ctx->ev_in[i], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ctx->ev_done[i], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ctx->ev_out[i], cudaEventDisableTiming));
        }
        CK(cudaHostAlloc(&ctx->h_carry, 2 * sizeof(LexCarry), cudaHostAllocDefault));
    }
    // nothing from an earlier call may still use the slots
    CK(cudaStreamSynchronize(ctx->cp_out));
    CK(cudaStreamSynchronize(ctx->cp_in));
    LexCarry* d_carry = reinterpret_cast<LexCarry*>(ctx->carry.p);
    const LexCarry c0 = carry_init();
    ctx->h_carry[0] = c0;
    CK(cudaMemcpyAsync(d_carry, &ctx->h_carry[0], sizeof c0, cudaMemcpyHostToDevice, ctx->stream));
    uint8_t* slots = reinterpret_cast<uint8_t*>(ctx->pipe.p);
    auto in_of = [&](int k) { return slots + k * b_slot; };
    auto term_of = [&](int k) { return reinterpret_cast<uint32_t*>(slots + k * b_slot + b_in); };
    auto start_of = [&](int k) { return reinterpret_cast<int64_t*>(slots + k * b_slot + b_in + b_term); };
    auto end_of = [&](int k) { return reinterpret_cast<int64_t*>(slots + k * b_slot + b_in + b_term + b_pos); };
    auto s32_of = [&](int k) { return reinterpret_cast<int32_t*>(slots + k * b_slot + b_in + b_term + 2 * b_pos); };
    auto e32_of = [&](int k) {
        return reinterpret_cast<int32_t*>(slots + k * b_slot + b_in + 2 * b_term + 2 * b_pos);
    };
    ctx->last_h2d = n;
    ctx->last_d2h = 0;
    const long long np = (n + P - 1) / P;
    long long copied = 0;  // tokens handed to the host so far
    bool overflow = false;
    // piece i-1's tokens out, once its lexing is done
    auto retire = [&](long long i) -> int {
        const int k = (int)(i & 1);
        CK(cudaEventSynchronize(ctx->ev_done[k]));
        const LexCarry c = ctx->h_carry[k];
        if (c.error & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "lexer look-back timed out");
        if (c.error & ALP_DEV_ERR_CAPACITY) return fail(ctx, ALP_ERR_CAPACITY, "piece token buffer too small");
        const long long m = c.piece;
        if (copied + m > cap) overflow = true;
        if (!overflow && m > 0 && narrow) {
            // the piece's tokens out through the ring, widened before the next piece's
            ctx->copies.clear();
            for (long long o = 0; o < m; o += RING_CHUNK) {
                const size_t len = (size_t)std::min(RING_CHUNK, m - o);
                ctx->copies.push_back({s32_of(k) + o, h_start + copied + o, len, true});
                ctx->copies.push_back({e32_of(k) + o, h_end + copied + o, len, true});
                ctx->copies.push_back({term_of(k) + o, h_term + copied + o, len * 4, false});
            }
            int r2 = send_to_host(ctx, ctx->cp_out);
            if (r2) return r2;
            ctx->last_d2h += m * 12;
        } else if (!overflow && m > 0) {
            CK(cudaMemcpyAsync(h_term + copied, term_of(k), (size_t)m * 4, cudaMemcpyDeviceToHost, ctx->cp_out));
            CK(cudaMemcpyAsync(h_start + copied, start_of(k), (size_t)m * 8, cudaMemcpyDeviceToHost, ctx->cp_out));
            CK(cudaMemcpyAsync(h_end + copied, end_of(k), (size_t)m * 8, cudaMemcpyDeviceToHost, ctx->cp_out));
            ctx->last_d2h += m * 20;
        }
        CK(cudaEventRecord(ctx->ev_out[k], ctx->cp_out));
        copied += m;
        if (i == np - 1) *valid = c.valid;
        return ALP_OK;
    };
    for (long long i = 0; i < np; ++i) {
        const int k = (int)(i & 1);
        const long long off = i * P, len = (n - off < P) ? n - off : P;
        if (i >= 2) CK(cudaStreamWaitEvent(ctx->cp_in, ctx->ev_done[k], 0));  // slot k's piece i-2 is lexed
        CK(cudaMemcpyAsync(in_of(k), h_in + off, (size_t)len, cudaMemcpyHostToDevice, ctx->cp_in));
        CK(cudaEventRecord(ctx->ev_in[k], ctx->cp_in));
        CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_in[k], 0));
        if (i >= 2) CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_out[k], 0));  // piece i-2's tokens are out
        if ((rc = stream_piece(ctx, d_carry, in_of(k), len, off, 0, 0, term_of(k), start_of(k), end_of(k), tcap)))
            return rc;
        if (i == np - 1 && (rc = stream_end(ctx, d_carry, n, 0, 0, term_of(k), start_of(k), end_of(k), tcap)))
            return rc;
        if (narrow) {
            narrow_i64_kernel<<<NARROW_GRID, 256, 0, ctx->stream>>>(start_of(k), end_of(k), tcap, s32_of(k), e32_of(k),
                                                                     &d_carry->piece);
            CK(cudaGetLastError());
        }
        CK(cudaMemcpyAsync(&ctx->h_carry[k], d_carry, sizeof(LexCarry), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaEventRecord(ctx->ev_done[k], ctx->stream));
        if (i >= 1 && (rc = retire(i - 1))) return rc;
    }
    if ((rc = retire(np - 1))) return rc;
    CK(cudaStreamSynchronize(ctx->cp_out));
    *n_tok = *valid ? copied : 0;  // a rejected input has no tokens
    ctx->last_tokens = *n_tok;
    if (overflow && *valid) return fail(ctx, ALP_ERR_CAPACITY, "host token buffer too small");
    return ALP_OK;
}



// ---- shards: one document lexed by several GPUs ---------------------------------
// Each GPU holds one byte range.  begin: the range's state function (32 bytes);
// the ranks exchange functions and compose the prefix to get each range's
// entry state; count: the range's token count and last token start from that
// state; the ranks exchange those to get each range's first token index and
// carried token start; emit: the range's tokens with document positions.
struct alp_lex_shard {
    alp_ctx* ctx = nullptr;
    const uint8_t* d_in = nullptr;
    long long n = 0, pos = 0;
    int last = 0;
    int stage = 0;                 // 1 after begin, 2 after count, 3 after emit
    LexCarry* d_carry = nullptr;   // device: carry in, [2] totals
    long long* d_tot = nullptr;
    uint8_t* d_fn = nullptr;       // [blocks + 1][32]
    uint8_t* d_valid = nullptr;
    long long* h = nullptr;        // pinned staging
    Lex3Run r;
};

static int shard_prepare(alp_lex_shard* s) {
    alp_ctx* ctx = s->ctx;
    int rc;
    if ((rc = grow(ctx, ctx->tmp[T_TOKOFF], 64))) return rc;
    if ((rc = lex3_prepare(ctx, s->d_in, s->n, nullptr, 1, 0, nullptr, nullptr, nullptr, 0, s->d_valid, s->r)))
        return rc;
    s->r.sg.cont = 1;
    s->r.sg.end1 = s->last ? s->n : s->n + 1;  // only the last range ends the document
    s->r.a.carry = s->d_carry;
    s->r.a.pos_base = s->pos;
    s->r.a.carry_tokens = 1;
    s->r.a.tok_first = 0;
    return ALP_OK;
}

int alp_lex_shard_begin(alp_ctx* ctx, const uint8_t* d_in, int64_t n, int64_t pos, int is_last, uint8_t* h_fn,
                        alp_lex_shard** out) {
    int rc;
    if ((rc = stream_ok(ctx))) return rc;
    if (!out || !h_fn || pos < 0) return fail(ctx, ALP_ERR_ARG, "bad argument");
    *out = nullptr;
    if ((rc = check_in(ctx, d_in, n, true))) return rc;
    if (n < 1) return fail(ctx, ALP_ERR_ARG, "a shard holds at least one byte");
    CK(cudaSetDevice(ctx->device));
    alp_lex_shard* s = new alp_lex_shard();
    s->ctx = ctx;
    s->d_in = d_in;
    s->n = n;
    s->pos = pos;
    s->last = is_last ? 1 : 0;
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const int blocks = sms * 16;  // short sequential runs per warp; the final kernel composes the blocks
    cudaError_t e = cudaMalloc(&s->d_carry, sizeof(LexCarry) + 64);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_fn, (size_t)(blocks + 1) * 32 + 64);
    if (e == cudaSuccess) e = cudaMallocHost(&s->h, 64);
    if (e != cudaSuccess) {
        alp_lex_shard_free(s);
        return fail(ctx, ALP_ERR_CUDA, "shard set-up: %s", cudaGetErrorString(e));
    }
    s->d_tot = reinterpret_cast<long long*>(reinterpret_cast<uint8_t*>(s->d_carry) + sizeof(LexCarry));
    s->d_valid = reinterpret_cast<uint8_t*>(s->d_tot + 4);
    if ((rc = shard_prepare(s))) { alp_lex_shard_free(s); return rc; }
    if ((rc = lex3_fold(ctx, s->r))) { alp_lex_shard_free(s); return rc; }
    const int rows = ctx->E + ctx->S;
    const size_t fsm = (size_t)rows * 32;
    CK(cudaFuncSetAttribute(lex3_fn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm));
    lex3_fn_kernel<<<blocks, LF_WARPS * 32, fsm, ctx->stream>>>(s->r.a.chunk_f, s->r.chunks, ctx->l3.app8, rows,
                                                                 s->d_fn);
    CK(cudaGetLastError());
    lex3_fn_final_kernel<<<1, 1024, 0, ctx->stream>>>(s->d_fn, blocks, s->d_fn + (size_t)blocks * 32);
    CK(cudaGetLastError());
    mark(ctx, "lex3_fn_kernel+lex3_fn_final_kernel");
    CK(cudaMemcpyAsync(s->h, s->d_fn + (size_t)blocks * 32, 32, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    memcpy(h_fn, s->h, 32);
    s->stage = 1;
    *out = s;
    return ALP_OK;
}

int alp_lex_shard_count(alp_lex_shard* s, uint32_t entry_state, int64_t* n_tok, int64_t* last_start) {
    if (!s || !n_tok || !last_start) return ALP_ERR_ARG;
    alp_ctx* ctx = s->ctx;
    if (s->stage != 1) return fail(ctx, ALP_ERR_ARG, "count follows begin, once");
    if (entry_state >= (uint32_t)ctx->S) return fail(ctx, ALP_ERR_ARG, "entry state out of range");
    CK(cudaSetDevice(ctx->device));
    LexCarry c{};
    c.state = entry_state;
    memcpy(s->h, &c, sizeof c);
    CK(cudaMemcpyAsync(s->d_carry, s->h, sizeof c, cudaMemcpyHostToDevice, ctx->stream));
    int rc;
    if ((rc = lex3_front(ctx, s->r, true)) || (rc = lex3_tiles(ctx, s->r))) return rc;
    lex3_shard_totals_kernel<<<1, LX_THREADS, 0, ctx->stream>>>(s->r.a, s->d_tot);
    CK(cudaGetLastError());
    mark(ctx, "lex3_tile_reduce+lex3_tile_scan+lex3_shard_totals_kernel");
    CK(cudaMemcpyAsync(s->h, s->d_tot, 16, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(s->h + 2, &s->r.a.res->error, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if ((unsigned int)s->h[2] & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "lexer look-back timed out");
    *n_tok = s->h[0];
    *last_start = s->h[1] < 0 ? -1 : s->pos + s->h[1];
    s->stage = 2;
    return ALP_OK;
}

int alp_lex_shard_emit(alp_lex_shard* s, int64_t carried_start, uint32_t* d_term, int64_t* d_start, int64_t* d_end,
                       int64_t cap, int64_t* n_tok, int* valid) {
    if (!s || !n_tok || !valid) return ALP_ERR_ARG;
    alp_ctx* ctx = s->ctx;
    if (s->stage != 2) return fail(ctx, ALP_ERR_ARG, "emit follows count, once");
    if (cap < 0 || (cap > 0 && (!d_term || !d_start || !d_end)) || carried_start < 0)
        return fail(ctx, ALP_ERR_ARG, "bad argument");
    CK(cudaSetDevice(ctx->device));
    // the carry's state stays (the scan already used it); tokens from 0, the carried start
    LexCarry c{};
    CK(cudaMemcpyAsync(&c, s->d_carry, sizeof c, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    c.start = carried_start;
    c.tokens = 0;
    memcpy(s->h, &c, sizeof c);
    CK(cudaMemcpyAsync(s->d_carry, s->h, sizeof c, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(s->d_valid, 0, 1, ctx->stream));
    s->r.a.out_term = d_term;
    s->r.a.out_start = d_start;
    s->r.a.out_end = d_end;
    s->r.a.cap = cap;
    int rc;
    if ((rc = lex3_emit<uint32_t, int64_t>(ctx, s->r, true))) return rc;
    CK(cudaMemcpyAsync(ctx->h_res, s->r.a.res, sizeof(AlpResult), cudaMemcpyDeviceToHost, ctx->stream));
    uint8_t v = 0;
    CK(cudaMemcpyAsync(s->h, s->d_valid, 1, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    v = *reinterpret_cast<uint8_t*>(s->h);
    s->stage = 3;
    if (ctx->h_res->error & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "lexer look-back timed out");
    *n_tok = ctx->h_res->count;
    *valid = s->last ? (int)v : 1;
    if (ctx->h_res->error & ALP_DEV_ERR_CAPACITY) return fail(ctx, ALP_ERR_CAPACITY, "token buffer too small");
    return ALP_OK;
}

void alp_lex_shard_free(alp_lex_shard* s) {
    if (!s) return;
    if (s->ctx) cudaSetDevice(s->ctx->device);
    if (s->d_carry) cudaFree(s->d_carry);
    if (s->d_fn) cudaFree(s->d_fn);
    if (s->h) cudaFreeHost(s->h);
    delete s;
}

}  // extern "C"

// ---- shards of one document's parse ---------------------------------------
// Rank r holds a contiguous slice of the document's tokens.  Three small
// all-gathers join the ranks: (1) the terminals at each slice's edges, from
// which every rank has the key windows across its edges (futhark/parser.fut:
// 117-122) and the pair ids just outside it; (2) each slice's position sums
// (nodes, brackets, depth, exscan(arity - 1), terminal productions, pairs
// closed at its first position), from which every rank has the sums of the
// slices before it (futhark/parser.fut:153-166, 286-290); (3) each slice's
// staircases of node values and bracket depth values, which answer the
// previous-smaller-or-equal searches that leave a slice (futhark/parser.fut:
// 72-108, 174-184, 291-298).
struct alp_parse_shard {
    alp_ctx* ctx = nullptr;
    long long m = 0, L = 0;
    int first = 0, last = 0;
    uint32_t halo_l[PS_HALO], halo_r[PS_HALO];
    uint32_t prev_pair = NO_PAIR, next_pair = NO_PAIR;
    long long sums[10] = {};
    long long N = 0, K = 0, node_base = 0, br_base = 0, pos_base = 0;
    long long n_stair_n = 0, n_stair_b = 0;
    DevBuf xq_n, xq_b, st_n_val, st_n_idx, st_b_val, st_b_sym, st_scratch, counts, prev_n, prev_b, seg, halo;
    int expanded = 0;
};

namespace {

// The pair at position p of a window of terminals `at` (parse_pairs_kernel's
// pair_at on the host).
template <typename At>
uint32_t host_pair(const ParseHost& ph, At at, long long p) {
    const int q = ph.q, W = ph.q + ph.k;
    uint32_t pw[17];
    uint32_t x = 1;
    for (int j = 0; j < W; ++j) { pw[W - 1 - j] = x; x *= ph.T; }
    const uint32_t c = at(p);
    uint32_t key = c * pw[q];
    bool ok = c != ph.start;
    for (int jj = q - 1; jj >= 0; --jj) {
        const uint32_t t = at(p - q + jj);
        key += (ok ? t : ph.empty) * pw[jj];
        ok = ok && t != ph.start;
    }
    ok = c != ph.end;
    for (int jj = q + 1; jj < W; ++jj) {
        const uint32_t t = at(p - q + jj);
        key += (ok ? t : ph.empty) * pw[jj];
        ok = ok && t != ph.end;
    }
    return key < ph.key_index.size() ? ph.key_index[key] : NO_PAIR;
}

uint32_t host_closed(const ParseHost& ph, uint32_t prev, uint32_t cur) {
    if (prev == NO_PAIR || cur == NO_PAIR) return 0;
    const PairInfo& a = ph.pairs[prev];
    const PairInfo& b = ph.pairs[cur];
    const uint32_t la = (uint32_t)(((int32_t)a.n_br + (int32_t)a.d_depth) >> 1);
    const uint32_t lb = (uint32_t)(((int32_t)b.n_br + (int32_t)b.d_depth) >> 1);
    return std::min(la, (uint32_t)b.n_br - lb);
}

void shard_args(alp_parse_shard* s, ParseArgs& a, AlpResult* d_res) {
    alp_ctx* ctx = s->ctx;
    memset(&a, 0, sizeof a);
    a.t = ctx->pt;
    a.P = (const uint16_t*)ctx->tmp[T_TTERM].p;
    a.pstart = (const uint32_t*)ctx->tmp[T_TSTART].p;
    a.pend = (const uint32_t*)ctx->tmp[T_TEND].p;
    a.L = s->L;
    a.n_docs = 1;
    a.pid = (uint16_t*)ctx->tmp[T_PID].p;
    a.tile_sums = (PosSums*)ctx->tmp[T_TSUMS].p;
    a.res = d_res;
    a.node_off = (long long*)ctx->tmp[T_NODEOFF].p;
    a.br_off = (long long*)ctx->tmp[T_BROFF].p;
    a.doc_valid = (uint8_t*)ctx->tmp[T_DVALID].p;
    a.subst_terminals = 1;
    a.shard = 1;
    a.halo = (const uint32_t*)s->halo.p;
    a.prev_pair = s->prev_pair;
    a.next_pair = s->next_pair;
}

}  // namespace

extern "C" {

int alp_parse_shard_begin(alp_ctx* ctx, const uint32_t* d_term, const int64_t* d_start, const int64_t* d_end,
                          int64_t m, int is_first, int is_last, uint32_t* h_edge, int64_t* n_pos,
                          alp_parse_shard** out) {
    if (!ctx || !out || !h_edge || !n_pos || m < 0 || (m > 0 && (!d_term || !d_start || !d_end)))
        return fail(ctx, ALP_ERR_ARG, "alp_parse_shard_begin: bad arguments");
    if (!ctx->has_parser || !ctx->has_lexer) return fail(ctx, ALP_ERR_MODE, "these tables are not lexer+parser tables");
    if (ctx->ph.q + ctx->ph.k > PS_HALO) return fail(ctx, ALP_ERR_ARG, "lookback + lookahead above %d", PS_HALO);
    CK(cudaSetDevice(ctx->device));
    *out = nullptr;
    alp_parse_shard* s = new alp_parse_shard();
    s->ctx = ctx;
    s->m = m;
    s->first = is_first ? 1 : 0;
    s->last = is_last ? 1 : 0;
    s->L = m + s->first + s->last;
    const long long L = s->L;
    int rc;
    if (L >= 0x7fffffffLL) { delete s; return fail(ctx, ALP_ERR_ARG, "too many positions (%lld)", L); }
    if ((rc = grow(ctx, ctx->tmp[T_TTERM], (size_t)L * 2 + 16)) || (rc = grow(ctx, ctx->tmp[T_TSTART], (size_t)L * 4 + 16)) ||
        (rc = grow(ctx, ctx->tmp[T_TEND], (size_t)L * 4 + 16)) || (rc = grow(ctx, ctx->scratch, 256)) ||
        (rc = grow(ctx, ctx->tmp[T_DVALID], 16))) {
        delete s;
        return rc;
    }
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    if ((rc = set_result(ctx, d_res, 1))) { delete s; return rc; }
    if (L > 0) {
        shard_positions_kernel<<<grid_for(L), 256, 0, ctx->stream>>>(d_term, d_start, d_end, m, s->first, s->last,
                                                                    (uint16_t*)ctx->tmp[T_TTERM].p,
                                                                    (uint32_t*)ctx->tmp[T_TSTART].p,
                                                                    (uint32_t*)ctx->tmp[T_TEND].p, ctx->pt.start,
                                                                    ctx->pt.end, d_res);
        CK(cudaGetLastError());
    }
    if ((rc = read_result(ctx, d_res))) { delete s; return rc; }
    if (!ctx->h_res->valid) { delete s; return fail(ctx, ALP_ERR_ARG, "terminal id out of range"); }
    CK(cudaMemsetAsync(ctx->tmp[T_DVALID].p, 1, 1, ctx->stream));
    // the terminals of the first and last PS_HALO positions, empty where the slice is shorter
    uint16_t hh[2 * PS_HALO];
    const long long e = L < PS_HALO ? L : PS_HALO;
    for (int i = 0; i < 2 * PS_HALO; ++i) h_edge[i] = ctx->pt.empty;
    if (e > 0) {
        CK(cudaMemcpy(hh, ctx->tmp[T_TTERM].p, (size_t)e * 2, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hh + PS_HALO, (uint16_t*)ctx->tmp[T_TTERM].p + (L - e), (size_t)e * 2, cudaMemcpyDeviceToHost));
        for (long long i = 0; i < e; ++i) {
            h_edge[i] = hh[i];
            h_edge[2 * PS_HALO - e + i] = hh[PS_HALO + i];
        }
    }
    *n_pos = L;
    *out = s;
    return ALP_OK;
}

int alp_parse_shard_sums(alp_parse_shard* s, const uint32_t* halo_l, const uint32_t* halo_r, int64_t* sums) {
    if (!s || !halo_l || !halo_r || !sums) return ALP_ERR_ARG;
    alp_ctx* ctx = s->ctx;
    CK(cudaSetDevice(ctx->device));
    memcpy(s->halo_l, halo_l, sizeof s->halo_l);
    memcpy(s->halo_r, halo_r, sizeof s->halo_r);
    int rc0;
    if ((rc0 = grow(ctx, s->halo, 2 * PS_HALO * sizeof(uint32_t)))) return rc0;
    CK(cudaMemcpy(s->halo.p, s->halo_l, PS_HALO * sizeof(uint32_t), cudaMemcpyHostToDevice));
    CK(cudaMemcpy((uint32_t*)s->halo.p + PS_HALO, s->halo_r, PS_HALO * sizeof(uint32_t), cudaMemcpyHostToDevice));
    const long long L = s->L;
    // the slice's own terminals at its edges, then the pair ids just outside it
    std::vector<uint16_t> head((size_t)std::min<long long>(L, PS_HALO)), tail(head.size());
    if (!head.empty()) {
        CK(cudaMemcpy(head.data(), ctx->tmp[T_TTERM].p, head.size() * 2, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(tail.data(), (uint16_t*)ctx->tmp[T_TTERM].p + (L - (long long)tail.size()), tail.size() * 2,
                      cudaMemcpyDeviceToHost));
    }
    auto at = [&](long long p) -> uint32_t {
        if (p < 0) return p >= -PS_HALO ? s->halo_l[PS_HALO + p] : ctx->pt.empty;
        if (p >= L) return p - L < PS_HALO ? s->halo_r[p - L] : ctx->pt.empty;
        if (p < (long long)head.size()) return head[(size_t)p];
        if (p >= L - (long long)tail.size()) return tail[(size_t)(p - (L - (long long)tail.size()))];
        return ctx->pt.empty;  // not reached: windows stay within PS_HALO of an edge
    };
    s->prev_pair = s->first ? NO_PAIR : host_pair(ctx->ph, at, -1);
    s->next_pair = s->last ? NO_PAIR : host_pair(ctx->ph, at, L);
    const long long tiles = (L + PP_TILE - 1) / PP_TILE;
    int rc;
    if ((rc = grow(ctx, ctx->tmp[T_PID], (size_t)L * 2 + 64)) ||
        (rc = grow(ctx, ctx->tmp[T_TSUMS], (tiles + tiles / ST_CHUNK + 2) * sizeof(PosSums))) ||
        (rc = grow(ctx, ctx->tmp[T_NODEOFF], 16)) || (rc = grow(ctx, ctx->tmp[T_BROFF], 16)))
        return rc;
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    if ((rc = set_result(ctx, d_res, 1))) return rc;
    ParseArgs a;
    shard_args(s, a, d_res);
    long long first_pair = NO_PAIR;
    if (L > 0) {
        const size_t sm1 = pairs_smem_bytes(ctx->pt.n_pairs, ctx->pt.q + ctx->pt.k);
        const void* fn = pairs_kernel_for(ctx->pt.q, ctx->pt.k);
        CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
        int sms = 0, per1 = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per1, fn, PP_THREADS, sm1));
        const long long x = (long long)persistent_ctas(per1, ctx->tune.pairs_ctas) * sms;
        {
            void* args[] = {&a};
            CK(cudaLaunchKernel(fn, dim3((unsigned)(x < tiles ? x : tiles)), dim3(PP_THREADS), args, sm1, ctx->stream));
        }
        const long long chunks = (tiles + ST_CHUNK - 1) / ST_CHUNK;
        PosSums* csum = a.tile_sums + tiles;
        scan_tiles_reduce_kernel<<<(unsigned)chunks, ST_CHUNK, 0, ctx->stream>>>(a.tile_sums, tiles, csum, nullptr);
        CK(cudaGetLastError());
        scan_tiles_kernel<<<(unsigned)chunks, ST_CHUNK, 0, ctx->stream>>>(a.tile_sums, tiles, csum, d_res, a.node_off,
                                                                         a.br_off, 1, nullptr);
        CK(cudaGetLastError());
        uint16_t p0 = NO_PAIR;
        CK(cudaMemcpyAsync(ctx->h_stage, a.pid, 2, cudaMemcpyDeviceToHost, ctx->stream));
        if ((rc = read_result(ctx, d_res))) return rc;
        memcpy(&p0, ctx->h_stage, 2);
        first_pair = p0;
    }
    const AlpResult& r = *ctx->h_res;
    // nodes, brackets, depth, v, terminal productions, heads, last head (global) or -1, closed pairs
    // (with those at the first position), the pairs closed at the first position, first pair id
    s->sums[0] = L > 0 ? r.aux[0] : 0;
    s->sums[1] = L > 0 ? r.aux[1] : 0;
    s->sums[2] = L > 0 ? r.aux[2] : 0;
    s->sums[3] = L > 0 ? r.aux[3] : 0;
    s->sums[4] = L > 0 ? r.aux[4] : 0;
    s->sums[5] = L > 0 ? r.aux[5] : 0;
    s->sums[6] = s->first ? 0 : -1;
    s->sums[7] = L > 0 ? r.aux[7] : 0;
    s->sums[8] = s->first ? 0 : host_closed(ctx->ph, s->prev_pair, (uint32_t)first_pair);
    s->sums[9] = first_pair;
    if (s->sums[0] > 0xffffffffLL || s->sums[1] > 0xffffffffLL) return fail(ctx, ALP_ERR_ARG, "tree too large");
    memcpy(sums, s->sums, sizeof s->sums);
    return ALP_OK;
}

int alp_parse_shard_expand(alp_parse_shard* s, const int64_t* pre, int64_t pos_base, int64_t closed_next,
                           int64_t* n_node, int64_t* n_stair_nodes, int64_t* n_stair_brackets) {
    if (!s || !pre || !n_node || !n_stair_nodes || !n_stair_brackets) return ALP_ERR_ARG;
    alp_ctx* ctx = s->ctx;
    CK(cudaSetDevice(ctx->device));
    PosSums p;
    p.nodes = (uint32_t)pre[0]; p.brs = (uint32_t)pre[1]; p.depth = (int32_t)pre[2]; p.v = (int32_t)pre[3];
    p.terms = (uint32_t)pre[4]; p.heads = (uint32_t)pre[5]; p.hpos = (int32_t)pre[6]; p.cls = (uint32_t)pre[7];
    s->pos_base = pos_base;
    s->node_base = pre[0];
    s->br_base = pre[1] - 2 * pre[7] - s->sums[8];
    s->N = s->sums[0];
    s->K = s->L > 0 ? s->sums[1] - 2 * s->sums[7] + s->sums[8] - closed_next : 0;
    if (s->K < 0) return fail(ctx, ALP_ERR_ARG, "inconsistent closed-pair counts between shards");
    const long long L = s->L, N = s->N, K = s->K;
    int rc;
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    if ((rc = set_result(ctx, d_res, 1))) return rc;
    ParseArgs a;
    shard_args(s, a, d_res);
    a.pre = p;
    a.node_base = s->node_base;
    a.br_base = s->br_base;
    a.pos_base = pos_base;
    ParseOut o{};
    if ((rc = parse_buffers(ctx, &o, 1, N, K, a))) return rc;
    const size_t sm2 = expand_smem_bytes(ctx->pt.n_pairs, ctx->pt.n_pseq, ctx->pt.n_stack);
    if (L > 0) {
        const long long tiles = (L + PP_TILE - 1) / PP_TILE;
        unsigned g = 1;
        if ((rc = expand_grid(ctx, (const void*)parse_expand_kernel<0, 0, false>, sm2, tiles, &g))) return rc;
        parse_expand_kernel<0, 0, false><<<g, PP_THREADS, sm2, ctx->stream>>>(a);
        CK(cudaGetLastError());
    }
    // one document: its first node is here only when no node comes before the shard (the
    // root, parent 0; -1: the document started before), likewise its first kept bracket
    const bool root_here = s->node_base == 0;
    long long seg[4] = {root_here ? 0 : -1, N, s->br_base == 0 ? 0 : -1, K};
    if ((rc = grow(ctx, s->seg, sizeof seg)) || (rc = grow(ctx, s->xq_n, (size_t)N * 8 + 16)) ||
        (rc = grow(ctx, s->xq_b, (size_t)K * 8 + 16)) || (rc = grow(ctx, s->counts, 64)))
        return rc;
    CK(cudaMemcpyAsync(s->seg.p, seg, sizeof seg, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(s->counts.p, 0, 64, ctx->stream));
    const long long* d_seg = (const long long*)s->seg.p;
    unsigned int* cnt = (unsigned int*)s->counts.p;  // [0] node queries, [1] bracket queries
    long long* lens = (long long*)((uint8_t*)s->counts.p + 16);  // [0] node staircase, [1] bracket staircase
    uint8_t* dvalid = a.doc_valid;
    if ((rc = run_ple(ctx, a.vbuf, N, nullptr, o.parent, T_N_TMIN, d_seg, 1, dvalid, d_res, nullptr,
                      root_here ? 0 : s->node_base - 1, (unsigned long long*)s->xq_n.p, cnt, N)) ||
        (rc = run_ple(ctx, a.dsbuf, K, a.brbuf, nullptr, T_B_TMIN, d_seg + 2, 1, dvalid, d_res, nullptr, 0,
                      (unsigned long long*)s->xq_b.p, cnt + 1, K)))
        return rc;
    // the shard's staircases from its tiles'
    const PleShape& sh = ple_shapes[ctx->tune.ple];
    const int tile = sh.threads * sh.items;
    if ((rc = grow(ctx, s->st_n_val, (size_t)N * 4 + 16)) || (rc = grow(ctx, s->st_n_idx, (size_t)N * 8 + 16)) ||
        (rc = grow(ctx, s->st_b_val, (size_t)K * 4 + 16)) || (rc = grow(ctx, s->st_b_sym, (size_t)K * 4 + 16)) ||
        (rc = grow(ctx, s->st_scratch, (size_t)((std::max(N, K) + tile - 1) / tile) * 4 + 16)))
        return rc;
    if (N > 0)
        shard_stair_kernel<<<1, 1024, 0, ctx->stream>>>(
            (const int32_t*)ctx->tmp[T_N_TMIN].p, (const int32_t*)ctx->tmp[T_N_SVAL].p,
            (const uint32_t*)ctx->tmp[T_N_SIDX].p, (const int32_t*)ctx->tmp[T_N_SLEN].p, (N + tile - 1) / tile, tile,
            nullptr, s->node_base, (int32_t*)s->st_scratch.p, (int32_t*)s->st_n_val.p, (long long*)s->st_n_idx.p,
            nullptr, lens);
    if (K > 0)
        shard_stair_kernel<<<1, 1024, 0, ctx->stream>>>(
            (const int32_t*)ctx->tmp[T_B_TMIN].p, (const int32_t*)ctx->tmp[T_B_SVAL].p,
            (const uint32_t*)ctx->tmp[T_B_SIDX].p, (const int32_t*)ctx->tmp[T_B_SLEN].p, (K + tile - 1) / tile, tile,
            a.brbuf, 0, (int32_t*)s->st_scratch.p, (int32_t*)s->st_b_val.p, nullptr, (uint32_t*)s->st_b_sym.p,
            lens + 1);
    CK(cudaGetLastError());
    long long h_lens[2] = {0, 0};
    CK(cudaMemcpyAsync(ctx->h_stage, lens, 16, cudaMemcpyDeviceToHost, ctx->stream));
    if ((rc = read_result(ctx, d_res))) return rc;
    memcpy(h_lens, ctx->h_stage, 16);
    s->n_stair_n = N > 0 ? h_lens[0] : 0;
    s->n_stair_b = K > 0 ? h_lens[1] : 0;
    s->expanded = 1;
    *n_node = N;
    *n_stair_nodes = s->n_stair_n;
    *n_stair_brackets = s->n_stair_b;
    return ALP_OK;
}

int alp_parse_shard_stairs(alp_parse_shard* s, int32_t* h_nval, int64_t* h_nidx, int32_t* h_bval, uint32_t* h_bsym) {
    if (!s || !s->expanded) return ALP_ERR_ARG;
    alp_ctx* ctx = s->ctx;
    CK(cudaSetDevice(ctx->device));
    if (s->n_stair_n) {
        if (!h_nval || !h_nidx) return fail(ctx, ALP_ERR_ARG, "null staircase buffer");
        CK(cudaMemcpy(h_nval, s->st_n_val.p, (size_t)s->n_stair_n * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(h_nidx, s->st_n_idx.p, (size_t)s->n_stair_n * 8, cudaMemcpyDeviceToHost));
    }
    if (s->n_stair_b) {
        if (!h_bval || !h_bsym) return fail(ctx, ALP_ERR_ARG, "null staircase buffer");
        CK(cudaMemcpy(h_bval, s->st_b_val.p, (size_t)s->n_stair_b * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(h_bsym, s->st_b_sym.p, (size_t)s->n_stair_b * 4, cudaMemcpyDeviceToHost));
    }
    return ALP_OK;
}

int alp_parse_shard_resolve(alp_parse_shard* s, int n_prev, const int64_t* n_off, const int32_t* nval,
                            const int64_t* nidx, const int64_t* b_off, const int32_t* bval, const uint32_t* bsym,
                            int* valid) {
    if (!s || !s->expanded || !valid || n_prev < 0 || (n_prev > 0 && (!n_off || !b_off))) return ALP_ERR_ARG;
    alp_ctx* ctx = s->ctx;
    CK(cudaSetDevice(ctx->device));
    int rc;
    const long long nn = n_prev > 0 ? n_off[n_prev] : 0, nb = n_prev > 0 ? b_off[n_prev] : 0;
    const size_t offb = 8 * ((size_t)n_prev + 1);
    if ((rc = grow(ctx, s->prev_n, 2 * offb + (size_t)nn * 12 + 64)) ||
        (rc = grow(ctx, s->prev_b, (size_t)nb * 8 + 64)))
        return rc;
    uint8_t* pn = (uint8_t*)s->prev_n.p;
    long long* d_noff = (long long*)pn;
    long long* d_boff = (long long*)(pn + offb);
    long long* d_nidx = (long long*)(pn + 2 * offb);
    int32_t* d_nval = (int32_t*)(pn + 2 * offb + (size_t)nn * 8);
    int32_t* d_bval = (int32_t*)s->prev_b.p;
    uint32_t* d_bsym = (uint32_t*)((uint8_t*)s->prev_b.p + (size_t)nb * 4);
    if (n_prev > 0) {
        CK(cudaMemcpy(d_noff, n_off, offb, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_boff, b_off, offb, cudaMemcpyHostToDevice));
        if (nn) {
            CK(cudaMemcpy(d_nidx, nidx, (size_t)nn * 8, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(d_nval, nval, (size_t)nn * 4, cudaMemcpyHostToDevice));
        }
        if (nb) {
            CK(cudaMemcpy(d_bval, bval, (size_t)nb * 4, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(d_bsym, bsym, (size_t)nb * 4, cudaMemcpyHostToDevice));
        }
    }
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    unsigned int* cnt = (unsigned int*)s->counts.p;
    uint8_t* dvalid = (uint8_t*)ctx->tmp[T_DVALID].p;
    shard_resolve_kernel<<<148 * 4, 256, 0, ctx->stream>>>((const unsigned long long*)s->xq_n.p, cnt, s->N, n_prev,
                                                          d_noff, d_nval, d_nidx, nullptr, (long long*)ctx->out[3].p,
                                                          nullptr, dvalid);
    CK(cudaGetLastError());
    shard_resolve_kernel<<<148 * 4, 256, 0, ctx->stream>>>((const unsigned long long*)s->xq_b.p, cnt + 1, s->K, n_prev,
                                                          d_boff, d_bval, nullptr, d_bsym, nullptr,
                                                          (const uint32_t*)ctx->tmp[T_BRBUF].p, dvalid);
    CK(cudaGetLastError());
    if ((rc = read_result(ctx, d_res))) return rc;
    return read_valid0(ctx, dvalid, valid);
}

int alp_parse_shard_tree(alp_parse_shard* s, int64_t** d_parent, uint32_t** d_tag, uint8_t** d_kind,
                         int64_t** d_start, int64_t** d_end, int64_t* n_node, int64_t* first_node) {
    if (!s || !s->expanded || !d_parent || !d_tag || !d_kind || !d_start || !d_end || !n_node || !first_node)
        return ALP_ERR_ARG;
    alp_ctx* ctx = s->ctx;
    *d_parent = (int64_t*)ctx->out[3].p;
    *d_tag = (uint32_t*)ctx->out[4].p;
    *d_kind = (uint8_t*)ctx->out[5].p;
    *d_start = (int64_t*)ctx->out[6].p;
    *d_end = (int64_t*)ctx->out[7].p;
    *n_node = s->N;
    *first_node = s->node_base;
    return ALP_OK;
}

void alp_parse_shard_free(alp_parse_shard* s) {
    if (!s) return;
    if (s->ctx) cudaSetDevice(s->ctx->device);
    for (DevBuf* b : {&s->xq_n, &s->xq_b, &s->st_n_val, &s->st_n_idx, &s->st_b_val, &s->st_b_sym, &s->st_scratch,
                      &s->counts, &s->prev_n, &s->prev_b, &s->seg, &s->halo})
        if (b->p) cudaFree(b->p);
    delete s;
}

int alp_parse(alp_ctx* ctx, const uint8_t* d_in, int64_t n, int64_t** d_parent, uint32_t** d_tag, uint8_t** d_kind,
              int64_t** d_start, int64_t** d_end, int64_t* n_node, int* valid) {
    int rc = check_in(ctx, d_in, n, true);
    if (rc) return rc;
    if (!d_parent || !d_tag || !d_kind || !d_start || !d_end || !n_node || !valid)
        return fail(ctx, ALP_ERR_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    ParseOut o{};
    rc = parse_core(ctx, d_in, n, &o, 0, 1, n_node, valid);
    if (rc) return rc;
    *d_parent = o.parent;
    *d_tag = o.tag;
    *d_kind = o.kind;
    *d_start = o.start;
    *d_end = o.end;
    return ALP_OK;
}

int alp_parse_into(alp_ctx* ctx, const uint8_t* d_in, int64_t n, int64_t* d_parent, uint32_t* d_tag, uint8_t* d_kind,
                   int64_t* d_start, int64_t* d_end, int64_t cap, int64_t* n_node, int* valid) {
    int rc = check_in(ctx, d_in, n, true);
    if (rc) return rc;
    if (!n_node || !valid || (cap > 0 && (!d_parent || !d_tag || !d_kind || !d_start || !d_end)))
        return fail(ctx, ALP_ERR_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    ParseOut o{d_parent, d_tag, d_kind, d_start, d_end};
    return parse_core(ctx, d_in, n, &o, cap, 0, n_node, valid);
}

int alp_parse_host(alp_ctx* ctx, const uint8_t* h_in, int64_t n, int64_t* h_parent, uint32_t* h_tag, uint8_t* h_kind,
                   int64_t* h_start, int64_t* h_end, int64_t cap, int64_t* n_node, int* valid) {
    int rc = check_in(ctx, h_in, n, true);
    if (rc) return rc;
    if (!n_node || !valid || cap < 0 || (cap > 0 && (!h_parent || !h_tag || !h_kind || !h_start || !h_end)))
        return fail(ctx, ALP_ERR_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    if ((rc = grow(ctx, ctx->tmp[T_HIN], (size_t)n + 16))) return rc;
    if (n) CK(cudaMemcpyAsync(ctx->tmp[T_HIN].p, h_in, (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    ParseOut o{};
    // spans may be narrowed for the host during the searches (on cp_out); every return
    // below waits for that stream, so that no copy outlives the call
    alp_ctx::HostTree ht{h_tag, h_kind, h_start, h_end, (long long)cap, false, false};
    ctx->host_tree = cap > 0 ? &ht : nullptr;
    ctx->copies.clear();
    ctx->last_h2d = n;
    ctx->last_d2h = 0;
    rc = parse_core(ctx, (const uint8_t*)ctx->tmp[T_HIN].p, n, &o, 0, 1, n_node, valid);
    ctx->host_tree = nullptr;
    return tree_to_host(ctx, rc, o, *n_node, cap, ht, h_parent);
}

int alp_parse_tokens(alp_ctx* ctx, const uint32_t* d_term, const int64_t* d_tstart, const int64_t* d_tend, int64_t m,
                     int64_t** d_parent, uint32_t** d_tag, uint8_t** d_kind, int64_t** d_start, int64_t** d_end,
                     int64_t* n_node, int* valid) {
    if (!ctx) return ALP_ERR_ARG;
    if (m < 0 || m > (int64_t)0x3fffffffLL || (m > 0 && (!d_term || !d_tstart || !d_tend)))
        return fail(ctx, ALP_ERR_ARG, "bad token arrays");
    if (!d_parent || !d_tag || !d_kind || !d_start || !d_end || !n_node || !valid)
        return fail(ctx, ALP_ERR_ARG, "null output");
    if (!ctx->has_parser) return fail(ctx, ALP_ERR_MODE, "these tables have no parser");
    CK(cudaSetDevice(ctx->device));
    int rc = tokens_in(ctx, d_term, d_tstart, d_tend, m);
    if (rc) return rc;
    ParseOut o{};
    uint8_t* dvalid = (uint8_t*)ctx->tmp[T_DVALID].p;
    int64_t N = 0;
    rc = parse_positions(ctx, m + 2, 1, dvalid, &o, 0, 1, &N, 1);
    if (rc) return rc;
    if ((rc = read_valid0(ctx, dvalid, valid))) return rc;
    *n_node = *valid ? N : 0;
    *d_parent = o.parent;
    *d_tag = o.tag;
    *d_kind = o.kind;
    *d_start = o.start;
    *d_end = o.end;
    return ALP_OK;
}

int alp_pre_productions(alp_ctx* ctx, const uint32_t* d_term, int64_t m, uint32_t** d_prod, int64_t* n_prod,
                        int* valid) {
    if (!ctx) return ALP_ERR_ARG;
    if (m < 0 || m > (int64_t)0x3fffffffLL || (m > 0 && !d_term)) return fail(ctx, ALP_ERR_ARG, "bad token array");
    if (!d_prod || !n_prod || !valid) return fail(ctx, ALP_ERR_ARG, "null output");
    if (!ctx->has_parser) return fail(ctx, ALP_ERR_MODE, "these tables have no parser");
    CK(cudaSetDevice(ctx->device));
    int rc = tokens_in(ctx, d_term, nullptr, nullptr, m);
    if (rc) return rc;
    ParseOut o{};
    uint8_t* dvalid = (uint8_t*)ctx->tmp[T_DVALID].p;
    int64_t N = 0;
    rc = parse_positions(ctx, m + 2, 1, dvalid, &o, 0, 1, &N, 0);
    if (rc) return rc;
    if ((rc = read_valid0(ctx, dvalid, valid))) return rc;
    *n_prod = *valid ? N : 0;
    *d_prod = o.tag;
    return ALP_OK;
}


int alp_lex_states(alp_ctx* ctx, const uint8_t* d_in, int64_t n, uint8_t* d_states) {
    int rc = check_in(ctx, d_in, n);
    if (rc) return rc;
    if (!d_states && n > 0) return fail(ctx, ALP_ERR_ARG, "null state buffer");
    uint32_t* t;
    int64_t *st, *en;
    int64_t m;
    int valid;
    ctx->state_out = d_states;
    rc = alp_lex(ctx, d_in, n, &t, &st, &en, &m, &valid);
    ctx->state_out = nullptr;
    return rc;
}

int alp_mlp_train_step(alp_ctx* ctx, float* params, uint16_t* wbf, float* grads, float* adam_m, float* adam_v,
                       int n_states, const uint8_t* d_win, const uint8_t* d_lab, int batch, float lr, float wd,
                       int step, int update, float* h_loss, float* h_acc) {
    if (!ctx) return ALP_ERR_ARG;
    if (!params || !wbf || !grads || !d_win || !d_lab || batch < 16 || (batch & 15) || n_states < 1 ||
        n_states > MLP_OUT || (update && (!adam_m || !adam_v || step < 1)))
        return fail(ctx, ALP_ERR_ARG, "bad MLP training arguments");
    CK(cudaSetDevice(ctx->device));
    const long long M = batch;
    int rc;
    static_assert(M_CNT <= 16, "scratch slots");
    DevBuf* sb = ctx->mlp;
    if ((rc = grow(ctx, sb[M_X], M * MLP_IN * 2)) || (rc = grow(ctx, sb[M_Z1], M * MLP_H * 4)) ||
        (rc = grow(ctx, sb[M_H1], M * MLP_H * 4)) || (rc = grow(ctx, sb[M_H1B], M * MLP_H * 2)) ||
        (rc = grow(ctx, sb[M_Z2], M * MLP_H * 4)) || (rc = grow(ctx, sb[M_H2], M * MLP_H * 4)) ||
        (rc = grow(ctx, sb[M_H2B], M * MLP_H * 2)) || (rc = grow(ctx, sb[M_Z3], M * MLP_OUT * 4)) ||
        (rc = grow(ctx, sb[M_DZ3], M * MLP_OUT * 4)) || (rc = grow(ctx, sb[M_DZ3B], M * MLP_OUT * 2)) ||
        (rc = grow(ctx, sb[M_DH], M * MLP_H * 4)) || (rc = grow(ctx, sb[M_DZ], M * MLP_H * 4)) ||
        (rc = grow(ctx, sb[M_DZB], M * MLP_H * 2)) || (rc = grow(ctx, sb[M_DX], M * MLP_IN * 4)) ||
        (rc = grow(ctx, sb[M_SCAL], 64)) || (rc = grow(ctx, ctx->scratch, 256)))
        return rc;
    // the GEMMs' bounded MMA waits report through the result block's error word
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    CK(cudaMemsetAsync(&d_res->error, 0, sizeof(unsigned int), ctx->stream));
    __nv_bfloat16* emb_b = reinterpret_cast<__nv_bfloat16*>(wbf);
    __nv_bfloat16* w1_b = emb_b + 256 * MLP_EMB;
    __nv_bfloat16* w2_b = w1_b + MLP_IN * MLP_H;
    __nv_bfloat16* w3_b = w2_b + MLP_H * MLP_H;
    auto bf = [&](int i) { return reinterpret_cast<__nv_bfloat16*>(sb[i].p); };
    auto f32 = [&](int i) { return reinterpret_cast<float*>(sb[i].p); };
    float* scal = f32(M_SCAL);
    CK(cudaMemsetAsync(scal, 0, 64, ctx->stream));
    const unsigned g1 = grid_for(M * MLP_IN);
    // forward
    gather_embed_kernel<<<g1, 256, 0, ctx->stream>>>(d_win, batch, emb_b, bf(M_X));
    if ((rc = gemm(ctx, bf(M_X), MLP_IN, 1, w1_b, MLP_H, 1, f32(M_Z1), MLP_H, batch, MLP_H, MLP_IN))) return rc;
    bias_relu_kernel<<<grid_for(M * MLP_H), 256, 0, ctx->stream>>>(f32(M_Z1), params + P_B1, batch, MLP_H, f32(M_H1), bf(M_H1B));
    if ((rc = gemm(ctx, bf(M_H1B), MLP_H, 1, w2_b, MLP_H, 1, f32(M_Z2), MLP_H, batch, MLP_H, MLP_H))) return rc;
    bias_relu_kernel<<<grid_for(M * MLP_H), 256, 0, ctx->stream>>>(f32(M_Z2), params + P_B2, batch, MLP_H, f32(M_H2), bf(M_H2B));
    if ((rc = gemm(ctx, bf(M_H2B), MLP_H, 1, w3_b, MLP_OUT, 1, f32(M_Z3), MLP_OUT, batch, MLP_OUT, MLP_H))) return rc;
    softmax_ce_kernel<<<grid_for(M * 32), 256, 0, ctx->stream>>>(f32(M_Z3), params + P_B3, d_lab, batch, n_states,
                                                                 f32(M_DZ3), bf(M_DZ3B), scal,
                                                                 reinterpret_cast<unsigned int*>(scal + 1));
    // backward
    if ((rc = gemm(ctx, bf(M_H2B), 1, MLP_H, bf(M_DZ3B), MLP_OUT, 1, grads + P_W3, MLP_OUT, MLP_H, MLP_OUT, batch))) return rc;
    colsum_kernel<<<MLP_OUT, 256, 0, ctx->stream>>>(f32(M_DZ3), batch, MLP_OUT, grads + P_B3);
    if ((rc = gemm(ctx, bf(M_DZ3B), MLP_OUT, 1, w3_b, 1, MLP_OUT, f32(M_DH), MLP_H, batch, MLP_H, MLP_OUT))) return rc;
    relu_back_kernel<<<grid_for(M * MLP_H), 256, 0, ctx->stream>>>(f32(M_DH), f32(M_H2), M * MLP_H, bf(M_DZB), f32(M_DZ));
    if ((rc = gemm(ctx, bf(M_H1B), 1, MLP_H, bf(M_DZB), MLP_H, 1, grads + P_W2, MLP_H, MLP_H, MLP_H, batch))) return rc;
    colsum_kernel<<<MLP_H, 256, 0, ctx->stream>>>(f32(M_DZ), batch, MLP_H, grads + P_B2);
    if ((rc = gemm(ctx, bf(M_DZB), MLP_H, 1, w2_b, 1, MLP_H, f32(M_DH), MLP_H, batch, MLP_H, MLP_H))) return rc;
    relu_back_kernel<<<grid_for(M * MLP_H), 256, 0, ctx->stream>>>(f32(M_DH), f32(M_H1), M * MLP_H, bf(M_DZB), f32(M_DZ));
    if ((rc = gemm(ctx, bf(M_X), 1, MLP_IN, bf(M_DZB), MLP_H, 1, grads + P_W1, MLP_H, MLP_IN, MLP_H, batch))) return rc;
    colsum_kernel<<<MLP_H, 256, 0, ctx->stream>>>(f32(M_DZ), batch, MLP_H, grads + P_B1);
    if ((rc = gemm(ctx, bf(M_DZB), MLP_H, 1, w1_b, 1, MLP_H, f32(M_DX), MLP_IN, batch, MLP_IN, MLP_H))) return rc;
    CK(cudaMemsetAsync(grads + P_EMB, 0, 256 * MLP_EMB * 4, ctx->stream));
    scatter_embed_kernel<<<g1, 256, 0, ctx->stream>>>(d_win, batch, f32(M_DX), grads + P_EMB);
    CK(cudaGetLastError());
    if (update) {
        const float b1 = 0.9f, b2 = 0.999f;
        const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
        adamw_kernel<<<grid_for(P_TOTAL), 256, 0, ctx->stream>>>(params, grads, adam_m, adam_v, P_TOTAL, lr, b1, b2,
                                                                 1e-8f, wd, bc1, bc2, emb_b, w1_b, w2_b, w3_b);
        CK(cudaGetLastError());
    }
    if (h_loss || h_acc) {
        float hs[2];
        unsigned int err = 0;
        CK(cudaMemcpyAsync(hs, scal, 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(&err, &d_res->error, sizeof err, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (err & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "tensor-core GEMM wait timed out");
        unsigned int corr;
        memcpy(&corr, &hs[1], 4);
        if (h_loss) *h_loss = hs[0] / (float)batch;
        if (h_acc) *h_acc = (float)corr / (float)batch;
    }
    return ALP_OK;
}

// Boundary-state predictions.  d_err: a device word for the tcgen05 kernel's
// timeout bit, read later by the caller; null = a word of its own, checked here.
static int mlp_predict(alp_ctx* ctx, const uint16_t* wbf, const float* wf32, int n_states, const uint8_t* d_in,
                       int64_t n, const int64_t* d_pos, int64_t count, uint8_t* d_pred, unsigned int* d_err) {
    if (!ctx) return ALP_ERR_ARG;
    if (!wbf || !wf32 || n_states < 1 || n_states > MLP_OUT || count < 0 || (count > 0 && (!d_pos || !d_pred)))
        return fail(ctx, ALP_ERR_ARG, "bad MLP arguments");
    CK(cudaSetDevice(ctx->device));
    if (count == 0) return ALP_OK;
    MlpWeights w;
    w.emb = reinterpret_cast<const __nv_bfloat16*>(wbf);
    w.w1 = w.emb + 256 * MLP_EMB;
    w.w2 = w.w1 + MLP_IN * MLP_H;
    w.w3 = w.w2 + MLP_H * MLP_H;
    w.b1 = wf32 + P_B1;
    w.b2 = wf32 + P_B2;
    w.b3 = wf32 + P_B3;
    w.n_states = n_states;
    int rc;
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    if (ctx->tune.mlp == 1) {  // mma.sync kernel
        if ((rc = grow(ctx, ctx->mlp[15], (size_t)MLP_IN * MLP_H * 2))) return rc;
        __nv_bfloat16* w1t = reinterpret_cast<__nv_bfloat16*>(ctx->mlp[15].p);
        CK(cudaFuncSetAttribute(mlp_infer2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)I2_SMEM));
        const long long tiles = (count + I2_ROWS - 1) / I2_ROWS;
        const long long grid = tiles < 2LL * sms ? tiles : 2LL * sms;
        mark(ctx, "start");
        mlp_w1t_kernel<<<128, 256, 0, ctx->stream>>>(w.w1, w1t);
        mlp_infer2_kernel<<<(unsigned)grid, I2_WARPS * 32, I2_SMEM, ctx->stream>>>(
            w, w1t, d_in, n, reinterpret_cast<const long long*>(d_pos), count, d_pred);
        CK(cudaGetLastError());
        mark(ctx, "mlp_w1t+mlp_infer2");
        return ALP_OK;
    }
    // tcgen05 kernel: weight image in the swizzled operand layout, one CTA per SM
    if ((rc = grow(ctx, ctx->mlp[14], (size_t)WIMG_BYTES)) || (rc = grow(ctx, ctx->mlp[13], 16))) return rc;
    unsigned int* own_err = reinterpret_cast<unsigned int*>(ctx->mlp[13].p);
    if (!d_err) {
        d_err = own_err;
        CK(cudaMemsetAsync(d_err, 0, 4, ctx->stream));
    }
    CK(cudaFuncSetAttribute(mlp_infer3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)I3_SMEM));
    const long long tiles = (count + I3_ROWS - 1) / I3_ROWS;
    const long long grid = tiles < (long long)sms ? tiles : (long long)sms;
    mark(ctx, "start");
    mlp_wimg_kernel<<<148, 256, 0, ctx->stream>>>(w, reinterpret_cast<__nv_bfloat16*>(ctx->mlp[14].p));
    mlp_infer3_kernel<<<(unsigned)grid, I3_THREADS, I3_SMEM, ctx->stream>>>(
        w, reinterpret_cast<const uint8_t*>(ctx->mlp[14].p), d_in, n, reinterpret_cast<const long long*>(d_pos),
        count, d_pred, d_err);
    CK(cudaGetLastError());
    mark(ctx, "mlp_wimg+mlp_infer3");
    if (d_err == own_err) {
        CK(cudaMemcpyAsync(ctx->h_stage, d_err, 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        unsigned int e = 0;
        memcpy(&e, ctx->h_stage, 4);
        if (e & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "MLP inference wait timed out");
    }
    return ALP_OK;
}

int alp_mlp_predict(alp_ctx* ctx, const uint16_t* wbf, const float* wf32, int n_states, const uint8_t* d_in, int64_t n,
                    const int64_t* d_pos, int64_t count, uint8_t* d_pred) {
    return mlp_predict(ctx, wbf, wf32, n_states, d_in, n, d_pos, count, d_pred, nullptr);
}

// Speculative lexing on the multi-kernel lexer: predicted block states
// replace the fold and scan kernels (spec3.cuh); the tile scan and the token
// pass are lex3's.  Block size `chunk` is a multiple of 256.
static int spec3_lex(alp_ctx* ctx, const uint16_t* wbf, const float* wf32, int n_states, const uint8_t* d_in, int64_t n,
                     int64_t chunk, uint32_t** d_term, int64_t** d_start, int64_t** d_end, int64_t* n_tok, int* valid,
                     int64_t* stats) {
    const long long K = (n + chunk - 1) / chunk;
    DevBuf* sb = ctx->spec;
    int rc;
    if ((rc = grow(ctx, sb[0], K + 16)) || (rc = grow(ctx, sb[1], K + 16)) || (rc = grow(ctx, sb[4], K * 4 + 16)) ||
        (rc = grow(ctx, sb[5], K * 4 + 16)) || (rc = grow(ctx, sb[10], K * 8 + 16)) || (rc = grow(ctx, sb[11], 64)) ||
        (rc = grow(ctx, sb[12], K + 16)) || (rc = grow(ctx, ctx->tmp[T_TOKOFF], 16)) ||
        (rc = grow(ctx, ctx->tmp[T_DVALID], 16)) || (rc = put_doc_off(ctx, n)))
        return rc;
    uint8_t* dvalid = (uint8_t*)ctx->tmp[T_DVALID].p;
    int64_t cap = n / 2 + 1024;
    for (int attempt = 0; attempt < 2; ++attempt) {
        if ((rc = grow(ctx, ctx->out[0], cap * 4)) || (rc = grow(ctx, ctx->out[1], cap * 8)) ||
            (rc = grow(ctx, ctx->out[2], cap * 8)))
            return rc;
        cap = (int64_t)(ctx->out[1].bytes / 8);
        Lex3Run r;
        if ((rc = lex3_prepare(ctx, d_in, n, (const long long*)ctx->tmp[T_DOCOFF].p, 1, 0, ctx->out[0].p,
                               ctx->out[1].p, ctx->out[2].p, cap, dvalid, r)))
            return rc;
        SpecArgs sa;
        memset(&sa, 0, sizeof sa);
        sa.in = d_in;
        sa.n = n;
        sa.C = chunk;
        sa.K = K;
        sa.st = (uint8_t*)sb[0].p;
        sa.en = (uint8_t*)sb[1].p;
        uint32_t* lists[2] = {(uint32_t*)sb[4].p, (uint32_t*)sb[5].p};
        unsigned int* next_n = (unsigned int*)sb[11].p;
        // 1) predictions at every block boundary; block 0 starts in the initial state
        CK(cudaMemsetAsync(sa.st, 1, 1, ctx->stream));
        if (K > 1) {
            long long* pos = (long long*)sb[10].p;
            positions_kernel<<<grid_for(K - 1), 256, 0, ctx->stream>>>(pos, K - 1, chunk);
            if ((rc = mlp_predict(ctx, wbf, wf32, n_states, d_in, n, reinterpret_cast<const int64_t*>(pos), K - 1,
                                  sa.st + 1, &r.a.res->error)))
                return rc;
        }
        // 2) every block from its predicted state, 3) re-run blocks until every start is exact
        const size_t smem = ctx->l3_count_smem;
        CK(cudaFuncSetAttribute(spec3_run_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CK(cudaFuncSetAttribute(spec3_fixup_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        mark(ctx, "start");
        spec3_run_kernel<<<grid_for((K + 1) / 2), 256, smem, ctx->stream>>>(sa, r.a);
        CK(cudaGetLastError());
        mark(ctx, "spec3_run_kernel");
        CK(cudaMemsetAsync(next_n, 0, 4, ctx->stream));
        sa.list = nullptr;
        sa.next_list = lists[0];
        sa.next_n = next_n;
        spec_flag_kernel<<<grid_for(K), 256, 0, ctx->stream>>>(sa, (uint8_t*)sb[12].p);
        spec_fix_kernel<<<grid_for(K), 256, 0, ctx->stream>>>(sa, (const uint8_t*)sb[12].p);
        spec3_fixup_kernel<<<1, 256, smem, ctx->stream>>>(sa, r.a, lists[0], next_n, (const uint8_t*)sb[12].p, 64);
        CK(cudaGetLastError());
        mark(ctx, "spec_flag+spec_fix+spec3_fixup");
        // 4) tile counts, tile scan, token pass
        spec3_tiles_kernel<<<(unsigned)(r.tiles < 148 * 16 ? r.tiles : 148 * 16), LX_THREADS, 0, ctx->stream>>>(r.a);
        CK(cudaGetLastError());
        mark(ctx, "spec3_tiles_kernel");
        long long total = 0;
        rc = lex3_back<uint32_t, int64_t>(ctx, r, &total);
        const long long rounds = ctx->h_res->aux[0], reruns = ctx->h_res->aux[1], first = ctx->h_res->aux[2];
        if (rounds < 0) {
            // predictions too poor for the fix-up rounds: the plain lexer decides
            rc = alp_lex(ctx, d_in, n, d_term, d_start, d_end, n_tok, valid);
            if (stats) { stats[0] = K; stats[1] = first; stats[2] = reruns; stats[3] = -1; }
            return rc;
        }
        if (rc == ALP_ERR_CAPACITY) {
            cap = total + 1;
            continue;
        }
        if (rc) return rc;
        int v = 0;
        if ((rc = read_valid0(ctx, dvalid, &v))) return rc;
        *valid = v;
        *n_tok = v ? total : 0;
        if (stats) { stats[0] = K; stats[1] = first; stats[2] = reruns; stats[3] = rounds; }
        break;
    }
    *d_term = (uint32_t*)ctx->out[0].p;
    *d_start = (int64_t*)ctx->out[1].p;
    *d_end = (int64_t*)ctx->out[2].p;
    return ALP_OK;
}

int alp_lex_speculative(alp_ctx* ctx, const uint16_t* wbf, const float* wf32, int n_states, const uint8_t* d_in,
                        int64_t n, int64_t chunk, uint32_t** d_term, int64_t** d_start, int64_t** d_end,
                        int64_t* n_tok, int* valid, int64_t* stats) {
    int rc = check_in(ctx, d_in, n);
    if (rc) return rc;
    if (!d_term || !d_start || !d_end || !n_tok || !valid) return fail(ctx, ALP_ERR_ARG, "null output");
    if (chunk < 64 || (chunk & 15)) return fail(ctx, ALP_ERR_ARG, "chunk must be a multiple of 16, at least 64");
    if (!ctx->has_lexer) return fail(ctx, ALP_ERR_MODE, "these tables have no lexer");
    if (ctx->S > 255) return fail(ctx, ALP_ERR_TABLE, "too many states for byte-sized predictions");
    CK(cudaSetDevice(ctx->device));
    *n_tok = 0;
    *valid = 0;
    if (stats) for (int i = 0; i < 4; ++i) stats[i] = 0;
    if (n == 0) {
        *valid = (ctx->h_tokinfo[1] & TOK_ACCEPT) ? 1 : 0;
        return ALP_OK;
    }
    if (ctx->lex3 && chunk % 256 == 0 && n <= 0x3fffffffLL)
        return spec3_lex(ctx, wbf, wf32, n_states, d_in, n, chunk, d_term, d_start, d_end, n_tok, valid, stats);
    const long long K = (n + chunk - 1) / chunk;
    const long long nb = (K + SPEC_SCAN_BLOCK - 1) / SPEC_SCAN_BLOCK;
    DevBuf* sb = ctx->spec;
    if ((rc = grow(ctx, sb[0], K + 16)) || (rc = grow(ctx, sb[1], K + 16)) || (rc = grow(ctx, sb[2], K * 4 + 16)) ||
        (rc = grow(ctx, sb[3], K * 4 + 16)) || (rc = grow(ctx, sb[4], K * 4 + 16)) || (rc = grow(ctx, sb[5], K * 4 + 16)) ||
        (rc = grow(ctx, sb[6], K * 4 + 16)) || (rc = grow(ctx, sb[7], K * 4 + 16)) || (rc = grow(ctx, sb[8], nb * 4 + 16)) ||
        (rc = grow(ctx, sb[9], nb * 4 + 16)) || (rc = grow(ctx, sb[10], K * 8 + 16)) || (rc = grow(ctx, sb[11], 64)) ||
        (rc = grow(ctx, sb[12], K + 16)))
        return rc;
    int64_t cap = n / 2 + 1024;
    for (int attempt = 0; attempt < 2; ++attempt) {
        if ((rc = grow(ctx, ctx->out[0], cap * 4)) || (rc = grow(ctx, ctx->out[1], cap * 8)) ||
            (rc = grow(ctx, ctx->out[2], cap * 8)))
            return rc;
        cap = (int64_t)(ctx->out[1].bytes / 8);
        SpecArgs a;
        memset(&a, 0, sizeof a);
        a.in = d_in;
        a.n = n;
        a.C = chunk;
        a.K = K;
        a.t = ctx->lt;
        a.st = (uint8_t*)sb[0].p;
        a.en = (uint8_t*)sb[1].p;
        a.cnt = (uint32_t*)sb[2].p;
        a.lastp = (uint32_t*)sb[3].p;
        uint32_t* lists[2] = {(uint32_t*)sb[4].p, (uint32_t*)sb[5].p};
        uint32_t* ex_c = (uint32_t*)sb[6].p;
        uint32_t* ex_p = (uint32_t*)sb[7].p;
        unsigned int* next_n = (unsigned int*)sb[11].p;
        const size_t ssm = spec_smem_bytes(ctx->S, ctx->C + 1);
        // 1) predictions at every chunk boundary; chunk 0 starts in the initial state
        CK(cudaMemsetAsync(a.st, 1, 1, ctx->stream));
        if (K > 1) {
            long long* pos = (long long*)sb[10].p;
            positions_kernel<<<grid_for(K - 1), 256, 0, ctx->stream>>>(pos, K - 1, chunk);
            if ((rc = alp_mlp_predict(ctx, wbf, wf32, n_states, d_in, n, reinterpret_cast<const int64_t*>(pos), K - 1, a.st + 1))) return rc;
        }
        // 2) run every chunk, 3) fix and re-run until every start is exact
        mark(ctx, "start");
        spec_run_kernel<<<grid_for(K), 256, ssm, ctx->stream>>>(a);
        CK(cudaGetLastError());
        mark(ctx, "spec_run_kernel");
        long long reruns = 0, first = -1, rounds = 0;
        int cur = 0;
        while (true) {
            CK(cudaMemsetAsync(next_n, 0, 4, ctx->stream));
            a.next_list = lists[cur];
            a.next_n = next_n;
            spec_flag_kernel<<<grid_for(K), 256, 0, ctx->stream>>>(a, (uint8_t*)sb[12].p);
            spec_fix_kernel<<<grid_for(K), 256, 0, ctx->stream>>>(a, (const uint8_t*)sb[12].p);
            CK(cudaGetLastError());
            unsigned int h_next = 0;
            CK(cudaMemcpyAsync(ctx->h_stage, next_n, 4, cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            memcpy(&h_next, ctx->h_stage, 4);
            if (first < 0) first = h_next;
            if (h_next == 0) break;
            ++rounds;
            reruns += h_next;
            a.list = lists[cur];
            a.list_n = h_next;
            spec_run_kernel<<<grid_for(h_next), 256, ssm, ctx->stream>>>(a);
            CK(cudaGetLastError());
            a.list = nullptr;
            cur ^= 1;
            if (rounds > 64) break;  // predictions too poor: the plain scan decides
        }
        if (rounds > 64) {
            rc = alp_lex(ctx, d_in, n, d_term, d_start, d_end, n_tok, valid);
            if (stats) { stats[0] = K; stats[1] = first; stats[2] = reruns; stats[3] = -1; }
            return rc;
        }
        mark(ctx, "spec_verify");
        // 4) token offsets per chunk, 5) emit
        spec_scan_local<<<(unsigned)nb, SPEC_SCAN_BLOCK, 0, ctx->stream>>>(a.cnt, a.lastp, K, ex_c, ex_p, (uint32_t*)sb[8].p,
                                                                          (uint32_t*)sb[9].p);
        spec_scan_blocks<<<1, 1024, 0, ctx->stream>>>((uint32_t*)sb[8].p, (uint32_t*)sb[9].p, nb);
        spec_scan_add<<<(unsigned)((K + 255) / 256), 256, 0, ctx->stream>>>(ex_c, ex_p, K, (uint32_t*)sb[8].p,
                                                                            (uint32_t*)sb[9].p);
        CK(cudaGetLastError());
        if ((rc = grow(ctx, ctx->scratch, 256))) return rc;
        AlpResult* res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
        CK(cudaMemsetAsync(res, 0, sizeof(AlpResult), ctx->stream));
        a.cnt_excl = ex_c;
        a.pos_excl = ex_p;
        a.out_term = (uint32_t*)ctx->out[0].p;
        a.out_start = (int64_t*)ctx->out[1].p;
        a.out_end = (int64_t*)ctx->out[2].p;
        a.cap = cap;
        a.res = res;
        spec_emit_kernel<<<grid_for(K), 256, ssm, ctx->stream>>>(a);
        CK(cudaGetLastError());
        mark(ctx, "spec_emit_kernel");
        if ((rc = read_result(ctx, res)) && rc != ALP_ERR_CAPACITY) return rc;
        if (rc == ALP_ERR_CAPACITY || ctx->h_res->count > cap) {
            cap = ctx->h_res->count + 1;
            continue;
        }
        *valid = ctx->h_res->valid;
        *n_tok = *valid ? ctx->h_res->count : 0;
        if (stats) { stats[0] = K; stats[1] = first; stats[2] = reruns; stats[3] = rounds; }
        break;
    }
    *d_term = (uint32_t*)ctx->out[0].p;
    *d_start = (int64_t*)ctx->out[1].p;
    *d_end = (int64_t*)ctx->out[2].p;
    return ALP_OK;
}

int alp_lex_batch(alp_ctx* ctx, const uint8_t* d_in, const int64_t* d_off, int64_t n_docs, uint32_t** d_term,
                  int64_t** d_start, int64_t** d_end, int64_t** d_tok_off, uint8_t** d_valid, int64_t* n_tok_total) {
    if (!ctx) return ALP_ERR_ARG;
    if (n_docs < 1 || !d_off || !d_term || !d_start || !d_end || !d_tok_off || !d_valid || !n_tok_total)
        return fail(ctx, ALP_ERR_ARG, "bad batch arguments");
    if (!ctx->has_lexer) return fail(ctx, ALP_ERR_MODE, "these tables have no lexer");
    CK(cudaSetDevice(ctx->device));
    int64_t n = 0;
    CK(cudaMemcpyAsync(ctx->h_stage, d_off + n_docs, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    n = ctx->h_stage[0];
    int rc = check_in(ctx, d_in, n, true);
    if (rc) return rc;
    if ((rc = grow(ctx, ctx->out[0], (size_t)n * 4 + 16)) || (rc = grow(ctx, ctx->out[1], (size_t)n * 8 + 16)) ||
        (rc = grow(ctx, ctx->out[2], (size_t)n * 8 + 16)) || (rc = grow(ctx, ctx->tmp[T_DVALID], (size_t)n_docs + 16)))
        return rc;
    long long total = 0;
    rc = lex_seg<uint32_t, int64_t>(ctx, d_in, n, (const long long*)d_off, n_docs, 0, (uint32_t*)ctx->out[0].p,
                                    (int64_t*)ctx->out[1].p, (int64_t*)ctx->out[2].p, n + 1,
                                    (uint8_t*)ctx->tmp[T_DVALID].p, &total);
    if (rc) return rc;
    *d_term = (uint32_t*)ctx->out[0].p;
    *d_start = (int64_t*)ctx->out[1].p;
    *d_end = (int64_t*)ctx->out[2].p;
    *d_tok_off = (int64_t*)ctx->tmp[T_TOKOFF].p;
    *d_valid = (uint8_t*)ctx->tmp[T_DVALID].p;
    *n_tok_total = total;
    return ALP_OK;
}

int alp_parse_batch(alp_ctx* ctx, const uint8_t* d_in, const int64_t* d_off, int64_t n_docs, int64_t** d_parent,
                    uint32_t** d_tag, uint8_t** d_kind, int64_t** d_start, int64_t** d_end, int64_t** d_node_off,
                    uint8_t** d_valid, int64_t* n_node_total) {
    if (!ctx) return ALP_ERR_ARG;
    if (n_docs < 1 || !d_off || !d_parent || !d_tag || !d_kind || !d_start || !d_end || !d_node_off || !d_valid ||
        !n_node_total)
        return fail(ctx, ALP_ERR_ARG, "bad batch arguments");
    if (!ctx->has_lexer || !ctx->has_parser) return fail(ctx, ALP_ERR_MODE, "these tables are not lexer+parser tables");
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(ctx->h_stage, d_off + n_docs, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const int64_t n = ctx->h_stage[0];
    int rc = check_in(ctx, d_in, n, true);
    if (rc) return rc;
    ParseOut o{};
    int64_t N = 0;
    if ((rc = parse_batch_core(ctx, d_in, d_off, n_docs, n, &o, &N))) return rc;
    uint8_t* dvalid = (uint8_t*)ctx->tmp[T_DVALID].p;
    *d_parent = o.parent;
    *d_tag = o.tag;
    *d_kind = o.kind;
    *d_start = o.start;
    *d_end = o.end;
    *d_node_off = (int64_t*)ctx->tmp[T_NODEOFF].p;
    *d_valid = dvalid;
    *n_node_total = N;
    return ALP_OK;
}

int alp_parse_batch_host(alp_ctx* ctx, const uint8_t* h_in, const int64_t* h_off, int64_t n_docs, int64_t* h_parent,
                         uint32_t* h_tag, uint8_t* h_kind, int64_t* h_start, int64_t* h_end, int64_t* h_node_off,
                         uint8_t* h_valid, int64_t cap, int64_t* n_node_total) {
    if (!ctx) return ALP_ERR_ARG;
    if (n_docs < 1 || !h_off || !h_node_off || !h_valid || !n_node_total || cap < 0 ||
        (cap > 0 && (!h_parent || !h_tag || !h_kind || !h_start || !h_end)))
        return fail(ctx, ALP_ERR_ARG, "bad batch arguments");
    if (!ctx->has_lexer || !ctx->has_parser) return fail(ctx, ALP_ERR_MODE, "these tables are not lexer+parser tables");
    *n_node_total = 0;
    if (h_off[0] != 0) return fail(ctx, ALP_ERR_ARG, "offsets must start at 0");
    for (int64_t i = 0; i < n_docs; ++i)
        if (h_off[i + 1] < h_off[i]) return fail(ctx, ALP_ERR_ARG, "offsets must not decrease");
    const int64_t n = h_off[n_docs];
    int rc = check_in(ctx, h_in, n, true);
    if (rc) return rc;
    CK(cudaSetDevice(ctx->device));
    const size_t b_off = (size_t)(n_docs + 1) * 8;
    if ((rc = grow(ctx, ctx->tmp[T_HIN], (size_t)n + 16)) || (rc = grow(ctx, ctx->tmp[T_HOFF], b_off))) return rc;
    if (n) CK(cudaMemcpyAsync(ctx->tmp[T_HIN].p, h_in, (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->tmp[T_HOFF].p, h_off, b_off, cudaMemcpyHostToDevice, ctx->stream));
    ParseOut o{};
    alp_ctx::HostTree ht{h_tag, h_kind, h_start, h_end, (long long)cap, false, false};
    ctx->host_tree = cap > 0 ? &ht : nullptr;
    ctx->copies.clear();
    ctx->last_h2d = n + (long long)b_off;
    ctx->last_d2h = 0;
    int64_t N = 0;
    rc = parse_batch_core(ctx, (const uint8_t*)ctx->tmp[T_HIN].p, (const int64_t*)ctx->tmp[T_HOFF].p, n_docs, n, &o,
                          &N);
    ctx->host_tree = nullptr;
    *n_node_total = N;
    if ((rc = tree_to_host(ctx, rc, o, N, cap, ht, h_parent))) return rc;
    // the per-document node offsets and validity
    CK(cudaMemcpyAsync(h_node_off, ctx->tmp[T_NODEOFF].p, b_off, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(h_valid, ctx->tmp[T_DVALID].p, (size_t)n_docs, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->last_d2h += (long long)b_off + n_docs;
    return ALP_OK;
}

}  // extern "C"

// ---- batched parse as a CUDA graph ---------------------------------------------
// The same kernels as alp_parse_batch, sized by capacities known on the host
// (bytes, documents, nodes, brackets) and reading the actual counts from device
// memory, so that the whole sequence runs with no host round trip and can be
// captured once and replayed with one cudaGraphLaunch.

namespace {

// positions of the batch from the token pass; the result block reset for the parser
__global__ void batch_sizes_kernel(AlpResult* res, long long n_docs, long long* sizes) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    sizes[0] = res->count + 2 * n_docs;
    sizes[1] = (long long)res->error;
    res->count = 0;
    res->valid = 1;
    res->error = 0;
    for (int i = 0; i < 8; ++i) res->aux[i] = 0;
}

// counts[0] nodes, [1] brackets, [2] positions, [3] ALP_DEV_ERR_* bits
__global__ void batch_status_kernel(const AlpResult* res, const long long* sizes, long long cap_nodes,
                                    long long cap_brs, long long* counts) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned int err = res->error | (unsigned int)sizes[1];
    if (res->aux[0] > cap_nodes || res->aux[1] > cap_brs) err |= ALP_DEV_ERR_CAPACITY;
    counts[0] = res->aux[0];
    counts[1] = res->aux[1];
    counts[2] = sizes[0];
    counts[3] = (long long)err;
}

// parse_positions with the position count in device memory (dL), L_cap
// positions at most, and caller capacities for nodes and brackets.
int parse_positions_dev(alp_ctx* ctx, long long Lcap, const long long* dL, long long nd, uint8_t* dvalid,
                        const ParseOut& o, long long cap_nodes, long long cap_brs, long long* node_off) {
    const long long tiles = (Lcap + PP_TILE - 1) / PP_TILE;
    int rc;
    if ((rc = grow(ctx, ctx->tmp[T_PID], (size_t)Lcap * 2 + 64)) ||
        (rc = grow(ctx, ctx->tmp[T_TSUMS], (tiles + tiles / ST_CHUNK + 2) * sizeof(PosSums))) ||
        (rc = grow(ctx, ctx->tmp[T_BROFF], (size_t)(nd + 1) * 8)) || (rc = grow(ctx, ctx->scratch, 256)) ||
        (rc = grow(ctx, ctx->tmp[T_VBUF], (size_t)cap_nodes * 4 + 8)) ||
        (rc = grow(ctx, ctx->tmp[T_BRBUF], (size_t)cap_brs * 4 + 8)) ||
        (rc = grow(ctx, ctx->tmp[T_DSBUF], (size_t)cap_brs * 4 + 8)))
        return rc;
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    ParseArgs a;
    memset(&a, 0, sizeof a);
    a.t = ctx->pt;
    a.P = (const uint16_t*)ctx->tmp[T_TTERM].p;
    a.pstart = (const uint32_t*)ctx->tmp[T_TSTART].p;
    a.pend = (const uint32_t*)ctx->tmp[T_TEND].p;
    a.L = Lcap;
    a.dL = dL;
    a.n_docs = nd;
    a.pid = (uint16_t*)ctx->tmp[T_PID].p;
    a.tile_sums = (PosSums*)ctx->tmp[T_TSUMS].p;
    a.res = d_res;
    a.node_off = node_off;
    a.br_off = (long long*)ctx->tmp[T_BROFF].p;
    a.doc_valid = dvalid;
    a.tag = o.tag;
    a.kind = o.kind;
    a.nstart = o.start;
    a.nend = o.end;
    a.subst_terminals = 1;
    a.vbuf = (int32_t*)ctx->tmp[T_VBUF].p;
    a.brbuf = (uint32_t*)ctx->tmp[T_BRBUF].p;
    a.dsbuf = (int32_t*)ctx->tmp[T_DSBUF].p;
    a.cap_nodes = cap_nodes;
    a.cap_brs = cap_brs;
    int sms = 0, per1 = 0, per2 = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const size_t sm1 = pairs_smem_bytes(ctx->pt.n_pairs, ctx->pt.q + ctx->pt.k);
    if (expand_smem_bytes(ctx->pt.n_pairs, ctx->pt.n_pseq, ctx->pt.n_stack) > 220 * 1024)
        return fail(ctx, ALP_ERR_TABLE, "parser tables too large for shared memory");
    size_t sm2 = 0;
    if ((rc = expand_smem(ctx, (const void*)parse_expand_kernel<0, 0, false>, a, &sm2))) return rc;
    CK(cudaFuncSetAttribute(pairs_kernel_for(ctx->pt.q, ctx->pt.k), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per1, pairs_kernel_for(ctx->pt.q, ctx->pt.k), PP_THREADS, sm1));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, parse_expand_kernel<0, 0, false>, PP_THREADS, sm2));
    const long long x1 = (long long)persistent_ctas(per1, ctx->tune.pairs_ctas) * sms,
                    x2 = (long long)persistent_ctas(per2, ctx->tune.expand_ctas) * sms;
    {
        void* args[] = {&a};
        CK(cudaLaunchKernel(pairs_kernel_for(ctx->pt.q, ctx->pt.k), dim3((unsigned)(x1 < tiles ? x1 : tiles)),
                            dim3(PP_THREADS), args, sm1, ctx->stream));
    }
    {
        const long long chunks = (tiles + ST_CHUNK - 1) / ST_CHUNK;
        PosSums* csum = a.tile_sums + tiles;
        scan_tiles_reduce_kernel<<<(unsigned)chunks, ST_CHUNK, 0, ctx->stream>>>(a.tile_sums, tiles, csum, dL);
        CK(cudaGetLastError());
        scan_tiles_kernel<<<(unsigned)chunks, ST_CHUNK, 0, ctx->stream>>>(a.tile_sums, tiles, csum, d_res, a.node_off,
                                                                         a.br_off, nd, dL);
        CK(cudaGetLastError());
    }
    parse_expand_kernel<0, 0, false><<<(unsigned)(x2 < tiles ? x2 : tiles), PP_THREADS, sm2, ctx->stream>>>(a);
    CK(cudaGetLastError());
    if ((rc = run_ple(ctx, a.vbuf, cap_nodes, nullptr, o.parent, T_N_TMIN, a.node_off, nd, dvalid, d_res,
                      &d_res->aux[0])))
        return rc;
    return run_ple(ctx, a.dsbuf, cap_brs, a.brbuf, nullptr, T_B_TMIN, a.br_off, nd, dvalid, d_res, &d_res->aux[6]);
}

}  // namespace

struct alp_parse_graph {
    alp_ctx* child = nullptr;        // tables shared with the parent context, buffers of its own
    cudaStream_t stream = nullptr;   // capture stream
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t last = nullptr;     // stream of the last launch
    long long* sizes = nullptr;      // device: positions, lexer error bits
    long long* h_counts = nullptr;   // pinned
    int64_t* d_counts = nullptr;
    long long cap_nodes = 0, cap_brs = 0;
    // the captured call
    const uint8_t* d_in = nullptr;
    long long n = 0, nd = 0;
    const int64_t* d_off = nullptr;
    ParseOut o{};
    int64_t* d_node_off = nullptr;
    uint8_t* d_valid = nullptr;
};

namespace {

// the whole batched parse, enqueued on child->stream with no host wait
int graph_enqueue(alp_parse_graph* g) {
    alp_ctx* ctx = g->child;
    const long long n = g->n, nd = g->nd;
    const size_t tcap = (size_t)n + 2 * (size_t)nd + 16;
    int rc;
    if ((rc = grow(ctx, ctx->tmp[T_TTERM], tcap * 2)) || (rc = grow(ctx, ctx->tmp[T_TSTART], tcap * 4)) ||
        (rc = grow(ctx, ctx->tmp[T_TEND], tcap * 4)) || (rc = grow(ctx, ctx->tmp[T_TOKOFF], (size_t)(nd + 1) * 8)))
        return rc;
    Lex3Run r;
    if ((rc = lex3_prepare(ctx, g->d_in, n, (const long long*)g->d_off, nd, 1, ctx->tmp[T_TTERM].p,
                           ctx->tmp[T_TSTART].p, ctx->tmp[T_TEND].p, (long long)tcap, g->d_valid, r)) ||
        (rc = lex3_front(ctx, r)) || (rc = lex3_emit<uint16_t, uint32_t>(ctx, r)))
        return rc;
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    batch_sizes_kernel<<<1, 32, 0, ctx->stream>>>(d_res, nd, g->sizes);
    CK(cudaGetLastError());
    if ((rc = parse_positions_dev(ctx, n + 2 * nd, g->sizes, nd, g->d_valid, g->o, g->cap_nodes, g->cap_brs,
                                  (long long*)g->d_node_off)))
        return rc;
    batch_status_kernel<<<1, 32, 0, ctx->stream>>>(d_res, g->sizes, g->cap_nodes, g->cap_brs,
                                                   (long long*)g->d_counts);
    CK(cudaGetLastError());
    return ALP_OK;
}

alp_ctx* child_ctx(const alp_ctx* p) {
    alp_ctx* c = new alp_ctx();
    c->device = p->device;
    c->has_lexer = p->has_lexer;
    c->S = p->S; c->C = p->C; c->E = p->E;
    c->ignore_term = p->ignore_term; c->dead_term = p->dead_term; c->n_terms = p->n_terms;
    c->h_tokinfo = p->h_tokinfo;
    c->lt = p->lt;
    c->lex_smem = p->lex_smem;
    c->lex3 = p->lex3;
    c->l3 = p->l3;
    c->l3_fold_smem = p->l3_fold_smem; c->l3_scan_smem = p->l3_scan_smem;
    c->l3_count_smem = p->l3_count_smem; c->l3_emit_smem = p->l3_emit_smem;
    c->has_parser = p->has_parser;
    c->pt = p->pt;
    c->ph = p->ph;
    c->tune = p->tune;
    return c;
}

void graph_free(alp_parse_graph* g) {
    if (!g) return;
    if (g->child) cudaSetDevice(g->child->device);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->sizes) cudaFree(g->sizes);
    if (g->h_counts) cudaFreeHost(g->h_counts);
    if (g->child) {
        g->child->stream = nullptr;
        alp_ctx_destroy(g->child);  // its own buffers only: the tables belong to the parent
    }
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
}

}  // namespace

extern "C" {

int alp_parse_graph_create(alp_ctx* ctx, const uint8_t* d_in, int64_t n, const int64_t* d_off, int64_t n_docs,
                           int64_t cap_nodes, int64_t cap_brackets, int64_t* d_parent, uint32_t* d_tag,
                           uint8_t* d_kind, int64_t* d_start, int64_t* d_end, int64_t* d_node_off, uint8_t* d_valid,
                           int64_t* d_counts, alp_parse_graph** out) {
    if (!ctx || !out) return ALP_ERR_ARG;
    *out = nullptr;
    if (!ctx->has_lexer || !ctx->has_parser) return fail(ctx, ALP_ERR_MODE, "these tables are not lexer+parser tables");
    if (!ctx->lex3) return fail(ctx, ALP_ERR_TABLE, "graphs need a DFA of at most 32 states");
    if (n < 1 || n > 0x7ff00000LL || n_docs < 1 || n + 2 * n_docs >= 0x7fffffffLL || cap_nodes < 0 ||
        cap_brackets < 0 || cap_nodes > 0xffffffffLL || cap_brackets > 0xffffffffLL)
        return fail(ctx, ALP_ERR_ARG, "graph sizes out of range");
    if (!d_in || !d_off || !d_parent || !d_tag || !d_kind || !d_start || !d_end || !d_node_off || !d_valid ||
        !d_counts)
        return fail(ctx, ALP_ERR_ARG, "null buffer");
    CK(cudaSetDevice(ctx->device));
    alp_parse_graph* g = new alp_parse_graph();
    g->child = child_ctx(ctx);
    g->d_in = d_in; g->n = n; g->d_off = d_off; g->nd = n_docs;
    g->o.parent = d_parent; g->o.tag = d_tag; g->o.kind = d_kind; g->o.start = d_start; g->o.end = d_end;
    g->d_node_off = d_node_off; g->d_valid = d_valid; g->d_counts = d_counts;
    g->cap_nodes = cap_nodes; g->cap_brs = cap_brackets;
    auto bad = [&](int rc, const char* what) {
        const std::string m = g->child->err.empty() ? std::string(what) : g->child->err;
        graph_free(g);
        return fail(ctx, rc, "%s", m.c_str());
    };
    if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&g->sizes, 64) != cudaSuccess || cudaMallocHost(&g->h_counts, 64) != cudaSuccess ||
        cudaMallocHost(&g->child->h_res, sizeof(AlpResult)) != cudaSuccess ||
        cudaMallocHost(&g->child->h_stage, 256) != cudaSuccess)
        return bad(ALP_ERR_CUDA, "graph set-up failed");
    g->child->stream = g->stream;
    // one plain run sizes every buffer and sets every kernel attribute, so
    // that the captured run allocates nothing
    int rc = graph_enqueue(g);
    if (rc) return bad(rc, "graph warm-up failed");
    if (cudaStreamSynchronize(g->stream) != cudaSuccess) return bad(ALP_ERR_CUDA, "graph warm-up failed");
    if (cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess)
        return bad(ALP_ERR_CUDA, "stream capture failed to start");
    rc = graph_enqueue(g);
    const cudaError_t ec = cudaStreamEndCapture(g->stream, &g->graph);
    if (rc) return bad(rc, "graph capture failed");
    if (ec != cudaSuccess) return bad(ALP_ERR_CUDA, cudaGetErrorString(ec));
    if (cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess) return bad(ALP_ERR_CUDA, "graph instantiation failed");
    g->last = g->stream;
    *out = g;
    return ALP_OK;
}

int alp_parse_graph_launch(alp_parse_graph* g, void* stream) {
    if (!g) return ALP_ERR_ARG;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);  // NULL: the legacy default stream
    alp_ctx* ctx = g->child;
    CK(cudaSetDevice(ctx->device));
    CK(cudaGraphLaunch(g->exec, s));
    g->last = s;
    return ALP_OK;
}

int alp_parse_graph_result(alp_parse_graph* g, int64_t* n_nodes) {
    if (!g || !n_nodes) return ALP_ERR_ARG;
    alp_ctx* ctx = g->child;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMemcpyAsync(g->h_counts, g->d_counts, 32, cudaMemcpyDeviceToHost, g->last));
    CK(cudaStreamSynchronize(g->last));
    *n_nodes = g->h_counts[0];
    const unsigned int err = (unsigned int)g->h_counts[3];
    if (err & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "kernel wait timed out");
    if (err & ALP_DEV_ERR_CAPACITY) return fail(ctx, ALP_ERR_CAPACITY, "node or bracket capacity too small");
    return ALP_OK;
}

const char* alp_parse_graph_error(const alp_parse_graph* g) { return g ? g->child->err.c_str() : "null graph"; }

void alp_parse_graph_destroy(alp_parse_graph* g) { graph_free(g); }

}  // extern "C"
