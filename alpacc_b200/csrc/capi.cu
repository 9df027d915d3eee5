// C ABI of alpacc_b200 (include/alpacc_b200.h): context, table upload, and
// the host side of every entry point.  Kernels live in the .cuh files.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/alpacc_b200.h"
#include "common.cuh"
#include "lexer.cuh"
#include "parser.cuh"

using namespace alp;

namespace {

constexpr uint32_t BLOB_MAGIC = 0x42504C41u;
constexpr int LEX_ITEMS = 16;
constexpr int LEX_TILE = LEX_THREADS * LEX_ITEMS;

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

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
    // ---- parser tables ----
    bool has_parser = false;
    ParseTables pt{};
    ParseHost ph{};
    // ---- memory ----
    std::vector<void*> owned;             // table allocations
    DevBuf scratch;                       // look-back status words, results
    DevBuf out[8];                        // context-owned outputs
    DevBuf tmp[24];                       // intermediates
    AlpResult* h_res = nullptr;           // pinned
    // optional per-kernel timing (alp_ctx_profile)
    int prof = 0;
    std::vector<std::pair<const char*, cudaEvent_t>> marks;
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

int grow(alp_ctx* ctx, DevBuf& b, size_t bytes) {
    if (b.bytes >= bytes && b.p) return ALP_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    size_t want = bytes < 256 ? 256 : bytes;
    CK(cudaMalloc(&b.p, want));
    b.bytes = want;
    return ALP_OK;
}

template <typename T>
int upload(alp_ctx* ctx, const T* h, size_t count, const T** d) {
    void* p = nullptr;
    size_t bytes = count * sizeof(T);
    CK(cudaMalloc(&p, bytes < 16 ? 16 : bytes));
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
    auto k = lex_kernel<ITEMS, TermT, PosT>;
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->lex_smem));
    mark(ctx, "start");
    k<<<(unsigned)tiles, LEX_THREADS, ctx->lex_smem, ctx->stream>>>(a);
    CK(cudaGetLastError());
    mark(ctx, "lex_kernel");
    CK(cudaMemcpyAsync(ctx->h_res, a.res, sizeof(AlpResult), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->h_res->error & ALP_DEV_ERR_TIMEOUT) return fail(ctx, ALP_ERR_TIMEOUT, "lexer look-back timed out");
    return ALP_OK;
}

int check_in(alp_ctx* ctx, const void* p, int64_t n) {
    if (!ctx) return ALP_ERR_ARG;
    if (n < 0 || n > (int64_t)0x3fffffffLL) return fail(ctx, ALP_ERR_ARG, "input size %lld out of range", (long long)n);
    if (n > 0 && !p) return fail(ctx, ALP_ERR_ARG, "null input");
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
    int rc = launch_lex<LEX_ITEMS, TermT, PosT>(ctx, d_in, n, term, start, end, cap);
    if (rc) return rc;
    *valid = ctx->h_res->valid;
    *count = ctx->h_res->count;
    if (ctx->h_res->error & ALP_DEV_ERR_CAPACITY) return fail(ctx, ALP_ERR_CAPACITY, "token buffer too small");
    if (!*valid) *count = 0;
    return ALP_OK;
}


// Buffers of one parse (indices into ctx->tmp).
enum {
    T_HIN = 0, T_TTERM, T_TSTART, T_TEND, T_PID, T_TSUMS, T_VBUF, T_BRBUF, T_DSBUF,
    T_N_TMIN, T_N_M32, T_N_M1024, T_N_SVAL, T_N_SIDX, T_N_SLEN, T_N_ESC,
    T_B_TMIN, T_B_M32, T_B_M1024, T_B_SVAL, T_B_SIDX, T_B_SLEN, T_B_ESC, T_CNT
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
int run_ple(alp_ctx* ctx, const int32_t* val, long long n, const uint32_t* sym, int64_t* parent, int first,
            AlpResult* d_res) {
    if (n == 0) return ALP_OK;
    const long long tiles = (n + PLE_TILE - 1) / PLE_TILE;
    const long long n32 = (tiles + 31) / 32, n1024 = (tiles + 1023) / 1024;
    int rc;
    if ((rc = grow(ctx, ctx->tmp[first + 0], tiles * 4)) || (rc = grow(ctx, ctx->tmp[first + 1], n32 * 4)) ||
        (rc = grow(ctx, ctx->tmp[first + 2], n1024 * 4)) ||
        (rc = grow(ctx, ctx->tmp[first + 3], (size_t)tiles * PLE_TILE * 4)) ||
        (rc = grow(ctx, ctx->tmp[first + 4], (size_t)tiles * PLE_TILE * 4)) ||
        (rc = grow(ctx, ctx->tmp[first + 5], tiles * 4)) ||
        (rc = grow(ctx, ctx->tmp[first + 6], (size_t)n * 8 + 64)))
        return rc;
    unsigned int* esc_count = reinterpret_cast<unsigned int*>(reinterpret_cast<uint8_t*>(ctx->tmp[first + 6].p) +
                                                              (size_t)n * 8);
    CK(cudaMemsetAsync(esc_count, 0, 16, ctx->stream));
    PleArgs a;
    a.val = val;
    a.n = n;
    a.sym = sym;
    a.out_parent = reinterpret_cast<long long*>(parent);
    a.tile_min = (int32_t*)ctx->tmp[first + 0].p;
    a.stair_val = (int32_t*)ctx->tmp[first + 3].p;
    a.stair_idx = (uint32_t*)ctx->tmp[first + 4].p;
    a.stair_len = (int32_t*)ctx->tmp[first + 5].p;
    a.esc = (unsigned long long*)ctx->tmp[first + 6].p;
    a.esc_count = esc_count;
    a.esc_cap = n;
    a.res = d_res;
    CK(cudaFuncSetAttribute(ple_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PLE_SMEM));
    mark(ctx, "start");
    ple_tile_kernel<<<(unsigned)tiles, PLE_THREADS, PLE_SMEM, ctx->stream>>>(a);
    CK(cudaGetLastError());
    mark(ctx, sym ? "ple_tile_kernel(brackets)" : "ple_tile_kernel(nodes)");
    tile_min_levels_kernel<<<(unsigned)((n32 + 255) / 256), 256, 0, ctx->stream>>>(
        a.tile_min, tiles, (int32_t*)ctx->tmp[first + 1].p, (int32_t*)ctx->tmp[first + 2].p);
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
    e.res = d_res;
    ple_escape_kernel<<<148 * 4, 256, 0, ctx->stream>>>(e);
    CK(cudaGetLastError());
    mark(ctx, sym ? "tile_min+ple_escape(brackets)" : "tile_min+ple_escape(nodes)");
    return ALP_OK;
}

// Tokens already in tmp[T_TTERM..T_TEND] (m of them) -> tree.  `want_tree`
// 0 gives the production sequence only (tags, subst off, no parents).
int parse_tokens_core(alp_ctx* ctx, long long m, ParseOut* o, int64_t cap, int ctx_out, int64_t* n_node,
                      int* valid, int want_tree) {
    *n_node = 0;
    *valid = 0;
    const long long L = m + 2;
    const long long tiles = (L + PP_TILE - 1) / PP_TILE;
    int rc;
    if ((rc = grow(ctx, ctx->tmp[T_PID], (size_t)L * 2 + 64)) || (rc = grow(ctx, ctx->tmp[T_TSUMS], tiles * sizeof(PosSums))))
        return rc;
    if ((rc = grow(ctx, ctx->scratch, 256))) return rc;
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    if ((rc = set_result(ctx, d_res, 1))) return rc;
    ParseArgs a;
    memset(&a, 0, sizeof a);
    a.t = ctx->pt;
    a.tterm = (const uint16_t*)ctx->tmp[T_TTERM].p;
    a.tstart = (const uint32_t*)ctx->tmp[T_TSTART].p;
    a.tend = (const uint32_t*)ctx->tmp[T_TEND].p;
    a.m = m;
    a.L = L;
    a.pid = (uint16_t*)ctx->tmp[T_PID].p;
    a.tile_sums = (PosSums*)ctx->tmp[T_TSUMS].p;
    a.res = d_res;
    const size_t sm1 = sizeof(PairInfo) * ctx->pt.n_pairs + (size_t)(PP_TILE + ctx->pt.q + ctx->pt.k) * 4;
    CK(cudaFuncSetAttribute(parse_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
    mark(ctx, "start");
    parse_pairs_kernel<<<(unsigned)tiles, PP_THREADS, sm1, ctx->stream>>>(a);
    CK(cudaGetLastError());
    mark(ctx, "parse_pairs_kernel");
    scan_tiles_kernel<<<1, 1024, 0, ctx->stream>>>(a.tile_sums, tiles, d_res);
    CK(cudaGetLastError());
    mark(ctx, "scan_tiles_kernel");
    if ((rc = read_result(ctx, d_res))) return rc;
    const long long N = ctx->h_res->aux[0], B = ctx->h_res->aux[1], D = ctx->h_res->aux[2], NT = ctx->h_res->aux[4];
    if (!ctx->h_res->valid || D != 0) return ALP_OK;  // rejected
    if (N > 0xffffffffLL || B > 0xffffffffLL) return fail(ctx, ALP_ERR_ARG, "tree too large");
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
    } else if (N > cap) {
        *n_node = N;
        return fail(ctx, ALP_ERR_CAPACITY, "node buffer too small (%lld needed)", (long long)N);
    }
    if ((rc = grow(ctx, ctx->tmp[T_VBUF], N * 4 + 8)) || (rc = grow(ctx, ctx->tmp[T_BRBUF], B * 4 + 8)) ||
        (rc = grow(ctx, ctx->tmp[T_DSBUF], B * 4 + 8)))
        return rc;
    a.subst_terminals = (want_tree && NT == m) ? 1 : 0;
    a.tag = o->tag;
    a.kind = want_tree ? o->kind : (uint8_t*)ctx->tmp[T_VBUF].p;  // kind unused for productions only
    a.nstart = o->start;
    a.nend = o->end;
    a.vbuf = (int32_t*)ctx->tmp[T_VBUF].p;
    a.brbuf = (uint32_t*)ctx->tmp[T_BRBUF].p;
    a.dsbuf = (int32_t*)ctx->tmp[T_DSBUF].p;
    a.cap_nodes = N;
    a.cap_brs = B;
    const size_t sm2 = sizeof(PairInfo) * ctx->pt.n_pairs + (size_t)ctx->pt.n_prods * 8;
    CK(cudaFuncSetAttribute(parse_expand_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
    mark(ctx, "start");
    parse_expand_kernel<<<(unsigned)tiles, PP_THREADS, sm2, ctx->stream>>>(a);
    CK(cudaGetLastError());
    mark(ctx, "parse_expand_kernel");
    if (want_tree) {
        if ((rc = run_ple(ctx, a.vbuf, N, nullptr, o->parent, T_N_TMIN, d_res))) return rc;
    }
    if ((rc = run_ple(ctx, a.dsbuf, B, a.brbuf, nullptr, T_B_TMIN, d_res))) return rc;
    if ((rc = read_result(ctx, d_res))) return rc;
    if (!ctx->h_res->valid) return ALP_OK;
    *valid = 1;
    *n_node = N;
    return ALP_OK;
}

int parse_core(alp_ctx* ctx, const uint8_t* d_in, int64_t n, ParseOut* o, int64_t cap, int ctx_out,
               int64_t* n_node, int* valid) {
    *n_node = 0;
    *valid = 0;
    if (!ctx->has_lexer || !ctx->has_parser) return fail(ctx, ALP_ERR_MODE, "these tables are not lexer+parser tables");
    int rc;
    if ((rc = grow(ctx, ctx->tmp[T_TTERM], (size_t)n * 2 + 16)) || (rc = grow(ctx, ctx->tmp[T_TSTART], (size_t)n * 4 + 16)) ||
        (rc = grow(ctx, ctx->tmp[T_TEND], (size_t)n * 4 + 16)))
        return rc;
    int64_t m = 0;
    int lv = 0;
    rc = lex_core<uint16_t, uint32_t>(ctx, d_in, n, (uint16_t*)ctx->tmp[T_TTERM].p, (uint32_t*)ctx->tmp[T_TSTART].p,
                                      (uint32_t*)ctx->tmp[T_TEND].p, n + 1, &m, &lv);
    if (rc) return rc;
    if (!lv) return ALP_OK;
    return parse_tokens_core(ctx, m, o, cap, ctx_out, n_node, valid, 1);
}

// Token arrays from the caller (uint32 ids, int64 spans) -> internal form.
__global__ void tokens_in_kernel(const uint32_t* term, const int64_t* ts, const int64_t* te, long long m, uint16_t* t16,
                                 uint32_t* s32, uint32_t* e32, AlpResult* res) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t t = term[i];
        if (t > 0xffffu) res->valid = 0;
        t16[i] = (uint16_t)t;
        s32[i] = ts ? (uint32_t)ts[i] : 0u;
        e32[i] = te ? (uint32_t)te[i] : 0u;
    }
}

int tokens_in(alp_ctx* ctx, const uint32_t* term, const int64_t* ts, const int64_t* te, int64_t m) {
    int rc;
    if ((rc = grow(ctx, ctx->tmp[T_TTERM], (size_t)m * 2 + 16)) || (rc = grow(ctx, ctx->tmp[T_TSTART], (size_t)m * 4 + 16)) ||
        (rc = grow(ctx, ctx->tmp[T_TEND], (size_t)m * 4 + 16)) || (rc = grow(ctx, ctx->scratch, 256)))
        return rc;
    if (m == 0) return ALP_OK;
    AlpResult* d_res = reinterpret_cast<AlpResult*>(ctx->scratch.p);
    if ((rc = set_result(ctx, d_res, 1))) return rc;
    tokens_in_kernel<<<148 * 4, 256, 0, ctx->stream>>>(term, ts, te, m, (uint16_t*)ctx->tmp[T_TTERM].p,
                                                      (uint32_t*)ctx->tmp[T_TSTART].p, (uint32_t*)ctx->tmp[T_TEND].p, d_res);
    CK(cudaGetLastError());
    if ((rc = read_result(ctx, d_res))) return rc;
    if (!ctx->h_res->valid) return fail(ctx, ALP_ERR_ARG, "terminal id out of range");
    return ALP_OK;
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
    if (!rc && cudaMallocHost(&ctx->h_res, sizeof(AlpResult)) != cudaSuccess)
        rc = fail(ctx, ALP_ERR_CUDA, "cudaMallocHost failed");
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
    if (ctx->h_res) cudaFreeHost(ctx->h_res);
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
    int64_t v[8] = {ctx->has_lexer, ctx->has_parser, ctx->has_parser ? ctx->ph.n_terms : ctx->n_terms,
                    ctx->ph.n_prods, ctx->ph.q, ctx->ph.k, ctx->ph.max_prods, ctx->ph.max_brackets};
    for (int i = 0; i < n_out && i < 8; ++i) out[i] = v[i];
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
    int rc = check_in(ctx, d_in, n);
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
// owns every byte of the device through its own pool, code on a latency-bound
// path where cudaMalloc/cudaFree would synchronise the device, or a host
// callback that must not enter the allocator.  alp_lex_noalloc serves them:
// the look-back status words and the result block live in the fixed array
// below, compiled into the library, instead of in context scratch that grows
// with cudaMalloc.  The caller still passes the input and the output buffers.
// ---------------------------------------------------------------------------
namespace {

constexpr long long NOALLOC_MAX_BYTES = 128ll << 20;                    // largest input
constexpr long long NOALLOC_MAX_TILES = NOALLOC_MAX_BYTES / LEX_TILE;  // 32768 tiles
constexpr size_t NOALLOC_SCRATCH_BYTES = 256 + 12 * (size_t)NOALLOC_MAX_TILES;  // 393,472 bytes

// Every GPU that loads this library holds one copy until the process exits.
// Host code must not pass `g_noalloc_scratch` itself to a kernel: on the host
// the name is only a stand-in, so its device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::once_flag g_noalloc_once[NOALLOC_MAX_DEVICES];
void* g_noalloc_ptr[NOALLOC_MAX_DEVICES];
cudaError_t g_noalloc_err[NOALLOC_MAX_DEVICES];

// Device address of the fixed scratch on `device` (which must be current),
// looked up once per device.
void* noalloc_scratch(int device, cudaError_t* err) {
    std::call_once(g_noalloc_once[device], [device] {
        void* p = nullptr;
        g_noalloc_err[device] = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        g_noalloc_ptr[device] = g_noalloc_err[device] == cudaSuccess ? p : nullptr;
    });
    *err = g_noalloc_err[device];
    return g_noalloc_ptr[device];
}

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
    if (ctx->device < 0 || ctx->device >= NOALLOC_MAX_DEVICES) return fail(ctx, ALP_ERR_ARG, "device id too large");
    *n_tok = 0;
    *valid = 0;
    CK(cudaSetDevice(ctx->device));
    if (n == 0) {
        *valid = (ctx->h_tokinfo[1] & TOK_ACCEPT) ? 1 : 0;
        return ALP_OK;
    }
    cudaError_t se;
    uint8_t* base = reinterpret_cast<uint8_t*>(noalloc_scratch(ctx->device, &se));
    if (!base) return fail(ctx, ALP_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(se));
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
    auto k = lex_kernel<LEX_ITEMS, uint32_t, int64_t>;
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ctx->lex_smem));
    k<<<(unsigned)tiles, LEX_THREADS, ctx->lex_smem, ctx->stream>>>(a);
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
    int rc = check_in(ctx, d_in, n);
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
    int rc = check_in(ctx, h_in, n);
    if (rc) return rc;
    if (!n_tok || !valid) return fail(ctx, ALP_ERR_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    if ((rc = grow(ctx, ctx->tmp[0], (size_t)n + 16))) return rc;
    if (n) CK(cudaMemcpyAsync(ctx->tmp[0].p, h_in, (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    uint32_t* dt;
    int64_t *ds, *de;
    rc = alp_lex(ctx, (const uint8_t*)ctx->tmp[0].p, n, &dt, &ds, &de, n_tok, valid);
    if (rc) return rc;
    if (*n_tok > cap) return fail(ctx, ALP_ERR_CAPACITY, "host token buffer too small");
    if (*n_tok) {
        CK(cudaMemcpyAsync(h_term, dt, (size_t)*n_tok * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(h_start, ds, (size_t)*n_tok * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(h_end, de, (size_t)*n_tok * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return ALP_OK;
}



int alp_parse(alp_ctx* ctx, const uint8_t* d_in, int64_t n, int64_t** d_parent, uint32_t** d_tag, uint8_t** d_kind,
              int64_t** d_start, int64_t** d_end, int64_t* n_node, int* valid) {
    int rc = check_in(ctx, d_in, n);
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
    int rc = check_in(ctx, d_in, n);
    if (rc) return rc;
    if (!n_node || !valid || (cap > 0 && (!d_parent || !d_tag || !d_kind || !d_start || !d_end)))
        return fail(ctx, ALP_ERR_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    ParseOut o{d_parent, d_tag, d_kind, d_start, d_end};
    return parse_core(ctx, d_in, n, &o, cap, 0, n_node, valid);
}

int alp_parse_host(alp_ctx* ctx, const uint8_t* h_in, int64_t n, int64_t* h_parent, uint32_t* h_tag, uint8_t* h_kind,
                   int64_t* h_start, int64_t* h_end, int64_t cap, int64_t* n_node, int* valid) {
    int rc = check_in(ctx, h_in, n);
    if (rc) return rc;
    if (!n_node || !valid) return fail(ctx, ALP_ERR_ARG, "null output");
    CK(cudaSetDevice(ctx->device));
    if ((rc = grow(ctx, ctx->tmp[T_HIN], (size_t)n + 16))) return rc;
    if (n) CK(cudaMemcpyAsync(ctx->tmp[T_HIN].p, h_in, (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    ParseOut o{};
    rc = parse_core(ctx, (const uint8_t*)ctx->tmp[T_HIN].p, n, &o, 0, 1, n_node, valid);
    if (rc) return rc;
    if (*n_node > cap) return fail(ctx, ALP_ERR_CAPACITY, "host node buffer too small");
    const size_t N = (size_t)*n_node;
    if (N) {
        CK(cudaMemcpyAsync(h_parent, o.parent, N * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(h_tag, o.tag, N * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(h_kind, o.kind, N, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(h_start, o.start, N * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaMemcpyAsync(h_end, o.end, N * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return ALP_OK;
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
    rc = parse_tokens_core(ctx, m, &o, 0, 1, n_node, valid, 1);
    if (rc) return rc;
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
    rc = parse_tokens_core(ctx, m, &o, 0, 1, n_prod, valid, 0);
    if (rc) return rc;
    *d_prod = o.tag;
    return ALP_OK;
}

// Entry points whose kernels are not in this build yet report ALP_ERR_MODE.
int alp_lex_batch(alp_ctx* ctx, const uint8_t*, const int64_t*, int64_t, uint32_t**, int64_t**, int64_t**,
                  int64_t**, uint8_t**, int64_t*) {
    return fail(ctx, ALP_ERR_MODE, "alp_lex_batch: not available in this build");
}
int alp_parse_batch(alp_ctx* ctx, const uint8_t*, const int64_t*, int64_t, int64_t**, uint32_t**, uint8_t**,
                    int64_t**, int64_t**, int64_t**, uint8_t**, int64_t*) {
    return fail(ctx, ALP_ERR_MODE, "alp_parse_batch: not available in this build");
}

}  // extern "C"
