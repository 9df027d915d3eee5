// LLP parser kernels (sm_100a) and the parser tables.
//
// Restates futhark/parser.fut:110-332 for one document:
//   K1 parse_pairs   -- keys over ⊢ tokens ⊣ (get_key, lines 117-122), the pair
//                       lookup (lines 130-148) and one decoupled look-back scan
//                       of every per-position count the later passes need;
//   K2 parse_expand  -- the segmented copies of stacks and productions
//                       (lines 216-233), node tags, terminal-node spans
//                       (lines 305-329), the value sequences of the two
//                       "previous smaller-or-equal" searches: bracket depths
//                       (lines 153-166) and exscan(arity-1) (lines 286-291);
//   K3 ple_tile      -- previous smaller-or-equal inside a tile with a
//                       shared-memory min tree (the template builds one
//                       min tree over the whole array, lines 72-108);
//   K4 ple_escape    -- the few elements whose answer lies in an earlier
//                       tile, through tile minima and each tile's staircase
//                       of suffix minima.
#pragma once
#include <string>
#include <vector>

#include "common.cuh"

namespace alp {

struct PairInfo {           // one admissible pair
    uint32_t stack_begin;   // into stack[]
    uint32_t prod_begin;    // into pseq[]
    uint16_t n_br;          // brackets
    uint16_t n_prod;        // productions (= nodes)
    int16_t d_depth;        // lefts - rights
    int16_t d_v;            // sum of (arity - 1) over its productions
    uint16_t n_term;        // terminal productions among them
    int16_t min_ds;         // least (depth before it - 1) over its right brackets; 0x7fff without any
};

struct ParseTables {
    const uint16_t* key_index;  // [T^(q+k)] pair id, 0xffff = no pair
    const PairInfo* pairs;      // [n_pairs]
    const uint32_t* stack;      // symbol | left<<31
    const uint32_t* pseq;       // production ids
    const int32_t* arity;       // [n_prods]
    const int32_t* prod_term;   // [n_prods] terminal id or -1
    const int16_t* pseq_v;      // [n_pseq] sum of (arity-1) over the pair's earlier productions
    const int16_t* pseq_t;      // [n_pseq] terminal productions among the pair's earlier productions
    const int16_t* stack_d;     // [n_stack] depth change before this bracket within its pair
    // per production-sequence entry: x = production | (terminal + 1) << 16 (0: not a terminal
    // production), y = (uint16) pseq_v | pseq_t << 16
    const uint2* pseq_rec;
    // per stack entry: x = symbol | left << 31, y = (uint16) stack_d
    const uint2* stack_rec;
    int q, k, T, n_pairs, n_prods, n_pseq, n_stack;
    uint32_t empty, start, end;
};

struct ParseHost {
    int q = 0, k = 0, n_terms = 0, n_prods = 0, n_pairs = 0, max_prods = 0, max_brackets = 0;
    long long key_space = 0;
    // host copies for the pairs at shard boundaries (alp_parse_shard_*)
    std::vector<uint16_t> key_index;
    std::vector<PairInfo> pairs;
    uint32_t T = 0, empty = 0, start = 0, end = 0;
};

inline int load_parser(ParseTables& pt, ParseHost& ph, const uint8_t* p, const uint8_t* e,
                       std::vector<void*>& owned, std::string& err) {
    auto u32 = [&](uint32_t& v) -> bool {
        if (p + 4 > e) return false;
        memcpy(&v, p, 4);
        p += 4;
        return true;
    };
    uint32_t q, k, T, empty, start, end, n_prods, n_terms;
    if (!u32(q) || !u32(k) || !u32(T) || !u32(empty) || !u32(start) || !u32(end) || !u32(n_prods) || !u32(n_terms)) {
        err = "truncated parser header";
        return 4;
    }
    if (q + k > 16 || k < 1 || T < 3 || T > 65535 || n_prods > 65535) {
        err = "parser tables out of range";
        return 4;
    }
    auto need = [&](size_t bytes) { return p + bytes <= e; };
    if (!need((size_t)n_prods * 8)) { err = "truncated arities"; return 4; }
    std::vector<int32_t> arity(n_prods), pterm(n_prods);
    memcpy(arity.data(), p, 4 * (size_t)n_prods); p += 4 * (size_t)n_prods;
    memcpy(pterm.data(), p, 4 * (size_t)n_prods); p += 4 * (size_t)n_prods;
    uint32_t n_pairs;
    if (!u32(n_pairs) || n_pairs >= 0xffff || !need((size_t)n_pairs * 16)) { err = "bad pair count"; return 4; }
    std::vector<uint32_t> raw((size_t)n_pairs * 4);
    memcpy(raw.data(), p, raw.size() * 4); p += raw.size() * 4;
    uint32_t n_stack;
    if (!u32(n_stack) || !need((size_t)n_stack * 4)) { err = "bad stack"; return 4; }
    std::vector<uint32_t> stack(n_stack);
    memcpy(stack.data(), p, 4 * (size_t)n_stack); p += 4 * (size_t)n_stack;
    uint32_t n_pseq;
    if (!u32(n_pseq) || !need((size_t)n_pseq * 4)) { err = "bad productions"; return 4; }
    std::vector<uint32_t> pseq(n_pseq);
    memcpy(pseq.data(), p, 4 * (size_t)n_pseq); p += 4 * (size_t)n_pseq;
    uint32_t n_keys;
    const uint32_t W = q + k;
    if (!u32(n_keys) || !need((size_t)n_keys * (W + 1) * 4)) { err = "bad keys"; return 4; }
    std::vector<uint32_t> keys((size_t)n_keys * W), key_pair(n_keys);
    memcpy(keys.data(), p, keys.size() * 4); p += keys.size() * 4;
    memcpy(key_pair.data(), p, key_pair.size() * 4); p += key_pair.size() * 4;

    long long space = 1;
    for (uint32_t j = 0; j < W; ++j) {
        space *= T;
        if (space > (1ll << 24)) { err = "key space too large for the direct key index"; return 4; }
    }
    std::vector<uint16_t> index((size_t)space, 0xffff);
    for (uint32_t i = 0; i < n_keys; ++i) {
        long long x = 0;
        for (uint32_t j = 0; j < W; ++j) {
            uint32_t t = keys[(size_t)i * W + j];
            if (t >= T) { err = "key symbol out of range"; return 4; }
            x = x * T + t;
        }
        if (key_pair[i] >= n_pairs) { err = "key names a pair out of range"; return 4; }
        index[(size_t)x] = (uint16_t)key_pair[i];
    }
    std::vector<PairInfo> info(n_pairs);
    int maxp = 0, maxb = 0;
    for (uint32_t i = 0; i < n_pairs; ++i) {
        uint32_t sb = raw[4 * i], se = raw[4 * i + 1], pb = raw[4 * i + 2], pe = raw[4 * i + 3];
        if (se < sb || pe < pb || se > n_stack || pe > n_pseq || se - sb > 60000 || pe - pb > 60000) {
            err = "bad pair span";
            return 4;
        }
        PairInfo& pi = info[i];
        pi.stack_begin = sb;
        pi.prod_begin = pb;
        pi.n_br = (uint16_t)(se - sb);
        pi.n_prod = (uint16_t)(pe - pb);
        int dd = 0, dv = 0, nt = 0;
        for (uint32_t j = sb; j < se; ++j) dd += (stack[j] >> 31) ? 1 : -1;
        for (uint32_t j = pb; j < pe; ++j) {
            if (pseq[j] >= n_prods) { err = "production id out of range"; return 4; }
            dv += arity[pseq[j]] - 1;
            if (pterm[pseq[j]] >= 0) ++nt;
        }
        pi.d_depth = (int16_t)dd;
        pi.d_v = (int16_t)dv;
        pi.n_term = (uint16_t)nt;
        int md = 0x7fff, acc = 0;
        for (uint32_t j = sb; j < se; ++j) {
            if (!(stack[j] >> 31) && acc - 1 < md) md = acc - 1;
            acc += (stack[j] >> 31) ? 1 : -1;
        }
        pi.min_ds = (int16_t)md;
        if ((int)pi.n_prod > maxp) maxp = pi.n_prod;
        if ((int)pi.n_br > maxb) maxb = pi.n_br;
    }
    std::vector<int16_t> pv(n_pseq, 0), ptm(n_pseq, 0), sd(n_stack, 0);
    for (uint32_t i = 0; i < n_pairs; ++i) {
        int acc_v = 0, acc_t = 0, acc_d = 0;
        for (uint32_t j = raw[4 * i + 2]; j < raw[4 * i + 3]; ++j) {
            pv[j] = (int16_t)acc_v;
            ptm[j] = (int16_t)acc_t;
            acc_v += arity[pseq[j]] - 1;
            acc_t += pterm[pseq[j]] >= 0 ? 1 : 0;
        }
        for (uint32_t j = raw[4 * i]; j < raw[4 * i + 1]; ++j) {
            sd[j] = (int16_t)acc_d;
            acc_d += (stack[j] >> 31) ? 1 : -1;
        }
    }
    std::vector<uint2> prec(n_pseq), srec(n_stack);
    for (uint32_t j = 0; j < n_pseq; ++j) {
        const int32_t tm = pterm[pseq[j]];
        if (tm >= 65535) { err = "terminal id too large"; return 4; }
        prec[j].x = pseq[j] | ((uint32_t)(tm >= 0 ? tm + 1 : 0) << 16);
        prec[j].y = (uint32_t)(uint16_t)pv[j] | ((uint32_t)(uint16_t)ptm[j] << 16);
    }
    for (uint32_t j = 0; j < n_stack; ++j) {
        srec[j].x = stack[j];
        srec[j].y = (uint32_t)(uint16_t)sd[j];
    }
    auto up = [&](const void* h, size_t bytes, const void** d) -> bool {
        void* x = nullptr;
        if (cudaMalloc(&x, bytes < 16 ? 16 : bytes) != cudaSuccess) return false;
        if (bytes && cudaMemcpy(x, h, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return false;
        owned.push_back(x);
        *d = x;
        return true;
    };
    bool ok = up(index.data(), index.size() * 2, (const void**)&pt.key_index) &&
              up(info.data(), info.size() * sizeof(PairInfo), (const void**)&pt.pairs) &&
              up(stack.data(), stack.size() * 4, (const void**)&pt.stack) &&
              up(pseq.data(), pseq.size() * 4, (const void**)&pt.pseq) &&
              up(arity.data(), arity.size() * 4, (const void**)&pt.arity) &&
              up(pterm.data(), pterm.size() * 4, (const void**)&pt.prod_term) &&
              up(pv.data(), pv.size() * 2, (const void**)&pt.pseq_v) &&
              up(ptm.data(), ptm.size() * 2, (const void**)&pt.pseq_t) &&
              up(sd.data(), sd.size() * 2, (const void**)&pt.stack_d) &&
              up(prec.data(), prec.size() * 8, (const void**)&pt.pseq_rec) &&
              up(srec.data(), srec.size() * 8, (const void**)&pt.stack_rec);
    if (!ok) { err = "cudaMalloc/cudaMemcpy failed for parser tables"; return 2; }
    pt.q = (int)q; pt.k = (int)k; pt.T = (int)T; pt.n_pairs = (int)n_pairs; pt.n_prods = (int)n_prods;
    pt.n_pseq = (int)n_pseq; pt.n_stack = (int)n_stack;
    pt.empty = empty; pt.start = start; pt.end = end;
    ph.q = (int)q; ph.k = (int)k; ph.n_terms = (int)n_terms; ph.n_prods = (int)n_prods; ph.n_pairs = (int)n_pairs;
    ph.max_prods = maxp; ph.max_brackets = maxb; ph.key_space = space;
    ph.key_index = std::move(index);
    ph.pairs = info;
    ph.T = T; ph.empty = empty; ph.start = start; ph.end = end;
    return 0;
}

}  // namespace alp

namespace alp {

constexpr int PP_THREADS = 512;
constexpr int PP_ITEMS = 4;                        // positions per thread
constexpr int PP_TILE = PP_THREADS * PP_ITEMS;     // positions per tile
// previous-smaller-or-equal tiles: the default shape (threads x elements per
// thread); ple_tile_kernel is instantiated for the shapes ple_shapes lists
constexpr int PLE_THREADS = 256;
constexpr int PLE_ITEMS = 16;
constexpr int PLE_TILE = PLE_THREADS * PLE_ITEMS;  // elements per tile
constexpr uint16_t NO_PAIR = 0xffff;
constexpr int PS_HALO = 16;                        // halo terminals a shard keeps on each side (q + k <= 16)

// Running sums over positions.  Positions are the documents' ⊢ tokens ⊣
// sequences back to back; nodes, brackets and heads (⊢ count) run over all
// documents, depth / v / terminals restart at every ⊢ (a segmented scan).
// All fields are 32-bit: node and bracket totals are checked below 2^32 and
// positions below 2^31 before any launch.
struct __align__(16) PosSums {
    uint32_t nodes;   // productions
    uint32_t brs;     // brackets
    int32_t depth;    // lefts - rights since the last ⊢
    int32_t v;        // sum of (arity - 1) since the last ⊢
    uint32_t terms;   // terminal productions since the last ⊢
    uint32_t heads;   // ⊢ positions
    int32_t hpos;     // position of the last ⊢ (-1: none)
    uint32_t cls;     // bracket pairs closed between a position and the one before it
};

__device__ __forceinline__ void possums_zero(PosSums& s) {
    s.nodes = 0; s.brs = 0; s.depth = 0; s.v = 0; s.terms = 0; s.heads = 0; s.hpos = -1; s.cls = 0;
}
__device__ __forceinline__ PosSums ps_combine(const PosSums& a, const PosSums& b) {
    PosSums r;
    r.nodes = a.nodes + b.nodes;
    r.brs = a.brs + b.brs;
    r.heads = a.heads + b.heads;
    const bool h = b.heads != 0;
    r.depth = h ? b.depth : a.depth + b.depth;
    r.v = h ? b.v : a.v + b.v;
    r.terms = h ? b.terms : a.terms + b.terms;
    r.hpos = h ? b.hpos : a.hpos;
    r.cls = a.cls + b.cls;
    return r;
}
// ps_combine where all positions belong to one document: its only ⊢ is position 0,
// before which every sum is zero, so that restarting there is the same as adding.
// The ⊢ count and position are then not needed (left 0).
template <bool ONE>
__device__ __forceinline__ PosSums ps_join(const PosSums& a, const PosSums& b) {
    if (!ONE) return ps_combine(a, b);
    PosSums r;
    r.nodes = a.nodes + b.nodes;
    r.brs = a.brs + b.brs;
    r.heads = 0;
    r.depth = a.depth + b.depth;
    r.v = a.v + b.v;
    r.terms = a.terms + b.terms;
    r.hpos = 0;
    r.cls = a.cls + b.cls;
    return r;
}
// The one-document forms of the warp scan and shift: no ⊢ anywhere but position 0
// (whose sums before it are zero), so the six counted fields are plain prefix sums
// and the ⊢ fields stay 0.
__device__ __forceinline__ PosSums ps_warp_scan_one(PosSums x, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t on = __shfl_up_sync(ALP_FULL_MASK, x.nodes, d);
        const uint32_t ob = __shfl_up_sync(ALP_FULL_MASK, x.brs, d);
        const int32_t od = __shfl_up_sync(ALP_FULL_MASK, x.depth, d);
        const int32_t ov = __shfl_up_sync(ALP_FULL_MASK, x.v, d);
        const uint32_t ot = __shfl_up_sync(ALP_FULL_MASK, x.terms, d);
        const uint32_t oc = __shfl_up_sync(ALP_FULL_MASK, x.cls, d);
        if (lane >= d) { x.nodes += on; x.brs += ob; x.depth += od; x.v += ov; x.terms += ot; x.cls += oc; }
    }
    x.heads = 0;
    x.hpos = 0;
    return x;
}
__device__ __forceinline__ PosSums ps_shfl_up_one(const PosSums& x, int d) {
    PosSums r;
    r.nodes = __shfl_up_sync(ALP_FULL_MASK, x.nodes, d);
    r.brs = __shfl_up_sync(ALP_FULL_MASK, x.brs, d);
    r.depth = __shfl_up_sync(ALP_FULL_MASK, x.depth, d);
    r.v = __shfl_up_sync(ALP_FULL_MASK, x.v, d);
    r.terms = __shfl_up_sync(ALP_FULL_MASK, x.terms, d);
    r.cls = __shfl_up_sync(ALP_FULL_MASK, x.cls, d);
    r.heads = 0;
    r.hpos = 0;
    return r;
}
__device__ __forceinline__ PosSums ps_shfl_up(const PosSums& x, int d) {
    PosSums r;
    r.nodes = __shfl_up_sync(ALP_FULL_MASK, x.nodes, d);
    r.brs = __shfl_up_sync(ALP_FULL_MASK, x.brs, d);
    r.depth = __shfl_up_sync(ALP_FULL_MASK, x.depth, d);
    r.v = __shfl_up_sync(ALP_FULL_MASK, x.v, d);
    r.terms = __shfl_up_sync(ALP_FULL_MASK, x.terms, d);
    r.heads = __shfl_up_sync(ALP_FULL_MASK, x.heads, d);
    r.hpos = __shfl_up_sync(ALP_FULL_MASK, x.hpos, d);
    r.cls = __shfl_up_sync(ALP_FULL_MASK, x.cls, d);
    return r;
}
// inclusive warp scan (lanes in order); a warp without a ⊢ needs plain sums
__device__ __forceinline__ PosSums ps_warp_scan(PosSums x, int lane) {
    if (!__any_sync(ALP_FULL_MASK, x.heads != 0)) {
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t on = __shfl_up_sync(ALP_FULL_MASK, x.nodes, d);
            const uint32_t ob = __shfl_up_sync(ALP_FULL_MASK, x.brs, d);
            const int32_t od = __shfl_up_sync(ALP_FULL_MASK, x.depth, d);
            const int32_t ov = __shfl_up_sync(ALP_FULL_MASK, x.v, d);
            const uint32_t ot = __shfl_up_sync(ALP_FULL_MASK, x.terms, d);
            const uint32_t oc = __shfl_up_sync(ALP_FULL_MASK, x.cls, d);
            if (lane >= d) { x.nodes += on; x.brs += ob; x.depth += od; x.v += ov; x.terms += ot; x.cls += oc; }
        }
        return x;
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        PosSums o = ps_shfl_up(x, d);
        if (lane >= d) x = ps_combine(o, x);
    }
    return x;
}
__device__ __forceinline__ PosSums ps_elem(const PairInfo* s_pi, uint16_t p, bool head, long long i) {
    PosSums e;
    possums_zero(e);
    if (p != NO_PAIR) {
        const PairInfo& pi = s_pi[p];
        e.nodes = pi.n_prod; e.brs = pi.n_br; e.depth = pi.d_depth; e.v = pi.d_v; e.terms = pi.n_term;
    }
    if (head) { e.heads = 1; e.hpos = (int32_t)i; }
    return e;
}

// Brackets closed between adjacent positions: a pair's brackets are its
// rights, then its lefts, so position p's first rights close position p-1's
// top lefts, min(lefts of p-1, rights of p) of them, unless p starts a
// document or either has no pair.
__device__ __forceinline__ uint32_t pair_lefts(const PairInfo& p) {
    return (uint32_t)(((int32_t)p.n_br + (int32_t)p.d_depth) >> 1);
}
__device__ __forceinline__ uint32_t adj_closed(const PairInfo* s_pi, uint32_t prev, uint32_t cur, bool head) {
    if (head || prev == NO_PAIR || cur == NO_PAIR) return 0;
    const PairInfo& b = s_pi[cur];
    return min(pair_lefts(s_pi[prev]), (uint32_t)b.n_br - pair_lefts(b));
}

struct ParseArgs {
    ParseTables t;
    const uint16_t* P;          // [L] ⊢ tokens ⊣ per document: terminal ids
    const uint32_t* pstart;     // [L] token spans (document-relative), same layout
    const uint32_t* pend;
    long long L;                // positions
    long long n_docs;
    uint16_t* pid;              // [L] pair id per position
    PosSums* tile_sums;         // [tiles] K1 output, scanned in place to exclusive prefixes
    AlpResult* res;             // aux: totals (0 nodes, 1 brackets, 6 brackets kept, 7 adjacent pairs closed)
    // K2 outputs
    uint32_t* tag;
    uint8_t* kind;
    int64_t* nstart;
    int64_t* nend;
    int32_t* vbuf;              // node values exscan(arity-1), per document
    uint32_t* brbuf;            // bracket symbol | left<<31
    int32_t* dsbuf;             // bracket depth value (before a left, after a right), per document
                                //   (the brackets kept after closing adjacent pairs, aux[6] of them)
    long long* node_off;        // [n_docs + 1] first node of each document
    long long* br_off;          // [n_docs + 1] first kept bracket of each document
    uint8_t* doc_valid;         // [n_docs] cleared on rejection
    int subst_terminals;        // 1: wrapper productions become terminal nodes (parse_int); 0: production ids
    long long cap_nodes;
    long long cap_brs;
    const long long* dL;        // when set: the position count, in device memory (L is then its capacity)
    // the fused pair + expand pass: tile tickets and look-back over the position sums
    unsigned int* ticket;       // [1], zero before the launch
    uint32_t* lb_flag;          // [tiles] ST_X / ST_A / ST_P << 30, zero before the launch
    PosSums* lb_agg;            // [tiles] the tile's own sums
    PosSums* lb_inc;            // [tiles] the sums up to and including the tile
    // one shard of a document's positions (alp_parse_shard_*, two-pass form):
    // the terminals around it, the pair ids of the positions just outside it,
    // the sums of the shards before it and where its outputs start
    int shard;
    // [2 * PS_HALO] in device memory: terminals of positions -PS_HALO .. -1, then of
    // positions L .. L + PS_HALO - 1 (empty past the document)
    const uint32_t* halo;
    uint32_t prev_pair, next_pair;  // NO_PAIR: no position there
    PosSums pre;
    long long node_base;        // global index of the shard's first node
    long long br_base;          // global index of its first kept bracket
    long long pos_base;         // global position of its position 0
    // token spans the expand kernel's span stage holds per array (0: none): the shared
    // memory past the node-owner array, 8 bytes per span
    int span_cap;
};

__device__ __forceinline__ uint32_t pos_term(const ParseArgs& a, long long i) {
    if (i < 0) return (a.shard && i >= -PS_HALO) ? __ldg(&a.halo[PS_HALO + i]) : a.t.empty;
    if (i >= a.L) return (a.shard && i - a.L < PS_HALO) ? __ldg(&a.halo[PS_HALO + (i - a.L)]) : a.t.empty;
    return (uint32_t)a.P[i];
}

// ---------------------------------------------------------------------------
// K1: pair ids and per-tile (segmented) sums
// ---------------------------------------------------------------------------
// The pair kernel's shared memory: the pair infos, then the window of terminals.
__host__ __device__ inline size_t pairs_smem_bytes(int n_pairs, int window) {
    return sizeof(PairInfo) * (size_t)n_pairs + ((size_t)PP_TILE + window + 1) * 4;
}

// QT, KT > 0: the lookback and lookahead fixed at compile time (window loops
// unrolled); 0: read from the tables.
template <int QT, int KT>
__global__ void __launch_bounds__(PP_THREADS, 3) parse_pairs_kernel(ParseArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    PairInfo* s_pi = reinterpret_cast<PairInfo*>(smem);
    uint32_t* s_term = reinterpret_cast<uint32_t*>(smem + sizeof(PairInfo) * a.t.n_pairs);
    __shared__ PosSums s_w[PP_THREADS / 32];
    __shared__ uint32_t s_pow[17];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = QT > 0 ? QT : a.t.q, k = KT > 0 ? KT : a.t.k, W = q + k;
    if (a.dL) a.L = *a.dL;
    for (int i = tid; i < a.t.n_pairs * (int)(sizeof(PairInfo) / 4); i += PP_THREADS)
        reinterpret_cast<uint32_t*>(s_pi)[i] = reinterpret_cast<const uint32_t*>(a.t.pairs)[i];
    if (tid == 0) {
        uint32_t pw = 1;
        for (int j = 0; j < W; ++j) { s_pow[W - 1 - j] = pw; pw *= (uint32_t)a.t.T; }
    }
    const long long n_tiles = (a.L + PP_TILE - 1) / PP_TILE;
    // The window of a tile, one tile ahead in registers (its loads in flight while the
    // block works on the tile before): this thread's four terminals, and for the first
    // W + 1 threads one of the window's edge terminals (q + 1 before the tile, k after).
    // Terminal ids fit 16 bits: the four are kept as two words.
    auto window_loads = [&](long long b, uint2& t4, uint32_t& te) {
        const long long i0 = b + (long long)tid * PP_ITEMS;
        if (i0 >= 0 && i0 + PP_ITEMS <= a.L && (reinterpret_cast<uintptr_t>(a.P) & 7) == 0) {
            t4 = __ldg(reinterpret_cast<const uint2*>(a.P + i0));
        } else {
            t4 = make_uint2(pos_term(a, i0) | (pos_term(a, i0 + 1) << 16), pos_term(a, i0 + 2) | (pos_term(a, i0 + 3) << 16));
        }
        te = 0;
        if (tid <= q) te = pos_term(a, b - q - 1 + tid);
        else if (tid <= W) te = pos_term(a, b + PP_TILE + (tid - q - 1));
    };
    uint2 nt4 = make_uint2(0, 0);
    uint32_t nte = 0;
    if ((long long)blockIdx.x < n_tiles) window_loads((long long)blockIdx.x * PP_TILE, nt4, nte);
    for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const long long base = tile * PP_TILE;
    __syncthreads();  // the previous tile is done with s_term and s_w
    // window [base - q - 1, base + PP_TILE + k): s_term[q + 1 + pl] is position base + pl
    {
        uint32_t* d = s_term + q + 1 + tid * PP_ITEMS;
        d[0] = nt4.x & 0xffffu; d[1] = nt4.x >> 16; d[2] = nt4.y & 0xffffu; d[3] = nt4.y >> 16;
        if (tid <= q) s_term[tid] = nte;
        else if (tid <= W) s_term[PP_TILE + tid] = nte;
    }
    if (tile + gridDim.x < n_tiles) window_loads(base + (long long)gridDim.x * PP_TILE, nt4, nte);
    __syncthreads();
    const uint32_t SL = a.t.start, SR = a.t.end, EMPTY = a.t.empty;
    // the pair id at tile-local position pl (-1: the position before the tile);
    // s_term[pl + 1 + jj] is position base + pl - q + jj
    auto pair_at = [&](int pl, bool& head) -> uint16_t {
        const int o = pl + 1;
        const uint32_t c = s_term[o + q];
        head = c == SL;
        // a window never reaches past its document's ⊢ (left) or ⊣ (right)
        uint32_t x = c * s_pow[q];
        bool ok = c != SL;
#pragma unroll
        for (int jj = q - 1; jj >= 0; --jj) {
            const uint32_t t = s_term[o + jj];
            x += (ok ? t : EMPTY) * s_pow[jj];
            ok = ok && t != SL;
        }
        ok = c != SR;
#pragma unroll
        for (int jj = q + 1; jj < W; ++jj) {
            const uint32_t t = s_term[o + jj];
            x += (ok ? t : EMPTY) * s_pow[jj];
            ok = ok && t != SR;
        }
        return __ldg(&a.t.key_index[x]);
    };
    // the pair before this thread's first position: a warp's first lane computes it
    // from the window (which starts one position early), first, so that its table
    // load is in flight with the four below; the other lanes take the previous lane's last
    uint32_t before = NO_PAIR;
    if (lane == 0) {
        const long long ip = base + (long long)tid * PP_ITEMS - 1;
        bool h;
        if (ip >= 0 && ip < a.L) before = pair_at(tid * PP_ITEMS - 1, h);
        else if (ip == -1 && a.shard) before = a.prev_pair;  // the last position of the shard before
    }
    uint16_t ids[PP_ITEMS];
    uint32_t hb = 0;
#pragma unroll
    for (int j = 0; j < PP_ITEMS; ++j) {
        const long long i = base + tid * PP_ITEMS + j;
        uint16_t p = NO_PAIR;
        bool head = false;
        if (i < a.L) p = pair_at(tid * PP_ITEMS + j, head);
        ids[j] = p;
        if (head) hb |= 1u << j;
    }
    const uint32_t up = __shfl_up_sync(ALP_FULL_MASK, (uint32_t)ids[PP_ITEMS - 1], 1);
    const uint32_t prev = lane == 0 ? before : up;
    PosSums acc;
    possums_zero(acc);
    {
        uint32_t lprev = prev != NO_PAIR ? pair_lefts(s_pi[prev]) : 0u;  // the previous position's lefts
        bool pv = prev != NO_PAIR;
#pragma unroll
        for (int j = 0; j < PP_ITEMS; ++j) {
            const long long i = base + tid * PP_ITEMS + j;
            if (i < a.L) {
                const bool head = (hb >> j) & 1u;
                PosSums e;
                possums_zero(e);
                uint32_t nl = 0;
                if (ids[j] != NO_PAIR) {
                    const PairInfo& pi = s_pi[ids[j]];
                    e.nodes = pi.n_prod; e.brs = pi.n_br; e.depth = pi.d_depth; e.v = pi.d_v; e.terms = pi.n_term;
                    nl = pair_lefts(pi);
                    if (!head && pv) e.cls = min(lprev, (uint32_t)pi.n_br - nl);  // adj_closed
                }
                if (head) { e.heads = 1; e.hpos = (int32_t)i; }
                acc = ps_combine(acc, e);
                lprev = nl;
                pv = ids[j] != NO_PAIR;
            }
        }
    }
    const long long i0 = base + tid * PP_ITEMS;
    if (i0 + PP_ITEMS <= a.L && ((i0 & 3) == 0)) {
        static_assert(PP_ITEMS == 4, "pair ids are stored as one 8-byte word per thread");
        uint2 w;
        w.x = ids[0] | ((uint32_t)ids[1] << 16);
        w.y = ids[2] | ((uint32_t)ids[3] << 16);
        *reinterpret_cast<uint2*>(a.pid + i0) = w;
    } else {
        for (int j = 0; j < PP_ITEMS; ++j)
            if (i0 + j < a.L) a.pid[i0 + j] = ids[j];
    }
    // ordered block reduce: the warps' totals, then warp 0 over them; a warp without a
    // document head adds its fields with one warp reduction each
    PosSums inc;
    if (!__any_sync(ALP_FULL_MASK, acc.heads != 0)) {
        inc.nodes = __reduce_add_sync(ALP_FULL_MASK, acc.nodes);
        inc.brs = __reduce_add_sync(ALP_FULL_MASK, acc.brs);
        inc.depth = __reduce_add_sync(ALP_FULL_MASK, acc.depth);
        inc.v = __reduce_add_sync(ALP_FULL_MASK, acc.v);
        inc.terms = __reduce_add_sync(ALP_FULL_MASK, acc.terms);
        inc.cls = __reduce_add_sync(ALP_FULL_MASK, acc.cls);
        inc.heads = 0;
        inc.hpos = -1;
    } else {
        inc = ps_warp_scan(acc, lane);
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        PosSums w;
        if (lane < PP_THREADS / 32) w = s_w[lane]; else possums_zero(w);
        const PosSums t = ps_warp_scan(w, lane);
        if (lane == PP_THREADS / 32 - 1) a.tile_sums[tile] = t;
    }
    }
}

// The pair kernel for a grammar's (q, k): an unrolled instantiation for the
// small ones, the generic kernel otherwise.
inline const void* pairs_kernel_for(int q, int k) {
    if (q == 1 && k == 1) return (const void*)parse_pairs_kernel<1, 1>;
    if (q == 1 && k == 2) return (const void*)parse_pairs_kernel<1, 2>;
    if (q == 1 && k == 3) return (const void*)parse_pairs_kernel<1, 3>;
    if (q == 2 && k == 1) return (const void*)parse_pairs_kernel<2, 1>;
    if (q == 2 && k == 2) return (const void*)parse_pairs_kernel<2, 2>;
    return (const void*)parse_pairs_kernel<0, 0>;
}

// Exclusive segmented scan of the tile sums in place, in two launches:
// scan_tiles_reduce_kernel sums each chunk of ST_CHUNK tiles, then
// scan_tiles_kernel (one CTA per chunk) scans the chunk sums before its own
// and its own tiles.  Totals go to res->aux (nodes, brackets, final depth, -,
// -, heads) and the closing entries of node_off / br_off.
constexpr int ST_CHUNK = 1024;

__device__ __forceinline__ PosSums ps_block_reduce(PosSums v, PosSums* s_w) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    PosSums inc = ps_warp_scan(v, lane);
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    PosSums t = s_w[0];
    for (int w = 1; w < (int)(blockDim.x / 32); ++w) t = ps_combine(t, s_w[w]);
    return t;
}

__global__ void __launch_bounds__(ST_CHUNK) scan_tiles_reduce_kernel(const PosSums* s, long long tiles,
                                                                     PosSums* chunk_sums, const long long* dL) {
    __shared__ PosSums s_w[ST_CHUNK / 32];
    if (dL) tiles = (*dL + PP_TILE - 1) / PP_TILE;  // the grid covers the capacity
    const long long idx = (long long)blockIdx.x * ST_CHUNK + threadIdx.x;
    PosSums v;
    if (idx < tiles) v = s[idx]; else possums_zero(v);
    const PosSums t = ps_block_reduce(v, s_w);
    if (threadIdx.x == 0) chunk_sums[blockIdx.x] = t;
}

__global__ void __launch_bounds__(ST_CHUNK) scan_tiles_kernel(PosSums* s, long long tiles, const PosSums* chunk_sums,
                                                              AlpResult* res, long long* node_off, long long* br_off,
                                                              long long n_docs, const long long* dL) {
    __shared__ PosSums s_w[ST_CHUNK / 32];
    __shared__ PosSums s_carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long chunk = blockIdx.x;
    if (dL) tiles = (*dL + PP_TILE - 1) / PP_TILE;  // the grid covers the capacity
    const long long last = (tiles + ST_CHUNK - 1) / ST_CHUNK - 1;
    if (chunk > last) return;
    if (warp == 0) {
        PosSums carry;
        possums_zero(carry);
        for (long long b = 0; b < chunk; b += 32) {
            PosSums v;
            if (b + lane < chunk) v = chunk_sums[b + lane]; else possums_zero(v);
            const PosSums inc = ps_warp_scan(v, lane);
            PosSums last;
            last.nodes = __shfl_sync(ALP_FULL_MASK, inc.nodes, 31);
            last.brs = __shfl_sync(ALP_FULL_MASK, inc.brs, 31);
            last.depth = __shfl_sync(ALP_FULL_MASK, inc.depth, 31);
            last.v = __shfl_sync(ALP_FULL_MASK, inc.v, 31);
            last.terms = __shfl_sync(ALP_FULL_MASK, inc.terms, 31);
            last.heads = __shfl_sync(ALP_FULL_MASK, inc.heads, 31);
            last.hpos = __shfl_sync(ALP_FULL_MASK, inc.hpos, 31);
            last.cls = __shfl_sync(ALP_FULL_MASK, inc.cls, 31);
            carry = ps_combine(carry, last);
        }
        if (lane == 0) s_carry = carry;
    }
    const long long idx = chunk * ST_CHUNK + tid;
    PosSums v;
    if (idx < tiles) v = s[idx]; else possums_zero(v);
    PosSums inc = ps_warp_scan(v, lane);
    PosSums ex = ps_shfl_up(inc, 1);
    if (lane == 0) possums_zero(ex);
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        PosSums w = s_w[lane];
        PosSums wi = ps_warp_scan(w, lane);
        PosSums we = ps_shfl_up(wi, 1);
        if (lane == 0) possums_zero(we);
        s_w[lane] = we;
    }
    __syncthreads();
    const PosSums pre = ps_combine(s_carry, s_w[warp]);
    if (idx < tiles) s[idx] = ps_combine(pre, ex);
    if (chunk == last) {
        __syncthreads();
        if (tid == ST_CHUNK - 1) s_carry = ps_combine(pre, inc);
        if (warp == 0) {
            // node, bracket and closed-pair totals in 64 bits, so that a total past 2^32 is seen
            unsigned long long tn = 0, tb = 0, tc = 0;
            for (long long b = lane; b <= chunk; b += 32) {
                if (b < chunk) { tn += chunk_sums[b].nodes; tb += chunk_sums[b].brs; tc += chunk_sums[b].cls; }
            }
            for (int d = 16; d >= 1; d >>= 1) {
                tn += __shfl_down_sync(ALP_FULL_MASK, tn, d);
                tb += __shfl_down_sync(ALP_FULL_MASK, tb, d);
                tc += __shfl_down_sync(ALP_FULL_MASK, tc, d);
            }
            if (lane == 0) { res->aux[0] = (long long)tn; res->aux[1] = (long long)tb; res->aux[7] = (long long)tc; }
        }
        __syncthreads();
        if (tid == 0) {
            const PosSums tot = s_carry;
            // the last chunk's own sums on top of the 64-bit totals of the earlier chunks
            const PosSums own = chunk_sums[chunk];
            res->aux[0] += own.nodes;
            res->aux[1] += own.brs;
            res->aux[7] += own.cls;
            res->aux[2] = tot.depth;
            res->aux[3] = tot.v;
            res->aux[4] = (long long)tot.terms;
            res->aux[5] = (long long)tot.heads;
            res->aux[6] = res->aux[1] - 2 * res->aux[7];  // brackets left for the search
            node_off[n_docs] = res->aux[0];
            br_off[n_docs] = res->aux[6];
        }
    }
}

// ---------------------------------------------------------------------------
// K2: expand every position's productions and brackets
//
// One tile = PP_TILE positions.  The block scans the per-position sums and
// records, per position, its pair, first node, first bracket, depth, value
// and first token index in shared memory, and checks the document rules that
// one position decides alone (an admissible pair, a depth that never goes
// below zero, depth zero at ⊣).  Nodes are then produced in windows of EX_WIN:
// each thread marks its positions as the owners of their nodes in the window
// (16-bit position indices), and the block emits the window one node per
// thread, in order, with coalesced stores.  No thread walks another
// position's productions, so warps stay converged whatever the sizes of the
// pairs.
//
// Brackets: a pair's brackets are its rights, then its lefts (the stack it
// pops, then the one it pushes), so a position's first rights close the
// previous position's top lefts, min(lefts before, rights here) of them, in
// the same document.  Those pairs are checked here (equal symbols) and
// dropped: removing matched adjacent pairs leaves every other bracket's
// match (the previous smaller-or-equal of futhark/parser.fut:153-184) as it
// was.  The rest -- about half of json's brackets -- is written by the
// position's own thread, at the front of the tile's bracket range, for the
// search that follows.
// ---------------------------------------------------------------------------
constexpr int EX_WIN = 8192;                     // nodes per window
constexpr int EX_SPAN_BYTES = 18432;             // shared bytes for the tile's token spans, where they fit
constexpr int EX_U = 1;                          // nodes a thread emits at once (2 and 4 measured slower
                                                 // once the token spans come from shared memory)
constexpr uint32_t EX_NO_TOKEN = 0xffffffffu;
// per position: a node record, one unused slot after every thread's four
// positions, so that the 32 lanes of a warp writing their first position
// (64 bytes apart without the pad) hit distinct banks
constexpr size_t EX_POS_BYTES = (size_t)PP_TILE * 5 / 4 * 16;
__device__ __forceinline__ int ex_slot(int pl) { return pl + (pl >> 2); }

// 16 bytes from global to shared memory without registers (cp.async; `bytes` < 16
// reads that many and zero-fills the rest)
__device__ __forceinline__ void ex_cp16(void* dst, const void* src, uint32_t bytes) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void ex_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void ex_cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// pair infos (20 bytes each), then the 8-byte records from a 16-byte boundary
__host__ __device__ inline size_t expand_rec_off(int n_pairs) {
    return (sizeof(PairInfo) * n_pairs + 15) & ~(size_t)15;
}
__host__ __device__ inline size_t expand_tables_bytes(int n_pairs, int n_pseq, int n_stack) {
    return (expand_rec_off(n_pairs) + 8 * ((size_t)n_pseq + n_stack) + 15) & ~(size_t)15;
}
__host__ __device__ inline size_t expand_smem_bytes(int n_pairs, int n_pseq, int n_stack) {
    return expand_tables_bytes(n_pairs, n_pseq, n_stack) + EX_POS_BYTES + 2 * (size_t)EX_WIN;
}

// Pair ids and (TERMS) terminals of the PP_ITEMS positions from i0 as two
// 8-byte words (one vector load each when all are in range; ids past the end
// read as no pair).
template <bool TERMS>
__device__ __forceinline__ void ex_words(const ParseArgs& a, long long i0, uint2& w, uint2& t) {
    static_assert(PP_ITEMS == 4, "a thread's positions are one 8-byte word");
    if (i0 + PP_ITEMS <= a.L) {
        w = __ldg(reinterpret_cast<const uint2*>(a.pid + i0));
        if (TERMS) t = __ldg(reinterpret_cast<const uint2*>(a.P + i0));
    } else {
        uint32_t x[PP_ITEMS], y[PP_ITEMS];
#pragma unroll
        for (int j = 0; j < PP_ITEMS; ++j) {
            x[j] = i0 + j < a.L ? a.pid[i0 + j] : NO_PAIR;
            y[j] = (TERMS && i0 + j < a.L) ? a.P[i0 + j] : 0xffffu;
        }
        w = make_uint2(x[0] | (x[1] << 16), x[2] | (x[3] << 16));
        t = make_uint2(y[0] | (y[1] << 16), y[2] | (y[3] << 16));
    }
}

// The fused form's look-back over tiles: warp 0 publishes the tile's own
// sums, combines the sums of earlier tiles (nearest first, 32 at a time) until
// it meets an inclusive prefix, and publishes this tile's inclusive prefix.
// Payloads are written before their flag with a fence in between; a reader
// fences after it sees the flag.
__device__ __forceinline__ PosSums ps_ld(const PosSums* p) {
    const volatile uint4* v = reinterpret_cast<const volatile uint4*>(p);
    const uint4 x = make_uint4(v[0].x, v[0].y, v[0].z, v[0].w), y = make_uint4(v[1].x, v[1].y, v[1].z, v[1].w);
    PosSums r;
    r.nodes = x.x; r.brs = x.y; r.depth = (int32_t)x.z; r.v = (int32_t)x.w;
    r.terms = y.x; r.heads = y.y; r.hpos = (int32_t)y.z; r.cls = y.w;
    return r;
}
__device__ __forceinline__ void ps_st(PosSums* p, const PosSums& r) {
    volatile uint4* v = reinterpret_cast<volatile uint4*>(p);
    v[0].x = r.nodes; v[0].y = r.brs; v[0].z = (uint32_t)r.depth; v[0].w = (uint32_t)r.v;
    v[1].x = r.terms; v[1].y = r.heads; v[1].z = (uint32_t)r.hpos; v[1].w = r.cls;
}
__device__ __forceinline__ PosSums ps_shfl_down(const PosSums& x, int d) {
    PosSums r;
    r.nodes = __shfl_down_sync(ALP_FULL_MASK, x.nodes, d);
    r.brs = __shfl_down_sync(ALP_FULL_MASK, x.brs, d);
    r.depth = __shfl_down_sync(ALP_FULL_MASK, x.depth, d);
    r.v = __shfl_down_sync(ALP_FULL_MASK, x.v, d);
    r.terms = __shfl_down_sync(ALP_FULL_MASK, x.terms, d);
    r.heads = __shfl_down_sync(ALP_FULL_MASK, x.heads, d);
    r.hpos = __shfl_down_sync(ALP_FULL_MASK, x.hpos, d);
    r.cls = __shfl_down_sync(ALP_FULL_MASK, x.cls, d);
    return r;
}
__device__ __forceinline__ PosSums ps_lookback(const ParseArgs& a, long long tile, const PosSums& agg) {
    const int lane = threadIdx.x & 31;
    PosSums acc;
    possums_zero(acc);
    if (tile == 0) {
        if (lane == 0) {
            ps_st(&a.lb_inc[0], agg);
            __threadfence();
            st_volatile32(&a.lb_flag[0], ST_P << 30);
        }
        return acc;
    }
    if (lane == 0) {
        ps_st(&a.lb_agg[tile], agg);
        __threadfence();
        st_volatile32(&a.lb_flag[tile], ST_A << 30);
    }
    long long end = tile;
    for (;;) {
        const long long idx = end - 32 + lane;
        uint32_t f = ST_P;
        if (idx >= 0) f = wait32(&a.lb_flag[idx], &a.res->error) >> 30;
        const uint32_t pm = __ballot_sync(ALP_FULL_MASK, f == ST_P && idx >= 0);
        const int p = pm ? 31 - __clz(pm) : -1;
        __threadfence();
        PosSums x;
        possums_zero(x);
        if (idx >= 0 && lane >= p) x = lane == p ? ps_ld(&a.lb_inc[idx]) : ps_ld(&a.lb_agg[idx]);
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {  // lanes in order
            const PosSums o = ps_shfl_down(x, d);
            if (lane + d < 32) x = ps_combine(x, o);
        }
        PosSums win;
        win.nodes = __shfl_sync(ALP_FULL_MASK, x.nodes, 0);
        win.brs = __shfl_sync(ALP_FULL_MASK, x.brs, 0);
        win.depth = __shfl_sync(ALP_FULL_MASK, x.depth, 0);
        win.v = __shfl_sync(ALP_FULL_MASK, x.v, 0);
        win.terms = __shfl_sync(ALP_FULL_MASK, x.terms, 0);
        win.heads = __shfl_sync(ALP_FULL_MASK, x.heads, 0);
        win.hpos = __shfl_sync(ALP_FULL_MASK, x.hpos, 0);
        win.cls = __shfl_sync(ALP_FULL_MASK, x.cls, 0);
        acc = ps_combine(win, acc);
        if (pm) break;
        end -= 32;
    }
    if (lane == 0) {
        ps_st(&a.lb_inc[tile], ps_combine(acc, agg));
        __threadfence();
        st_volatile32(&a.lb_flag[tile], ST_P << 30);
    }
    return acc;
}

// FUSED (QT, KT as in parse_pairs_kernel): the pair ids come from the key
// windows of a shared-memory copy of the tile's terminals, and the tile's
// exclusive position sums from a look-back over earlier tiles (tiles taken in
// ticket order, so every tile a look-back waits for is running or done).  The
// pair kernel, the tile-sum scans and the pair-id array are then not needed.
// ONE: the positions are one document (not a shard of one): the thread-level
// sums are plain sums and every position's document is document 0.
template <int QT, int KT, bool FUSED, bool ONE = false>
__global__ void __launch_bounds__(PP_THREADS, 2) parse_expand_kernel(ParseArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    PairInfo* s_pi = reinterpret_cast<PairInfo*>(smem);
    uint2* s_prec = reinterpret_cast<uint2*>(smem + expand_rec_off(a.t.n_pairs));
    uint2* s_srec = s_prec + a.t.n_pseq;
    // per position: x = its first production record minus its first (tile-local)
    // node, so that node g reads record g + x; y = exscan(arity - 1) before it;
    // z = token index of its first terminal production; w = depth before it (not read by
    // the node windows; a record stays one 16-byte store)
    int4* s_pos = reinterpret_cast<int4*>(smem + expand_tables_bytes(a.t.n_pairs, a.t.n_pseq, a.t.n_stack));
    uint16_t* s_own = reinterpret_cast<uint16_t*>(s_pos + PP_TILE * 5 / 4);  // [EX_WIN] owner of each node
    // FUSED: the tile's terminals [base - q - 1, base + PP_TILE + k), before s_own is used
    uint32_t* s_term = reinterpret_cast<uint32_t*>(s_own);
    static_assert((PP_TILE + 17 + 1) * 4 <= 2 * EX_WIN, "the key window fits the owner array");
    __shared__ PosSums s_w[PP_THREADS / 32];
    __shared__ PosSums s_tp;
    __shared__ uint32_t s_tn, s_tile, s_slo, s_shi;
    __shared__ uint32_t s_pow[17];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = QT > 0 ? QT : a.t.q, k = KT > 0 ? KT : a.t.k, W = q + k;
    if (a.dL) a.L = *a.dL;
    for (int i = tid; i < a.t.n_pairs * (int)(sizeof(PairInfo) / 4); i += PP_THREADS)
        reinterpret_cast<uint32_t*>(s_pi)[i] = reinterpret_cast<const uint32_t*>(a.t.pairs)[i];
    for (int i = tid; i < a.t.n_pseq; i += PP_THREADS) s_prec[i] = a.t.pseq_rec[i];
    for (int i = tid; i < a.t.n_stack; i += PP_THREADS) s_srec[i] = a.t.stack_rec[i];
    if (FUSED && tid == 0) {
        uint32_t pw = 1;
        for (int j = 0; j < W; ++j) { s_pow[W - 1 - j] = pw; pw *= (uint32_t)a.t.T; }
    }
    const uint32_t SL = a.t.start, SR = a.t.end, EMPTY = a.t.empty;
    const long long n_tiles = (a.L + PP_TILE - 1) / PP_TILE;
    // (not fused) this thread's pair ids and terminals, one tile ahead (loads in
    // flight while the block works on the current tile)
    uint2 nw = make_uint2(0, 0), nt = make_uint2(0, 0);
    if (!FUSED) ex_words<!ONE>(a, (long long)blockIdx.x * PP_TILE + tid * PP_ITEMS, nw, nt);
    for (long long it = blockIdx.x;; it += gridDim.x) {
        __syncthreads();  // the previous tile is done with the shared arrays
        long long tile = it;
        if (FUSED) {
            if (tid == 0) s_tile = atomicAdd(a.ticket, 1u);
            __syncthreads();
            tile = s_tile;
        }
        if (tile >= n_tiles) break;
        const long long i0 = tile * PP_TILE + tid * PP_ITEMS;
        PosSums tp;
        uint16_t ids[PP_ITEMS];
        uint32_t hm = 0, em = 0;  // head / end bits of this thread's positions
        uint32_t prev_id = NO_PAIR, next_id = NO_PAIR;
        bool next_head = false;
        if (FUSED) {
            const long long base = tile * PP_TILE;
            for (int i = tid; i < PP_TILE + W + 1; i += PP_THREADS) s_term[i] = pos_term(a, base - q - 1 + i);
            __syncthreads();
            // the pair id at tile-local position pl; s_term[pl + 1 + jj] is position base + pl - q + jj
            auto pair_at = [&](int pl) -> uint16_t {
                const int o = pl + 1;
                const uint32_t c = s_term[o + q];
                uint32_t x = c * s_pow[q];
                bool ok = c != SL;  // a window never reaches past its document's ⊢ (left) or ⊣ (right)
#pragma unroll
                for (int jj = q - 1; jj >= 0; --jj) {
                    const uint32_t t = s_term[o + jj];
                    x += (ok ? t : EMPTY) * s_pow[jj];
                    ok = ok && t != SL;
                }
                ok = c != SR;
#pragma unroll
                for (int jj = q + 1; jj < W; ++jj) {
                    const uint32_t t = s_term[o + jj];
                    x += (ok ? t : EMPTY) * s_pow[jj];
                    ok = ok && t != SR;
                }
                return __ldg(&a.t.key_index[x]);
            };
            const int pl0 = tid * PP_ITEMS;
            if (lane == 0 && i0 > 0 && i0 - 1 < a.L) prev_id = pair_at(pl0 - 1);
            if (lane == 31 && i0 + PP_ITEMS < a.L) {
                next_id = pair_at(pl0 + PP_ITEMS);
                next_head = s_term[pl0 + PP_ITEMS + 1 + q] == SL;
            }
#pragma unroll
            for (int j = 0; j < PP_ITEMS; ++j) {
                ids[j] = NO_PAIR;
                if (i0 + j < a.L) {
                    ids[j] = pair_at(pl0 + j);
                    const uint32_t c = s_term[pl0 + j + 1 + q];
                    if (c == SL) hm |= 1u << j;
                    if (c == SR) em |= 1u << j;
                }
            }
            possums_zero(tp);
        } else {
            tp = a.shard ? ps_combine(a.pre, a.tile_sums[tile]) : a.tile_sums[tile];
            ids[0] = (uint16_t)nw.x; ids[1] = (uint16_t)(nw.x >> 16); ids[2] = (uint16_t)nw.y; ids[3] = (uint16_t)(nw.y >> 16);
            if (ONE) {
                // one document: its ⊢ is position 0 and its ⊣ position L - 1
                if (i0 == 0) hm = 1u;
                if (a.L - 1 >= i0 && a.L - 1 < i0 + PP_ITEMS) em = 1u << (uint32_t)(a.L - 1 - i0);
            } else {
                const uint32_t c[PP_ITEMS] = {nt.x & 0xffffu, nt.x >> 16, nt.y & 0xffffu, nt.y >> 16};
#pragma unroll
                for (int j = 0; j < PP_ITEMS; ++j) {
                    if (i0 + j < a.L) {
                        if (c[j] == SL) hm |= 1u << j;
                        if (c[j] == SR) em |= 1u << j;
                    }
                }
            }
            if (tile + gridDim.x < n_tiles) ex_words<!ONE>(a, i0 + (long long)gridDim.x * PP_TILE, nw, nt);
            if (lane == 0 && i0 > 0 && i0 - 1 < a.L) prev_id = a.pid[i0 - 1];
            else if (lane == 0 && i0 == 0 && a.shard) prev_id = a.prev_pair;
            if (lane == 31 && i0 + PP_ITEMS < a.L) {
                next_id = a.pid[i0 + PP_ITEMS];
                next_head = !ONE && (uint32_t)a.P[i0 + PP_ITEMS] == SL;  // one document: no ⊢ after position 0
            } else if (lane == 31 && i0 + PP_ITEMS == a.L && a.shard) {
                next_id = a.next_pair;  // the next shard's first position (never a document head)
            }
        }
        // ---- pairs closed between each position and the one before it (adj_closed),
        // with the previous lefts carried along; cl[PP_ITEMS] is the next thread's cl[0]
        {
            const uint32_t up = __shfl_up_sync(ALP_FULL_MASK, (uint32_t)ids[PP_ITEMS - 1], 1);
            if (lane > 0) prev_id = up;
        }
        uint32_t cl[PP_ITEMS + 1];
        PosSums mine;
        possums_zero(mine);
        {
            uint32_t lprev = prev_id != NO_PAIR ? pair_lefts(s_pi[prev_id]) : 0u;
            bool pv = prev_id != NO_PAIR;
#pragma unroll
            for (int j = 0; j < PP_ITEMS; ++j) {
                cl[j] = 0;
                if (i0 + j < a.L) {
                    const bool head = (hm >> j) & 1u;
                    PosSums e;
                    possums_zero(e);
                    uint32_t nl = 0;
                    if (ids[j] != NO_PAIR) {
                        const PairInfo& pi = s_pi[ids[j]];
                        e.nodes = pi.n_prod; e.brs = pi.n_br; e.depth = pi.d_depth; e.v = pi.d_v; e.terms = pi.n_term;
                        nl = pair_lefts(pi);
                        if (!head && pv) e.cls = min(lprev, (uint32_t)pi.n_br - nl);
                    }
                    if (head && !ONE) { e.heads = 1; e.hpos = (int32_t)(i0 + j); }
                    cl[j] = e.cls;
                    mine = ps_join<ONE>(mine, e);
                    lprev = nl;
                    pv = ids[j] != NO_PAIR;
                } else if (a.shard && i0 + j == a.L && pv && a.next_pair != NO_PAIR) {
                    // the next shard's first position closes this shard's last lefts
                    const PairInfo& pn = s_pi[a.next_pair];
                    cl[j] = min(lprev, (uint32_t)pn.n_br - pair_lefts(pn));
                }
            }
            const uint32_t dn = __shfl_down_sync(ALP_FULL_MASK, cl[0], 1);
            cl[PP_ITEMS] = dn;
            if (lane == 31) {  // the next warp's first position
                cl[PP_ITEMS] = (i0 + PP_ITEMS < a.L || (a.shard && i0 + PP_ITEMS == a.L))
                                   ? adj_closed(s_pi, ids[PP_ITEMS - 1], next_id, next_head) : 0u;
            }
        }
        const PosSums inc = ONE ? ps_warp_scan_one(mine, lane) : ps_warp_scan(mine, lane);
        PosSums ex = ONE ? ps_shfl_up_one(inc, 1) : ps_shfl_up(inc, 1);
        if (lane == 0) possums_zero(ex);
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            PosSums w;
            if (lane < PP_THREADS / 32) w = s_w[lane]; else possums_zero(w);
            const PosSums wi = ONE ? ps_warp_scan_one(w, lane) : ps_warp_scan(w, lane);
            PosSums we = ONE ? ps_shfl_up_one(wi, 1) : ps_shfl_up(wi, 1);
            if (lane == 0) possums_zero(we);
            if (lane < PP_THREADS / 32) s_w[lane] = we;
            if (lane == PP_THREADS / 32 - 1) {
                s_tn = wi.nodes;
                if (!FUSED) {
                    // the tile's terminal nodes take the spans of positions [s_slo, s_shi): the
                    // first terminal index after the last head before the tile, and after the tile
                    const PosSums tot = ps_join<ONE>(tp, wi);
                    // (one document: the last ⊢ is position 0)
                    s_slo = (ONE ? 0u : (uint32_t)tp.hpos) + 1u + tp.terms;
                    s_shi = (ONE ? 0u : (uint32_t)tot.hpos) + 1u + tot.terms;
                }
            }
            if (FUSED) {
                // the tile's own sums: the last warp's inclusive value
                constexpr int LW = PP_THREADS / 32 - 1;
                PosSums agg;
                agg.nodes = __shfl_sync(ALP_FULL_MASK, wi.nodes, LW);
                agg.brs = __shfl_sync(ALP_FULL_MASK, wi.brs, LW);
                agg.depth = __shfl_sync(ALP_FULL_MASK, wi.depth, LW);
                agg.v = __shfl_sync(ALP_FULL_MASK, wi.v, LW);
                agg.terms = __shfl_sync(ALP_FULL_MASK, wi.terms, LW);
                agg.heads = __shfl_sync(ALP_FULL_MASK, wi.heads, LW);
                agg.hpos = __shfl_sync(ALP_FULL_MASK, wi.hpos, LW);
                agg.cls = __shfl_sync(ALP_FULL_MASK, wi.cls, LW);
                const PosSums pre = ps_lookback(a, tile, agg);
                if (lane == 0) {
                    s_tp = pre;
                    if (tile == n_tiles - 1) {
                        // totals (the host checks beforehand that they fit 32 bits)
                        const PosSums tot = ps_combine(pre, agg);
                        a.res->aux[0] = (long long)tot.nodes;
                        a.res->aux[1] = (long long)tot.brs;
                        a.res->aux[2] = tot.depth;
                        a.res->aux[3] = tot.v;
                        a.res->aux[4] = (long long)tot.terms;
                        a.res->aux[5] = (long long)tot.heads;
                        a.res->aux[7] = (long long)tot.cls;
                        a.res->aux[6] = (long long)tot.brs - 2 * (long long)tot.cls;
                        a.node_off[a.n_docs] = a.res->aux[0];
                        a.br_off[a.n_docs] = a.res->aux[6];
                    }
                }
            }
        }
        __syncthreads();
        if (FUSED) tp = s_tp;
        // ---- the tile's token spans, copied into shared memory (past the node owners)
        // while the positions and brackets are processed; the node windows read them there
        uint32_t* s_span = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(s_own) + 2 * EX_WIN);
        long long sp_lo = 0;
        uint32_t sp_n = 0;
        if (!FUSED && a.span_cap > 0 && !a.shard &&
            ((reinterpret_cast<uintptr_t>(a.pstart) | reinterpret_cast<uintptr_t>(a.pend)) & 15) == 0) {
            const long long lo = (long long)(s_slo & ~3u), hi = min((long long)s_shi, a.L);
            if (hi > lo && ((hi - lo + 3) & ~3ll) <= (long long)a.span_cap) {  // the same in every thread
                sp_lo = lo;
                sp_n = (uint32_t)(hi - lo);
                const uint32_t chunks = (sp_n + 3) / 4;
                for (uint32_t c = tid; c < 2 * chunks; c += PP_THREADS) {
                    const bool e = c >= chunks;
                    const uint32_t cc = e ? c - chunks : c;
                    const long long idx = lo + 4 * (long long)cc;
                    ex_cp16(s_span + (e ? a.span_cap : 0) + 4 * cc, (e ? a.pend : a.pstart) + idx,
                            (uint32_t)min(16ll, 4 * (a.L - idx)));
                }
                ex_cp_commit();
            }
        }
        // ---- per position: records and the one-position document rules --------
        uint32_t nof[PP_ITEMS], cnt[PP_ITEMS];  // first node (tile-local), n_prod
        // brackets: the depth before each position and where its kept brackets go
        uint32_t kof[PP_ITEMS];
        int32_t depj[PP_ITEMS];
        {
            PosSums run = ps_join<ONE>(ps_join<ONE>(tp, s_w[warp]), ex);  // before this thread's first position
#pragma unroll
            for (int j = 0; j < PP_ITEMS; ++j) {
                const long long i = i0 + j;
                const int pl = tid * PP_ITEMS + j;
                nof[j] = run.nodes - tp.nodes;
                cnt[j] = 0;
                kof[j] = 0;
                depj[j] = 0;
                if (i < a.L) {
                    const bool head = (hm >> j) & 1u;
                    // (one document: every sum before position 0 is zero, the last ⊢ is position 0)
                    const int32_t dep = (head && !ONE) ? 0 : run.depth;
                    const long long doc = ONE ? 0 : (long long)run.heads + (head ? 1 : 0) - 1;
                    const bool dok = ONE || (doc >= 0 && doc < a.n_docs);
                    depj[j] = dep;
                    // the previous position's top lefts against this position's first rights
                    const uint32_t pid_prev = j == 0 ? prev_id : (uint32_t)ids[j - 1];
                    const uint32_t m = cl[j];
                    if (m) {
                        const PairInfo pa = s_pi[pid_prev], pb = s_pi[ids[j]];
                        bool bad = false;
                        for (uint32_t t = 0; t < m; ++t)
                            bad |= ((s_srec[pa.stack_begin + pa.n_br - 1 - t].x ^ s_srec[pb.stack_begin + t].x) &
                                    0x7fffffffu) != 0;
                        if (bad && dok) a.doc_valid[doc] = 0;  // a right and its left differ
                    }
                    // brackets kept before this position's: all before it, less both sides of
                    // every closed pair before it, less the lefts it closes here
                    kof[j] = run.brs - 2u * run.cls - m;
                    if (head && dok) {
                        a.node_off[doc] = (long long)run.nodes;
                        a.br_off[doc] = (long long)kof[j];
                    }
                    PosSums e;
                    possums_zero(e);
                    if (ids[j] == NO_PAIR) {
                        if (dok) a.doc_valid[doc] = 0;  // no admissible pair
                    } else {
                        const PairInfo pi = s_pi[ids[j]];
                        s_pos[ex_slot(pl)] =
                            ONE ? make_int4((int32_t)pi.prod_begin - (int32_t)nof[j], run.v, (int32_t)(1u + run.terms), dep)
                                : make_int4((int32_t)pi.prod_begin - (int32_t)nof[j], head ? 0 : run.v,
                                            (int32_t)((uint32_t)(head ? i : run.hpos) + 1u + (head ? 0u : run.terms)),
                                            dep);
                        if (dep + (int32_t)pi.min_ds < 0 && dok) a.doc_valid[doc] = 0;  // depth below zero
                        e.nodes = pi.n_prod; e.brs = pi.n_br; e.depth = pi.d_depth; e.v = pi.d_v; e.terms = pi.n_term;
                        cnt[j] = (uint32_t)pi.n_prod | ((uint32_t)pi.n_br << 16);
                    }
                    if (((em >> j) & 1u) && (dep + e.depth != 0) && dok) a.doc_valid[doc] = 0;  // unbalanced at the end
                    if (head && !ONE) { e.heads = 1; e.hpos = (int32_t)i; }
                    e.cls = m;
                    run = ps_join<ONE>(run, e);
                }
            }
        }
        // ---- the kept brackets, each position's by its own thread
#pragma unroll
        for (int j = 0; j < PP_ITEMS; ++j) {
            const uint32_t nb = cnt[j] >> 16;
            if (nb) {
                const PairInfo pi = s_pi[ids[j]];
                const uint32_t hi = nb - cl[j + 1];
                for (uint32_t r = cl[j]; r < hi; ++r) {
                    const uint2 rec = s_srec[pi.stack_begin + r];
                    const int32_t before = depj[j] + (int32_t)(int16_t)(rec.y & 0xffffu);
                    const long long g = (long long)kof[j] + (r - cl[j]) - (a.shard ? a.br_base : 0);
                    if (g >= 0 && g < a.cap_brs) {
                        a.brbuf[g] = rec.x;
                        a.dsbuf[g] = (rec.x >> 31) ? before : before - 1;  // after a right bracket, before a left
                    }
                }
            }
        }
        const uint32_t tn = s_tn;
        if (sp_n) ex_cp_wait_all();  // this thread's span copies; the window barrier publishes them
        // ---- nodes, one window at a time ---------------------------------------------
        for (uint32_t w0 = 0; w0 < tn; w0 += EX_WIN) {
            const uint32_t wn = min(tn - w0, (uint32_t)EX_WIN);
#pragma unroll
            for (int j = 0; j < PP_ITEMS; ++j) {
                const uint32_t b = nof[j], n = cnt[j] & 0xffffu;
                const uint32_t lo = max(b, w0), hi = min(b + n, w0 + wn);
                for (uint32_t x = lo; x < hi; ++x) s_own[x - w0] = (uint16_t)(tid * PP_ITEMS + j);
            }
            __syncthreads();
            for (uint32_t e0 = tid; e0 < wn; e0 += EX_U * PP_THREADS) {
                uint32_t tg[EX_U], kd[EX_U];
                long long gi[EX_U];
                int32_t vv[EX_U];
                int64_t st[EX_U], en[EX_U];
#pragma unroll
                for (int u = 0; u < EX_U; ++u) {
                    const uint32_t e = e0 + u * PP_THREADS;
                    tg[u] = 0; kd[u] = 0; vv[u] = 0; st[u] = 0; en[u] = 0; gi[u] = -1;
                    if (e < wn) {
                        const uint32_t g = w0 + e;
                        const int4 ps = s_pos[ex_slot(s_own[e])];
                        const uint2 rec = s_prec[(int32_t)g + ps.x];
                        const uint32_t tm1 = rec.x >> 16;  // terminal + 1, 0: not a terminal production
                        vv[u] = ps.y + (int32_t)(int16_t)(rec.y & 0xffffu);
                        tg[u] = rec.x & 0xffffu;
                        gi[u] = (long long)tp.nodes + g - (a.shard ? a.node_base : 0);
                        if (tm1 && a.subst_terminals) {
                            // the k-th terminal production of a document takes its k-th token's span
                            tg[u] = tm1 - 1;
                            kd[u] = 1;
                            const long long ti = (long long)((uint32_t)ps.z + (rec.y >> 16)) - (a.shard ? a.pos_base : 0);
                            const long long d = ti - sp_lo;
                            if (d >= 0 && d < (long long)sp_n) {
                                st[u] = s_span[d];
                                en[u] = s_span[a.span_cap + d];
                            } else if (ti >= 0 && ti < a.L) {
                                st[u] = __ldg(&a.pstart[ti]);
                                en[u] = __ldg(&a.pend[ti]);
                            }
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < EX_U; ++u) {
                    if (gi[u] >= 0 && gi[u] < a.cap_nodes) {
                        const size_t g = gi[u];
                        a.vbuf[g] = vv[u];
                        a.tag[g] = tg[u];
                        a.kind[g] = (uint8_t)kd[u];
                        a.nstart[g] = st[u];
                        a.nend[g] = en[u];
                    }
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// K3: previous smaller-or-equal inside a tile
// ---------------------------------------------------------------------------
struct PleArgs {
    const int32_t* val;          // [n] values
    long long n;
    const uint32_t* sym;         // brackets: symbol|left<<31 (queries only at rights); nodes: null
    long long* out_parent;       // nodes: parent index relative to its document (root 0)
    const long long* seg_off;    // [n_seg + 1] first element of each document
    long long n_seg;
    uint8_t* seg_valid;          // brackets: cleared for a document with a mismatch
    int32_t* tile_min;           // [tiles]
    int32_t* stair_val;          // [tiles * tile elements]
    uint32_t* stair_idx;         // [tiles * tile elements] global index
    int32_t* stair_len;          // [tiles]
    unsigned long long* esc;     // escapees: index << 32 | (uint32)value
    unsigned int* esc_count;
    long long esc_cap;
    AlpResult* res;
    const long long* dn;         // when set: the element count, in device memory (n is then its capacity)
    long long out_off;           // nodes: added to every parent written (a shard's global node numbering)
    unsigned long long* xq;      // when set (a shard): elements with no answer in the shard, index << 32 | value,
    unsigned int* xq_count;      //   for the shards before it to answer
    long long xq_cap;
};

// Shared memory: the tile's values and a second array (bracket symbols, or
// node results) with one pad word after every thread's PI elements, so that a
// warp reading element k of its threads' chunks hits 32 different banks; the
// minima of each chunk's quarters; a min tree over the PT chunk minima (leaves
// at PT..2*PT-1); a query queue per warp.
// PT threads with PI elements each (PI a multiple of 4): one tile of PT * PI.
__host__ __device__ constexpr size_t ple_smem(int PT, int PI) {
    return (size_t)(2 * PT * (PI + 1) + 2 * PT) * 4 + (size_t)PT * (PI / 4) * 4 + (size_t)PT * PI * 2;
}

// largest d in [lo, hi] with off[d] <= g
__device__ __forceinline__ long long seg_upper(const long long* off, long long lo, long long hi, long long g) {
    while (lo < hi) {
        const long long mid = (lo + hi + 1) >> 1;
        if (off[mid] <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <int PI>
__device__ __forceinline__ int ple_pad(int e) { return (e / PI) * (PI + 1) + (e % PI); }

// Each thread owns PI consecutive elements.  An element's answer is
// (1) its thread's last earlier element <= x (branch-free compares in
// registers), else (2) the last element <= x in the nearest earlier chunk
// whose minimum is <= x: a per-warp queue of these queries runs 32 at a time
// through one copy of the search (min tree up and down, then the chunk's
// quarter minima, then four elements), else (3) in an earlier tile:
// ple_escape_kernel.  Node parents are staged in shared memory and written
// with coalesced stores.
template <int PT, int PI>
__global__ void __launch_bounds__(PT, 1024 / PT) ple_tile_kernel(PleArgs a) {
    static_assert(PI % 4 == 0 && PT % 32 == 0 && PT * PI <= 65536, "tile shape");
    constexpr int NQ = PI / 4;  // quarters of four elements
    extern __shared__ __align__(16) uint8_t smem[];
    int32_t* s_val = reinterpret_cast<int32_t*>(smem);                        // [PT * (PI + 1)]
    int32_t* s_aux = s_val + PT * (PI + 1);                         // symbols / results
    int32_t* tree = s_aux + PT * (PI + 1);                          // [2 * PT]
    int32_t* s_sub = tree + 2 * PT;                                   // [PT][NQ] quarter minima
    uint16_t* s_q = reinterpret_cast<uint16_t*>(s_sub + PT * NQ);     // [(PT * PI)] query queues
    __shared__ int32_t s_suf[PT];
    __shared__ int32_t s_wm[PT / 32];
    __shared__ uint32_t s_cnt[PT / 32];
    __shared__ long long s_sd0, s_sd1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long base = (long long)blockIdx.x * (PT * PI);
    if (a.dn) {
        a.n = min(a.n, *a.dn);
        if (base >= a.n) return;  // the grid covers the capacity
    }
    const bool brackets = a.sym != nullptr;
    const long long gfirst = base + (long long)tid * PI;
    const int lim = (int)max(0ll, min((long long)PI, a.n - gfirst));  // valid elements of this thread

    // ---- this thread's values (and symbols) --------------------------------
    int32_t v[PI];
    if (lim == PI) {
        const int4* src = reinterpret_cast<const int4*>(a.val + gfirst);
#pragma unroll
        for (int q = 0; q < PI / 4; ++q) {
            const int4 x = __ldg(src + q);
            v[4 * q] = x.x; v[4 * q + 1] = x.y; v[4 * q + 2] = x.z; v[4 * q + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < PI; ++i) v[i] = i < lim ? a.val[gfirst + i] : INT32_MAX;
    }
#pragma unroll
    for (int i = 0; i < PI; ++i) s_val[tid * (PI + 1) + i] = v[i];
    if (brackets) {
        if (lim == PI) {
            const uint4* src = reinterpret_cast<const uint4*>(a.sym + gfirst);
#pragma unroll
            for (int q = 0; q < PI / 4; ++q) {
                const uint4 x = __ldg(src + q);
                s_aux[tid * (PI + 1) + 4 * q] = (int32_t)x.x;
                s_aux[tid * (PI + 1) + 4 * q + 1] = (int32_t)x.y;
                s_aux[tid * (PI + 1) + 4 * q + 2] = (int32_t)x.z;
                s_aux[tid * (PI + 1) + 4 * q + 3] = (int32_t)x.w;
            }
        } else {
#pragma unroll
            for (int i = 0; i < PI; ++i) s_aux[tid * (PI + 1) + i] = i < lim ? (int32_t)a.sym[gfirst + i] : 0;
        }
    }
    if (tid == 0) {
        s_sd0 = seg_upper(a.seg_off, 0, a.n_seg - 1, base);
        s_sd1 = seg_upper(a.seg_off, 0, a.n_seg - 1, min(base + (PT * PI), a.n) - 1);
    }
    int32_t cm = INT32_MAX;
#pragma unroll
    for (int qq = 0; qq < NQ; ++qq) {
        const int32_t m = min(min(v[4 * qq], v[4 * qq + 1]), min(v[4 * qq + 2], v[4 * qq + 3]));
        s_sub[tid * NQ + qq] = m;
        cm = min(cm, m);
    }

    // ---- min tree over chunk minima: warp levels by shuffles, top by thread 0
    {
        int32_t m = cm;
        int node = PT + tid;
        tree[node] = m;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            m = min(m, __shfl_xor_sync(ALP_FULL_MASK, m, d));
            node >>= 1;
            if ((lane & (2 * d - 1)) == 0) tree[node] = m;
        }
    }
    __syncthreads();
    if (tid == 0) {
        for (int node = PT / 32 - 1; node >= 1; --node) tree[node] = min(tree[2 * node], tree[2 * node + 1]);
    }
    __syncthreads();
    const long long sd0 = s_sd0, sd1 = s_sd1;

    // ---- (1) answers inside the thread ---------------------------------------
    long long doc = lim > 0 ? seg_upper(a.seg_off, sd0, sd1, gfirst) : 0;
    long long dbase = lim > 0 ? a.seg_off[doc] : 0;
    long long dnext = lim > 0 ? a.seg_off[doc + 1] : 0;
    uint32_t unres = 0;
#pragma unroll
    for (int j = 0; j < PI; ++j) {
        if (j < lim) {
            const long long g = gfirst + j;
            while (sd0 != sd1 && g >= dnext && doc + 1 < a.n_seg) {  // (a tile in one document: never)
                ++doc;
                dbase = a.seg_off[doc];
                dnext = a.seg_off[doc + 1];
            }
            const int e = tid * PI + j;
            int ans = -1;
#pragma unroll
            for (int i = 0; i < j; ++i) ans = v[i] <= v[j] ? tid * PI + i : ans;
            if (brackets) {
                const uint32_t my_sym = (uint32_t)s_aux[tid * (PI + 1) + j];
                if (!(my_sym >> 31)) {  // rights ask; lefts do not
                    if (ans >= 0) {
                        const uint32_t l = (uint32_t)s_aux[tid * (PI + 1) + (ans - tid * PI)];
                        if (base + ans < dbase || (l & 0x7fffffffu) != (my_sym & 0x7fffffffu) || !(l >> 31)) {
                            a.seg_valid[doc] = 0;
                        }
                    } else {
                        unres |= 1u << j;
                    }
                }
            } else {
                int32_t r = 0;  // a document's root: parent 0
                if (g != dbase) {
                    if (ans >= 0) r = (int32_t)(base + ans - dbase);
                    else unres |= 1u << j;
                }
                s_aux[tid * (PI + 1) + j] = r;
                (void)e;
            }
        }
    }

    // ---- (2) the warp's remaining queries, 32 at a time -----------------------
    {
        const uint32_t cnt = __popc(unres);
        const uint32_t incl = warp_scan_add(cnt, lane);
        const uint32_t total = __shfl_sync(ALP_FULL_MASK, incl, 31);
        uint16_t* q = s_q + warp * (32 * PI);
        uint32_t o = incl - cnt;
        for (uint32_t m = unres; m; m &= m - 1) q[o++] = (uint16_t)(tid * PI + __ffs(m) - 1);
        __syncwarp();
        for (uint32_t qb = 0; qb < total; qb += 32) {
            if (qb + lane < total) {
                const int e = q[qb + lane];
                const int32_t x = s_val[ple_pad<PI>(e)];
                const long long g = base + e;
                // the nearest earlier chunk with minimum <= x: the few chunks just
                // before the element's first (most answers are near), then the tree
                const int ce = e / PI;
                // the four chunk minima read at once (clamped indices), the nearest fitting one kept
                int32_t near[4];
#pragma unroll
                for (int back = 1; back <= 4; ++back) near[back - 1] = tree[PT + max(ce - back, 0)];
                int c = -1;
#pragma unroll
                for (int back = 4; back >= 1; --back)
                    if (ce - back >= 0 && near[back - 1] <= x) c = ce - back;
                bool found = c >= 0;
                if (!found && ce > 4) {
                    int node = PT + ce - 4;  // chunks left of those
                    while (node > 1) {
                        if ((node & 1) && tree[node - 1] <= x) { node = node - 1; found = true; break; }
                        node >>= 1;
                    }
                    if (found) {
                        while (node < PT) node = (tree[2 * node + 1] <= x) ? 2 * node + 1 : 2 * node;
                        c = node - PT;
                    }
                }
                const long long dq = sd0 == sd1 ? sd0 : seg_upper(a.seg_off, sd0, sd1, g);
                const long long dqb = a.seg_off[dq];
                if (found) {
                    int qq = 0;
#pragma unroll
                    for (int t2 = 1; t2 < NQ; ++t2)
                        if (s_sub[c * NQ + t2] <= x) qq = t2;
                    const int32_t* cv = s_val + c * (PI + 1) + 4 * qq;
                    const int k = cv[3] <= x ? 3 : (cv[2] <= x ? 2 : (cv[1] <= x ? 1 : 0));
                    const int ans = c * PI + 4 * qq + k;
                    if (brackets) {
                        const uint32_t l = (uint32_t)s_aux[ple_pad<PI>(ans)];
                        const uint32_t r = (uint32_t)s_aux[ple_pad<PI>(e)];
                        if (base + ans < dqb || (l & 0x7fffffffu) != (r & 0x7fffffffu) || !(l >> 31)) {
                            a.seg_valid[dq] = 0;
                        }
                    } else {
                        s_aux[ple_pad<PI>(e)] = (int32_t)(base + ans - dqb);
                    }
                } else {
                    const unsigned int slot = atomicAdd(a.esc_count, 1u);
                    if ((long long)slot < a.esc_cap) a.esc[slot] = ((unsigned long long)g << 32) | (uint32_t)x;
                    else atomicOr(&a.res->error, ALP_DEV_ERR_CAPACITY);
                }
            }
        }
    }
    __syncthreads();

    // ---- node parents, coalesced --------------------------------------------------
    if (!brackets) {
        for (int e = tid; e < (PT * PI); e += PT) {
            const long long g = base + e;
            if (g < a.n) a.out_parent[g] = (long long)s_aux[ple_pad<PI>(e)] + a.out_off;
        }
    }

    // ---- tile minimum and staircase of suffix minima (values strictly below every later one)
    s_suf[tid] = cm;
    __syncthreads();
    int32_t after;
    {
        int32_t y = s_suf[PT - 1 - tid];  // reversed order
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int32_t o = __shfl_up_sync(ALP_FULL_MASK, y, d);
            if (lane >= d) y = min(y, o);
        }
        if (lane == 31) s_wm[warp] = y;
        __syncthreads();
        int32_t pre = INT32_MAX;
        for (int w = 0; w < warp; ++w) pre = min(pre, s_wm[w]);
        y = min(y, pre);
        s_suf[PT - 1 - tid] = y;  // s_suf[t] = min over threads t..end
        __syncthreads();
        after = tid + 1 < PT ? s_suf[tid + 1] : INT32_MAX;
    }
    uint32_t flags = 0;
    int32_t run = after;
#pragma unroll
    for (int i = PI - 1; i >= 0; --i) {
        if (i < lim && v[i] < run) flags |= 1u << i;
        run = min(run, v[i]);
    }
    const uint32_t cnt = __popc(flags);
    const uint32_t incl = warp_scan_add(cnt, lane);
    if (lane == 31) s_cnt[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0, total = 0;
    for (int w = 0; w < PT / 32; ++w) {
        if (w < warp) wpre += s_cnt[w];
        total += s_cnt[w];
    }
    uint32_t o = wpre + incl - cnt;
    const long long sbase = (long long)blockIdx.x * (PT * PI);
#pragma unroll
    for (int i = 0; i < PI; ++i) {
        if (flags & (1u << i)) {
            a.stair_val[sbase + o] = v[i];
            a.stair_idx[sbase + o] = (uint32_t)(gfirst + i);
            ++o;
        }
    }
    if (tid == 0) {
        a.stair_len[blockIdx.x] = (int32_t)total;
        a.tile_min[blockIdx.x] = tree[1];
    }
}

// Level-1/2 minima over groups of 32 / 1024 tiles.
// Thread g: the minimum of tiles [32g, 32g + 32); lane 0 of each warp: the minimum of
// its 32 lanes' groups, tiles [1024w, 1024w + 1024) (warps hold 32 consecutive groups).
__global__ void tile_min_levels_kernel(const int32_t* tmin, long long tiles, int32_t* m32, int32_t* m1024,
                                       const long long* dn, int tile) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (dn) tiles = min(tiles, (*dn + tile - 1) / tile);  // tiles is then the capacity
    const long long n32 = (tiles + 31) / 32;
    int32_t m = INT32_MAX;
    if (g < n32) {
#pragma unroll 8
        for (int k = 0; k < 32; ++k) {
            const long long t = g * 32 + k;
            if (t < tiles) m = min(m, __ldg(&tmin[t]));
        }
        m32[g] = m;
    }
    m = __reduce_min_sync(ALP_FULL_MASK, m);
    if ((threadIdx.x & 31) == 0 && g / 32 < (tiles + 1023) / 1024) m1024[g / 32] = m;
}

// Nearest tile before `t` whose minimum is <= x, or -1.
__device__ __forceinline__ long long prev_tile_leq(const int32_t* tmin, const int32_t* m32, const int32_t* m1024,
                                                   long long t, int32_t x) {
    long long u = t - 1;
    // within the 32-group of t
    while (u >= 0 && (u & 31) != 31) {
        if (tmin[u] <= x) return u;
        --u;
    }
    if (u < 0) return -1;
    long long g = (u + 1) / 32 - 1;  // group index of u (u is the last tile of its group)
    // groups within the current 1024-block
    while (g >= 0 && (g & 31) != 31) {
        if (m32[g] <= x) break;
        --g;
    }
    if (g >= 0 && (g & 31) == 31 && m32[g] > x) {
        long long h = (g + 1) / 32 - 1;
        while (h >= 0 && m1024[h] > x) --h;
        if (h < 0) return -1;
        g = h * 32 + 31;
        while (m32[g] > x) --g;
    }
    if (g < 0) return -1;
    u = g * 32 + 31;
    while (tmin[u] > x) --u;
    return u;
}

struct EscArgs {
    const unsigned long long* esc;
    const unsigned int* esc_count;
    long long esc_cap;
    const int32_t* tile_min;
    const int32_t* m32;
    const int32_t* m1024;
    const int32_t* stair_val;
    const uint32_t* stair_idx;
    const int32_t* stair_len;
    const uint32_t* sym;         // brackets mode when non-null
    long long* out_parent;       // nodes mode
    const long long* seg_off;
    long long n_seg;
    uint8_t* seg_valid;
    AlpResult* res;
    int tile;                    // elements per tile
    long long out_off;           // as PleArgs
    unsigned long long* xq;
    unsigned int* xq_count;
    long long xq_cap;
};

__global__ void ple_escape_kernel(EscArgs a) {
    const long long cnt = min((long long)*a.esc_count, a.esc_cap);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += (long long)gridDim.x * blockDim.x) {
        const unsigned long long r = a.esc[e];
        const long long g = (long long)(r >> 32);
        const int32_t x = (int32_t)(uint32_t)r;
        const long long t = g / a.tile;
        const long long u = prev_tile_leq(a.tile_min, a.m32, a.m1024, t, x);
        long long ans = -1;
        if (u >= 0) {
            const int32_t* sv = a.stair_val + u * a.tile;
            int lo = 0, hi = a.stair_len[u] - 1;  // largest k with sv[k] <= x (values ascend)
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (sv[mid] <= x) lo = mid; else hi = mid - 1;
            }
            ans = a.stair_idx[u * a.tile + lo];
        }
        const long long doc = seg_upper(a.seg_off, 0, a.n_seg - 1, g);
        const long long dbase = a.seg_off[doc];
        if (ans < 0 && a.xq) {
            // a shard: the answer lies in a shard before this one
            const unsigned int slot = atomicAdd(a.xq_count, 1u);
            if ((long long)slot < a.xq_cap) a.xq[slot] = r;
            else atomicOr(&a.res->error, ALP_DEV_ERR_CAPACITY);
            if (!a.sym) a.out_parent[g] = -1;
        } else if (a.sym) {
            if (ans < dbase) {
                a.seg_valid[doc] = 0;
            }
            else {
                const uint32_t l = a.sym[ans], rr = a.sym[g];
                if (!(l >> 31) || (l & 0x7fffffffu) != (rr & 0x7fffffffu)) a.seg_valid[doc] = 0;
            }
        } else {
            a.out_parent[g] = ans < 0 ? -1 : ans - dbase + a.out_off;
        }
    }
}

// ---------------------------------------------------------------------------
// Shards of one document (alp_parse_shard_*): cross-shard previous-smaller-or-equal
// ---------------------------------------------------------------------------
// A shard's staircase: the elements strictly smaller than every element after
// them in the shard, left to right (so ascending values).  Built from the
// tiles' staircases: tile t contributes the first of its entries that lie
// below the minimum of every later tile.  One CTA; `scratch` holds a count per
// tile.  Nodes take a global index (local + idx_off), brackets their symbol.
__global__ void __launch_bounds__(1024) shard_stair_kernel(const int32_t* tile_min, const int32_t* stair_val,
                                                           const uint32_t* stair_idx, const int32_t* stair_len,
                                                           long long tiles, int tile, const uint32_t* sym,
                                                           long long idx_off, int32_t* scratch, int32_t* out_val,
                                                           long long* out_idx, uint32_t* out_sym, long long* out_len) {
    __shared__ int32_t s_w[32];
    __shared__ long long s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int32_t carry = INT32_MAX;  // minimum of the tiles after the current chunk
    for (long long c0 = ((tiles - 1) / 1024) * 1024; c0 >= 0; c0 -= 1024) {
        const long long t = c0 + tid;
        int32_t x = t < tiles ? tile_min[t] : INT32_MAX;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {  // x = minimum over this lane and the lanes after it
            const int32_t o = __shfl_down_sync(ALP_FULL_MASK, x, d);
            if (lane + d < 32) x = min(x, o);
        }
        if (lane == 0) s_w[warp] = x;
        __syncthreads();
        int32_t after = carry, chunk = INT32_MAX;
        for (int w2 = 0; w2 < 32; ++w2) {
            if (w2 > warp) after = min(after, s_w[w2]);
            chunk = min(chunk, s_w[w2]);
        }
        int32_t ex = __shfl_down_sync(ALP_FULL_MASK, x, 1);
        if (lane == 31) ex = INT32_MAX;
        const int32_t below = min(ex, after);  // minimum of every tile after t
        if (t < tiles) {
            const int32_t* sv = stair_val + t * (long long)tile;
            int lo = 0, hi = stair_len[t];  // first entry not below `below` (entries ascend)
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (sv[mid] < below) lo = mid + 1; else hi = mid;
            }
            scratch[t] = lo;
        }
        carry = min(carry, chunk);
        __syncthreads();
    }
    if (tid == 0) s_base = 0;
    __syncthreads();
    for (long long c0 = 0; c0 < tiles; c0 += 1024) {
        const long long t = c0 + tid;
        const uint32_t cnt = t < tiles ? (uint32_t)scratch[t] : 0u;
        const uint32_t incl = warp_scan_add(cnt, lane);
        if (lane == 31) s_w[warp] = (int32_t)incl;
        __syncthreads();
        uint32_t wpre = 0, total = 0;
        for (int w2 = 0; w2 < 32; ++w2) {
            if (w2 < warp) wpre += (uint32_t)s_w[w2];
            total += (uint32_t)s_w[w2];
        }
        const long long o = s_base + wpre + incl - cnt;
        for (uint32_t k = 0; k < cnt; ++k) {
            const long long src = t * (long long)tile + k;
            const uint32_t ix = stair_idx[src];
            out_val[o + k] = stair_val[src];
            if (out_idx) out_idx[o + k] = (long long)ix + idx_off;
            if (out_sym) out_sym[o + k] = sym[ix];
        }
        __syncthreads();
        if (tid == 0) s_base += total;
        __syncthreads();
    }
    if (tid == 0) *out_len = s_base;
}

// Answers from the shards before this one for the elements that found none
// inside it (xq: index << 32 | value): the nearest earlier shard whose
// staircase starts at or below the value, and in it the last entry at or
// below the value (futhark/parser.fut:72-108 over the whole document).
// Nodes get that entry's global index as parent; a right bracket's entry must
// be a left of its symbol (futhark/parser.fut:168-184), else the document is
// rejected.
__global__ void shard_resolve_kernel(const unsigned long long* xq, const unsigned int* xq_count, long long xq_cap,
                                     int n_prev, const long long* prev_off, const int32_t* pval,
                                     const long long* pidx, const uint32_t* psym, long long* out_parent,
                                     const uint32_t* sym, uint8_t* valid) {
    const long long cnt = min((long long)*xq_count, xq_cap);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt;
         e += (long long)gridDim.x * blockDim.x) {
        const unsigned long long r = xq[e];
        const long long g = (long long)(r >> 32);
        const int32_t x = (int32_t)(uint32_t)r;
        long long ans = -1;
        for (int rk = n_prev - 1; rk >= 0 && ans < 0; --rk) {
            long long lo = prev_off[rk], hi = prev_off[rk + 1] - 1;
            if (hi < lo || pval[lo] > x) continue;
            while (lo < hi) {  // last entry at or below x
                const long long mid = (lo + hi + 1) >> 1;
                if (pval[mid] <= x) lo = mid; else hi = mid - 1;
            }
            ans = lo;
        }
        if (sym) {
            if (ans < 0) {
                valid[0] = 0;
            } else {
                const uint32_t l = psym[ans], rr = sym[g];
                if (!(l >> 31) || (l & 0x7fffffffu) != (rr & 0x7fffffffu)) valid[0] = 0;
            }
        } else {
            out_parent[g] = ans < 0 ? -1 : pidx[ans];
        }
    }
}

// A shard's positions: its tokens, with ⊢ before them on the document's first
// shard and ⊣ after them on its last (spans stay the document's).
__global__ void shard_positions_kernel(const uint32_t* term, const int64_t* ts, const int64_t* te, long long m,
                                       int first, int last, uint16_t* P, uint32_t* s32, uint32_t* e32, uint32_t sl,
                                       uint32_t sr, AlpResult* res) {
    const long long L = m + first + last;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L; i += (long long)gridDim.x * blockDim.x) {
        if ((first && i == 0) || (last && i == L - 1)) {
            P[i] = (uint16_t)(first && i == 0 ? sl : sr);
            s32[i] = 0;
            e32[i] = 0;
            continue;
        }
        const long long k = i - first;
        const uint32_t t = term[k];
        if (t > 0xffffu || t == sl || t == sr) res->valid = 0;
        P[i] = (uint16_t)t;
        s32[i] = (uint32_t)ts[k];
        e32[i] = (uint32_t)te[k];
    }
}

}  // namespace alp
