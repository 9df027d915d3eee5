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
    uint16_t pad;
};

struct ParseTables {
    const uint16_t* key_index;  // [T^(q+k)] pair id, 0xffff = no pair
    const PairInfo* pairs;      // [n_pairs]
    const uint32_t* stack;      // symbol | left<<31
    const uint32_t* pseq;       // production ids
    const int32_t* arity;       // [n_prods]
    const int32_t* prod_term;   // [n_prods] terminal id or -1
    int q, k, T, n_pairs, n_prods;
    uint32_t empty, start, end;
};

struct ParseHost {
    int q = 0, k = 0, n_terms = 0, n_prods = 0, n_pairs = 0, max_prods = 0, max_brackets = 0;
    long long key_space = 0;
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
        pi.pad = 0;
        if ((int)pi.n_prod > maxp) maxp = pi.n_prod;
        if ((int)pi.n_br > maxb) maxb = pi.n_br;
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
              up(pterm.data(), pterm.size() * 4, (const void**)&pt.prod_term);
    if (!ok) { err = "cudaMalloc/cudaMemcpy failed for parser tables"; return 2; }
    pt.q = (int)q; pt.k = (int)k; pt.T = (int)T; pt.n_pairs = (int)n_pairs; pt.n_prods = (int)n_prods;
    pt.empty = empty; pt.start = start; pt.end = end;
    ph.q = (int)q; ph.k = (int)k; ph.n_terms = (int)n_terms; ph.n_prods = (int)n_prods; ph.n_pairs = (int)n_pairs;
    ph.max_prods = maxp; ph.max_brackets = maxb; ph.key_space = space;
    return 0;
}

}  // namespace alp

namespace alp {

constexpr int PP_THREADS = 256;
constexpr int PP_ITEMS = 8;                        // positions per thread
constexpr int PP_TILE = PP_THREADS * PP_ITEMS;     // positions per tile
constexpr int PLE_THREADS = 256;
constexpr int PLE_ITEMS = 16;
constexpr int PLE_TILE = PLE_THREADS * PLE_ITEMS;  // elements per tile
constexpr uint16_t NO_PAIR = 0xffff;

// Per-tile sums of the per-position counts (and, after the scan, the
// exclusive prefixes).  Field order is the scan order.
struct __align__(16) PosSums {
    unsigned long long nodes;   // productions
    unsigned long long brs;     // brackets
    long long depth;            // lefts - rights
    long long v;                // sum of (arity - 1)
    unsigned long long terms;   // terminal productions
    unsigned long long pad[3];
};

__device__ __forceinline__ void possums_zero(PosSums& s) {
    s.nodes = 0; s.brs = 0; s.depth = 0; s.v = 0; s.terms = 0;
}

struct ParseArgs {
    ParseTables t;
    const uint16_t* tterm;      // [m] token terminal ids
    const uint32_t* tstart;     // [m]
    const uint32_t* tend;       // [m]
    long long m;                // tokens
    long long L;                // positions = m + 2
    uint16_t* pid;              // [L] pair id per position
    PosSums* tile_sums;         // [tiles] K1 output, scanned in place to exclusive prefixes
    AlpResult* res;             // valid flag, error bits; aux[0..4] totals
    // K2 outputs
    int subst_terminals;
    uint32_t* tag;
    uint8_t* kind;
    int64_t* nstart;
    int64_t* nend;
    int32_t* vbuf;              // node values exscan(arity-1)
    uint32_t* brbuf;            // bracket symbol | left<<31
    int32_t* dsbuf;             // bracket depth value (before a left, after a right)
    long long cap_nodes;
    long long cap_brs;
};

// Terminal symbol at padded position i of ⊢ tokens ⊣ (empty outside).
__device__ __forceinline__ uint32_t pos_term(const ParseArgs& a, long long i) {
    if (i < 0 || i >= a.L) return a.t.empty;
    if (i == 0) return a.t.start;
    if (i == a.L - 1) return a.t.end;
    return a.tterm[i - 1];
}

// ---------------------------------------------------------------------------
// K1: pair ids and per-tile sums
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(PP_THREADS) parse_pairs_kernel(ParseArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    PairInfo* s_pi = reinterpret_cast<PairInfo*>(smem);
    uint32_t* s_term = reinterpret_cast<uint32_t*>(smem + sizeof(PairInfo) * a.t.n_pairs);
    __shared__ PosSums s_w[PP_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = a.t.q, k = a.t.k, W = q + k, T = a.t.T;
    for (int i = tid; i < a.t.n_pairs * (int)(sizeof(PairInfo) / 4); i += PP_THREADS)
        reinterpret_cast<uint32_t*>(s_pi)[i] = reinterpret_cast<const uint32_t*>(a.t.pairs)[i];
    const long long base = (long long)blockIdx.x * PP_TILE;
    const int span = PP_TILE + W;  // window [base - q, base + PP_TILE + k)
    for (int i = tid; i < span; i += PP_THREADS) s_term[i] = pos_term(a, base - q + i);
    __syncthreads();
    PosSums acc;
    possums_zero(acc);
    bool bad = false;
    uint16_t ids[PP_ITEMS];
#pragma unroll
    for (int j = 0; j < PP_ITEMS; ++j) {
        const long long i = base + tid * PP_ITEMS + j;
        uint16_t p = NO_PAIR;
        if (i < a.L) {
            long long x = 0;
            const int o = tid * PP_ITEMS + j;  // s_term[o + jj] is position i - q + jj
            for (int jj = 0; jj < W; ++jj) x = x * T + s_term[o + jj];
            p = __ldg(&a.t.key_index[x]);
            if (p == NO_PAIR) bad = true;
            else {
                const PairInfo& pi = s_pi[p];
                acc.nodes += pi.n_prod;
                acc.brs += pi.n_br;
                acc.depth += pi.d_depth;
                acc.v += pi.d_v;
                acc.terms += pi.n_term;
            }
        }
        ids[j] = p;
    }
    const long long i0 = base + tid * PP_ITEMS;
    if (i0 + PP_ITEMS <= a.L && ((i0 & 7) == 0)) {
        uint4 w;
        w.x = ids[0] | ((uint32_t)ids[1] << 16);
        w.y = ids[2] | ((uint32_t)ids[3] << 16);
        w.z = ids[4] | ((uint32_t)ids[5] << 16);
        w.w = ids[6] | ((uint32_t)ids[7] << 16);
        *reinterpret_cast<uint4*>(a.pid + i0) = w;
    } else {
        for (int j = 0; j < PP_ITEMS; ++j)
            if (i0 + j < a.L) a.pid[i0 + j] = ids[j];
    }
    if (__any_sync(ALP_FULL_MASK, bad) && lane == 0) a.res->valid = 0;
    // block reduce
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        acc.nodes += __shfl_down_sync(ALP_FULL_MASK, acc.nodes, d);
        acc.brs += __shfl_down_sync(ALP_FULL_MASK, acc.brs, d);
        acc.depth += __shfl_down_sync(ALP_FULL_MASK, acc.depth, d);
        acc.v += __shfl_down_sync(ALP_FULL_MASK, acc.v, d);
        acc.terms += __shfl_down_sync(ALP_FULL_MASK, acc.terms, d);
    }
    if (lane == 0) s_w[warp] = acc;
    __syncthreads();
    if (tid == 0) {
        PosSums t;
        possums_zero(t);
        for (int w = 0; w < PP_THREADS / 32; ++w) {
            t.nodes += s_w[w].nodes; t.brs += s_w[w].brs; t.depth += s_w[w].depth;
            t.v += s_w[w].v; t.terms += s_w[w].terms;
        }
        a.tile_sums[blockIdx.x] = t;
    }
}

// Exclusive scan of the tile sums in place (one block); totals to res->aux.
__global__ void __launch_bounds__(1024) scan_tiles_kernel(PosSums* s, long long tiles, AlpResult* res) {
    __shared__ PosSums s_w[32];
    __shared__ PosSums s_carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) possums_zero(s_carry);
    __syncthreads();
    for (long long b = 0; b < tiles; b += 1024) {
        PosSums v;
        if (b + tid < tiles) v = s[b + tid]; else possums_zero(v);
        PosSums inc = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            unsigned long long n1 = __shfl_up_sync(ALP_FULL_MASK, inc.nodes, d);
            unsigned long long n2 = __shfl_up_sync(ALP_FULL_MASK, inc.brs, d);
            long long n3 = __shfl_up_sync(ALP_FULL_MASK, inc.depth, d);
            long long n4 = __shfl_up_sync(ALP_FULL_MASK, inc.v, d);
            unsigned long long n5 = __shfl_up_sync(ALP_FULL_MASK, inc.terms, d);
            if (lane >= d) { inc.nodes += n1; inc.brs += n2; inc.depth += n3; inc.v += n4; inc.terms += n5; }
        }
        if (lane == 31) s_w[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            PosSums w = s_w[lane];
            PosSums wi = w;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                unsigned long long n1 = __shfl_up_sync(ALP_FULL_MASK, wi.nodes, d);
                unsigned long long n2 = __shfl_up_sync(ALP_FULL_MASK, wi.brs, d);
                long long n3 = __shfl_up_sync(ALP_FULL_MASK, wi.depth, d);
                long long n4 = __shfl_up_sync(ALP_FULL_MASK, wi.v, d);
                unsigned long long n5 = __shfl_up_sync(ALP_FULL_MASK, wi.terms, d);
                if (lane >= d) { wi.nodes += n1; wi.brs += n2; wi.depth += n3; wi.v += n4; wi.terms += n5; }
            }
            // exclusive warp prefix
            PosSums we;
            we.nodes = wi.nodes - w.nodes; we.brs = wi.brs - w.brs; we.depth = wi.depth - w.depth;
            we.v = wi.v - w.v; we.terms = wi.terms - w.terms;
            s_w[lane] = we;
        }
        __syncthreads();
        PosSums c = s_carry, wp = s_w[warp];
        if (b + tid < tiles) {
            PosSums o;
            o.nodes = c.nodes + wp.nodes + inc.nodes - v.nodes;
            o.brs = c.brs + wp.brs + inc.brs - v.brs;
            o.depth = c.depth + wp.depth + inc.depth - v.depth;
            o.v = c.v + wp.v + inc.v - v.v;
            o.terms = c.terms + wp.terms + inc.terms - v.terms;
            o.pad[0] = o.pad[1] = o.pad[2] = 0;
            s[b + tid] = o;
        }
        __syncthreads();
        if (tid == 1023) {
            PosSums nc;
            nc.nodes = c.nodes + wp.nodes + inc.nodes;
            nc.brs = c.brs + wp.brs + inc.brs;
            nc.depth = c.depth + wp.depth + inc.depth;
            nc.v = c.v + wp.v + inc.v;
            nc.terms = c.terms + wp.terms + inc.terms;
            s_carry = nc;
        }
        __syncthreads();
    }
    if (tid == 0) {
        res->aux[0] = (long long)s_carry.nodes;
        res->aux[1] = (long long)s_carry.brs;
        res->aux[2] = s_carry.depth;
        res->aux[3] = s_carry.v;
        res->aux[4] = (long long)s_carry.terms;
    }
}

// ---------------------------------------------------------------------------
// K2: expand every position's productions and brackets
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(PP_THREADS) parse_expand_kernel(ParseArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    PairInfo* s_pi = reinterpret_cast<PairInfo*>(smem);
    int32_t* s_ar = reinterpret_cast<int32_t*>(smem + sizeof(PairInfo) * a.t.n_pairs);
    int32_t* s_pt = s_ar + a.t.n_prods;
    __shared__ PosSums s_w[PP_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < a.t.n_pairs * (int)(sizeof(PairInfo) / 4); i += PP_THREADS)
        reinterpret_cast<uint32_t*>(s_pi)[i] = reinterpret_cast<const uint32_t*>(a.t.pairs)[i];
    for (int i = tid; i < a.t.n_prods; i += PP_THREADS) { s_ar[i] = a.t.arity[i]; s_pt[i] = a.t.prod_term[i]; }
    __syncthreads();
    const long long i0 = (long long)blockIdx.x * PP_TILE + tid * PP_ITEMS;
    uint16_t ids[PP_ITEMS];
#pragma unroll
    for (int j = 0; j < PP_ITEMS; ++j) ids[j] = (i0 + j < a.L) ? a.pid[i0 + j] : NO_PAIR;
    PosSums mine;
    possums_zero(mine);
#pragma unroll
    for (int j = 0; j < PP_ITEMS; ++j) {
        if (ids[j] == NO_PAIR) continue;
        const PairInfo& pi = s_pi[ids[j]];
        mine.nodes += pi.n_prod; mine.brs += pi.n_br; mine.depth += pi.d_depth; mine.v += pi.d_v;
        mine.terms += pi.n_term;
    }
    PosSums inc = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        unsigned long long n1 = __shfl_up_sync(ALP_FULL_MASK, inc.nodes, d);
        unsigned long long n2 = __shfl_up_sync(ALP_FULL_MASK, inc.brs, d);
        long long n3 = __shfl_up_sync(ALP_FULL_MASK, inc.depth, d);
        long long n4 = __shfl_up_sync(ALP_FULL_MASK, inc.v, d);
        unsigned long long n5 = __shfl_up_sync(ALP_FULL_MASK, inc.terms, d);
        if (lane >= d) { inc.nodes += n1; inc.brs += n2; inc.depth += n3; inc.v += n4; inc.terms += n5; }
    }
    if (lane == 31) s_w[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        PosSums w = lane < PP_THREADS / 32 ? s_w[lane] : PosSums{};
        if (lane >= PP_THREADS / 32) possums_zero(w);
        PosSums wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            unsigned long long n1 = __shfl_up_sync(ALP_FULL_MASK, wi.nodes, d);
            unsigned long long n2 = __shfl_up_sync(ALP_FULL_MASK, wi.brs, d);
            long long n3 = __shfl_up_sync(ALP_FULL_MASK, wi.depth, d);
            long long n4 = __shfl_up_sync(ALP_FULL_MASK, wi.v, d);
            unsigned long long n5 = __shfl_up_sync(ALP_FULL_MASK, wi.terms, d);
            if (lane >= d) { wi.nodes += n1; wi.brs += n2; wi.depth += n3; wi.v += n4; wi.terms += n5; }
        }
        if (lane < PP_THREADS / 32) {
            PosSums we;
            we.nodes = wi.nodes - w.nodes; we.brs = wi.brs - w.brs; we.depth = wi.depth - w.depth;
            we.v = wi.v - w.v; we.terms = wi.terms - w.terms;
            s_w[lane] = we;
        }
    }
    __syncthreads();
    const PosSums tp = a.tile_sums[blockIdx.x];
    const PosSums wp = s_w[warp];
    unsigned long long nd = tp.nodes + wp.nodes + inc.nodes - mine.nodes;
    unsigned long long bi = tp.brs + wp.brs + inc.brs - mine.brs;
    long long depth = tp.depth + wp.depth + inc.depth - mine.depth;
    long long v = tp.v + wp.v + inc.v - mine.v;
    unsigned long long tr = tp.terms + wp.terms + inc.terms - mine.terms;
    bool neg = false;
    for (int j = 0; j < PP_ITEMS; ++j) {
        if (ids[j] == NO_PAIR) continue;
        const PairInfo pi = s_pi[ids[j]];
        for (int t = 0; t < pi.n_br; ++t, ++bi) {
            const uint32_t sym = __ldg(&a.t.stack[pi.stack_begin + t]);
            int32_t ds;
            if (sym >> 31) { ds = (int32_t)depth; ++depth; }
            else { --depth; ds = (int32_t)depth; if (depth < 0) neg = true; }
            if ((long long)bi < a.cap_brs) { a.brbuf[bi] = sym; a.dsbuf[bi] = ds; }
        }
        for (int t = 0; t < pi.n_prod; ++t, ++nd) {
            const uint32_t p = __ldg(&a.t.pseq[pi.prod_begin + t]);
            const int32_t pt = s_pt[p];
            if ((long long)nd < a.cap_nodes) {
                a.vbuf[nd] = (int32_t)v;
                if (pt >= 0 && a.subst_terminals && (long long)tr < a.m) {
                    a.tag[nd] = (uint32_t)pt;
                    a.kind[nd] = 1;
                    a.nstart[nd] = (int64_t)a.tstart[tr];
                    a.nend[nd] = (int64_t)a.tend[tr];
                } else {
                    a.tag[nd] = p;
                    a.kind[nd] = 0;
                    a.nstart[nd] = 0;
                    a.nend[nd] = 0;
                }
            }
            v += s_ar[p] - 1;
            if (pt >= 0) ++tr;
        }
    }
    if (__any_sync(ALP_FULL_MASK, neg) && lane == 0) a.res->valid = 0;
}

// ---------------------------------------------------------------------------
// K3: previous smaller-or-equal inside a tile
// ---------------------------------------------------------------------------
struct PleArgs {
    const int32_t* val;          // [n] values
    long long n;
    const uint32_t* sym;         // brackets: symbol|left<<31 (queries only at rights); nodes: null
    long long* out_parent;       // nodes: answer index per element (root 0)
    int32_t* tile_min;           // [tiles]
    int32_t* stair_val;          // [tiles * PLE_TILE]
    uint32_t* stair_idx;         // [tiles * PLE_TILE] global index
    int32_t* stair_len;          // [tiles]
    unsigned long long* esc;     // escapees: index << 32 | (uint32)value
    unsigned int* esc_count;
    long long esc_cap;
    AlpResult* res;
};

// Escapee record: element index in the high 32 bits, its value in the low 32.
constexpr size_t PLE_SMEM = (2 * PLE_TILE + PLE_TILE) * 4;  // min tree + symbols

__global__ void __launch_bounds__(PLE_THREADS) ple_tile_kernel(PleArgs a) {
    extern __shared__ __align__(16) uint8_t smem[];
    int32_t* tree = reinterpret_cast<int32_t*>(smem);
    uint32_t* s_sym = reinterpret_cast<uint32_t*>(smem + 2 * PLE_TILE * 4);
    __shared__ int32_t s_suf[PLE_THREADS];
    __shared__ uint32_t s_cnt[PLE_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long base = (long long)blockIdx.x * PLE_TILE;
    const bool brackets = a.sym != nullptr;
    for (int j = tid; j < PLE_TILE; j += PLE_THREADS) {
        const long long g = base + j;
        tree[PLE_TILE + j] = g < a.n ? a.val[g] : INT32_MAX;
        if (brackets) s_sym[j] = g < a.n ? a.sym[g] : 0u;
    }
    __syncthreads();
    for (int width = PLE_TILE / 2; width >= 1; width >>= 1) {
        for (int i = tid; i < width; i += PLE_THREADS) {
            const int node = width + i;
            tree[node] = min(tree[2 * node], tree[2 * node + 1]);
        }
        __syncthreads();
    }
    // local answers
    bool mismatch = false;
    for (int jj = 0; jj < PLE_ITEMS; ++jj) {
        const int j = tid * PLE_ITEMS + jj;
        const long long g = base + j;
        if (g >= a.n) break;
        if (brackets && (s_sym[j] >> 31)) continue;  // lefts ask nothing
        const int32_t v = tree[PLE_TILE + j];
        int node = PLE_TILE + j;
        bool found = false;
        while (node > 1) {
            if ((node & 1) && tree[node - 1] <= v) { node = node - 1; found = true; break; }
            node >>= 1;
        }
        if (found) {
            while (node < PLE_TILE) node = (tree[2 * node + 1] <= v) ? 2 * node + 1 : 2 * node;
            const int ans = node - PLE_TILE;
            if (brackets) {
                if ((s_sym[ans] & 0x7fffffffu) != (s_sym[j] & 0x7fffffffu) || !(s_sym[ans] >> 31)) mismatch = true;
            } else {
                a.out_parent[g] = base + ans;
            }
        } else if (g == 0 && !brackets) {
            a.out_parent[0] = 0;
        } else {
            const unsigned int slot = atomicAdd(a.esc_count, 1u);
            if ((long long)slot < a.esc_cap) a.esc[slot] = ((unsigned long long)g << 32) | (uint32_t)v;
            else atomicOr(&a.res->error, ALP_DEV_ERR_CAPACITY);
        }
    }
    if (mismatch) a.res->valid = 0;
    // tile minimum and staircase of suffix minima (values strictly below every later one)
    int32_t tmin = INT32_MAX;
    for (int jj = PLE_ITEMS - 1; jj >= 0; --jj) tmin = min(tmin, tree[PLE_TILE + tid * PLE_ITEMS + jj]);
    s_suf[tid] = tmin;
    __syncthreads();
    // suffix min over the threads after this one
    int32_t after = INT32_MAX;
    {
        // inclusive suffix scan over s_suf (256 entries) by warps of reversed order
        int32_t x = s_suf[PLE_THREADS - 1 - tid];  // reversed
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            int32_t o = __shfl_up_sync(ALP_FULL_MASK, x, d);
            if (lane >= d) x = min(x, o);
        }
        __shared__ int32_t s_wm[PLE_THREADS / 32];
        if (lane == 31) s_wm[warp] = x;
        __syncthreads();
        int32_t pre = INT32_MAX;
        for (int w = 0; w < warp; ++w) pre = min(pre, s_wm[w]);
        x = min(x, pre);  // inclusive min of reversed[0..tid] = min of s_suf[255-tid .. 255]
        __syncthreads();
        s_suf[PLE_THREADS - 1 - tid] = x;  // now s_suf[t] = min over threads t..255
        __syncthreads();
        after = tid + 1 < PLE_THREADS ? s_suf[tid + 1] : INT32_MAX;
    }
    uint32_t flags = 0;
    int32_t run = after;
    for (int jj = PLE_ITEMS - 1; jj >= 0; --jj) {
        const long long g = base + tid * PLE_ITEMS + jj;
        const int32_t v = tree[PLE_TILE + tid * PLE_ITEMS + jj];
        if (g < a.n && v < run) flags |= 1u << jj;
        run = min(run, v);
    }
    const uint32_t cnt = __popc(flags);
    const uint32_t incl = warp_scan_add(cnt, lane);
    if (lane == 31) s_cnt[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0, total = 0;
    for (int w = 0; w < PLE_THREADS / 32; ++w) {
        if (w < warp) wpre += s_cnt[w];
        total += s_cnt[w];
    }
    uint32_t o = wpre + incl - cnt;
    const long long sbase = (long long)blockIdx.x * PLE_TILE;
    for (int jj = 0; jj < PLE_ITEMS; ++jj) {
        if (flags & (1u << jj)) {
            a.stair_val[sbase + o] = tree[PLE_TILE + tid * PLE_ITEMS + jj];
            a.stair_idx[sbase + o] = (uint32_t)(base + tid * PLE_ITEMS + jj);
            ++o;
        }
    }
    if (tid == 0) {
        a.stair_len[blockIdx.x] = (int32_t)total;
        a.tile_min[blockIdx.x] = tree[1];
    }
}

// Level-1/2 minima over groups of 32 / 1024 tiles.
__global__ void tile_min_levels_kernel(const int32_t* tmin, long long tiles, int32_t* m32, int32_t* m1024) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n32 = (tiles + 31) / 32;
    if (g < n32) {
        int32_t m = INT32_MAX;
        for (long long t = g * 32; t < tiles && t < g * 32 + 32; ++t) m = min(m, tmin[t]);
        m32[g] = m;
    }
    const long long n1024 = (tiles + 1023) / 1024;
    if (g < n1024) {
        int32_t m = INT32_MAX;
        for (long long t = g * 1024; t < tiles && t < g * 1024 + 1024; ++t) m = min(m, tmin[t]);
        m1024[g] = m;
    }
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
    AlpResult* res;
};

__global__ void ple_escape_kernel(EscArgs a) {
    const long long cnt = min((long long)*a.esc_count, a.esc_cap);
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += (long long)gridDim.x * blockDim.x) {
        const unsigned long long r = a.esc[e];
        const long long g = (long long)(r >> 32);
        const int32_t x = (int32_t)(uint32_t)r;
        const long long t = g / PLE_TILE;
        const long long u = prev_tile_leq(a.tile_min, a.m32, a.m1024, t, x);
        long long ans = -1;
        if (u >= 0) {
            const int32_t* sv = a.stair_val + u * PLE_TILE;
            int lo = 0, hi = a.stair_len[u] - 1;  // largest k with sv[k] <= x (values ascend)
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (sv[mid] <= x) lo = mid; else hi = mid - 1;
            }
            ans = a.stair_idx[u * PLE_TILE + lo];
        }
        if (a.sym) {
            if (ans < 0) a.res->valid = 0;
            else {
                const uint32_t l = a.sym[ans], rr = a.sym[g];
                if (!(l >> 31) || (l & 0x7fffffffu) != (rr & 0x7fffffffu)) a.res->valid = 0;
            }
        } else {
            a.out_parent[g] = g == 0 ? 0 : ans;
        }
    }
}

}  // namespace alp
