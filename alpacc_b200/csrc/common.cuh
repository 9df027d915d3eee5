// Shared device helpers for the alpacc B200 kernels: tile status words for
// decoupled look-back, bounded spin waits, warp/block scans.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define ALP_FULL_MASK 0xffffffffu

// Error bits a kernel records in its result block (host turns them into
// ALP_ERR_TIMEOUT / ALP_ERR_CAPACITY).
enum : uint32_t {
    ALP_DEV_ERR_TIMEOUT = 1u,
    ALP_DEV_ERR_CAPACITY = 2u,
};

// A look-back wait gives up after this many polls (with nanosleep backoff,
// well over a second) and records ALP_DEV_ERR_TIMEOUT.
#ifndef ALP_SPIN_LIMIT
#define ALP_SPIN_LIMIT (1u << 22)
#endif

struct __align__(16) AlpResult {
    long long count;        // tokens or nodes written
    int valid;              // 1 accepted, 0 rejected
    unsigned int error;     // ALP_DEV_ERR_* bits
    long long aux[8];       // kernel-specific extras (counts for sizing, etc.)
};

// ---- status words ---------------------------------------------------------
// 32-bit: [31:30] flag, [29:0] value.   64-bit: [63:62] flag, [61:0] payload.
enum : uint32_t { ST_X = 0u, ST_A = 1u, ST_P = 2u };

__device__ __forceinline__ uint32_t ld_volatile32(const uint32_t* p) {
    return *reinterpret_cast<const volatile uint32_t*>(p);
}
__device__ __forceinline__ unsigned long long ld_volatile64(const unsigned long long* p) {
    return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ void st_volatile32(uint32_t* p, uint32_t v) {
    *reinterpret_cast<volatile uint32_t*>(p) = v;
}
__device__ __forceinline__ void st_volatile64(unsigned long long* p, unsigned long long v) {
    *reinterpret_cast<volatile unsigned long long*>(p) = v;
}

// Poll a 32-bit status word until its flag is not X.  Returns the word; on
// timeout sets *err and returns a P word with value 0 so the caller finishes.
__device__ __forceinline__ uint32_t wait32(const uint32_t* p, unsigned int* err) {
    uint32_t v = ld_volatile32(p);
    unsigned int ns = 32;
    for (uint32_t it = 0; (v >> 30) == ST_X; ++it) {
        if (it >= ALP_SPIN_LIMIT) {
            atomicOr(err, ALP_DEV_ERR_TIMEOUT);
            return (ST_P << 30);
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
        v = ld_volatile32(p);
    }
    return v;
}

__device__ __forceinline__ unsigned long long wait64(const unsigned long long* p, unsigned int* err) {
    unsigned long long v = ld_volatile64(p);
    unsigned int ns = 32;
    for (uint32_t it = 0; (v >> 62) == ST_X; ++it) {
        if (it >= ALP_SPIN_LIMIT) {
            atomicOr(err, ALP_DEV_ERR_TIMEOUT);
            return ((unsigned long long)ST_P << 62);
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
        v = ld_volatile64(p);
    }
    return v;
}

// ---- (count, last position) pair monoid ---------------------------------
// Sum of counts; the position keeps the right operand unless it is NONE.
// Packed in a 64-bit payload: [61:32] count (30 bits), [31:0] position.
#define ALP_NONE32 0xffffffffu

__device__ __forceinline__ unsigned long long cs_pack(uint32_t flag, uint32_t count, uint32_t pos) {
    return ((unsigned long long)flag << 62) | ((unsigned long long)(count & 0x3fffffffu) << 32) | pos;
}
__device__ __forceinline__ uint32_t cs_count(unsigned long long w) { return (uint32_t)(w >> 32) & 0x3fffffffu; }
__device__ __forceinline__ uint32_t cs_pos(unsigned long long w) { return (uint32_t)w; }

// Inclusive warp scan of (count, pos) pairs.
__device__ __forceinline__ void warp_scan_cs(uint32_t& c, uint32_t& p, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t oc = __shfl_up_sync(ALP_FULL_MASK, c, d);
        uint32_t op = __shfl_up_sync(ALP_FULL_MASK, p, d);
        if (lane >= d) {
            c += oc;
            if (p == ALP_NONE32) p = op;
        }
    }
}

// Inclusive warp scan of 32-bit sums.
__device__ __forceinline__ uint32_t warp_scan_add(uint32_t v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t o = __shfl_up_sync(ALP_FULL_MASK, v, d);
        if (lane >= d) v += o;
    }
    return v;
}
