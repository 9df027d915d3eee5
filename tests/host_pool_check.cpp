// CPU check of the host widening and its thread pool (alpacc_b200/csrc/host_pool.h):
// every value sign-extended, destinations at every alignment the AVX2 path's head
// and tail loops meet, partial slices, several jobs in flight with their slice
// counters, pools of zero to five workers, and help() from the calling thread.
// Prints "ok" and exits 0, else names the first failure and exits 1.
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "../alpacc_b200/csrc/host_pool.h"

using alp_host::HostPool;
using alp_host::WIDEN_SLICE;

static int fails = 0;

static void expect(bool ok, const char* what, long long a, long long b) {
    if (!ok && fails++ < 5) std::printf("FAIL %s (%lld, %lld)\n", what, a, b);
}

int main() {
    std::mt19937_64 rng(7);
    // widen() alone: lengths around the vector width, destinations off 32-byte boundaries
    for (size_t n : {0ul, 1ul, 3ul, 4ul, 5ul, 31ul, 32ul, 33ul, 1000ul, 4099ul}) {
        for (int shift = 0; shift < 4; ++shift) {
            std::vector<int32_t> src(n);
            for (auto& v : src) v = (int32_t)(rng() >> 32);
            if (n) src[0] = -1;
            std::vector<int64_t> buf(n + 8, 0x5a5a5a5a5a5a5a5aLL);
            alp_host::widen(src.data(), buf.data() + shift, n);
            for (size_t i = 0; i < n; ++i) expect(buf[shift + i] == (int64_t)src[i], "widen value", (long long)i, shift);
            for (int i = 0; i < shift; ++i) expect(buf[i] == 0x5a5a5a5a5a5a5a5aLL, "widen wrote before", i, shift);
            for (size_t i = shift + n; i < buf.size(); ++i)
                expect(buf[i] == 0x5a5a5a5a5a5a5a5aLL, "widen wrote after", (long long)i, shift);
        }
    }
    // the pool: jobs of several slices (a partial last one), three in flight at once
    for (int workers : {0, 1, 2, 5}) {
        HostPool pool(workers);
        for (int round = 0; round < 3; ++round) {
            const size_t lens[3] = {WIDEN_SLICE * 3 + 17, 5, WIDEN_SLICE};
            std::vector<int32_t> src[3];
            std::vector<int64_t> dst[3];
            std::atomic<int> left[3];
            for (int j = 0; j < 3; ++j) {
                src[j].resize(lens[j]);
                for (auto& v : src[j]) v = (int32_t)(rng() >> 32);
                dst[j].assign(lens[j] + 1, -7);
                left[j].store(HostPool::slices(lens[j]));
                pool.push(src[j].data(), dst[j].data() + (j == 1), lens[j], &left[j]);
            }
            if (round == 1)
                while (pool.help()) {
                }
            pool.wait();
            for (int j = 0; j < 3; ++j) {
                expect(left[j].load() == 0, "slices left", j, left[j].load());
                const int64_t* d = dst[j].data() + (j == 1);
                for (size_t i = 0; i < lens[j]; ++i) {
                    if (d[i] != (int64_t)src[j][i]) {
                        expect(false, "pool value", (long long)i, workers);
                        break;
                    }
                }
            }
            expect(HostPool::slices(lens[0]) == 4, "slice count", HostPool::slices(lens[0]), 4);
        }
    }
    if (fails) return 1;
    std::printf("ok\n");
    return 0;
}
