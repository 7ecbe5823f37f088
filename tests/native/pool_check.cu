// Stress check of the library's host worker pool (parallel_chunks /
// parallel_for in tmpm_host.h): several threads run parallel passes at once,
// some passes run a nested pass inside a chunk, and every pass's sum must equal
// the serial sum.  Prints OK and exits 0, or prints FAIL and exits 1; a
// deadlock is caught by the caller's timeout.
#include <cstdio>
#include <thread>
#include <vector>

#include "../../tessera_b200/csrc/tmpm_host.h"

int main() {
    using namespace tmpm;
    const size_t n = size_t(1) << 20;
    std::vector<uint64_t> data(n);
    uint64_t expect = 0;
    for (size_t i = 0; i < n; ++i) {
        data[i] = (i * 2654435761ull) % 1000003ull;
        expect += data[i];
    }
    std::atomic<int> bad{0};
    auto pass = [&](int rep) {
        std::vector<uint64_t> part(host_threads() + 1, 0);
        parallel_chunks(
            n,
            [&](size_t c, size_t lo, size_t hi) {
                uint64_t s = 0;
                for (size_t i = lo; i < hi; ++i) s += data[i];
                if (rep % 3 == 0 && c == 0) {  // a pass nested inside a chunk
                    std::atomic<size_t> inner{0};
                    parallel_chunks(
                        size_t(40000), [&](size_t, size_t a, size_t b) { inner += b - a; }, 1000);
                    if (inner != 40000) ++bad;
                }
                part[c] = s;
            },
            1024);
        uint64_t total = 0;
        for (uint64_t v : part) total += v;
        if (total != expect) ++bad;
    };
    std::vector<std::thread> callers;
    for (int t = 0; t < 4; ++t)
        callers.emplace_back([&, t] {
            for (int r = 0; r < 150; ++r) pass(r + t);
        });
    for (std::thread &c : callers) c.join();
    for (int r = 0; r < 50; ++r) pass(r);  // and one caller alone afterwards
    std::printf("%s\n", bad ? "FAIL" : "OK");
    return bad ? 1 : 0;
}
