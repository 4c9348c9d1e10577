// Shared host-side helpers: error codes, the per-thread last-error message, thread fan-out.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

#include "../../include/sprout_b200.h"

namespace spb {

// Records msg as the calling thread's last error and returns code.
int32_t fail(int32_t code, char const* fmt, ...) __attribute__((format(printf, 2, 3)));

void clear_error();

uint32_t resolve_threads(uint32_t requested);

// Runs fn(thread_index, begin, end) over [0, count) split into num_threads contiguous ranges.
template <typename F>
void parallel_ranges(uint64_t count, uint32_t num_threads, F&& fn) {
    if (count == 0) {
        return;
    }
    uint64_t const workers = std::min<uint64_t>(num_threads, count);
    if (workers <= 1) {
        fn(0u, uint64_t(0), count);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(workers);
    for (uint64_t w = 0; w < workers; ++w) {
        uint64_t const begin = count * w / workers;
        uint64_t const end   = count * (w + 1) / workers;
        pool.emplace_back([&fn, w, begin, end]() { fn(uint32_t(w), begin, end); });
    }
    for (auto& t : pool) {
        t.join();
    }
}

}  // namespace spb
