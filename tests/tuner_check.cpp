// Drives the render autotuner (sprout_b200/csrc/tuner.hpp) with synthetic wave timings and
// prints "ok <name>" per passed check.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "tuner.hpp"

using spb::render::Tuner;

static int failures = 0;
#define CHECK(name, cond)                                      \
    do {                                                       \
        if (cond) {                                            \
            std::printf("ok %s\n", name);                      \
        } else {                                               \
            std::printf("FAILED %s (line %d)\n", name, __LINE__); \
            ++failures;                                        \
        }                                                      \
    } while (0)

// Runs the tuner to completion with cost(wave_paths, per_sm) ns per path; returns the candidates
// it asked for, in order.
template <class Cost>
std::vector<std::pair<uint32_t, uint32_t>> drive(Tuner& t, Cost cost) {
    std::vector<std::pair<uint32_t, uint32_t>> asked;
    for (int i = 0; i < 32 && !t.done(); ++i) {
        asked.emplace_back(t.wave_paths, t.per_sm);
        t.report(cost(t.wave_paths, t.per_sm));
    }
    return asked;
}

int main() {
    {
        // Larger waves and full occupancy are cheaper: the tuner ends on the largest of both.
        Tuner t;
        t.reset(9);
        auto const asked = drive(t, [](uint32_t w, uint32_t sm) { return 10.0 - 1e-7 * w - 0.1 * sm; });
        CHECK("sizes_first_at_full_occupancy", asked.size() >= 5 && asked[0] == std::make_pair(1u << 20, 9u) &&
                                                    asked[4] == std::make_pair(1u << 24, 9u));
        CHECK("occupancies_after_at_best_size",
              asked.size() == 7 && asked[5] == std::make_pair(1u << 24, 6u) && asked[6] == std::make_pair(1u << 24, 4u));
        CHECK("keeps_best", t.done() && t.best_wave == (1u << 24) && t.best_sm == 9u);
    }
    {
        // A middle wave size and a lower occupancy win.
        Tuner t;
        t.reset(8);
        drive(t, [](uint32_t w, uint32_t sm) { return (w == (1u << 22) ? 1.0 : 2.0) + (sm == 6 ? 0.0 : 0.5); });
        CHECK("picks_interior_optimum", t.done() && t.best_wave == (1u << 22) && t.best_sm == 6u);
    }
    {
        // With one block per SM there is no lower occupancy to try.
        Tuner t;
        t.reset(1);
        auto const asked = drive(t, [](uint32_t, uint32_t) { return 1.0; });
        CHECK("single_block_skips_occupancy", t.done() && asked.size() == 5 && t.best_sm == 1u);
    }
    {
        // reset() starts over (a new scene).
        Tuner t;
        t.reset(4);
        drive(t, [](uint32_t, uint32_t) { return 1.0; });
        t.reset(4);
        CHECK("reset_restarts", !t.done() && t.wave_paths == (1u << 20) && t.per_sm == 4u);
    }
    return failures ? EXIT_FAILURE : EXIT_SUCCESS;
}
