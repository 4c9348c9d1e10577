// Online autotuner of the path tracer's launch shapes (render.cu); host code only.
#pragma once

#include <algorithm>
#include <cstdint>

namespace spb::render {

// Online autotuner of the wave size (paths per wave) and the traversal kernels' grid (blocks
// per SM).  The waves of a frame try the candidates in turn -- wave sizes at the largest
// occupancy first, then lower occupancies at the best size -- each timed with CUDA events
// (device time per path of the whole wave); the best is kept for the rest of the frame and for
// later frames of the scene.  Which samples are drawn does not depend on the wave size (each
// sample's stream is fixed by its pixel and sample index), so tuning renders no extra work.
struct Tuner {
    static constexpr uint32_t Wave_sizes[5] = {1u << 20, 1u << 21, 1u << 22, 1u << 23, 1u << 24};
    static constexpr uint32_t Sizes          = 5;
    static constexpr uint32_t Max_wave_paths = 1u << 24;
    uint32_t max_per_sm = 1;   // most traversal blocks an SM holds
    uint32_t stage      = 0;   // 0: wave sizes, 1: occupancies, 2: done
    uint32_t candidate  = 0;
    uint32_t wave_paths = 1u << 22;
    uint32_t per_sm     = 1;
    double   best_ns    = 1e300;  // device ns per path of the best candidate so far
    uint32_t best_wave  = 1u << 22;
    uint32_t best_sm    = 1;

    void reset(uint32_t max_blocks) {
        *this      = Tuner();
        max_per_sm = std::max(1u, max_blocks);
        per_sm     = max_per_sm;
        best_sm    = max_per_sm;
        wave_paths = Wave_sizes[0];
    }
    bool     done() const { return stage == 2; }
    uint32_t occupancy(uint32_t i) const {  // 3/4 and 1/2 of the largest
        return std::max(1u, i == 0 ? max_per_sm * 3 / 4 : max_per_sm / 2);
    }
    // Result of a full wave of the current candidate.
    void report(double ns_per_path) {
        if (ns_per_path < best_ns) {
            best_ns   = ns_per_path;
            best_wave = wave_paths;
            best_sm   = per_sm;
        }
        if (stage == 0 && ++candidate < Sizes) {
            wave_paths = Wave_sizes[candidate];
            return;
        }
        if (stage == 0) {
            stage = 1;
            candidate = 0;
        } else {
            ++candidate;
        }
        wave_paths = best_wave;
        if (candidate < 2 && occupancy(candidate) < max_per_sm) {
            per_sm = occupancy(candidate);
        } else {
            stage  = 2;
            per_sm = best_sm;
        }
    }
};

}  // namespace spb::render
