// Reads the lines tests/golden/make_phase_golden.py sends the reference's harness and prints this
// renderer's answers (sprout_b200/csrc/material.cuh: phase_hg, sample_hg,
// van_de_hulst_anisotropy, similarity_relation_scale) in the same form; compiled and run by
// tests/test_phase.py.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "../sprout_b200/csrc/material.cuh"

using namespace spb::shading;

int main() {
    char kind[4];
    while (std::scanf("%3s", kind) == 1) {
        if (std::strcmp(kind, "p") == 0) {
            float c, g;
            if (std::scanf("%f %f", &c, &g) != 2) {
                return 1;
            }
            std::printf("%.9g\n", double(phase_hg(c, g)));
        } else if (std::strcmp(kind, "s") == 0) {
            float w[3], r0, r1, g;
            if (std::scanf("%f %f %f %f %f %f", w, w + 1, w + 2, &r0, &r1, &g) != 6) {
                return 1;
            }
            V3 const wo = v3(w[0], w[1], w[2]);
            float    pdf;
            V3 const wi = sample_hg(wo, g, r0, r1, pdf);
            std::printf("%.9g %.9g %.9g\n", double(-dot(wi, wo)), double(pdf), double(std::sqrt(dot(wi, wi))));
        } else {
            float    g;
            unsigned depth;
            if (std::scanf("%f %u", &g, &depth) != 2) {
                return 1;
            }
            std::printf("%.9g %.9g\n", double(van_de_hulst_anisotropy(g, depth)),
                        double(similarity_relation_scale(g, depth)));
        }
    }
    return 0;
}
