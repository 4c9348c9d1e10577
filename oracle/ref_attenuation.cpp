// Medium-coefficient harness (test infrastructure, not part of the product): reads lines of
// "ac.r ac.g ac.b ssc.r ssc.g ssc.b distance anisotropy" from standard input and prints, per
// line, the reference's attenuation(ac, ssc, distance, anisotropy)
// (source/core/scene/material/collision_coefficients.inl:50-71) as "mu_a.rgb mu_s.rgb", built
// by oracle/Makefile against the reference's own sources.
#include <cstdio>

#include "base/math/vector3.inl"
#include "scene/material/collision_coefficients.inl"

int main() {
    float v[8];
    while (std::scanf("%f %f %f %f %f %f %f %f", v, v + 1, v + 2, v + 3, v + 4, v + 5, v + 6, v + 7) == 8) {
        auto const cc = scene::material::attenuation(float3(v[0], v[1], v[2]), float3(v[3], v[4], v[5]), v[6], v[7]);
        std::printf("%.9g %.9g %.9g %.9g %.9g %.9g\n", double(cc.a[0]), double(cc.a[1]), double(cc.a[2]),
                    double(cc.s[0]), double(cc.s[1]), double(cc.s[2]));
    }
    return 0;
}
