// Reads lines of "ac.r ac.g ac.b ssc.r ssc.g ssc.b distance anisotropy" from standard input and
// prints this renderer's medium coefficients (sprout_b200/csrc/material.cuh, attenuation) as
// "mu_a.rgb mu_s.rgb"; compiled and run by tests/test_attenuation.py.
#include <cstdio>

#include "../sprout_b200/csrc/material.cuh"

int main() {
    float v[8];
    while (std::scanf("%f %f %f %f %f %f %f %f", v, v + 1, v + 2, v + 3, v + 4, v + 5, v + 6, v + 7) == 8) {
        spb::shading::V3 a, s;
        spb::shading::attenuation(spb::shading::v3(v[0], v[1], v[2]), spb::shading::v3(v[3], v[4], v[5]), v[6], v[7],
                                  a, s);
        std::printf("%.9g %.9g %.9g %.9g %.9g %.9g\n", double(a.x), double(a.y), double(a.z), double(s.x),
                    double(s.y), double(s.z));
    }
    return 0;
}
