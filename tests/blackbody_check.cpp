// Prints this renderer's black-body colour (sprout_b200/csrc/spectral.cuh, blackbody) for each
// temperature given in kelvin on the command line, one "kelvin r g b" line each, or with the
// single argument "matrix" its XYZ -> linear sRGB matrix (row-major, one line); compiled and
// run by tests/test_blackbody.py.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../sprout_b200/csrc/spectral.cuh"

int main(int argc, char** argv) {
    if (argc == 2 && std::strcmp(argv[1], "matrix") == 0) {
        double m[9];
        spb::spectral::xyz_to_srgb(m);
        for (double x : m) {
            std::printf("%.9f ", x);
        }
        std::printf("\n");
        return 0;
    }
    for (int i = 1; i < argc; ++i) {
        double const t = std::atof(argv[i]);
        double       c[3];
        spb::spectral::blackbody(t, c);
        std::printf("%.3f %.9g %.9g %.9g\n", t, c[0], c[1], c[2]);
    }
    return 0;
}
