// Black-body harness (test infrastructure, not part of the product): prints the reference's
// spectrum::blackbody (source/base/spectrum/mapping.cpp:125-147) for each temperature given in
// kelvin on the command line, one "kelvin r g b" line each, built by oracle/Makefile against
// the reference's own library.
#include <cstdio>
#include <cstdlib>

#include "base/math/vector3.inl"
#include "base/spectrum/mapping.hpp"

int main(int argc, char** argv) {
    for (int i = 1; i < argc; ++i) {
        float const  t = float(std::atof(argv[i]));
        float3 const c = spectrum::blackbody(t);
        std::printf("%.3f %.9g %.9g %.9g\n", double(t), double(c[0]), double(c[1]), double(c[2]));
    }
    return 0;
}
