// Driver for the CPU tests of sprout_b200/csrc/postprocess.cpp (the product's tonemappers, half
// conversion and EXR/RGBE writers), built by tests/test_postprocess.py with g++.
//
// usage: postprocess_check tonemap KIND AUTO_EXPOSE EXPOSURE P0 P1 P2 P3 P4 WIDTH HEIGHT IN OUT
//        postprocess_check half IN OUT            (float32 -> uint16 binary16)
//        postprocess_check exr WIDTH HEIGHT IN OUT  (float32 RGBA -> EXR file)
//        postprocess_check rgbe WIDTH HEIGHT IN OUT (float32 RGBA -> Radiance RGBE file)
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "postprocess.hpp"

static std::vector<float> read_floats(char const* path) {
    std::vector<float> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        std::exit(2);
    }
    float x;
    while (std::fread(&x, 4, 1, f) == 1) {
        v.push_back(x);
    }
    std::fclose(f);
    return v;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        return 2;
    }
    std::string const mode = argv[1];
    if (mode == "half" && argc == 4) {
        std::vector<float> const in = read_floats(argv[2]);
        std::vector<uint16_t>    out(in.size());
        for (size_t i = 0; i < in.size(); ++i) {
            out[i] = spb::post::float_to_half(in[i]);
        }
        FILE* f = std::fopen(argv[3], "wb");
        std::fwrite(out.data(), 2, out.size(), f);
        std::fclose(f);
        return 0;
    }
    if ((mode == "exr" || mode == "rgbe") && argc == 6) {
        uint32_t const           w  = uint32_t(std::atoi(argv[2]));
        uint32_t const           h  = uint32_t(std::atoi(argv[3]));
        std::vector<float> const in = read_floats(argv[4]);
        bool const ok = mode == "exr" ? spb::post::write_exr(argv[5], w, h, in.data(), false)
                                      : spb::post::write_rgbe(argv[5], w, h, in.data());
        return ok ? 0 : 1;
    }
    if (mode == "tonemap" && argc == 14) {
        std::string const      kind = argv[2];
        spb::post::Tonemapper t;
        t.auto_expose = std::atoi(argv[3]) != 0;
        t.exposure    = float(std::atof(argv[4]));
        float p[5];
        for (int i = 0; i < 5; ++i) {
            p[i] = float(std::atof(argv[5 + i]));
        }
        if (kind == "Linear") {
            t.kind = spb::post::Tonemapper::Kind::Linear;
        } else if (kind == "ACES") {
            t.kind = spb::post::Tonemapper::Kind::Aces;
        } else if (kind == "Generic") {
            t.kind = spb::post::Tonemapper::Kind::Generic;
            t.contrast = p[0], t.shoulder = p[1], t.mid_in = p[2], t.mid_out = p[3], t.hdr_max = p[4];
        } else if (kind == "Piecewise") {
            t.kind         = spb::post::Tonemapper::Kind::Piecewise;
            t.toe_strength = p[0], t.toe_length = p[1], t.shoulder_strength = p[2], t.shoulder_length = p[3];
            t.shoulder_angle = p[4];
        } else {
            return 2;
        }
        std::vector<float> px = read_floats(argv[12]);
        spb::post::apply(t, px.data(), px.size() / 4);
        FILE* f = std::fopen(argv[13], "wb");
        std::fwrite(px.data(), 4, px.size(), f);
        std::fclose(f);
        return 0;
    }
    return 2;
}
