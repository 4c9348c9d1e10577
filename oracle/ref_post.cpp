// Postprocessing harness around the reference's own code: TEST INFRASTRUCTURE, not product.
//
// tonemap: applies one of the reference's tonemappers (rendering/postprocessor/tonemapping:
//   Linear, ACES, Generic, Piecewise) to a float RGBA image, through Postprocessor::apply as
//   the reference's pipeline does (postprocessor_pipeline.cpp:69-102).
// read_exr: reads an EXR file with the reference's reader (image/encoding/exr/exr_reader.cpp)
//   and writes its pixels as float RGB (half channels widened by the reference's half_to_float).
//
// usage: ref_post tonemap KIND AUTO_EXPOSE EXPOSURE P0 P1 P2 P3 P4 WIDTH HEIGHT IN OUT
//          KIND: Linear | ACES | Generic (P: contrast shoulder mid_in mid_out hdr_max)
//                | Piecewise (P: toe_strength toe_length shoulder_strength shoulder_length
//                  shoulder_angle); IN/OUT: float32 RGBA, WIDTH * HEIGHT * 4
//        ref_post read_exr FILE OUT    (prints "width height"; OUT: float32 RGB)
#include "base/math/half.inl"
#include "base/math/vector4.inl"
#include "base/thread/thread_pool.hpp"
#include "image/encoding/exr/exr_reader.hpp"
#include "image/image.hpp"
#include "image/typed_image.hpp"
#include "rendering/postprocessor/tonemapping/aces.hpp"
#include "rendering/postprocessor/tonemapping/generic.hpp"
#include "rendering/postprocessor/tonemapping/linear.hpp"
#include "rendering/postprocessor/tonemapping/piecewise.hpp"
#include "scene/scene.hpp"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

using namespace rendering::postprocessor::tonemapping;

int main(int argc, char** argv) {
    if (argc >= 4 && std::string(argv[1]) == "read_exr") {
        std::ifstream stream(argv[2], std::ios::binary);
        std::unique_ptr<image::Image> img(image::encoding::exr::Reader::read(stream, false));  // raw: no sRGB -> AP1
        if (!img) {
            std::fprintf(stderr, "reference EXR reader refused %s\n", argv[2]);
            return 1;
        }
        int2 const d = img->description().dimensions().xy();
        std::vector<float> out;
        for (int32_t y = 0; y < d[1]; ++y) {
            for (int32_t x = 0; x < d[0]; ++x) {
                float c[3];
                if (image::Image::Type::Short3 == img->type()) {  // half channels, as stored
                    ushort3 const h = img->short3().at(x, y);
                    for (int k = 0; k < 3; ++k) {
                        c[k] = half_to_float(h[k]);
                    }
                } else {
                    packed_float3 const f = img->float3().at(x, y);
                    for (int k = 0; k < 3; ++k) {
                        c[k] = f[k];
                    }
                }
                out.push_back(c[0]);
                out.push_back(c[1]);
                out.push_back(c[2]);
            }
        }
        FILE* f = std::fopen(argv[3], "wb");
        std::fwrite(out.data(), sizeof(float), out.size(), f);
        std::fclose(f);
        std::printf("%d %d\n", d[0], d[1]);
        return 0;
    }
    if (argc < 14 || std::string(argv[1]) != "tonemap") {
        std::fprintf(stderr, "usage: see ref_post.cpp\n");
        return 2;
    }
    std::string const kind     = argv[2];
    bool const        auto_exp = std::atoi(argv[3]) != 0;
    float const       exposure = float(std::atof(argv[4]));
    float             p[5];
    for (int i = 0; i < 5; ++i) {
        p[i] = float(std::atof(argv[5 + i]));
    }
    int const w = std::atoi(argv[10]);
    int const h = std::atoi(argv[11]);

    std::unique_ptr<rendering::postprocessor::Postprocessor> pp;
    if (kind == "Linear") {
        pp.reset(new Linear(auto_exp, exposure));
    } else if (kind == "ACES") {
        pp.reset(new Aces(auto_exp, exposure));
    } else if (kind == "Generic") {
        pp.reset(new Generic(auto_exp, exposure, p[0], p[1], p[2], p[3], p[4]));
    } else if (kind == "Piecewise") {
        pp.reset(new Piecewise(auto_exp, exposure, p[0], p[1], p[2], p[3], p[4]));
    } else {
        return 2;
    }
    image::Float4 source(image::Description(int2(w, h)));
    image::Float4 destination(image::Description(int2(w, h)));
    std::vector<float> in(size_t(w) * h * 4);
    FILE* f = std::fopen(argv[12], "rb");
    if (!f || std::fread(in.data(), sizeof(float), in.size(), f) != in.size()) {
        return 2;
    }
    std::fclose(f);
    for (int i = 0; i < w * h; ++i) {
        source.store(i, float4(in[4 * i], in[4 * i + 1], in[4 * i + 2], in[4 * i + 3]));
    }
    thread::Pool threads(1);
    std::vector<image::Image*>    images;
    std::vector<scene::material::Material*> materials;
    std::vector<scene::shape::Shape*>       shapes;
    scene::Scene scene(images, materials, shapes, 0);
    pp->apply(source, destination, scene, threads);
    std::vector<float> out(in.size());
    for (int i = 0; i < w * h; ++i) {
        float4 const c = destination.at(i);
        for (int k = 0; k < 4; ++k) {
            out[4 * i + k] = c[k];
        }
    }
    f = std::fopen(argv[13], "wb");
    std::fwrite(out.data(), sizeof(float), out.size(), f);
    std::fclose(f);
    return 0;
}
