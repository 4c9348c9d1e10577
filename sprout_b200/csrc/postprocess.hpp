// Postprocessing and export of a resolved frame (host side): the tonemappers of a take's "post"
// pipeline and the image writers of its "export" object.
//
// The film holds linear ACEScg (AP1) RGB (the reference's SU_ACESCG build).  Tonemappers follow
// rendering/postprocessor/tonemapping/*.cpp: an exposure factor (2^exposure, or with
// auto_expose 0.18 / (2^mean(log2(1 + luminance)) - 1), tonemapper.cpp:16-58), then
//   Linear:    AP1 -> linear sRGB (linear.cpp:10-27);
//   ACES:      AP1 -> RRT_SAT, the RRT + ODT rational fit, ODT_SAT -> sRGB (aces.cpp:10-32);
//   Generic:   x^a / ((x^a)^d b + c) per channel on min(x, hdr_max), b and c from the contrast a,
//              shoulder d, mid-grey in/out and HDR maximum (generic.cpp:8-58; Lottes, "Advanced
//              Techniques and Optimization of HDR Color Pipelines", GDC 2016);
//   Piecewise: AP1 -> RRT_SAT, a toe / linear / shoulder curve of power segments, ODT_SAT -> sRGB
//              (piecewise.cpp; Hable, "Filmic Tonemapping with Piecewise Power Curves", 2017).
// Writers: EXR (OpenEXR 2 scanline file, half channels, ZIP compression), RGBE (Radiance HDR,
// flat scanlines); the PNG writer lives with the C API.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

namespace spb::post {

struct Tonemapper {
    enum class Kind { Linear, Aces, Generic, Piecewise };
    Kind  kind        = Kind::Linear;
    bool  auto_expose = false;
    float exposure    = 0.f;  // stops
    // Generic (take_loader.cpp:873-884 defaults)
    float contrast = 1.15f;
    float shoulder = 0.99f;
    float mid_in   = 0.18f;
    float mid_out  = 0.18f;
    float hdr_max  = 1.f;
    // Piecewise (take_loader.cpp:890-899 defaults)
    float toe_strength      = 0.1f;
    float toe_length        = 0.5f;
    float shoulder_strength = 2.f;
    float shoulder_length   = 0.5f;
    float shoulder_angle    = 0.5f;
};

// Applies the tonemapper to count pixels of rgba (alpha untouched), in place.
void apply(Tonemapper const& t, float* rgba, size_t count);

// IEEE half (binary16) of f, rounded to nearest even; infinities and NaN kept.
uint16_t float_to_half(float f);

// An OpenEXR file: R, G, B (and A) as half, scanlines top to bottom (increasing y), ZIP
// compressed in blocks of 16 scanlines.
bool write_exr(std::string const& path, uint32_t width, uint32_t height, float const* rgba, bool alpha);

// A Radiance RGBE file, flat (not run-length encoded) scanlines.
bool write_rgbe(std::string const& path, uint32_t width, uint32_t height, float const* rgba);

}  // namespace spb::post
