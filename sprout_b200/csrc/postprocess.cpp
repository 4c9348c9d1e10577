// Tonemappers and HDR image writers for a resolved frame; see postprocess.hpp.
#include "postprocess.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <zlib.h>

namespace spb::post {

namespace {

struct Rgb {
    float r, g, b;
};

// 3x3 colour transforms of the ACEScg pipeline (the colour spaces' definitions, as the
// reference's base/spectrum/aces.hpp states them).
Rgb ap1_to_srgb(Rgb c) {
    return {1.70505155f * c.r - 0.62179068f * c.g - 0.08325840f * c.b,
            -0.13025714f * c.r + 1.14080289f * c.g - 0.01054853f * c.b,
            -0.02400328f * c.r - 0.12896877f * c.g + 1.15297171f * c.b};
}

Rgb ap1_to_rrt_sat(Rgb c) {
    return {0.970889f * c.r + 0.026963f * c.g + 0.002148f * c.b,
            0.010889f * c.r + 0.986963f * c.g + 0.002148f * c.b,
            0.010889f * c.r + 0.026963f * c.g + 0.962148f * c.b};
}

Rgb odt_sat_to_srgb(Rgb c) {
    return {1.60475f * c.r - 0.53108f * c.g - 0.07367f * c.b,
            -0.10208f * c.r + 1.10813f * c.g - 0.00605f * c.b,
            -0.00327f * c.r - 0.07276f * c.g + 1.07602f * c.b};
}

// The RRT and ODT of ACES as one rational function per channel (Hill's fit).
float rrt_odt(float x) {
    float const a = x * (x + 0.0245786f) - 0.000090537f;
    float const b = x * (0.983729f * x + 0.4329510f) + 0.238081f;
    return a / b;
}

// Relative luminance of AP1 RGB (Y row of AP1 -> XYZ).
float luminance(Rgb c) {
    return 0.2722287168f * c.r + 0.6740817658f * c.g + 0.0536895174f * c.b;
}

float exposure_factor(Tonemapper const& t, float const* rgba, size_t count) {
    if (!t.auto_expose) {
        return std::exp2(t.exposure);
    }
    // mean of log2(1 + luminance), brought back to a factor that maps it to mid grey
    double sum = 0.0;
    for (size_t i = 0; i < count; ++i) {
        sum += std::log2(1.0 + double(luminance(Rgb{rgba[4 * i], rgba[4 * i + 1], rgba[4 * i + 2]})));
    }
    double const average = count ? sum / double(count) : 0.0;
    return float(0.18 / (std::exp2(average) - 1.0));
}

// Lottes' curve: contrast a, shoulder d, mid grey mapped from mid_in to mid_out, saturating at
// hdr_max; b and c solve the two constraints.
struct Generic_curve {
    float a, d, b, c, hdr_max;

    explicit Generic_curve(Tonemapper const& t) : a(t.contrast), d(t.shoulder), hdr_max(t.hdr_max) {
        float const ad       = a * d;
        float const mid_a    = std::pow(t.mid_in, a);
        float const mid_ad   = std::pow(t.mid_in, ad);
        float const max_a    = std::pow(t.hdr_max, a);
        float const max_ad   = std::pow(t.hdr_max, ad);
        float const u        = max_ad * t.mid_out - mid_ad * t.mid_out;
        float const v        = mid_ad * t.mid_out;
        float const cross    = max_ad * mid_a - max_a * v;
        c                    = cross / u;
        b                    = -((-mid_a + (t.mid_out * cross) / u) / v);
    }

    float operator()(float x) const {
        float const z = std::pow(std::min(x, hdr_max), a);
        return z / (std::pow(z, d) * b + c);
    }
};

// Hable's piecewise power curve: a toe and a shoulder of the form y = e^(ln_a + b ln x) around a
// linear middle, in coordinates normalised to the white point w.
struct Piecewise_curve {
    struct Segment {
        float offset_x = 0.f, offset_y = 0.f, scale_x = 1.f, scale_y = 1.f, ln_a = 0.f, b = 1.f;

        float eval(float x) const {
            float const x0 = (x - offset_x) * scale_x;
            float const y0 = x0 > 0.f ? std::exp(ln_a + b * std::log(x0)) : 0.f;
            return y0 * scale_y + offset_y;
        }
    };

    Segment segments[3];
    float   x0 = 0.f, x1 = 0.f, w_inv = 1.f;

    // ln_a and b of the power segment through (x, y) with slope m there
    static void power_through(float x, float y, float m, float& ln_a, float& b) {
        b    = (m * x) / y;
        ln_a = std::log(y) - b * std::log(x);
    }

    static float saturate(float x) { return std::min(std::max(x, 0.f), 1.f); }

    explicit Piecewise_curve(Tonemapper const& t) {
        // the user-facing lengths are in a perceptual (gamma 2.2) space
        float const toe_length        = std::pow(saturate(t.toe_length), 2.2f);
        float const toe_strength      = saturate(t.toe_strength);
        float const shoulder_angle    = saturate(t.shoulder_angle);
        float const shoulder_length   = std::max(1e-5f, saturate(t.shoulder_length));
        float const shoulder_strength = std::max(0.f, t.shoulder_strength);

        float const px0         = toe_length * 0.5f;
        float const py0         = (1.f - toe_strength) * px0;
        float const remaining_y = 1.f - py0;
        float const y1_offset   = (1.f - shoulder_length) * remaining_y;
        float const px1         = px0 + y1_offset;
        float const py1         = py0 + y1_offset;
        float const w           = px0 + remaining_y + (std::exp2(shoulder_strength) - 1.f);
        float const over_x      = (w * 2.f) * shoulder_angle * shoulder_strength / w;
        float const over_y      = 0.5f * shoulder_angle * shoulder_strength;

        w_inv       = 1.f / w;
        x0          = px0 / w;
        x1          = px1 / w;
        // linear middle through (x0, y0) and (x1, y1)
        float const dx = x1 - x0;
        float const m  = dx == 0.f ? 1.f : (py1 - py0) / dx;
        float const c0 = py0 - x0 * m;
        segments[1].offset_x = -(c0 / m);
        segments[1].ln_a     = std::log(m);
        segments[1].b        = 1.f;
        // toe through (x0, y0) with the middle's slope
        power_through(x0, py0, m, segments[0].ln_a, segments[0].b);
        // shoulder: mirrored about (1 + overshoot), through the middle's end with its slope
        power_through((1.f + over_x) - x1, (1.f + over_y) - py1, m, segments[2].ln_a, segments[2].b);
        segments[2].offset_x = 1.f + over_x;
        segments[2].offset_y = 1.f + over_y;
        segments[2].scale_x  = -1.f;
        segments[2].scale_y  = -1.f;
        // normalise so that the white point maps to 1
        float const inv = 1.f / segments[2].eval(1.f);
        for (Segment& s : segments) {
            s.offset_y *= inv;
            s.scale_y *= inv;
        }
    }

    float operator()(float x) const {
        float const n = x * w_inv;
        return segments[n < x0 ? 0 : (n < x1 ? 1 : 2)].eval(n);
    }
};

bool put(FILE* f, void const* data, size_t bytes) {
    return std::fwrite(data, 1, bytes, f) == bytes;
}

template <typename T>
void append(std::vector<uint8_t>& out, T v) {
    uint8_t b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));  // little-endian hosts, as EXR stores
    out.insert(out.end(), b, b + sizeof(T));
}

void append_str(std::vector<uint8_t>& out, char const* s) {
    out.insert(out.end(), s, s + std::strlen(s) + 1);
}

}  // namespace

void apply(Tonemapper const& t, float* rgba, size_t count) {
    float const factor = exposure_factor(t, rgba, count);
    switch (t.kind) {
        case Tonemapper::Kind::Linear:
            for (size_t i = 0; i < count; ++i) {
                float* p = rgba + 4 * i;
                Rgb const s = ap1_to_srgb({factor * p[0], factor * p[1], factor * p[2]});
                p[0] = s.r, p[1] = s.g, p[2] = s.b;
            }
            break;
        case Tonemapper::Kind::Aces:
            for (size_t i = 0; i < count; ++i) {
                float* p = rgba + 4 * i;
                Rgb const r = ap1_to_rrt_sat({factor * p[0], factor * p[1], factor * p[2]});
                Rgb const s = odt_sat_to_srgb({rrt_odt(r.r), rrt_odt(r.g), rrt_odt(r.b)});
                p[0] = s.r, p[1] = s.g, p[2] = s.b;
            }
            break;
        case Tonemapper::Kind::Generic: {
            Generic_curve const curve(t);
            for (size_t i = 0; i < count; ++i) {
                float* p = rgba + 4 * i;
                p[0] = curve(factor * p[0]), p[1] = curve(factor * p[1]), p[2] = curve(factor * p[2]);
            }
            break;
        }
        case Tonemapper::Kind::Piecewise: {
            Piecewise_curve const curve(t);
            for (size_t i = 0; i < count; ++i) {
                float* p = rgba + 4 * i;
                Rgb const r = ap1_to_rrt_sat({factor * p[0], factor * p[1], factor * p[2]});
                Rgb const s = odt_sat_to_srgb({curve(r.r), curve(r.g), curve(r.b)});
                p[0] = s.r, p[1] = s.g, p[2] = s.b;
            }
            break;
        }
    }
}

uint16_t float_to_half(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    uint32_t const sign = (x >> 16) & 0x8000u;
    uint32_t const abs  = x & 0x7FFFFFFFu;
    if (abs >= 0x7F800000u) {  // infinity or NaN
        return uint16_t(sign | 0x7C00u | (abs > 0x7F800000u ? 0x200u | ((abs >> 13) & 0x3FFu) : 0u));
    }
    if (abs >= 0x477FF000u) {  // rounds to beyond 65504: infinity
        return uint16_t(sign | 0x7C00u);
    }
    if (abs < 0x38800000u) {  // below 2^-14: a subnormal half (or zero)
        if (abs < 0x33000000u) {  // below half of the smallest subnormal
            return uint16_t(sign);
        }
        uint32_t const e        = abs >> 23;
        uint32_t const mantissa = (abs & 0x7FFFFFu) | 0x800000u;
        uint32_t const shift    = 126u - e;  // the value in units of 2^-24: mantissa * 2^(e - 126)
        uint32_t const q        = mantissa >> shift;
        uint32_t const rem      = mantissa & ((1u << shift) - 1u);
        uint32_t const half     = 1u << (shift - 1u);
        uint32_t const rounded  = q + (rem > half || (rem == half && (q & 1u)) ? 1u : 0u);
        return uint16_t(sign | rounded);
    }
    // normal: rebias the exponent, round the mantissa to 10 bits, nearest even
    uint32_t const rebiased = abs - 0x38000000u;  // exponent 127 -> 15
    uint32_t const q        = rebiased >> 13;
    uint32_t const rem      = rebiased & 0x1FFFu;
    uint32_t const rounded  = q + (rem > 0x1000u || (rem == 0x1000u && (q & 1u)) ? 1u : 0u);
    return uint16_t(sign | rounded);
}

bool write_exr(std::string const& path, uint32_t width, uint32_t height, float const* rgba, bool alpha) {
    if (width == 0 || height == 0) {
        return false;
    }
    // OpenEXR file layout: magic, version (2: single-part scanline), header attributes
    // (name, type, size, value) ending in an empty name, the offset table (one entry per block
    // of 16 scanlines), and the blocks (first y, byte count, data).  A block's data is its
    // scanlines one after the other, each the rows of the channels in alphabetical order, ZIP
    // compressed: bytes split into even and odd positions, then each byte replaced by its
    // difference to the previous one (+128), then zlib (the format's definition; the
    // reference writes ZIP too, exr_writer.cpp).
    std::vector<uint8_t> head;
    append<uint32_t>(head, 20000630u);  // magic 0x762f3101
    append<uint32_t>(head, 2u);
    char const* names[4] = {"A", "B", "G", "R"};
    uint32_t const first = alpha ? 0u : 1u;
    uint32_t const channels = 4u - first;
    append_str(head, "channels");
    append_str(head, "chlist");
    append<int32_t>(head, int32_t(channels * 18 + 1));
    for (uint32_t c = first; c < 4; ++c) {
        append_str(head, names[c]);
        append<int32_t>(head, 1);  // HALF
        append<uint8_t>(head, 0);  // pLinear
        append<uint8_t>(head, 0);
        append<uint8_t>(head, 0);
        append<uint8_t>(head, 0);
        append<int32_t>(head, 1);  // x sampling
        append<int32_t>(head, 1);  // y sampling
    }
    append<uint8_t>(head, 0);
    append_str(head, "compression");
    append_str(head, "compression");
    append<int32_t>(head, 1);
    append<uint8_t>(head, 3);  // ZIP_COMPRESSION: blocks of 16 scanlines
    for (char const* window : {"dataWindow", "displayWindow"}) {
        append_str(head, window);
        append_str(head, "box2i");
        append<int32_t>(head, 16);
        append<int32_t>(head, 0);
        append<int32_t>(head, 0);
        append<int32_t>(head, int32_t(width - 1));
        append<int32_t>(head, int32_t(height - 1));
    }
    append_str(head, "lineOrder");
    append_str(head, "lineOrder");
    append<int32_t>(head, 1);
    append<uint8_t>(head, 0);  // INCREASING_Y
    append_str(head, "pixelAspectRatio");
    append_str(head, "float");
    append<int32_t>(head, 4);
    append<float>(head, 1.f);
    append_str(head, "screenWindowCenter");
    append_str(head, "v2f");
    append<int32_t>(head, 8);
    append<float>(head, 0.f);
    append<float>(head, 0.f);
    append_str(head, "screenWindowWidth");
    append_str(head, "float");
    append<int32_t>(head, 4);
    append<float>(head, 1.f);
    append<uint8_t>(head, 0);

    constexpr uint32_t Lines = 16;
    uint32_t const     num_blocks = (height + Lines - 1) / Lines;
    int const          channel_of[4] = {3, 2, 1, 0};  // A, B, G, R in rgba
    std::vector<std::vector<uint8_t>> blocks(num_blocks);
    std::vector<uint8_t> raw, split;
    for (uint32_t b = 0; b < num_blocks; ++b) {
        uint32_t const y0 = b * Lines;
        uint32_t const y1 = std::min(height, y0 + Lines);
        raw.clear();
        for (uint32_t y = y0; y < y1; ++y) {
            for (uint32_t c = first; c < 4; ++c) {
                for (uint32_t x = 0; x < width; ++x) {
                    append<uint16_t>(raw, float_to_half(rgba[4 * (size_t(y) * width + x) + channel_of[c]]));
                }
            }
        }
        size_t const n = raw.size();
        split.resize(n);
        size_t const half_n = (n + 1) / 2;
        for (size_t i = 0; i < n; ++i) {
            split[(i & 1) ? half_n + i / 2 : i / 2] = raw[i];
        }
        for (size_t i = n; i-- > 1;) {
            split[i] = uint8_t(int(split[i]) - int(split[i - 1]) + 128);
        }
        uLongf packed_size = compressBound(uLong(n));
        std::vector<uint8_t>& out = blocks[b];
        out.resize(8 + packed_size);
        if (compress2(out.data() + 8, &packed_size, split.data(), uLong(n), Z_DEFAULT_COMPRESSION) != Z_OK) {
            return false;
        }
        // a block that does not shrink is stored as it is (raw, unpredicted)
        uint32_t const stored = packed_size < n ? uint32_t(packed_size) : uint32_t(n);
        if (packed_size >= n) {
            std::memcpy(out.data() + 8, raw.data(), n);
        }
        out.resize(8 + stored);
        int32_t const y_first = int32_t(y0);
        std::memcpy(out.data(), &y_first, 4);
        std::memcpy(out.data() + 4, &stored, 4);
    }
    uint64_t offset = head.size() + 8ull * num_blocks;
    for (uint32_t b = 0; b < num_blocks; ++b) {
        append<uint64_t>(head, offset);
        offset += blocks[b].size();
    }
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        return false;
    }
    bool ok = put(f, head.data(), head.size());
    for (uint32_t b = 0; ok && b < num_blocks; ++b) {
        ok = put(f, blocks[b].data(), blocks[b].size());
    }
    return std::fclose(f) == 0 && ok;
}

bool write_rgbe(std::string const& path, uint32_t width, uint32_t height, float const* rgba) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        return false;
    }
    bool ok = std::fprintf(f, "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %u +X %u\n", height, width) > 0;
    std::vector<uint8_t> row(4 * size_t(width));
    for (uint32_t y = 0; ok && y < height; ++y) {
        for (uint32_t x = 0; x < width; ++x) {
            float const* p = rgba + 4 * (size_t(y) * width + x);
            float const  r = std::max(p[0], 0.f), g = std::max(p[1], 0.f), b = std::max(p[2], 0.f);
            float const  v = std::max(r, std::max(g, b));
            uint8_t*     o = &row[4 * size_t(x)];
            if (v < 1e-32f) {
                o[0] = o[1] = o[2] = o[3] = 0;
            } else {
                // v = m 2^e with m in [0.5, 1): each channel c becomes c 256 / 2^e
                int         e;
                float const m     = std::frexp(v, &e);
                float const scale = m * 256.f / v;
                o[0]              = uint8_t(r * scale);
                o[1]              = uint8_t(g * scale);
                o[2]              = uint8_t(b * scale);
                o[3]              = uint8_t(e + 128);
            }
        }
        ok = put(f, row.data(), row.size());
    }
    return std::fclose(f) == 0 && ok;
}

}  // namespace spb::post
