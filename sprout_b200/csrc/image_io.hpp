// Image files for textures and density grids (host side): PNG and OpenEXR readers, the formats
// the reference's image providers read for surface textures (image/encoding/png, exr).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace spb::image_io {

// Pixels as floats, channels per pixel, x fastest then y.  Integer formats become unorm values
// in [0, 1] (encoded_bytes = true: the values are sRGB-encoded where the usage says colour).
struct Pixels {
    uint32_t           width         = 0;
    uint32_t           height        = 0;
    uint32_t           channels      = 0;
    bool               encoded_bytes = false;
    std::vector<float> values;
};

// PNG: 8- or 16-bit grey, grey + alpha, RGB, RGBA or 8-bit palette images, not interlaced.
bool read_png(std::string const& path, Pixels& out, std::string& error);

// OpenEXR: single-part scanline files, half or float channels, no or ZIP / ZIPS compression;
// channels in the order R, G, B, A of those present (others in name order after them).
bool read_exr(std::string const& path, Pixels& out, std::string& error);

// Either, by the file's magic bytes.
bool read_image(std::string const& path, Pixels& out, std::string& error);

}  // namespace spb::image_io
