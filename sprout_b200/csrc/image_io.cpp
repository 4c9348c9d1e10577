// PNG and OpenEXR readers; see image_io.hpp.  Both formats are read as their specifications
// define them (PNG 1.2: chunks, zlib stream, per-row filters; OpenEXR 2: header attributes,
// offset table, scanline blocks, ZIP predictor), with the system zlib for inflation.
#include "image_io.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>

#include <zlib.h>

namespace spb::image_io {

namespace {

bool read_file(std::string const& path, std::vector<uint8_t>& data) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        return false;
    }
    std::fseek(f, 0, SEEK_END);
    long const size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    data.resize(size > 0 ? size_t(size) : 0);
    bool const ok = data.empty() || std::fread(data.data(), 1, data.size(), f) == data.size();
    std::fclose(f);
    return ok;
}

uint32_t be32(uint8_t const* p) {
    return (uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) | p[3];
}

template <typename T>
T le(std::vector<uint8_t> const& d, size_t at) {
    T v;
    std::memcpy(&v, d.data() + at, sizeof(T));
    return v;
}

float half_to_float(uint16_t h) {
    uint32_t const sign = uint32_t(h & 0x8000u) << 16;
    uint32_t const e    = (h >> 10) & 0x1Fu;
    uint32_t const m    = h & 0x3FFu;
    uint32_t       bits;
    if (e == 0) {
        if (m == 0) {
            bits = sign;
        } else {  // subnormal: m 2^-24
            float const v = float(m) * (1.f / 16777216.f);
            std::memcpy(&bits, &v, 4);
            bits |= sign;
        }
    } else if (e == 31) {
        bits = sign | 0x7F800000u | (m << 13);
    } else {
        bits = sign | ((e + 112u) << 23) | (m << 13);
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

int paeth(int a, int b, int c) {
    int const p  = a + b - c;
    int const pa = std::abs(p - a);
    int const pb = std::abs(p - b);
    int const pc = std::abs(p - c);
    return (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
}

}  // namespace

bool read_png(std::string const& path, Pixels& out, std::string& error) {
    std::vector<uint8_t> d;
    if (!read_file(path, d)) {
        error = "cannot read " + path;
        return false;
    }
    static uint8_t const signature[8] = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
    if (d.size() < 8 || std::memcmp(d.data(), signature, 8) != 0) {
        error = path + " is not a PNG file";
        return false;
    }
    uint32_t             width = 0, height = 0, depth = 0, type = 0;
    std::vector<uint8_t> idat, palette;
    for (size_t at = 8; at + 12 <= d.size();) {
        uint32_t const len = be32(&d[at]);
        if (at + 12 + size_t(len) > d.size()) {
            error = path + ": truncated chunk";
            return false;
        }
        char const* kind = reinterpret_cast<char const*>(&d[at + 4]);
        uint8_t const* body = &d[at + 8];
        if (std::memcmp(kind, "IHDR", 4) == 0 && len >= 13) {
            width  = be32(body);
            height = be32(body + 4);
            depth  = body[8];
            type   = body[9];
            if (body[12] != 0) {
                error = path + ": interlaced PNG not supported";
                return false;
            }
        } else if (std::memcmp(kind, "PLTE", 4) == 0) {
            palette.assign(body, body + len);
        } else if (std::memcmp(kind, "IDAT", 4) == 0) {
            idat.insert(idat.end(), body, body + len);
        } else if (std::memcmp(kind, "IEND", 4) == 0) {
            break;
        }
        at += 12 + size_t(len);
    }
    uint32_t const channels = type == 0 ? 1 : type == 2 ? 3 : type == 3 ? 1 : type == 4 ? 2 : type == 6 ? 4 : 0;
    if (width == 0 || height == 0 || channels == 0 || (depth != 8 && depth != 16) || (type == 3 && depth != 8)) {
        error = path + ": unsupported PNG (bit depth " + std::to_string(depth) + ", colour type " +
                std::to_string(type) + ")";
        return false;
    }
    size_t const bpp      = channels * depth / 8;  // bytes per pixel, for the filters
    size_t const row      = size_t(width) * bpp;
    uLongf       raw_size = uLongf((row + 1) * height);
    std::vector<uint8_t> raw(raw_size);
    if (uncompress(raw.data(), &raw_size, idat.data(), uLong(idat.size())) != Z_OK || raw_size != raw.size()) {
        error = path + ": corrupt image data";
        return false;
    }
    std::vector<uint8_t> img(row * height);
    for (uint32_t y = 0; y < height; ++y) {
        uint8_t const  filter = raw[y * (row + 1)];
        uint8_t const* src    = &raw[y * (row + 1) + 1];
        uint8_t*       dst    = &img[y * row];
        uint8_t const* up     = y > 0 ? &img[(y - 1) * row] : nullptr;
        for (size_t i = 0; i < row; ++i) {
            int const a = i >= bpp ? dst[i - bpp] : 0;
            int const b = up ? up[i] : 0;
            int const c = (up && i >= bpp) ? up[i - bpp] : 0;
            int       v = src[i];
            switch (filter) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) / 2; break;
                case 4: v += paeth(a, b, c); break;
                default: error = path + ": bad PNG row filter"; return false;
            }
            dst[i] = uint8_t(v);
        }
    }
    out.width         = width;
    out.height        = height;
    out.encoded_bytes = true;
    if (type == 3) {
        out.channels = 3;
        out.values.resize(size_t(width) * height * 3);
        for (size_t p = 0; p < size_t(width) * height; ++p) {
            size_t const k = size_t(img[p]) * 3;
            for (int c = 0; c < 3; ++c) {
                out.values[3 * p + c] = k + c < palette.size() ? float(palette[k + c]) / 255.f : 0.f;
            }
        }
        return true;
    }
    out.channels = channels;
    out.values.resize(size_t(width) * height * channels);
    for (size_t i = 0; i < out.values.size(); ++i) {
        out.values[i] = depth == 8 ? float(img[i]) / 255.f
                                   : float((uint32_t(img[2 * i]) << 8) | img[2 * i + 1]) / 65535.f;
    }
    return true;
}

bool read_exr(std::string const& path, Pixels& out, std::string& error) {
    std::vector<uint8_t> d;
    if (!read_file(path, d)) {
        error = "cannot read " + path;
        return false;
    }
    if (d.size() < 8 || le<uint32_t>(d, 0) != 20000630u) {
        error = path + " is not an EXR file";
        return false;
    }
    if (le<uint32_t>(d, 4) & 0x1A00u) {  // tiled, long names with deep data, multi-part
        error = path + ": only single-part scanline EXR files are supported";
        return false;
    }
    struct Channel {
        std::string name;
        int32_t     type;  // 0 uint, 1 half, 2 float
    };
    std::vector<Channel> chans;
    int                  compression = -1;
    int32_t              box[4]      = {0, 0, -1, -1};
    size_t               at          = 8;
    auto const           cstring     = [&](std::string& s) {
        size_t const end = std::find(d.begin() + long(at), d.end(), uint8_t(0)) - d.begin();
        if (end >= d.size()) {
            return false;
        }
        s.assign(reinterpret_cast<char const*>(&d[at]), end - at);
        at = end + 1;
        return true;
    };
    for (;;) {
        std::string name, type;
        if (!cstring(name)) {
            error = path + ": truncated header";
            return false;
        }
        if (name.empty()) {
            break;
        }
        if (!cstring(type) || at + 4 > d.size()) {
            error = path + ": truncated header";
            return false;
        }
        int32_t const size = le<int32_t>(d, at);
        at += 4;
        size_t const end = at + size_t(size);
        if (size < 0 || end > d.size()) {
            error = path + ": bad attribute";
            return false;
        }
        if (type == "chlist") {
            while (at < end && d[at] != 0) {
                Channel c;
                cstring(c.name);
                c.type = le<int32_t>(d, at);
                chans.push_back(c);
                at += 16;
            }
        } else if (type == "compression") {
            compression = d[at];
        } else if (name == "dataWindow" && type == "box2i") {
            for (int k = 0; k < 4; ++k) {
                box[k] = le<int32_t>(d, at + 4 * size_t(k));
            }
        }
        at = end;
    }
    int32_t const width  = box[2] - box[0] + 1;
    int32_t const height = box[3] - box[1] + 1;
    int const     lines  = compression == 0 || compression == 2 ? 1 : (compression == 3 ? 16 : 0);
    if (width <= 0 || height <= 0 || chans.empty() || lines == 0) {
        error = path + ": unsupported EXR (compression " + std::to_string(compression) + ")";
        return false;
    }
    std::sort(chans.begin(), chans.end(), [](Channel const& a, Channel const& b) { return a.name < b.name; });
    // output order: R, G, B, A, Y (those present), then the rest
    std::vector<size_t> order;
    for (char const* want : {"R", "G", "B", "A", "Y"}) {
        for (size_t c = 0; c < chans.size(); ++c) {
            if (chans[c].name == want) {
                order.push_back(c);
            }
        }
    }
    for (size_t c = 0; c < chans.size(); ++c) {
        if (std::find(order.begin(), order.end(), c) == order.end()) {
            order.push_back(c);
        }
    }
    std::vector<size_t> slot(chans.size());
    for (size_t k = 0; k < order.size(); ++k) {
        slot[order[k]] = k;
    }
    size_t bytes_per_pixel = 0;
    for (Channel const& c : chans) {
        bytes_per_pixel += c.type == 1 ? 2 : 4;
    }
    out.width         = uint32_t(width);
    out.height        = uint32_t(height);
    out.channels      = uint32_t(chans.size());
    out.encoded_bytes = false;
    out.values.assign(size_t(width) * height * chans.size(), 0.f);
    int const            blocks = (height + lines - 1) / lines;
    size_t               table  = at;
    std::vector<uint8_t> raw, tmp;
    for (int b = 0; b < blocks; ++b) {
        uint64_t const off = le<uint64_t>(d, table + 8 * size_t(b));
        if (off + 8 > d.size()) {
            error = path + ": bad offset table";
            return false;
        }
        int32_t const y0   = le<int32_t>(d, off) - box[1];
        int32_t const size = le<int32_t>(d, off + 4);
        int32_t const n    = std::min(lines, height - y0);
        size_t const  need = size_t(n) * width * bytes_per_pixel;
        if (y0 < 0 || n <= 0 || size < 0 || off + 8 + size_t(size) > d.size()) {
            error = path + ": bad block";
            return false;
        }
        uint8_t const* src = &d[off + 8];
        if (compression != 0 && size_t(size) < need) {
            tmp.resize(need);
            uLongf got = uLongf(need);
            if (uncompress(tmp.data(), &got, src, uLong(size)) != Z_OK || got != need) {
                error = path + ": corrupt ZIP block";
                return false;
            }
            for (size_t i = 1; i < need; ++i) {
                tmp[i] = uint8_t(tmp[i - 1] + tmp[i] - 128);
            }
            raw.resize(need);
            size_t const half = (need + 1) / 2;
            for (size_t i = 0; i < need; ++i) {
                raw[i] = (i & 1) ? tmp[half + i / 2] : tmp[i / 2];
            }
            src = raw.data();
        } else if (size_t(size) < need) {
            error = path + ": short block";
            return false;
        }
        size_t pos = 0;
        for (int32_t y = y0; y < y0 + n; ++y) {
            for (size_t c = 0; c < chans.size(); ++c) {
                for (int32_t x = 0; x < width; ++x) {
                    float v;
                    if (chans[c].type == 1) {
                        uint16_t h;
                        std::memcpy(&h, src + pos, 2);
                        v = half_to_float(h);
                        pos += 2;
                    } else if (chans[c].type == 2) {
                        std::memcpy(&v, src + pos, 4);
                        pos += 4;
                    } else {
                        uint32_t u;
                        std::memcpy(&u, src + pos, 4);
                        v = float(u);
                        pos += 4;
                    }
                    out.values[(size_t(y) * width + x) * chans.size() + slot[c]] = v;
                }
            }
        }
    }
    return true;
}

bool read_image(std::string const& path, Pixels& out, std::string& error) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        error = "cannot read " + path;
        return false;
    }
    uint8_t magic[4] = {0, 0, 0, 0};
    size_t const got = std::fread(magic, 1, 4, f);
    std::fclose(f);
    if (got == 4 && magic[0] == 0x89 && magic[1] == 'P') {
        return read_png(path, out, error);
    }
    if (got == 4 && magic[0] == 0x76 && magic[1] == 0x2F && magic[2] == 0x31 && magic[3] == 0x01) {
        return read_exr(path, out, error);
    }
    error = path + ": not a PNG or EXR file";
    return false;
}

}  // namespace spb::image_io
