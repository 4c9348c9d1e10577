// Deterministic synthetic inputs for the cast benchmark: a displaced tetra-sphere mesh and
// uniformly distributed rays.  Every value is computed with IEEE add/sub/mul/div/sqrt and
// floor only (this file is compiled with -ffp-contract=off), so the same inputs are produced
// on any x86-64 host.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>

#include "common.hpp"

namespace {

// PCG32 (O'Neill 2014, XSH-RR output), seeded the way the reference's rnd::Generator::start
// seeds it (source/base/random/generator.inl:16-24): state 0, inc = 2*sequence+1, one step,
// add the seed, one step.
struct Pcg32 {
    uint64_t state = 0;
    uint64_t inc   = 1;

    Pcg32(uint64_t seed, uint64_t sequence) {
        inc = (sequence << 1u) | 1u;
        next();
        state += seed;
        next();
    }

    uint32_t next() {
        uint64_t const old = state;
        state              = old * 6364136223846793005ull + (inc | 1);
        uint32_t const xrs = uint32_t(((old >> 18u) ^ old) >> 27u);
        uint32_t const rot = uint32_t(old >> 59u);
        return (xrs >> rot) | (xrs << ((0u - rot) & 31u));
    }

    // Uniform in [0, 1) with 23 bits: the mantissa of a float in [1, 2), minus one.
    float uniform() {
        uint32_t const bits = (next() & 0x007FFFFFu) | 0x3F800000u;
        float          f;
        std::memcpy(&f, &bits, 4);
        return f - 1.f;
    }
};

// 3-D gradient noise with a seeded permutation and the 12 cube-edge gradients, quintic fade.
class Gradient_noise {
  public:
    explicit Gradient_noise(uint32_t seed) {
        for (uint32_t i = 0; i < 256; ++i) {
            perm_[i] = uint8_t(i);
        }
        Pcg32 rng(seed, 0x5eed);
        for (uint32_t i = 255; i > 0; --i) {
            uint32_t const j = rng.next() % (i + 1);
            std::swap(perm_[i], perm_[j]);
        }
    }

    double operator()(double x, double y, double z) const {
        double const fx = std::floor(x);
        double const fy = std::floor(y);
        double const fz = std::floor(z);

        int32_t const ix = int32_t(fx) & 255;
        int32_t const iy = int32_t(fy) & 255;
        int32_t const iz = int32_t(fz) & 255;

        double const rx = x - fx;
        double const ry = y - fy;
        double const rz = z - fz;

        double const u = fade(rx);
        double const v = fade(ry);
        double const w = fade(rz);

        double c[8];
        for (int32_t k = 0; k < 8; ++k) {
            int32_t const dx = k & 1;
            int32_t const dy = (k >> 1) & 1;
            int32_t const dz = (k >> 2) & 1;
            uint32_t const h = hash(ix + dx, iy + dy, iz + dz);
            c[k]             = grad(h, rx - dx, ry - dy, rz - dz);
        }

        double const x00 = lerp(c[0], c[1], u);
        double const x10 = lerp(c[2], c[3], u);
        double const x01 = lerp(c[4], c[5], u);
        double const x11 = lerp(c[6], c[7], u);
        double const y0  = lerp(x00, x10, v);
        double const y1  = lerp(x01, x11, v);
        return lerp(y0, y1, w);
    }

  private:
    static double fade(double t) {
        return t * t * t * (t * (t * 6. - 15.) + 10.);
    }

    static double lerp(double a, double b, double t) {
        return a + t * (b - a);
    }

    uint32_t hash(int32_t x, int32_t y, int32_t z) const {
        return perm_[(perm_[(perm_[x & 255] + y) & 255] + z) & 255];
    }

    static double grad(uint32_t h, double x, double y, double z) {
        switch (h % 12) {
            case 0: return x + y;
            case 1: return -x + y;
            case 2: return x - y;
            case 3: return -x - y;
            case 4: return x + z;
            case 5: return -x + z;
            case 6: return x - z;
            case 7: return -x - z;
            case 8: return y + z;
            case 9: return -y + z;
            case 10: return y - z;
            default: return -y - z;
        }
    }

    uint8_t perm_[256];
};

// fBm: 6 octaves, lacunarity 2, gain 0.5, base frequency 3, normalised by the sum of the
// octave weights so the result stays within about [-1, 1].
double fbm(Gradient_noise const& noise, double x, double y, double z) {
    double sum    = 0.;
    double norm   = 0.;
    double amp    = 1.;
    double freq   = 3.;
    for (int32_t o = 0; o < 6; ++o) {
        double const off = 17.0 * double(o);
        sum += amp * noise(x * freq + off, y * freq + 0.5 * off, z * freq + 0.25 * off);
        norm += amp;
        amp *= 0.5;
        freq *= 2.;
    }
    return sum / norm;
}

}  // namespace

extern "C" SPB_API int32_t spb_synth_sphere_mesh(uint32_t n, float amplitude, uint32_t seed,
                                                 uint32_t* num_vertices, uint32_t* num_triangles,
                                                 float* positions, uint32_t* indices) {
    spb::clear_error();
    if (n == 0 || n > 16384 || !num_vertices || !num_triangles) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_synth_sphere_mesh: n must be in [1, 16384]");
    }

    uint32_t const nv = 2 * n * n + 2;
    uint32_t const nt = 4 * n * n;
    *num_vertices     = nv;
    *num_triangles    = nt;
    if (!positions && !indices) {
        return SPB_OK;
    }
    if (!positions || !indices) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_synth_sphere_mesh: need both buffers");
    }

    static double const corners[4][3] = {{1., 1., 1.}, {1., -1., -1.}, {-1., 1., -1.},
                                         {-1., -1., 1.}};
    // Faces wound counter-clockwise seen from outside.
    static uint32_t const faces[4][3] = {{0, 2, 1}, {0, 1, 3}, {0, 3, 2}, {1, 2, 3}};

    Gradient_noise const noise(seed);

    // A lattice point is identified by its integer weights over the 4 corners (they sum to
    // n), so points on shared edges get one vertex whichever face reaches them first.
    std::unordered_map<uint64_t, uint32_t> ids;
    ids.reserve(size_t(nv) * 2);
    uint32_t next_vertex = 0;

    auto vertex = [&](uint32_t const w[4]) -> uint32_t {
        uint64_t const key = uint64_t(w[0]) | (uint64_t(w[1]) << 16) | (uint64_t(w[2]) << 32) |
                             (uint64_t(w[3]) << 48);
        auto const it = ids.find(key);
        if (it != ids.end()) {
            return it->second;
        }
        double p[3] = {0., 0., 0.};
        for (int32_t k = 0; k < 4; ++k) {
            for (int32_t a = 0; a < 3; ++a) {
                p[a] += double(w[k]) * corners[k][a];
            }
        }
        double const len = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        double const ux  = p[0] / len;
        double const uy  = p[1] / len;
        double const uz  = p[2] / len;
        double const r   = 1. + double(amplitude) * fbm(noise, ux, uy, uz);

        uint32_t const id      = next_vertex++;
        positions[3 * id + 0] = float(ux * r);
        positions[3 * id + 1] = float(uy * r);
        positions[3 * id + 2] = float(uz * r);
        ids.emplace(key, id);
        return id;
    };

    uint32_t tri = 0;
    auto lattice = [&](uint32_t const f[3], uint32_t i, uint32_t j) -> uint32_t {
        uint32_t w[4] = {0, 0, 0, 0};
        w[f[0]] += n - i - j;
        w[f[1]] += i;
        w[f[2]] += j;
        return vertex(w);
    };

    for (auto const& f : faces) {
        for (uint32_t i = 0; i < n; ++i) {
            for (uint32_t j = 0; i + j < n; ++j) {
                uint32_t const a = lattice(f, i, j);
                uint32_t const b = lattice(f, i + 1, j);
                uint32_t const c = lattice(f, i, j + 1);
                indices[3 * tri + 0] = a;
                indices[3 * tri + 1] = b;
                indices[3 * tri + 2] = c;
                ++tri;
                if (i + j + 1 < n) {
                    uint32_t const d = lattice(f, i + 1, j + 1);
                    indices[3 * tri + 0] = b;
                    indices[3 * tri + 1] = d;
                    indices[3 * tri + 2] = c;
                    ++tri;
                }
            }
        }
    }

    if (tri != nt || next_vertex != nv) {
        return spb::fail(SPB_ERROR_STATE, "spb_synth_sphere_mesh: lattice count mismatch");
    }
    return SPB_OK;
}

extern "C" SPB_API int32_t spb_synth_rays(uint64_t first, uint64_t count, uint32_t seed,
                                          float extent, float* rays, uint32_t num_threads) {
    spb::clear_error();
    if (count > 0 && !rays) {
        return spb::fail(SPB_ERROR_ARGUMENT, "spb_synth_rays: rays is null");
    }

    float const ray_max_t = 3.4027715434167032e+38f;

    spb::parallel_ranges(count, spb::resolve_threads(num_threads),
                         [&](uint32_t, uint64_t begin, uint64_t end) {
                             for (uint64_t k = begin; k < end; ++k) {
                                 Pcg32 rng(seed, first + k);
                                 float* r = rays + 8 * k;
                                 for (int32_t a = 0; a < 3; ++a) {
                                     r[a] = extent * (2.f * rng.uniform() - 1.f);
                                 }
                                 r[3] = 0.f;
                                 // z uniform in [-1, 1], azimuth from a point rejection-sampled in
                                 // the unit disk (no trigonometric functions involved).
                                 float const z = 1.f - 2.f * rng.uniform();
                                 float       a;
                                 float       b;
                                 float       s;
                                 do {
                                     a = 2.f * rng.uniform() - 1.f;
                                     b = 2.f * rng.uniform() - 1.f;
                                     s = a * a + b * b;
                                 } while (s > 1.f || s < 1e-12f);
                                 float const rr = std::sqrt(std::max(0.f, 1.f - z * z));
                                 float const k2 = rr / std::sqrt(s);
                                 r[4]           = a * k2;
                                 r[5]           = b * k2;
                                 r[6]           = z;
                                 r[7]           = ray_max_t;
                             }
                         });
    return SPB_OK;
}
