// Hero-wavelength spectral transport (no counterpart in the reference, which renders RGB): the
// colour arithmetic shared by the renderer's spectral mode (host and device) and restated by
// the FP64 oracle (oracle/spectral_oracle.c).
//
// A path carries Hero_count wavelengths: a hero wavelength drawn uniformly from
// [Lambda_min, Lambda_max] and the others at equal steps of the range, wrapped into it
// (Wilkie et al., "Hero Wavelength Spectral Sampling", EGSR 2014).  Every RGB quantity of the
// scene (emission, medium coefficients) is upsampled to a spectrum as a blend of three smooth
// basis functions that sum to one at every wavelength (so grey stays flat):
//     s(lambda) = r S_r(lambda) + g S_g(lambda) + b S_b(lambda),
// S_b = 1 - t1, S_g = t1 - t2, S_r = t2 with t1, t2 smoothsteps over [465, 515] and [560, 610] nm.
// The film reads a path's radiance through the CIE 1931 colour-matching functions (the
// multi-lobe Gaussian fit of Wyman, Sloan and Shirley, JCGT 2013), then XYZ -> linear sRGB
// (IEC 61966-2-1) -> ACEScg (the renderer's working space), and a 3x3 correction that makes
// the basis round-trip: an upsampled colour reads back as itself.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define SPB_SPEC_HD __host__ __device__ __forceinline__
#else
#define SPB_SPEC_HD inline
#endif

namespace spb::spectral {

constexpr int   Hero_count = 4;
// The renderer's sRGB -> ACEScg conversion (row-major; the same matrix converts material colours).
constexpr double Srgb_to_ap1[9] = {0.61309732, 0.33952285, 0.04737928, 0.07019422, 0.91635557,
                                   0.01345259, 0.02061560, 0.10956983, 0.86981512};
constexpr float Lambda_min = 380.f;
constexpr float Lambda_max = 720.f;
constexpr float Lambda_span = Lambda_max - Lambda_min;

// A value per carried wavelength.
struct V4 {
    float v[Hero_count];
};

SPB_SPEC_HD V4 splat(float x) {
    V4 r;
    for (int k = 0; k < Hero_count; ++k) {
        r.v[k] = x;
    }
    return r;
}
SPB_SPEC_HD V4 mul(V4 a, V4 b) {
    for (int k = 0; k < Hero_count; ++k) {
        a.v[k] *= b.v[k];
    }
    return a;
}
SPB_SPEC_HD V4 scale(float s, V4 a) {
    for (int k = 0; k < Hero_count; ++k) {
        a.v[k] *= s;
    }
    return a;
}
SPB_SPEC_HD V4 add(V4 a, V4 b) {
    for (int k = 0; k < Hero_count; ++k) {
        a.v[k] += b.v[k];
    }
    return a;
}
SPB_SPEC_HD float average(V4 a) {
    float s = 0.f;
    for (int k = 0; k < Hero_count; ++k) {
        s += a.v[k];
    }
    return s * (1.f / Hero_count);
}
SPB_SPEC_HD float maximum(V4 a) {
    float m = a.v[0];
    for (int k = 1; k < Hero_count; ++k) {
        m = a.v[k] > m ? a.v[k] : m;
    }
    return m;
}

// The carried wavelengths for a hero wavelength drawn as u in [0, 1).
SPB_SPEC_HD V4 wavelengths(float u) {
    V4 l;
    for (int k = 0; k < Hero_count; ++k) {
        float x = u + float(k) / Hero_count;
        x       = x >= 1.f ? x - 1.f : x;
        l.v[k]  = Lambda_min + Lambda_span * x;
    }
    return l;
}

SPB_SPEC_HD float smoothstep01(float x) {
    x = x < 0.f ? 0.f : (x > 1.f ? 1.f : x);
    return x * x * (3.f - 2.f * x);
}

// The basis at one wavelength: (S_r, S_g, S_b).
SPB_SPEC_HD void basis(float lambda, float& r, float& g, float& b) {
    float const t1 = smoothstep01((lambda - 465.f) * (1.f / 50.f));
    float const t2 = smoothstep01((lambda - 560.f) * (1.f / 50.f));
    r              = t2;
    g              = t1 - t2;
    b              = 1.f - t1;
}

// An RGB triple upsampled at the carried wavelengths.
SPB_SPEC_HD V4 upsample(float r, float g, float b, V4 lambdas) {
    V4 s;
    for (int k = 0; k < Hero_count; ++k) {
        float sr, sg, sb;
        basis(lambdas.v[k], sr, sg, sb);
        s.v[k] = r * sr + g * sg + b * sb;
    }
    return s;
}

// One lobe of the colour-matching fit: a Gaussian with different widths left and right of mu.
SPB_SPEC_HD double lobe(double lambda, double mu, double left, double right) {
    double const t = (lambda - mu) / (lambda < mu ? left : right);
    return std::exp(-0.5 * t * t);
}

// CIE 1931 2-degree colour-matching functions (Wyman, Sloan and Shirley 2013, multi-lobe fit).
SPB_SPEC_HD void cmf(double lambda, double& x, double& y, double& z) {
    x = 1.056 * lobe(lambda, 599.8, 37.9, 31.0) + 0.362 * lobe(lambda, 442.0, 16.0, 26.7) -
        0.065 * lobe(lambda, 501.1, 20.4, 26.2);
    y = 0.821 * lobe(lambda, 568.8, 46.9, 40.5) + 0.286 * lobe(lambda, 530.9, 16.3, 31.1);
    z = 1.217 * lobe(lambda, 437.0, 11.8, 36.0) + 0.681 * lobe(lambda, 459.0, 26.0, 13.8);
}

// The film's response to one wavelength, before the round-trip correction: XYZ -> linear
// sRGB -> ACEScg.  srgb_to_ap1 is the renderer's conversion (row-major 3x3).
SPB_SPEC_HD void response(double lambda, double const srgb_to_ap1[9], double out[3]) {
    double x, y, z;
    cmf(lambda, x, y, z);
    double const s[3] = {3.2406 * x - 1.5372 * y - 0.4986 * z, -0.9689 * x + 1.8758 * y + 0.0415 * z,
                         0.0557 * x - 0.2040 * y + 1.0570 * z};
    for (int i = 0; i < 3; ++i) {
        out[i] = srgb_to_ap1[3 * i] * s[0] + srgb_to_ap1[3 * i + 1] * s[1] + srgb_to_ap1[3 * i + 2] * s[2];
    }
}

// The readout matrix C with C G = I, G[i][j] = integral over [Lambda_min, Lambda_max] of
// response_i(lambda) basis_j(lambda) (midpoint rule, 0.25 nm), so that a path carrying the
// upsampled spectrum of an RGB colour reads back as that colour:
//     rgb = C * (Lambda_span / Hero_count) * sum_k L(lambda_k) response(lambda_k).
inline void readout_matrix(double const srgb_to_ap1[9], double c[9]) {
    double       g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double const step = 0.25;
    for (double l = Lambda_min + 0.5 * step; l < Lambda_max; l += step) {
        double resp[3];
        response(l, srgb_to_ap1, resp);
        float br, bg, bb;
        basis(float(l), br, bg, bb);
        double const b[3] = {br, bg, bb};
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) {
                g[3 * i + j] += resp[i] * b[j] * step;
            }
        }
    }
    // inverse of the 3x3 g
    double const det = g[0] * (g[4] * g[8] - g[5] * g[7]) - g[1] * (g[3] * g[8] - g[5] * g[6]) +
                       g[2] * (g[3] * g[7] - g[4] * g[6]);
    double const id = 1.0 / det;
    c[0]            = (g[4] * g[8] - g[5] * g[7]) * id;
    c[1]            = (g[2] * g[7] - g[1] * g[8]) * id;
    c[2]            = (g[1] * g[5] - g[2] * g[4]) * id;
    c[3]            = (g[5] * g[6] - g[3] * g[8]) * id;
    c[4]            = (g[0] * g[8] - g[2] * g[6]) * id;
    c[5]            = (g[2] * g[3] - g[0] * g[5]) * id;
    c[6]            = (g[3] * g[7] - g[4] * g[6]) * id;
    c[7]            = (g[1] * g[6] - g[0] * g[7]) * id;
    c[8]            = (g[0] * g[4] - g[1] * g[3]) * id;
}

// XYZ -> linear sRGB, derived from the sRGB primaries' chromaticities (0.64, 0.33), (0.30, 0.60),
// (0.15, 0.06) and the D65 white point (0.3127, 0.3290) (IEC 61966-2-1): the matrix whose
// inverse maps each primary to its XYZ, scaled so that RGB (1, 1, 1) is the white of luminance 1.
inline void xyz_to_srgb(double out[9]) {
    double const xr = 0.64, yr = 0.33, xg = 0.30, yg = 0.60, xb = 0.15, yb = 0.06, xw = 0.3127, yw = 0.3290;
    double const p[9] = {xr / yr, xg / yg, xb / yb, 1.0, 1.0, 1.0, (1.0 - xr - yr) / yr, (1.0 - xg - yg) / yg,
                         (1.0 - xb - yb) / yb};
    double const w[3] = {xw / yw, 1.0, (1.0 - xw - yw) / yw};
    auto const   inverse = [](double const a[9], double r[9]) {
        double const det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                           a[2] * (a[3] * a[7] - a[4] * a[6]);
        r[0] = (a[4] * a[8] - a[5] * a[7]) / det;
        r[1] = (a[2] * a[7] - a[1] * a[8]) / det;
        r[2] = (a[1] * a[5] - a[2] * a[4]) / det;
        r[3] = (a[5] * a[6] - a[3] * a[8]) / det;
        r[4] = (a[0] * a[8] - a[2] * a[6]) / det;
        r[5] = (a[2] * a[3] - a[0] * a[5]) / det;
        r[6] = (a[3] * a[7] - a[4] * a[6]) / det;
        r[7] = (a[1] * a[6] - a[0] * a[7]) / det;
        r[8] = (a[0] * a[4] - a[1] * a[3]) / det;
    };
    double pi[9];
    inverse(p, pi);
    double s[3];
    for (int i = 0; i < 3; ++i) {
        s[i] = pi[3 * i] * w[0] + pi[3 * i + 1] * w[1] + pi[3 * i + 2] * w[2];
    }
    double m[9];  // RGB -> XYZ: the primaries' columns scaled by s
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            m[3 * r + c] = p[3 * r + c] * s[c];
        }
    }
    inverse(m, out);
}

// The colour of a black body at `kelvin` as linear sRGB with its largest XYZ component 1,
// negative components clamped (spectrum::blackbody, mapping.cpp:84-147): Planck's law summed
// at 5 nm steps over 380-780 nm against the colour-matching functions.  The reference sums
// against a 5 nm tabulation of the CIE 1931 observer; here the functions are the multi-lobe
// fit above, whose colours agree within 0.4 % from 4000 to 5000 K and differ by up to 3 % (and
// 6 % of a blue near 0) at 2000 K.
inline void blackbody(double kelvin, double out[3]) {
    double const h = 6.62606896e-34, c = 2.99792458e8, k = 1.3806488e-23;
    double       xyz[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i <= 80; ++i) {
        double const nm = 380.0 + 5.0 * i;
        double const wl = nm * 1e-9;
        double const p  = (2.0 * 3.14159265358979323846 * h * c * c) / (wl * wl * wl * wl * wl) /
                         (std::exp(h * c / (wl * k * kelvin)) - 1.0);
        double x, y, z;
        cmf(nm, x, y, z);
        xyz[0] += p * x;
        xyz[1] += p * y;
        xyz[2] += p * z;
    }
    double const mx = std::fmax(xyz[0], std::fmax(xyz[1], xyz[2]));
    double       m[9];
    xyz_to_srgb(m);
    for (int i = 0; i < 3; ++i) {
        double const v = (m[3 * i] * xyz[0] + m[3 * i + 1] * xyz[1] + m[3 * i + 2] * xyz[2]) / mx;
        out[i]         = v > 0.0 ? v : 0.0;
    }
}

}  // namespace spb::spectral
