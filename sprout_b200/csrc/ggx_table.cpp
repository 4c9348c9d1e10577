// Directional albedo of the GGX lobe without Fresnel, E(cos_theta_o, alpha), on a 32 x 32
// grid over [0, 1]^2 -- the table the energy compensation ilm_ep_conductor reads
// (reference: material/ggx/ggx.inl:27-29).  Computed here with the estimator the
// reference's table generator uses (material/ggx/ggx_integrate.cpp:17-48, table layout
// :199-230): 1024 Hammersley points, visible-normal sampling, weight n.wi * D V / pdf, and
// E = 1 below the minimum alpha.  Evaluated in double precision.
#include <cmath>
#include <cstdint>
#include <mutex>

#include "ggx_table.hpp"

namespace spb {

namespace {

double radical_inverse2(uint32_t i) {
    i = (i << 16u) | (i >> 16u);
    i = ((i & 0x55555555u) << 1u) | ((i & 0xAAAAAAAAu) >> 1u);
    i = ((i & 0x33333333u) << 2u) | ((i & 0xCCCCCCCCu) >> 2u);
    i = ((i & 0x0F0F0F0Fu) << 4u) | ((i & 0xF0F0F0F0u) >> 4u);
    i = ((i & 0x00FF00FFu) << 8u) | ((i & 0xFF00FF00u) >> 8u);
    return double(i) * 2.3283064365386963e-10;
}

double clamp_cos(double x) {
    return std::fmin(std::fmax(x, 0.00001), 1.0);
}

double albedo(double alpha, double n_dot_wo, uint32_t num_samples) {
    double const min_alpha = 0.01314 * 0.01314;
    if (alpha < min_alpha) {
        return 1.0;
    }
    double const pi = 3.14159265358979323846;
    n_dot_wo        = clamp_cos(n_dot_wo);
    // wo = (sin, 0, cos) in the tangent frame
    double const wo[3] = {std::sqrt(1.0 - n_dot_wo * n_dot_wo), 0.0, n_dot_wo};
    double const a2    = alpha * alpha;

    double sum = 0.0;
    for (uint32_t i = 0; i < num_samples; ++i) {
        double const xi0 = double(i) / double(num_samples);
        double const xi1 = radical_inverse2(i);

        // visible-normal sample (stretch, sample the projected disk, unstretch)
        double v[3] = {alpha * wo[0], alpha * wo[1], wo[2]};
        double const vl = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        for (double& c : v) {
            c /= vl;
        }
        double t1[3] = {1.0, 0.0, 0.0};
        if (v[2] < 0.9999) {
            double const l = std::sqrt(v[1] * v[1] + v[0] * v[0]);
            t1[0]          = v[1] / l;
            t1[1]          = -v[0] / l;
            t1[2]          = 0.0;
        }
        double const t2[3] = {t1[1] * v[2], -t1[0] * v[2], t1[0] * v[1] - t1[1] * v[0]};
        double const a     = 1.0 / (1.0 + v[2]);
        double const r     = std::sqrt(xi0);
        double const phi   = xi1 < a ? xi1 / a * pi : pi + (xi1 - a) / (1.0 - a) * pi;
        double const p1    = r * std::cos(phi);
        double const p2    = r * std::sin(phi) * (xi1 < a ? 1.0 : v[2]);
        double const p3    = std::sqrt(std::fmax(1.0 - p1 * p1 - p2 * p2, 0.0));
        double m[3];
        for (int k = 0; k < 3; ++k) {
            m[k] = p1 * t1[k] + p2 * t2[k] + p3 * v[k];
        }
        double h[3]      = {alpha * m[0], alpha * m[1], std::fmax(m[2], 0.0)};
        double const hl  = std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
        for (double& c : h) {
            c /= hl;
        }
        double const n_dot_h  = std::fmin(std::fmax(h[2], 0.0), 1.0);
        double const wo_dot_h = clamp_cos(wo[0] * h[0] + wo[1] * h[1] + wo[2] * h[2]);
        double wi[3];
        for (int k = 0; k < 3; ++k) {
            wi[k] = 2.0 * wo_dot_h * h[k] - wo[k];
        }
        double const wl = std::sqrt(wi[0] * wi[0] + wi[1] * wi[1] + wi[2] * wi[2]);
        double const n_dot_wi = clamp_cos(wi[2] / wl);

        double const dd  = (n_dot_h * n_dot_h) * (a2 - 1.0) + 1.0;
        double const d   = a2 / (pi * dd * dd);
        double const twi = std::sqrt(a2 + (1.0 - a2) * n_dot_wi * n_dot_wi);
        double const two = std::sqrt(a2 + (1.0 - a2) * n_dot_wo * n_dot_wo);
        double const vis = 0.5 / (n_dot_wi * two + n_dot_wo * twi);
        double const pdf = 0.5 * d / (two + n_dot_wo);
        sum += n_dot_wi * d * vis / pdf;
    }
    return sum / double(num_samples);
}

}  // namespace

float const* ggx_albedo_table() {
    static float         table[Ggx_table_size * Ggx_table_size];
    static std::once_flag once;
    std::call_once(once, []() {
        double const step = 1.0 / double(Ggx_table_size - 1);
        for (int a = 0; a < Ggx_table_size; ++a) {
            for (int i = 0; i < Ggx_table_size; ++i) {
                table[a * Ggx_table_size + i] = float(albedo(a * step, i * step, 1024));
            }
        }
    });
    return table;
}

}  // namespace spb

extern "C" SPB_API int32_t spb_ggx_albedo_table(float* out) {
    if (!out) {
        return SPB_ERROR_ARGUMENT;
    }
    float const* t = spb::ggx_albedo_table();
    for (int i = 0; i < spb::Ggx_table_size * spb::Ggx_table_size; ++i) {
        out[i] = t[i];
    }
    return SPB_OK;
}
