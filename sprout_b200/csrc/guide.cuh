// Learned path guiding: the network's fixed shape, its input encoding and the mixture of
// von Mises-Fisher lobes it predicts.  The reference has no path guiding; this is the
// project's own addition (the directional distribution follows Dong et al., "Neural
// Parametric Mixtures for Path Guiding", SIGGRAPH 2023; the training objective is the
// KL-divergence estimator of Mueller et al., "Neural Importance Sampling", 2019).
//
// Network: 32 inputs -> 64 -> 64 -> 64 -> 64 (ReLU) -> 40 outputs.  Outputs 4j..4j+2 are the
// unnormalised mean direction of lobe j, 4j+3 its log-concentration, 32..39 the mixture
// logits.  GEMM operands are BF16, accumulation FP32; biases FP32.
#pragma once

#include <cstdint>

#include "material.cuh"

namespace spb::guide {

constexpr int Inputs     = 32;
constexpr int Width      = 64;
constexpr int Outputs    = 40;
constexpr int Lobes      = 8;
constexpr int Layers     = 5;
constexpr int Tile       = 128;  // samples per thread block (the tensor-core tile height)
constexpr float Log_kappa_min = -3.f;  // concentration in [e^-3, e^6]
constexpr float Log_kappa_max = 6.f;

// Layer l maps in_dim(l) to out_dim(l).
SPB_HD constexpr int in_dim(int l) { return l == 0 ? Inputs : Width; }
SPB_HD constexpr int out_dim(int l) { return l == Layers - 1 ? Outputs : Width; }

// Offsets into the packed parameter vector: per layer W (out x in, row-major) then b (out).
SPB_HD constexpr int weight_offset(int l) {
    int o = 0;
    for (int k = 0; k < l; ++k) {
        o += out_dim(k) * in_dim(k) + out_dim(k);
    }
    return o;
}
SPB_HD constexpr int bias_offset(int l) { return weight_offset(l) + out_dim(l) * in_dim(l); }
constexpr int Parameters = weight_offset(Layers);  // 17,192

// Input encoding: position p in the scene's bounding box mapped to [0, 1]^3 with sin and cos
// at 4 frequencies per axis (24), the normal n (3), the outgoing direction wo (3), their
// cosine (1) and a constant 1 (1).
SPB_HD void encode(shading::V3 p01, shading::V3 n, shading::V3 wo, float out[Inputs]) {
    float const c[3] = {p01.x, p01.y, p01.z};
    int         k    = 0;
    for (int a = 0; a < 3; ++a) {
        float f = 3.14159265358979f;
        for (int o = 0; o < 4; ++o) {
            out[k++] = sinf(f * c[a]);
            out[k++] = cosf(f * c[a]);
            f *= 2.f;
        }
    }
    out[k++] = n.x;
    out[k++] = n.y;
    out[k++] = n.z;
    out[k++] = wo.x;
    out[k++] = wo.y;
    out[k++] = wo.z;
    out[k++] = n.x * wo.x + n.y * wo.y + n.z * wo.z;
    out[k++] = 1.f;
}

// One lobe: unit mean direction, concentration, mixture weight.
struct Lobe {
    shading::V3 mu;
    float       kappa;
    float       weight;
};

// Maps the network's 40 outputs to the mixture (normalised means, clamped concentrations,
// softmax weights).
SPB_HD void mixture(float const out[Outputs], Lobe lobes[Lobes]) {
    float mx = out[32];
    for (int j = 1; j < Lobes; ++j) {
        mx = fmaxf(mx, out[32 + j]);
    }
    float sum = 0.f;
    for (int j = 0; j < Lobes; ++j) {
        float const e = expf(out[32 + j] - mx);
        lobes[j].weight = e;
        sum += e;
    }
    for (int j = 0; j < Lobes; ++j) {
        shading::V3 m  = shading::v3(out[4 * j], out[4 * j + 1], out[4 * j + 2]);
        float const l2 = shading::dot(m, m);
        lobes[j].mu     = l2 > 1e-20f ? (1.f / sqrtf(l2)) * m : shading::v3(0.f, 0.f, 1.f);
        lobes[j].kappa  = expf(fminf(fmaxf(out[4 * j + 3], Log_kappa_min), Log_kappa_max));
        lobes[j].weight /= sum;
    }
}

// vMF density on the sphere: kappa / (2 pi (1 - e^{-2 kappa})) exp(kappa (mu.w - 1)).
SPB_HD float vmf_pdf(Lobe const& l, shading::V3 w) {
    float const norm = l.kappa / (2.f * 3.14159265358979f * -expm1f(-2.f * l.kappa));
    return norm * expf(l.kappa * (shading::dot(l.mu, w) - 1.f));
}

// Samples one lobe with two uniform numbers: the cosine to the mean by the inverse CDF of the
// vMF (Wenzel Jakob, "Numerically stable sampling of the von Mises Fisher distribution on S2",
// 2012), clamped to [-1, 1], then the azimuth.
SPB_HD shading::V3 vmf_sample(Lobe const& l, float u1, float u2) {
    float const c = fminf(fmaxf(1.f + logf(u1 + (1.f - u1) * expf(-2.f * l.kappa)) / l.kappa, -1.f), 1.f);
    float const s = sqrtf(fmaxf(0.f, 1.f - c * c));
    float const phi = 2.f * 3.14159265358979f * u2;
    shading::Frame const f = shading::make_frame(l.mu);
    return (s * cosf(phi)) * f.t + (s * sinf(phi)) * f.b + c * f.n;
}

}  // namespace spb::guide
