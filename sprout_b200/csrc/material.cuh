// Surface materials of the path tracer, callable on host and device:
// the reference's "Substitute" material (Disney diffuse + GGX, one-sample 50/50 lobe choice;
// pure GGX when metallic == 1) and the constant-emission "Light" material.
//
// Follows (paths relative to the reference project):
//   substitute::Sample::evaluate / sample      material/substitute/substitute_sample.cpp:10-45
//   Base_closure::{base,pure_gloss}_evaluate,
//     {diffuse,gloss,pure_gloss}_sample          material/substitute/substitute_base_sample.inl:18-238
//   disney::Iso::evaluate / reflect              material/disney/disney.inl:21-77
//   ggx::Iso::reflection, visibility_and_g1_wo,
//     pdf_visible, distribution_isotropic        material/ggx/ggx.inl:51-236
//   ggx::Aniso::sample (visible-normal sampling,
//     Heitz 2018, JCGT 7(4))                     material/ggx/ggx.inl:469-503
//   ilm_ep_conductor (energy compensation)       material/ggx/ggx.inl:27-29
//   roughness -> alpha = max(r, 0.01314)^2       material/substitute/substitute_base_material.cpp:63-75
//   Schlick Fresnel                              material/fresnel/fresnel.inl:137-143
//   clamp of cosines to [1e-5, 1]                material/material_sample_helper.hpp:17-33
// The GGX directional-albedo table E (32 x 32 over cos(theta_o) and alpha) is computed by
// this project (ggx_table.cpp) with the estimator the reference's table generator uses.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define SPB_HD __host__ __device__ __forceinline__
#else
#define SPB_HD inline
#endif

namespace spb::shading {

constexpr float Pi           = 3.14159265358979323846f;
constexpr float Pi_inv       = 0.318309886183790671538f;
constexpr float Dot_min      = 0.00001f;
constexpr float Min_roughness = 0.01314f;
constexpr float Min_alpha    = Min_roughness * Min_roughness;
constexpr int   E_size       = 32;

struct V3 {
    float x, y, z;
};

SPB_HD V3 v3(float x, float y, float z) {
    return V3{x, y, z};
}
SPB_HD V3 operator+(V3 a, V3 b) {
    return v3(a.x + b.x, a.y + b.y, a.z + b.z);
}
SPB_HD V3 operator-(V3 a, V3 b) {
    return v3(a.x - b.x, a.y - b.y, a.z - b.z);
}
SPB_HD V3 operator-(V3 a) {
    return v3(-a.x, -a.y, -a.z);
}
SPB_HD V3 operator*(float s, V3 a) {
    return v3(s * a.x, s * a.y, s * a.z);
}
SPB_HD V3 operator*(V3 a, V3 b) {
    return v3(a.x * b.x, a.y * b.y, a.z * b.z);
}
SPB_HD V3 operator/(V3 a, float s) {
    return v3(a.x / s, a.y / s, a.z / s);
}
SPB_HD float dot(V3 a, V3 b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
SPB_HD V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
SPB_HD V3 normalize(V3 a) {
    return (1.f / std::sqrt(dot(a, a))) * a;
}
SPB_HD float max_component(V3 a) {
    return fmaxf(a.x, fmaxf(a.y, a.z));
}
SPB_HD float min_component(V3 a) {
    return fminf(a.x, fminf(a.y, a.z));
}
SPB_HD float clampf(float x, float lo, float hi) {
    return fminf(fmaxf(x, lo), hi);
}
SPB_HD float clamp_dot(V3 a, V3 b) {
    return clampf(dot(a, b), Dot_min, 1.f);
}
SPB_HD float clamp_abs_dot(V3 a, V3 b) {
    return clampf(fabsf(dot(a, b)), Dot_min, 1.f);
}
SPB_HD float saturate(float x) {
    return clampf(x, 0.f, 1.f);
}
SPB_HD float pow5(float x) {
    float const x2 = x * x;
    return x2 * x2 * x;
}
SPB_HD float lerp(float a, float b, float t) {
    return a + t * (b - a);
}

// Orthonormal frame around n (Duff et al. 2017, "Building an Orthonormal Basis, Revisited").
struct Frame {
    V3 t, b, n;
};

SPB_HD Frame make_frame(V3 n) {
    float const sign = copysignf(1.f, n.z);
    float const c    = -1.f / (sign + n.z);
    float const d    = n.x * n.y * c;
    Frame f;
    f.t = v3(1.f + sign * n.x * n.x * c, sign * d, -sign * n.x);
    f.b = v3(d, sign + n.y * n.y * c, -n.y);
    f.n = n;
    return f;
}

SPB_HD V3 to_world(Frame const& f, V3 v) {
    return v3(v.x * f.t.x + v.y * f.b.x + v.z * f.n.x, v.x * f.t.y + v.y * f.b.y + v.z * f.n.y,
              v.x * f.t.z + v.y * f.b.z + v.z * f.n.z);
}

SPB_HD V3 to_local(Frame const& f, V3 v) {
    return v3(dot(v, f.t), dot(v, f.b), dot(v, f.n));
}

// Material record shared by host and device (80 bytes).
struct Material {
    uint32_t type;       // Type_substitute, Type_light or Type_volume
    uint32_t two_sided;  // 1: back faces shade like front faces
    float    metallic;
    float    alpha;      // GGX alpha (roughness^2, roughness clamped below at 0.01314)
    V3       albedo;     // (1 - metallic) * color
    V3       f0;         // lerp(f0 of ior 1.46, color, metallic)
    V3       emission;   // radiance (Light) -- colours are ACEScg (AP1) linear
    float    g;          // Henyey-Greenstein anisotropy (Volume), clamped to [-0.999, 0.999]
    V3       mu_a;       // absorption coefficient per metre (Volume)
    V3       mu_s;       // scattering coefficient per metre (Volume)
    uint32_t medium;     // Volume: 0 homogeneous, else 1 + index of the density-grid medium
    // Volume: 0 when its emission is not a light's; else 1 + its light's position in the light
    // tree, or Volume_light_unsampled for a light whose shape next-event estimation cannot
    // sample (its emission then counts with weight 1 on every segment).
    uint32_t volume_light;
    // Substitute texture maps: the base colour and the dielectric F0 the per-hit parameters are
    // rebuilt from, and 1 + the index of the colour and surface textures (0: none); the surface
    // texture holds roughness, and metallic too when surface_channels is 2.
    V3       color;
    float    f0d;
    uint32_t color_map;
    uint32_t surface_map;
    uint32_t surface_channels;
    uint32_t pad2;
};

constexpr uint32_t Type_substitute = 0;
constexpr uint32_t Type_light      = 1;
constexpr uint32_t Type_volume     = 2;  // participating medium inside a closed mesh
constexpr uint32_t Volume_light_unsampled = 0xFFFFFFFFu;

// Absorption and scattering coefficients of a medium from its attenuation colour, subsurface
// colour (the multiple-scattering albedo), attenuation distance and anisotropy
// (attenuation_coefficient and scattering, collision_coefficients.inl:50-71): mu_t from the
// colour a ray keeps after the distance, split by the single-scattering albedo that gives ssc.
SPB_HD void attenuation(V3 ac, V3 ssc, float distance, float g, V3& mu_a, V3& mu_s) {
    float const acs[3] = {ac.x, ac.y, ac.z};
    float const xs[3]  = {ssc.x, ssc.y, ssc.z};
    float       a[3], s[3];
    for (int k = 0; k < 3; ++k) {
        float const ca     = fminf(fmaxf(acs[k], 0.01f), 0.991102f);
        float const mu_t   = -logf(ca) / distance;
        float const x      = xs[k];
        float const root   = sqrtf(9.59217f + 41.6808f * x + 17.7126f * x * x);
        float const factor = fminf(fmaxf(4.097125f + 4.20863f * x - root, 0.f), 1.f);
        float const fsq    = factor * factor;
        float const pss    = (1.f - fsq) / (1.f - g * fsq);
        a[k]               = mu_t * (1.f - pss);
        s[k]               = mu_t - a[k];
    }
    mu_a = v3(a[0], a[1], a[2]);
    mu_s = v3(s[0], s[1], s[2]);
}

// Henyey-Greenstein phase function of c = dot(wo, wi) (material.inl:15-19).
SPB_HD float phase_hg(float c, float g) {
    float const gg    = g * g;
    float const denom = 1.f + gg + 2.f * g * c;
    return (1.f / (4.f * Pi)) * (1.f - gg) / (denom * std::sqrt(denom));
}

// Samples the phase function around the forward direction -wo (material.inl:21-40); returns
// wi and sets pdf (= the phase value).
SPB_HD V3 sample_hg(V3 wo, float g, float xi0, float xi1, float& pdf) {
    float cos_theta;
    if (fabsf(g) < 0.001f) {
        cos_theta = 1.f - 2.f * xi0;
    } else {
        float const gg  = g * g;
        float const sqr = (1.f - gg) / (1.f - g + 2.f * g * xi0);
        cos_theta       = (1.f + gg - sqr * sqr) / (2.f * g);
    }
    float const sin_theta = std::sqrt(fmaxf(0.f, 1.f - cos_theta * cos_theta));
    float const phi       = xi1 * (2.f * Pi);
    Frame const f         = make_frame(-wo);
    V3 const    wi = (sin_theta * std::cos(phi)) * f.t + (sin_theta * std::sin(phi)) * f.b +
                  cos_theta * f.n;
    pdf = phase_hg(-cos_theta, g);
    return wi;
}

// Phase anisotropy after depth bounces (Material::van_de_hulst_anisotropy,
// material.cpp:128-140; similarity range 16..64 by default, take_loader.cpp:748-754).
SPB_HD float van_de_hulst_anisotropy(float g, uint32_t depth) {
    constexpr uint32_t low  = 16;
    constexpr uint32_t high = 64;
    if (depth < low) {
        return g;
    }
    if (depth < high) {
        return lerp(g, 0.f, float(depth - low) / float(high - low));
    }
    return 0.f;
}

// Scale of the scattering coefficient that goes with the reduced anisotropy
// (Material::similarity_relation_scale, material.cpp:108-112; van_de_hulst,
// collision_coefficients.inl:9-11): (1 - g) / (1 - g').
SPB_HD float similarity_relation_scale(float g, uint32_t depth) {
    return (1.f - g) / (1.f - van_de_hulst_anisotropy(g, depth));
}

// E table lookup: bilinear over x = cos(theta_o) (columns), y = alpha (rows), both in [0, 1]
// (interpolated_function_2d.inl:109-130).
SPB_HD float e_lookup(float const* table, float x, float y) {
    x            = fminf(x, 1.f);
    y            = fminf(y, 1.f);
    float const ox = x * float(E_size - 1);
    float const oy = y * float(E_size - 1);
    int const   ix = int(ox);
    int const   iy = int(oy);
    float const tx = ox - float(ix);
    float const ty = oy - float(iy);
    int const   x1 = ix + 1 < E_size ? ix + 1 : E_size - 1;
    int const   y1 = iy + 1 < E_size ? iy + 1 : E_size - 1;
    float const c00 = table[iy * E_size + ix];
    float const c10 = table[iy * E_size + x1];
    float const c01 = table[y1 * E_size + ix];
    float const c11 = table[y1 * E_size + x1];
    float const a   = c00 + tx * (c10 - c00);
    float const b   = c01 + tx * (c11 - c01);
    return a + ty * (b - a);
}

SPB_HD V3 ilm_ep_conductor(float const* table, V3 f0, float n_dot_wo, float alpha,
                           float metallic) {
    float const k = metallic / e_lookup(table, n_dot_wo, alpha) - 1.f;
    return v3(1.f + k * f0.x, 1.f + k * f0.y, 1.f + k * f0.z);
}

SPB_HD V3 schlick(float wo_dot_h, V3 f0) {
    float const p = pow5(1.f - wo_dot_h);
    return v3(f0.x + (1.f - f0.x) * p, f0.y + (1.f - f0.y) * p, f0.z + (1.f - f0.z) * p);
}

SPB_HD float distribution_isotropic(float n_dot_h, float a2) {
    float const d = (n_dot_h * n_dot_h) * (a2 - 1.f) + 1.f;
    return a2 / (Pi * d * d);
}

// Height-correlated Smith visibility G2 / (4 n.wi n.wo), and t_wo + n.wo for the VNDF pdf.
SPB_HD void visibility_and_g1_wo(float n_dot_wi, float n_dot_wo, float a2, float& vis,
                                 float& g1_wo) {
    float const t_wi = std::sqrt(a2 + (1.f - a2) * (n_dot_wi * n_dot_wi));
    float const t_wo = std::sqrt(a2 + (1.f - a2) * (n_dot_wo * n_dot_wo));
    vis              = 0.5f / (n_dot_wi * t_wo + n_dot_wo * t_wi);
    g1_wo            = t_wo + n_dot_wo;
}

struct Bxdf {
    V3    reflection;  // f * cos(theta_i)
    float pdf;
};

// GGX reflection with Schlick Fresnel: returns D * V * F and the visible-normal pdf.
SPB_HD Bxdf ggx_reflection(float n_dot_wi, float n_dot_wo, float wo_dot_h, float n_dot_h,
                           float alpha, V3 f0) {
    float const a2 = alpha * alpha;
    float const d  = distribution_isotropic(n_dot_h, a2);
    float       vis, g1;
    visibility_and_g1_wo(n_dot_wi, n_dot_wo, a2, vis, g1);
    V3 const f = schlick(wo_dot_h, f0);
    return Bxdf{(d * vis) * f, (0.5f * d) / g1};
}

// Energy-preserving Disney diffuse (disney.inl:56-77), without the cosine.
SPB_HD V3 disney_diffuse(float h_dot_wi, float n_dot_wi, float n_dot_wo, float alpha, V3 color) {
    float const energy_bias   = lerp(0.f, 0.5f, alpha);
    float const energy_factor = lerp(1.f, 1.f / 1.53f, alpha);
    float const f_d90         = energy_bias + (2.f * alpha) * (h_dot_wi * h_dot_wi);
    float const fmo           = f_d90 - 1.f;
    float const a             = 1.f + fmo * pow5(1.f - n_dot_wi);
    float const b             = 1.f + fmo * pow5(1.f - n_dot_wo);
    return (a * b * energy_factor) * (Pi_inv * color);
}

// Visible-normal sample of the isotropic GGX distribution (Heitz 2018); wo in world space.
SPB_HD V3 sample_visible_normal(Frame const& fr, V3 wo, float alpha, float xi0, float xi1,
                                float& n_dot_h) {
    V3 const lwo = to_local(fr, wo);
    V3 const v   = normalize(v3(alpha * lwo.x, alpha * lwo.y, lwo.z));
    V3 const t1  = (v.z < 0.9999f) ? normalize(v3(v.y, -v.x, 0.f)) : v3(1.f, 0.f, 0.f);
    V3 const t2  = v3(t1.y * v.z, -t1.x * v.z, t1.x * v.y - t1.y * v.x);
    float const a   = 1.f / (1.f + v.z);
    float const r   = std::sqrt(xi0);
    float const phi = (xi1 < a) ? (xi1 / a * Pi) : (Pi + (xi1 - a) / (1.f - a) * Pi);
    float const p1  = r * std::cos(phi);
    float const p2  = r * std::sin(phi) * ((xi1 < a) ? 1.f : v.z);
    V3 m = p1 * t1 + p2 * t2 + std::sqrt(fmaxf(1.f - p1 * p1 - p2 * p2, 0.f)) * v;
    m    = normalize(v3(alpha * m.x, alpha * m.y, fmaxf(m.z, 0.f)));
    n_dot_h = saturate(m.z);
    return to_world(fr, m);
}

// Cosine-weighted hemisphere direction in the frame (Malley's method on a concentric disk).
SPB_HD V3 sample_cosine(Frame const& fr, float xi0, float xi1) {
    float const ox = 2.f * xi0 - 1.f;
    float const oy = 2.f * xi1 - 1.f;
    float       r, phi;
    if (ox == 0.f && oy == 0.f) {
        r   = 0.f;
        phi = 0.f;
    } else if (fabsf(ox) > fabsf(oy)) {
        r   = ox;
        phi = (Pi * 0.25f) * (oy / ox);
    } else {
        r   = oy;
        phi = (Pi * 0.5f) - (Pi * 0.25f) * (ox / oy);
    }
    float const dx = r * std::cos(phi);
    float const dy = r * std::sin(phi);
    float const dz = std::sqrt(fmaxf(0.f, 1.f - dx * dx - dy * dy));
    return normalize(to_world(fr, v3(dx, dy, dz)));
}

// Shading context at a surface hit.
struct Context {
    Frame frame;  // shading frame (interpolated normal)
    V3    geo_n;  // geometric normal (flipped with the shading normal for two-sided materials)
    V3    wo;
};

SPB_HD bool same_hemisphere(Context const& c, V3 v) {
    return dot(c.geo_n, v) > 0.f;
}

// Substitute::evaluate (substitute_sample.cpp:10-24).
SPB_HD Bxdf substitute_evaluate(Material const& m, float const* e_table, Context const& c, V3 wi) {
    if (!same_hemisphere(c, c.wo)) {
        return Bxdf{v3(0.f, 0.f, 0.f), 0.f};
    }
    V3 const    h        = normalize(c.wo + wi);
    float const wo_dot_h = clamp_dot(c.wo, h);
    float const n_dot_wi = clamp_dot(c.frame.n, wi);
    float const n_dot_wo = clamp_abs_dot(c.frame.n, c.wo);
    float const n_dot_h  = saturate(dot(c.frame.n, h));

    Bxdf     g   = ggx_reflection(n_dot_wi, n_dot_wo, wo_dot_h, n_dot_h, m.alpha, m.f0);
    V3 const ilm = ilm_ep_conductor(e_table, m.f0, n_dot_wo, m.alpha, m.metallic);
    g.reflection = g.reflection * ilm;

    if (m.metallic == 1.f) {
        return Bxdf{n_dot_wi * g.reflection, g.pdf};
    }
    V3 const    d     = disney_diffuse(wo_dot_h, n_dot_wi, n_dot_wo, m.alpha, m.albedo);
    float const d_pdf = n_dot_wi * Pi_inv;
    return Bxdf{n_dot_wi * (d + g.reflection), 0.5f * (d_pdf + g.pdf)};
}

struct Sampled {
    V3    wi;
    V3    reflection;  // f * cos(theta_i)
    float pdf;         // 0: no sample
    bool  specular;
};

// Substitute::sample (substitute_sample.cpp:26-45): xi_lobe picks the lobe, (xi0, xi1) the
// direction within it.
SPB_HD Sampled substitute_sample(Material const& m, float const* e_table, Context const& c,
                                 float xi_lobe, float xi0, float xi1) {
    Sampled s{v3(0.f, 0.f, 0.f), v3(0.f, 0.f, 0.f), 0.f, false};
    if (!same_hemisphere(c, c.wo)) {
        return s;
    }
    float const n_dot_wo = clamp_abs_dot(c.frame.n, c.wo);
    V3 const    ilm      = ilm_ep_conductor(e_table, m.f0, n_dot_wo, m.alpha, m.metallic);

    bool const pure_gloss = m.metallic == 1.f;
    if (pure_gloss || xi_lobe >= 0.5f) {
        // gloss: visible-normal sample (ggx::Iso::reflect, ggx.inl:184-228)
        float    n_dot_h;
        V3 const h        = sample_visible_normal(c.frame, c.wo, m.alpha, xi0, xi1, n_dot_h);
        float const wo_dot_h = clamp_dot(c.wo, h);
        V3 const wi       = normalize((2.f * wo_dot_h) * h - c.wo);
        float const n_dot_wi = clamp_dot(c.frame.n, wi);
        Bxdf g            = ggx_reflection(n_dot_wi, n_dot_wo, wo_dot_h, n_dot_h, m.alpha, m.f0);
        g.reflection      = g.reflection * ilm;
        s.wi              = wi;
        s.specular        = m.alpha <= Min_alpha;
        if (pure_gloss) {
            s.reflection = n_dot_wi * g.reflection;
            s.pdf        = g.pdf;
        } else {
            V3 const d   = disney_diffuse(wo_dot_h, n_dot_wi, n_dot_wo, m.alpha, m.albedo);
            s.reflection = n_dot_wi * (g.reflection + d);
            s.pdf        = 0.5f * (g.pdf + n_dot_wi * Pi_inv);
        }
        return s;
    }

    // diffuse: cosine-weighted hemisphere (disney::Iso::reflect, disney.inl:32-50)
    V3 const    wi       = sample_cosine(c.frame, xi0, xi1);
    V3 const    h        = normalize(c.wo + wi);
    float const h_dot_wi = clamp_dot(h, wi);
    float const n_dot_wi = clamp_dot(c.frame.n, wi);
    V3 const    d        = disney_diffuse(h_dot_wi, n_dot_wi, n_dot_wo, m.alpha, m.albedo);
    float const n_dot_h  = saturate(dot(c.frame.n, h));
    Bxdf g = ggx_reflection(n_dot_wi, n_dot_wo, h_dot_wi, n_dot_h, m.alpha, m.f0);
    g.reflection = g.reflection * ilm;
    s.wi         = wi;
    s.reflection = n_dot_wi * (d + g.reflection);
    s.pdf        = 0.5f * (n_dot_wi * Pi_inv + g.pdf);
    return s;
}

}  // namespace spb::shading
