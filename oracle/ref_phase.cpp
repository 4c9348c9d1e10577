// Phase-function harness (test infrastructure, not part of the product): reads lines from
// standard input and prints the reference's answer to each, built by oracle/Makefile against
// the reference's own sources:
//   "p cos g"                  -> phase_hg(cos, g)                  (material.inl:15-19)
//   "s wo.x wo.y wo.z r0 r1 g" -> sample_phase(wo, (r0, r1), g): dot(wi, -wo), its pdf and |wi|
//                                 (material.inl:21-40)
//   "v g depth"                -> van_de_hulst_anisotropy(depth) and similarity_relation_scale(depth)
//                                 of a medium of anisotropy g (material.cpp:108-140)
#include <cstdio>
#include <cstring>

#include "base/math/vector3.inl"
#include "base/math/sampling.inl"
#include "scene/material/material.inl"
#include "scene/material/volumetric/volumetric_homogeneous.hpp"

namespace {

struct Medium : scene::material::volumetric::Homogeneous {
    Medium() : Homogeneous(scene::material::Sampler_settings()) {}
    using Homogeneous::van_de_hulst_anisotropy;
};

}  // namespace

int main() {
    char kind[4];
    while (std::scanf("%3s", kind) == 1) {
        if (std::strcmp(kind, "p") == 0) {
            float c, g;
            if (std::scanf("%f %f", &c, &g) != 2) {
                return 1;
            }
            std::printf("%.9g\n", double(scene::material::phase_hg(c, g)));
        } else if (std::strcmp(kind, "s") == 0) {
            float w[3], r0, r1, g;
            if (std::scanf("%f %f %f %f %f %f", w, w + 1, w + 2, &r0, &r1, &g) != 6) {
                return 1;
            }
            float3 const wo(w[0], w[1], w[2]);
            float4 const s  = scene::material::sample_phase(wo, float2(r0, r1), g);
            float3 const wi = s.xyz();
            std::printf("%.9g %.9g %.9g\n", double(-dot(wi, wo)), double(s[3]), double(length(wi)));
        } else {
            float    g;
            unsigned depth;
            if (std::scanf("%f %u", &g, &depth) != 2) {
                return 1;
            }
            Medium m;
            m.set_volumetric(float3(0.5f), float3(0.5f), 1.f, g);
            std::printf("%.9g %.9g\n", double(m.van_de_hulst_anisotropy(depth)),
                        double(m.similarity_relation_scale(depth)));
        }
    }
    return 0;
}
