// Light tree over the emissive triangles of a scene: the GPU counterpart of the reference's
// light::Tree + Primitive_tree (scene/light/light_tree.cpp:27-302, light_tree_builder.cpp),
// flattened to one binary tree whose leaves hold up to four triangles.
//
// Built on the host in double precision with a binned surface-area-orientation heuristic
// (Estevez and Kulla, "Importance Sampling of Many Lights with Adaptive Tree Splitting", 2018);
// each node bounds its lights by a sphere (centre, radius), a cone of normals (axis, cos of
// the spread; -1 for two-sided emitters) and their total power.  The device walks it top-down,
// choosing a child in proportion to an importance estimate seen from the shading point
// (light_tree.cuh).
#pragma once

#include <cstdint>
#include <vector>

namespace spb::render {

// One emissive triangle in world space.
struct Light_input {
    double   a[3], b[3], c[3];
    double   power = 0.0;  // area * mean radiance (twice that for two-sided emitters)
    bool     two_sided = false;
    uint32_t slot      = 0;  // index of its entry in Light_tree::order
    uint32_t material  = 0;  // its material (stored with it for the renderer's light sampling)
};

// Device-ready arrays, 4 floats per float4.
//   nodes:  3 float4 per node: (centre, radius), (axis, cos spread), (power, first, count,
//           middle) with first/count/middle stored as uint32 bits.  Inner nodes have count 0
//           and their children at first and first + 1; lights of the subtree [b, e) split at
//           middle (left child: order < middle).  Leaves hold lights first .. first+count-1.
//   cones:  3 float4 per light in tree order: (centre, radius), (normal, cos spread),
//           (power, 0, 0, 0)
//   tris:   3 float4 per light in tree order: (a, area), (b - a, 0), (c - a, material index bits)
//   order:  per light slot (Light_input::slot), its position in tree order, or 0xFFFFFFFF
struct Light_tree {
    std::vector<float>    nodes;
    std::vector<float>    cones;
    std::vector<float>    tris;
    std::vector<uint32_t> order;
    uint32_t              num_nodes  = 0;
    uint32_t              num_lights = 0;
    uint32_t              depth      = 0;
};

constexpr uint32_t Light_leaf_size = 4;

void build_light_tree(std::vector<Light_input> const& lights, uint32_t num_slots,
                      Light_tree& out);

}  // namespace spb::render
