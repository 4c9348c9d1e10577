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

// One emissive triangle in world space, or an emitting medium (volume != 0) whose world box
// runs from a to b (c its centre), emitting in all directions.
struct Light_input {
    double   a[3], b[3], c[3];
    double   power = 0.0;  // area * mean radiance (twice that for two-sided emitters)
    bool     two_sided = false;
    uint32_t slot      = 0;  // index of its entry in Light_tree::order
    uint32_t material  = 0;  // its material (stored with it for the renderer's light sampling)
    uint32_t volume    = 0;  // 1 + the renderer's index of an emitting medium's light; 0: a triangle
};

// Device-ready arrays, 4 floats per float4.
//   nodes:  4 float4 per node: (centre, radius), (axis, cos spread), (power, first, count,
//           middle), (variance, lights, variance + mean^2, 0 -- the renderer's split radius^2)
//           with first/count/middle/lights
//           stored as uint32 bits.  Inner nodes have count 0 and their children at first and
//           first + 1; lights of the subtree [b, e) split at middle (left child: order <
//           middle).  Leaves hold lights first .. first+count-1.  variance and mean are the
//           population variance and the mean of the subtree's light powers and lights their
//           number (the inputs of the splitting decision, light_tree.cpp:197-224 and
//           light_tree_builder.cpp:86-102).
//   cones:  3 float4 per light in tree order: (centre, radius), (normal, cos spread),
//           (power, 0, 0, 0)
//   tris:   3 float4 per light in tree order: (a, area), (b - a, 0), (c - a, material index bits);
//           for an emitting medium (centre, -volume), (0, 0), (0, material index bits)
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

constexpr uint32_t Light_leaf_size   = 4;
constexpr uint32_t Light_node_floats = 16;
// Splitting (Tree::random_light with split, light_tree.cpp:363-461): while a walk is above
// this depth, a node whose split test passes sends the walk into both children, and a leaf
// passes all its lights; at most Max_light_picks lights per walk (Tree::Max_lights).
constexpr uint32_t Max_split_depth = 5;
constexpr uint32_t Max_light_picks = 1u << (Max_split_depth + 1);

// The most lights one splitting walk that starts at depth `start` can return
// (Build_node::count_max_splits, light_tree.cpp:156-170, over this tree's shape): a leaf
// reached above Max_split_depth gives all its lights, a node at Max_split_depth - 1 gives two
// picks, a deeper node one.
uint32_t max_split_picks(Light_tree const& tree, uint32_t start);

void build_light_tree(std::vector<Light_input> const& lights, uint32_t num_slots,
                      Light_tree& out);

}  // namespace spb::render
