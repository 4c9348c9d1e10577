// Host-side BVH construction for the GPU cast: binned-SAH binary tree, greedy collapse to an
// 8-wide tree, and encoding into 80-byte nodes with 8-bit quantized child boxes.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace spb {

// One 8-wide node, 80 bytes = 5 x 16-byte words (loaded with five 128-bit loads).
//   w0: origin.xyz (float), exponents ex|ey|ez (biased by 127, one byte each) | imask << 24
//   w1: child_base, tri_base, meta[0..3], meta[4..7]
//   w2: qlo_x[0..7], qlo_y[0..7]
//   w3: qlo_z[0..7], qhi_x[0..7]
//   w4: qhi_y[0..7], qhi_z[0..7]
// Child slot i has the box origin + [qlo, qhi] * 2^(e - 127) per axis.  imask bit i marks an
// internal child.  meta[i]: 0 = empty slot; internal child = 0b001 << 5 | (24 + i);
// leaf = unary(triangle count) << 5 | offset, the leaf's triangles being
// tri_base + offset .. tri_base + offset + count - 1 (count 1..3, offset 0..23).
// Internal children are stored contiguously from child_base in slot order.
struct alignas(16) Wide_node {
    float    origin[3];
    uint8_t  exponent[3];
    uint8_t  imask;
    uint32_t child_base;
    uint32_t tri_base;
    uint8_t  meta[8];
    uint8_t  qlo[3][8];
    uint8_t  qhi[3][8];
};
static_assert(sizeof(Wide_node) == 80, "Wide_node must be 80 bytes");

// One triangle, 48 bytes: vertex a, edges b - a and c - a (exactly the values the
// Möller-Trumbore test computes first), the caller's triangle index and a class word the
// traversal can filter on (the path tracer marks participating-medium boundaries).
struct alignas(16) Wide_triangle {
    float    a[3];
    uint32_t id;
    float    e1[3];
    uint32_t tri_class;
    float    e2[3];
    uint32_t pad1;
};
static_assert(sizeof(Wide_triangle) == 48, "Wide_triangle must be 48 bytes");

struct Wide_bvh {
    std::vector<Wide_node>     nodes;
    std::vector<Wide_triangle> triangles;
    uint32_t                   num_leaves = 0;
    uint32_t                   max_depth  = 0;
    double                     sah_cost   = 0.;
    float                      hit_margin = 0.f;  // see hit_margin_for
    // Bounds of all triangles widened by 2^-10 of the scene size (rounded outward): a ray that
    // misses this box cannot hit a triangle (scene_box_pad).
    float                      scene_lo[3] = {0.f, 0.f, 0.f};
    float                      scene_hi[3] = {0.f, 0.f, 0.f};
};

// Padding of the scene box a ray is first tested against: 2^-10 * max(scene extent, largest
// coordinate magnitude), 128 times the hit margin, so that no ray whose hit point the
// traversal accepts (within the hit margin of a triangle) falls outside it.
double scene_box_pad(double extent, double magnitude);

// Margin around a triangle's bounds within which a hit point must lie:
// 2^-17 * max(scene extent, largest coordinate magnitude), at least FLT_MIN.  extent and
// magnitude come from the float bounds of all triangle vertices, converted to double.
float hit_margin_for(double extent, double magnitude);

// Deepest tree the traversal kernels accept (their stack holds one entry per level).
constexpr uint32_t Max_wide_depth = 48;

// Builds the 8-wide tree.  Returns false (with a message) if the input is unusable.
// tri_class (optional, one word per triangle) is stored with each triangle.
bool build_wide_bvh(uint32_t num_vertices, uint32_t num_triangles, float const* positions,
                    uint32_t const* indices, uint32_t num_threads, Wide_bvh& out,
                    std::string& error, uint32_t const* tri_class = nullptr);

// Builds a top-level 8-wide tree over instance boxes (6 floats each: lo.xyz, hi.xyz).  Its leaf
// records carry the instance index in Wide_triangle::id and instance_class in tri_class; their
// vertex fields are unused.
bool build_wide_instances(uint32_t num_instances, float const* boxes_lo_hi, uint32_t instance_class,
                          uint32_t num_threads, Wide_bvh& out, std::string& error);

}  // namespace spb
