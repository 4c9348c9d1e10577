// Cast harness around the reference's own BVH code: TEST INFRASTRUCTURE, not product.
//
// Builds the reference tree exactly as the reference's mesh loader does
// (scene::shape::triangle::bvh::Builder_SAH(16, 64, 4), triangle_mesh_provider.cpp:375-378)
// and casts rays through the reference traversal:
//   closest hit  Tree::intersect    (triangle_bvh_tree.cpp:41-90)
//   any hit      Tree::intersect_p  (triangle_bvh_tree.cpp:145-185)
// with one Node_stack per worker thread, as rendering::Worker does.
//
// The reference reports the leaf-slot index of the hit (Intersection::index), which is the
// triangle's position in the tree's DFS leaf order.  This harness maps each slot back to the
// caller's triangle index through the slot's three vertex positions, so its output is
// comparable with any other implementation.
//
// usage: ref_cast MESH RAYS OUT [threads=0 (all)] [mode=both|hit|occl] [repeats=1]
//   MESH: u32 num_vertices, u32 num_triangles, f32 positions[3*nv], u32 indices[3*nt]
//   RAYS: u64 num_rays, f32 rays[8*n]  (ox oy oz min_t dx dy dz max_t)
//   OUT : u32 id[n] (0xFFFFFFFF = miss), f32 t[n] (max_t after the call), u8 occluded[n]
// Prints one JSON line with build and cast times.

#include "base/math/aabb.inl"
#include "base/math/vector3.inl"
#include "base/thread/thread_pool.hpp"
#include "scene/shape/node_stack.inl"
#include "scene/shape/shape_vertex.hpp"
#include "scene/shape/triangle/bvh/triangle_bvh_builder_sah.hpp"
#include "scene/shape/triangle/bvh/triangle_bvh_tree.inl"
#include "scene/shape/triangle/triangle_primitive.hpp"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

using namespace scene::shape;
using namespace scene::shape::triangle;

namespace {

struct Key {
    uint32_t w[9];
    bool operator==(Key const& o) const {
        return 0 == std::memcmp(w, o.w, sizeof(w));
    }
};

struct Key_hash {
    size_t operator()(Key const& k) const {
        uint64_t h = 1469598103934665603ull;
        for (uint32_t x : k.w) {
            h = (h ^ x) * 1099511628211ull;
        }
        return size_t(h);
    }
};

Key make_key(float3 const& a, float3 const& b, float3 const& c) {
    Key   k;
    float f[9] = {a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2]};
    std::memcpy(k.w, f, sizeof(f));
    return k;
}

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

bool read_all(char const* path, std::vector<char>& buf) {
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        return false;
    }
    std::fseek(f, 0, SEEK_END);
    long const size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.resize(size_t(size));
    bool const ok = size == 0 || 1 == std::fread(buf.data(), size_t(size), 1, f);
    std::fclose(f);
    return ok;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: ref_cast MESH RAYS OUT [threads] [both|hit|occl]\n");
        return 2;
    }

    int32_t const     thread_request = argc > 4 ? std::atoi(argv[4]) : 0;
    std::string const mode           = argc > 5 ? argv[5] : "both";
    int32_t const     repeats        = argc > 6 ? std::max(1, std::atoi(argv[6])) : 1;

    std::vector<char> mesh_buf;
    std::vector<char> ray_buf;
    if (!read_all(argv[1], mesh_buf) || !read_all(argv[2], ray_buf)) {
        std::fprintf(stderr, "cannot read inputs\n");
        return 2;
    }

    uint32_t nv;
    uint32_t nt;
    std::memcpy(&nv, mesh_buf.data(), 4);
    std::memcpy(&nt, mesh_buf.data() + 4, 4);
    float const*    positions = reinterpret_cast<float const*>(mesh_buf.data() + 8);
    uint32_t const* indices   = reinterpret_cast<uint32_t const*>(mesh_buf.data() + 8 + 12 * nv);

    uint64_t n;
    std::memcpy(&n, ray_buf.data(), 8);
    float const* rays = reinterpret_cast<float const*>(ray_buf.data() + 8);

    // Vertex stream with positions and a unit normal per vertex (normals do not take part in
    // intersection; the builder only needs them to fill the tangent frames it stores).
    auto* p  = new packed_float3[nv];
    auto* nn = new packed_float3[nv];
    for (uint32_t i = 0; i < nv; ++i) {
        p[i] = packed_float3(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
        nn[i] = packed_float3(0.f, 0.f, 1.f);
    }
    Vertex_stream_separate_compact vertices(nv, p, nn);

    std::vector<Index_triangle> triangles(nt);
    for (uint32_t i = 0; i < nt; ++i) {
        triangles[i] = Index_triangle(indices[3 * i], indices[3 * i + 1], indices[3 * i + 2], 0);
    }

    thread::Pool threads(thread::Pool::num_threads(thread_request));

    bvh::Tree tree;

    double const b0 = now();
    {
        bvh::Builder_SAH builder(16, 64, 4);
        builder.build(tree, nt, triangles.data(), vertices, threads);
    }
    double const build_s = now() - b0;

    // slot -> caller triangle index, through the slot's vertex positions
    std::unordered_map<Key, uint32_t, Key_hash> by_position;
    by_position.reserve(nt * 2);
    for (uint32_t i = 0; i < nt; ++i) {
        float3 const a(positions + 3 * indices[3 * i]);
        float3 const b(positions + 3 * indices[3 * i + 1]);
        float3 const c(positions + 3 * indices[3 * i + 2]);
        by_position.emplace(make_key(a, b, c), i);
    }

    uint32_t const        num_slots = tree.num_triangles();
    std::vector<uint32_t> slot_to_id(num_slots, 0xFFFFFFFF);
    uint32_t              unmapped = 0;
    for (uint32_t s = 0; s < num_slots; ++s) {
        float3 a;
        float3 b;
        float3 c;
        tree.triangle(s, a, b, c);
        auto const it = by_position.find(make_key(a, b, c));
        if (it == by_position.end()) {
            ++unmapped;
        } else {
            slot_to_id[s] = it->second;
        }
    }

    std::vector<uint32_t> ids(n, 0xFFFFFFFF);
    std::vector<float>    ts(n, 0.f);
    std::vector<uint8_t>  occluded(n, 0);

    uint32_t const          num_threads = threads.num_threads();
    std::vector<Node_stack> stacks(num_threads);
    for (auto& s : stacks) {
        s.clear();
    }

    double              hit_s  = 0.;
    double              occl_s = 0.;
    std::vector<double> hit_list;

    for (int32_t rep = 0; rep < repeats && (mode == "both" || mode == "hit"); ++rep) {
        double const t0 = now();
        threads.run_range(
            [&](uint32_t id, int32_t begin, int32_t end) noexcept {
                Node_stack& stack = stacks[id];
                for (int32_t i = begin; i < end; ++i) {
                    float const* r = rays + 8 * size_t(i);

                    alignas(16) float o[4] = {r[0], r[1], r[2], 0.f};
                    alignas(16) float d[4] = {r[4], r[5], r[6], 0.f};

                    Simdf const  origin(o);
                    Simdf const  direction(d);
                    scalar const min_t(r[3]);
                    scalar       max_t(r[7]);

                    stack.clear();  // as prop_bvh_wrapper.cpp:40 does before each query

                    triangle::Intersection isec;
                    if (tree.intersect(origin, direction, min_t, max_t, stack, isec)) {
                        ids[size_t(i)] = slot_to_id[isec.index];
                    }
                    // the ray's max_t after the call: the hit t, or unchanged on a miss
                    ts[size_t(i)] = max_t.x();
                }
            },
            0, int32_t(n));
        hit_s = now() - t0;
        hit_list.push_back(hit_s);
    }

    if (mode == "both" || mode == "occl") {
        double const t0 = now();
        threads.run_range(
            [&](uint32_t id, int32_t begin, int32_t end) noexcept {
                Node_stack& stack = stacks[id];
                for (int32_t i = begin; i < end; ++i) {
                    float const* r = rays + 8 * size_t(i);

                    alignas(16) float o[4] = {r[0], r[1], r[2], 0.f};
                    alignas(16) float d[4] = {r[4], r[5], r[6], 0.f};

                    Simdf const  origin(o);
                    Simdf const  direction(d);
                    scalar const min_t(r[3]);
                    scalar const max_t(r[7]);

                    // intersect_p returns with entries left on the stack; the reference's
                    // caller clears it before every query (prop_bvh_wrapper.cpp:186)
                    stack.clear();

                    occluded[size_t(i)] = tree.intersect_p(origin, direction, min_t, max_t,
                                                           stack)
                                              ? 1
                                              : 0;
                }
            },
            0, int32_t(n));
        occl_s = now() - t0;
    }

    FILE* f = std::fopen(argv[3], "wb");
    if (!f) {
        std::fprintf(stderr, "cannot write %s\n", argv[3]);
        return 2;
    }
    std::fwrite(ids.data(), 4, n, f);
    std::fwrite(ts.data(), 4, n, f);
    std::fwrite(occluded.data(), 1, n, f);
    std::fclose(f);

    std::string list;
    for (size_t i = 0; i < hit_list.size(); ++i) {
        char buf[32];
        std::snprintf(buf, sizeof(buf), "%s%.6f", i ? ", " : "", hit_list[i]);
        list += buf;
    }
    std::printf(
        "{\"threads\": %u, \"triangles\": %u, \"slots\": %u, \"unmapped_slots\": %u, "
        "\"rays\": %llu, \"build_s\": %.6f, \"hit_s\": %.6f, \"occl_s\": %.6f, "
        "\"hit_s_list\": [%s]}\n",
        num_threads, nt, num_slots, unmapped, (unsigned long long)n, build_s, hit_s, occl_s,
        list.c_str());

    return 0;
}
