// The reference's C API (source/capi/capi.cpp) on top of the B200 path tracer.
//
// A single global engine, as in the reference (capi.cpp:64-110): meshes, materials and props
// are collected on the host; su_start_render_frame / su_render_frame flatten every prop into
// one world-space triangle set (the props' transformations applied to their meshes), build the
// 8-wide BVH and upload the scene; iterations then run entirely on the GPU (render.cu).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <list>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "../../include/sprout.h"
#include "../../include/sprout_b200.h"
#include "common.hpp"
#include "image_io.hpp"
#include "json.hpp"
#include "postprocess.hpp"
#include "render.hpp"
#include "spectral.cuh"

namespace {

using spb::shading::Material;
using spb::shading::V3;

constexpr uint32_t Null          = 0xFFFFFFFFu;
constexpr uint32_t First_mesh_id = 8;  // ids 0..7 are the built-in shapes (sprout.h:22-29)
constexpr uint32_t Shape_cube            = 1;
constexpr uint32_t Shape_disk            = 2;
constexpr uint32_t Shape_infinite_sphere = 4;
constexpr uint32_t Shape_rectangle       = 6;
constexpr uint32_t Shape_sphere          = 7;

struct Mesh {
    std::vector<float>    positions;  // 3 per vertex
    std::vector<float>    normals;    // 3 per vertex
    std::vector<float>    uvs;        // 2 per vertex (texture coordinates; zero when not given)
    std::vector<uint32_t> indices;    // 3 per triangle
    std::vector<uint32_t> part_of;    // part per triangle
    std::vector<uint32_t> part_slot;  // material slot per part
};

// su_create_image: pixels converted to float (Byte: unorm / 255, image_provider.cpp:90-170).
struct Image {
    uint32_t           dims[3]  = {0, 0, 0};
    uint32_t           channels = 0;
    std::vector<float> pixels;         // channels per pixel, x fastest
    bool               encoded_bytes = false;  // from 8- or 16-bit data: sRGB where used as colour
};

// Texture maps of a Substitute material (Material_base::set_sample,
// substitute_base_material.inl:36-96): colour, and surface (roughness, and metallic from a
// second channel) or roughness alone; images by id, sampled with the material's sampler
// settings and the texture's uv scale.
struct Material_maps {
    uint32_t color          = Null;  // image ids
    uint32_t surface        = Null;
    uint32_t surface_usage  = 0;     // 2: Surface (roughness, metallic), 1: Roughness
    float    color_scale[2] = {1.f, 1.f};
    float    surface_scale[2] = {1.f, 1.f};
    bool     nearest        = false;
    bool     clamp          = false;
};

// Host-side part of a Volumetric material with a density grid (Grid, volumetric_grid.cpp).
struct Grid_ref {
    uint32_t image       = Null;   // density image id, Null for homogeneous media
    uint32_t temperature = Null;   // temperature image id of an emitting grid, or Null
    uint32_t color       = Null;   // RGBA image id of a colour grid (Grid_color), or Null
    float    distance    = 1.f;    // attenuation distance (a colour grid's coefficients)
    bool     nearest     = false;  // "sampler": {"filter": "Nearest"}
    bool     repeat      = false;  // "sampler": {"address": "Repeat"}
};

struct Entity {
    bool                  camera = false;
    uint32_t              shape  = Null;
    std::vector<uint32_t> materials;
    float                 trafo[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    bool                  light = false;
};

struct Engine {
    explicit Engine(bool p) : progressive(p) {}

    bool                  progressive;
    std::vector<Mesh>     meshes;
    Mesh                  builtin[First_mesh_id];  // tessellated built-in shapes, made on first use
    std::vector<Material> materials;
    std::vector<Grid_ref> material_grids;  // parallel to materials
    std::vector<Material_maps> material_maps;  // parallel to materials
    std::vector<Image>    images;
    std::vector<Entity>   entities;
    uint32_t              camera_entity = Null;
    uint32_t              width         = 0;
    uint32_t              height        = 0;
    float                 fov           = 0.f;
    uint32_t              spp           = 1;
    bool                  have_integrator = false;
    spb::render::Settings settings;
    spb::render::Renderer renderer;
    bool                  frame_started = false;
    bool                  scene_dirty    = true;   // host scene changed since the last upload
    bool                  camera_dirty   = false;  // only the camera changed since then
    std::vector<spb::post::Tonemapper> pipeline;  // applied in order by su_postprocess
    std::vector<std::string>           exporters = {"PNG"};  // image formats su_export_frame writes
    int                   instancing     = -1;     // PTMIS "instancing": -1 auto, 0 off, 1 on
    bool                  sampler_golden = true;   // a take's "Random" sampler turns it off
    uint32_t              iteration     = 0;
    std::vector<float>    target;  // resolved rgba
    std::vector<std::string> mounts;  // su_mount folders, searched last mounted first
};

Engine* engine = nullptr;
Post    log_post = nullptr;
Progress_start progress_start = nullptr;
Progress_tick  progress_tick  = nullptr;

void log(uint32_t type, std::string const& text) {
    if (log_post) {
        log_post(type, text.c_str());
    }
}

// sRGB -> ACEScg (AP1) primaries, applied to every colour the material descriptions carry,
// as the reference does with SU_ACESCG (material_provider.cpp:1022-1028, spectrum/aces.hpp).
V3 srgb_to_ap1(V3 c) {
    return V3{0.61309732f * c.x + 0.33952285f * c.y + 0.04737928f * c.z,
              0.07019422f * c.x + 0.91635557f * c.y + 0.01345259f * c.z,
              0.02061560f * c.x + 0.10956983f * c.y + 0.86981512f * c.z};
}

bool read_color(spb::json::Value const* v, V3& out) {
    if (!v) {
        return false;
    }
    if (v->is_number()) {
        // a single number is a grey level; the reference keeps the mapped green channel
        float const g = srgb_to_ap1(V3{float(v->number), float(v->number), float(v->number)}).y;
        out           = V3{g, g, g};
        return true;
    }
    if (v->is_array() && v->array.size() >= 3) {
        out = srgb_to_ap1(V3{float(v->array[0].number), float(v->array[1].number),
                             float(v->array[2].number)});
        return true;
    }
    if (v->is_object()) {
        return read_color(v->find("value"), out);
    }
    return false;
}

// The reference's analytic unit shapes as triangle meshes, so that one traversal serves every
// prop: Rectangle [-1, 1]^2 at z = 0 facing +z (rectangle.cpp:25-64), Disk of radius 1 facing
// +z (disk.cpp), Cube [-1, 1]^3 (cube.cpp), Sphere of radius 1 (sphere.cpp).  The disk (256
// segments) and the sphere (icosphere, 20,480 triangles, smooth normals) are scaled to the
// exact areas, so emitters built from them carry the analytic shape's power.
Mesh make_builtin(uint32_t shape) {
    Mesh m;
    // Texture coordinates as the analytic shapes report them: planar shapes (0.5 (x + 1),
    // 0.5 (1 - y)) in their plane (rectangle.cpp:38-58, disk.cpp:50-58), the sphere
    // (phi / 2 pi, theta / pi) (sphere.cpp:55-60).
    auto vertex = [&m](double x, double y, double z, double nx, double ny, double nz, double u = 0.0,
                       double v = 0.0) {
        m.positions.insert(m.positions.end(), {float(x), float(y), float(z)});
        m.normals.insert(m.normals.end(), {float(nx), float(ny), float(nz)});
        m.uvs.insert(m.uvs.end(), {float(u), float(v)});
        return uint32_t(m.positions.size() / 3 - 1);
    };
    if (shape == Shape_rectangle) {
        for (auto [x, y] : {std::pair{-1, -1}, {1, -1}, {1, 1}, {-1, 1}}) {
            vertex(x, y, 0, 0, 0, 1, 0.5 * (x + 1), 0.5 * (1 - y));
        }
        m.indices = {0, 1, 2, 0, 2, 3};
    } else if (shape == Shape_disk) {
        int const    n = 256;
        double const r = std::sqrt(3.14159265358979323846 /
                                   (0.5 * n * std::sin(2.0 * 3.14159265358979323846 / n)));
        vertex(0, 0, 0, 0, 0, 1, 0.5, 0.5);
        for (int i = 0; i < n; ++i) {
            double const a = 2.0 * 3.14159265358979323846 * i / n;
            vertex(r * std::cos(a), r * std::sin(a), 0, 0, 0, 1, 0.5 * (std::cos(a) + 1), 0.5 * (1 - std::sin(a)));
        }
        for (uint32_t i = 0; i < uint32_t(n); ++i) {
            m.indices.insert(m.indices.end(), {0u, 1 + i, 1 + (i + 1) % n});
        }
    } else if (shape == Shape_cube) {
        for (int axis = 0; axis < 3; ++axis) {
            for (int sign = -1; sign <= 1; sign += 2) {
                int const u = (axis + 1) % 3, v = (axis + 2) % 3;
                uint32_t  base = uint32_t(m.positions.size() / 3);
                for (auto [a, b] : {std::pair{-1, -1}, {1, -1}, {1, 1}, {-1, 1}}) {
                    double p[3], nn[3] = {0, 0, 0};
                    p[axis]  = sign;
                    p[u]     = a;
                    p[v]     = b;
                    nn[axis] = sign;
                    vertex(p[0], p[1], p[2], nn[0], nn[1], nn[2], 0.5 * (a + 1), 0.5 * (1 - b));
                }
                // (u, v, axis) is right-handed: counter-clockwise in (u, v) faces +axis
                if (sign > 0) {
                    m.indices.insert(m.indices.end(), {base, base + 1, base + 2, base, base + 2, base + 3});
                } else {
                    m.indices.insert(m.indices.end(), {base, base + 2, base + 1, base, base + 3, base + 2});
                }
            }
        }
    } else if (shape == Shape_sphere) {
        double const t = (1.0 + std::sqrt(5.0)) / 2.0;
        std::vector<std::array<double, 3>> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0},
                                                {0, -1, t}, {0, 1, t}, {0, -1, -t}, {0, 1, -t},
                                                {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
        std::vector<std::array<uint32_t, 3>> f = {
            {0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
            {11, 10, 2}, {10, 7, 6}, {7, 1, 8},  {3, 9, 4},  {3, 4, 2},   {3, 2, 6}, {3, 6, 8},
            {3, 8, 9},  {4, 9, 5},  {2, 4, 11}, {6, 2, 10}, {8, 6, 7},   {9, 8, 1}};
        auto unit = [](std::array<double, 3> a) {
            double const l = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
            return std::array<double, 3>{a[0] / l, a[1] / l, a[2] / l};
        };
        for (auto& p : v) {
            p = unit(p);
        }
        for (int level = 0; level < 5; ++level) {
            std::map<std::pair<uint32_t, uint32_t>, uint32_t> mid;
            auto middle = [&](uint32_t a, uint32_t b) {
                auto const key = std::minmax(a, b);
                auto const it  = mid.find(key);
                if (it != mid.end()) {
                    return it->second;
                }
                v.push_back(unit({v[a][0] + v[b][0], v[a][1] + v[b][1], v[a][2] + v[b][2]}));
                return mid[key] = uint32_t(v.size() - 1);
            };
            std::vector<std::array<uint32_t, 3>> nf;
            for (auto const& [a, b, c] : f) {
                uint32_t const ab = middle(a, b), bc = middle(b, c), ca = middle(c, a);
                nf.insert(nf.end(), {{a, ab, ca}, {b, bc, ab}, {c, ca, bc}, {ab, bc, ca}});
            }
            f.swap(nf);
        }
        double area = 0.0;
        for (auto const& [a, b, c] : f) {
            double const e1[3] = {v[b][0] - v[a][0], v[b][1] - v[a][1], v[b][2] - v[a][2]};
            double const e2[3] = {v[c][0] - v[a][0], v[c][1] - v[a][1], v[c][2] - v[a][2]};
            double const x = e1[1] * e2[2] - e1[2] * e2[1], y = e1[2] * e2[0] - e1[0] * e2[2],
                         z = e1[0] * e2[1] - e1[1] * e2[0];
            area += 0.5 * std::sqrt(x * x + y * y + z * z);
        }
        double const s = std::sqrt(4.0 * 3.14159265358979323846 / area);
        double const pi = 3.14159265358979323846;
        for (auto const& p : v) {
            // per vertex; triangles across the u seam interpolate between 1 and 0
            vertex(s * p[0], s * p[1], s * p[2], p[0], p[1], p[2], (-std::atan2(p[0], p[2]) + pi) / (2.0 * pi),
                   std::acos(std::clamp(p[1], -1.0, 1.0)) / pi);
        }
        for (auto const& [a, b, c] : f) {
            m.indices.insert(m.indices.end(), {a, b, c});
        }
    }
    m.part_of.assign(m.indices.size() / 3, 0);
    m.part_slot = {0};
    return m;
}

bool ready() {
    return engine && engine->camera_entity != Null && engine->width > 0 && engine->fov > 0.f &&
           engine->have_integrator;
}

// Rotation rows (normalised) and translation of a row-major object-to-world matrix.
void decompose(float const* m, float rot[9], float pos[3]) {
    for (int r = 0; r < 3; ++r) {
        float const len = std::sqrt(m[4 * r] * m[4 * r] + m[4 * r + 1] * m[4 * r + 1] +
                                    m[4 * r + 2] * m[4 * r + 2]);
        float const inv = len > 0.f ? 1.f / len : 0.f;
        for (int c = 0; c < 3; ++c) {
            rot[3 * r + c] = m[4 * r + c] * inv;
        }
    }
    pos[0] = m[12];
    pos[1] = m[13];
    pos[2] = m[14];
}

// World -> texture-space map of a prop (texture_space_ray, tracking.inl:12-29): the inverse of
// the row-major object-to-world matrix m, then (local - mesh min) / mesh extent.  Computed in
// double; rows of a 3x4 affine map.
void texture_space(float const* m, Mesh const& mesh, float out[12]) {
    double lo[3] = {1e300, 1e300, 1e300};
    double hi[3] = {-1e300, -1e300, -1e300};
    for (size_t v = 0; v < mesh.positions.size() / 3; ++v) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], double(mesh.positions[3 * v + a]));
            hi[a] = std::max(hi[a], double(mesh.positions[3 * v + a]));
        }
    }
    // object-to-world: p_world[c] = sum_r p_obj[r] * m[4r + c] + m[12 + c]; A[c][r] = m[4r + c]
    double A[3][3];
    for (int c = 0; c < 3; ++c) {
        for (int r = 0; r < 3; ++r) {
            A[c][r] = m[4 * r + c];
        }
    }
    double const det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                       A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                       A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
    double const id = det != 0.0 ? 1.0 / det : 0.0;
    double       inv[3][3];
    inv[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) * id;
    inv[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id;
    inv[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
    inv[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) * id;
    inv[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
    inv[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id;
    inv[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) * id;
    inv[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id;
    inv[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
    double const t[3] = {m[12], m[13], m[14]};
    for (int a = 0; a < 3; ++a) {
        double const extent = hi[a] - lo[a];
        double const s      = extent > 0.0 ? 1.0 / extent : 0.0;
        double       off    = 0.0;
        for (int c = 0; c < 3; ++c) {
            out[4 * a + c] = float(inv[a][c] * s);
            off -= inv[a][c] * t[c];
        }
        out[4 * a + 3] = float((off - lo[a]) * s);
    }
}

int32_t apply_camera();

int32_t compile_scene() {
    spb::render::Scene_desc scene;
    scene.instancing = engine->instancing;
    scene.materials  = engine->materials;
    // fallback material for unassigned slots: grey Substitute
    Material fallback{};
    fallback.type     = spb::shading::Type_substitute;
    fallback.metallic = 0.f;
    fallback.alpha    = 1.f;
    fallback.albedo   = srgb_to_ap1(V3{0.5f, 0.5f, 0.5f});
    fallback.f0       = V3{0.03497f, 0.03497f, 0.03497f};
    uint32_t const fallback_id = uint32_t(scene.materials.size());
    scene.materials.push_back(fallback);
    std::vector<uint64_t> grid_images;  // image id << 2 | channel of each scene.grids entry
    std::list<std::vector<float>> grid_channels;  // one channel of a multi-channel image, until uploaded
    std::map<uint32_t, uint32_t> scene_mesh;  // engine shape id -> scene mesh index

    // Texture maps: each (image, use, sampler, scale) once, its texels decoded for the use.
    std::map<std::tuple<uint32_t, uint32_t, bool, bool, float, float>, uint32_t> textures;
    auto const texture = [&](uint32_t image, uint32_t use, Material_maps const& mm, float const scale[2]) {
        auto const key = std::make_tuple(image, use, mm.nearest, mm.clamp, scale[0], scale[1]);
        auto const it  = textures.find(key);
        if (it != textures.end()) {
            return it->second;
        }
        Image const&              img = engine->images[image];
        spb::render::Texture_desc t;
        t.width    = img.dims[0];
        t.height   = img.dims[1];
        t.nearest  = mm.nearest;
        t.clamp    = mm.clamp;
        t.scale[0] = scale[0];
        t.scale[1] = scale[1];
        size_t const texels = size_t(t.width) * t.height;
        uint32_t const c    = img.channels;
        if (use == 0) {
            // colour (Byte3_sRGB / Float3, texture.cpp:60-110): sRGB-encoded bytes to linear, then
            // sRGB -> AP1; one-channel images as grey
            t.channels = 3;
            t.texels.resize(3 * texels);
            for (size_t i = 0; i < texels; ++i) {
                float rgb[3];
                for (int k = 0; k < 3; ++k) {
                    float v = img.pixels[i * c + std::min<uint32_t>(k, c - 1)];
                    if (img.encoded_bytes) {
                        v = v <= 0.04045f ? v / 12.92f : std::pow((v + 0.055f) / 1.055f, 2.4f);
                    }
                    rgb[k] = v;
                }
                V3 const ap1 = img.encoded_bytes ? srgb_to_ap1(V3{rgb[0], rgb[1], rgb[2]}) : V3{rgb[0], rgb[1], rgb[2]};
                t.texels[3 * i]     = ap1.x;
                t.texels[3 * i + 1] = ap1.y;
                t.texels[3 * i + 2] = ap1.z;
            }
        } else {
            // surface: roughness (X) and, for the Surface use of a 2+ channel image, metallic (Y)
            t.channels = (use == 2 && c >= 2) ? 2 : 1;
            t.texels.resize(t.channels * texels);
            for (size_t i = 0; i < texels; ++i) {
                for (uint32_t k = 0; k < t.channels; ++k) {
                    t.texels[t.channels * i + k] = img.pixels[i * c + k];
                }
            }
        }
        scene.textures.push_back(std::move(t));
        return textures[key] = uint32_t(scene.textures.size());
    };
    for (size_t k = 0; k < engine->materials.size() && k < engine->material_maps.size(); ++k) {
        Material_maps const& mm = engine->material_maps[k];
        Material&            m  = scene.materials[k];
        if (mm.color != Null && mm.color < engine->images.size()) {
            m.color_map = texture(mm.color, 0, mm, mm.color_scale);
        }
        if (mm.surface != Null && mm.surface < engine->images.size()) {
            m.surface_map      = texture(mm.surface, mm.surface_usage, mm, mm.surface_scale);
            m.surface_channels = scene.textures[m.surface_map - 1].channels;
        }
    }

    for (Entity const& e : engine->entities) {
        if (e.camera || e.shape == Null) {
            continue;
        }
        if (e.shape == Shape_infinite_sphere) {
            // Uniform environment (Infinite_sphere with a Light material, infinite_sphere.cpp):
            // seen by rays that leave the scene; a light only after su_create_light.
            uint32_t const mat = e.materials.empty() ? Null : e.materials[0];
            if (mat < engine->materials.size() &&
                engine->materials[mat].type == spb::shading::Type_light) {
                V3 const em = engine->materials[mat].emission;
                scene.environment[0] += em.x;
                scene.environment[1] += em.y;
                scene.environment[2] += em.z;
                scene.environment_light |= e.light;
            }
            continue;
        }
        Mesh const& mesh =
            e.shape < First_mesh_id ? engine->builtin[e.shape] : engine->meshes[e.shape - First_mesh_id];
        auto it = scene_mesh.find(e.shape);
        if (it == scene_mesh.end()) {
            spb::render::Mesh_desc md;
            md.positions = mesh.positions;
            md.normals   = mesh.normals;
            md.uvs       = mesh.uvs;
            md.indices   = mesh.indices;
            md.tri_slot.resize(mesh.indices.size() / 3);
            for (size_t t = 0; t < md.tri_slot.size(); ++t) {
                md.tri_slot[t] = mesh.part_slot[mesh.part_of[t]];
            }
            it = scene_mesh.emplace(e.shape, uint32_t(scene.meshes.size())).first;
            scene.meshes.push_back(std::move(md));
        }
        spb::render::Instance_desc inst;
        inst.mesh     = it->second;
        inst.fallback = fallback_id;
        inst.light    = e.light;
        inst.cube     = e.shape == Shape_cube;
        std::copy(e.trafo, e.trafo + 16, inst.trafo);
        float pos[3];
        decompose(e.trafo, inst.rotation, pos);
        // A density-grid medium samples its grid in the prop's texture space, so each prop gets
        // its own copy of such a material (one per slot), pointing at its own medium record.
        inst.materials.assign(e.materials.size(), fallback_id);
        for (size_t k = 0; k < e.materials.size(); ++k) {
            uint32_t const mat = e.materials[k];
            if (mat >= engine->materials.size()) {
                continue;
            }
            inst.materials[k] = mat;
            Grid_ref const& gr = engine->material_grids[mat];
            Material const& em = engine->materials[mat];
            bool const emitting_light = e.light && em.type == spb::shading::Type_volume &&
                                        (em.emission.x > 0.f || em.emission.y > 0.f || em.emission.z > 0.f);
            if (gr.image == Null && gr.color == Null) {
                if (emitting_light) {
                    // the light of an emitting medium is named by its material: one per prop
                    inst.materials[k] = uint32_t(scene.materials.size());
                    scene.materials.push_back(em);
                }
                continue;
            }
            spb::render::Grid_medium gm;
            // index of the grid of an image's channel in the scene (each uploaded once; the
            // channels of a two-channel image as separate grids)
            // (channels 4 to 6: a byte colour image's red, green and blue decoded from sRGB to
            // linear ACEScg, as the reference's Byte4_sRGB texture reads them)
            auto const grid_of = [&](uint32_t image, uint32_t channel) {
                uint64_t const key = (uint64_t(image) << 3) | channel;
                auto const     gi  = std::find(grid_images.begin(), grid_images.end(), key);
                if (gi != grid_images.end()) {
                    return uint32_t(gi - grid_images.begin());
                }
                Image const&              img = engine->images[image];
                spb::render::Density_grid g;
                std::copy(img.dims, img.dims + 3, g.dims);
                if (img.channels == 1) {
                    g.density = img.pixels.data();
                } else {
                    size_t const n = size_t(img.dims[0]) * img.dims[1] * img.dims[2];
                    grid_channels.emplace_back(n);
                    for (size_t v = 0; v < n; ++v) {
                        if (channel < 4) {
                            grid_channels.back()[v] = img.pixels[v * img.channels + channel];
                            continue;
                        }
                        float rgb[3];
                        for (int k = 0; k < 3; ++k) {
                            float const e = img.pixels[v * img.channels + k];
                            rgb[k] = e <= 0.04045f ? e / 12.92f : std::pow((e + 0.055f) / 1.055f, 2.4f);
                        }
                        V3 const ap1 = srgb_to_ap1(V3{rgb[0], rgb[1], rgb[2]});
                        grid_channels.back()[v] = channel == 4 ? ap1.x : (channel == 5 ? ap1.y : ap1.z);
                    }
                    g.density = grid_channels.back().data();
                }
                scene.grids.push_back(g);
                grid_images.push_back(key);
                return uint32_t(grid_images.size() - 1);
            };
            if (gr.image != Null) {
                gm.grid = grid_of(gr.image, 0);
                if (engine->images[gr.image].channels == 2) {
                    gm.emission_scale = grid_of(gr.image, 1) + 1;
                }
            } else {
                // a colour grid: alpha is the density, rgb the colour its coefficients follow
                gm.grid = grid_of(gr.color, 3);
                for (uint32_t c = 0; c < 3; ++c) {
                    gm.color[c] = grid_of(gr.color, 4 + c) + 1;
                }
                gm.color_distance = gr.distance;
            }
            if (gr.temperature != Null) {
                // Grid_emission::commit (volumetric_grid.cpp:140-160): the emission times the
                // black-body colour at 16 temperatures from 2000 to 5000 K
                gm.temperature = grid_of(gr.temperature, 0) + 1;
                for (int k = 0; k < 16; ++k) {
                    double c[3];
                    spb::spectral::blackbody(2000.0 + double(k) / 15.0 * 3000.0, c);
                    gm.blackbody[3 * k]     = float(em.emission.x * c[0]);
                    gm.blackbody[3 * k + 1] = float(em.emission.y * c[1]);
                    gm.blackbody[3 * k + 2] = float(em.emission.z * c[2]);
                }
            }
            gm.nearest = gr.nearest;
            gm.repeat  = gr.repeat;
            texture_space(e.trafo, mesh, gm.world_to_uvw);
            scene.media.push_back(gm);
            Material copy = engine->materials[mat];
            copy.medium   = uint32_t(scene.media.size());
            inst.materials[k] = uint32_t(scene.materials.size());
            scene.materials.push_back(copy);
        }
        scene.instances.push_back(std::move(inst));
    }
    if (scene.instances.empty()) {
        log(SU_LOG_ERROR, "scene has no triangles");
        return -2;
    }
    if (int32_t const s = engine->renderer.set_scene(scene, 0)) {
        log(SU_LOG_ERROR, engine->renderer.error());
        return s == SPB_ERROR_CUDA ? -2 : -1;
    }
    return apply_camera();
}

// The camera entity's transformation, resolution and field of view, and the integrator
// settings, into the renderer (without touching the uploaded scene).
int32_t apply_camera() {
    spb::render::Camera_desc cam;
    cam.width  = engine->width;
    cam.height = engine->height;
    cam.fov    = engine->fov;
    decompose(engine->entities[engine->camera_entity].trafo, cam.rotation, cam.position);
    if (engine->renderer.set_camera(cam)) {
        log(SU_LOG_ERROR, engine->renderer.error());
        return -2;
    }
    // Batch rendering samples with golden ratio sequences, progressive rendering with
    // independent random numbers (su_create_sampler, capi.cpp:295-312; load_sampler_pool,
    // take_loader.cpp:531-556).
    spb::render::Settings settings = engine->settings;
    settings.golden_ratio          = !engine->progressive && engine->sampler_golden;
    engine->renderer.set_settings(settings);
    return 0;
}

int32_t render_samples(uint32_t first, uint32_t count) {
    if (progress_start) {
        progress_start(count);
    }
    if (engine->renderer.render(first, count)) {
        log(SU_LOG_ERROR, engine->renderer.error());
        return -2;
    }
    if (progress_tick) {
        for (uint32_t i = 0; i < count; ++i) {
            progress_tick();
        }
    }
    return 0;
}

// ---- take and scene files (take::Loader::load, take_loader.cpp:98-197; scene::Loader,
// scene_loader.cpp) -- the subset this renderer draws: a Perspective camera, the sampler's
// sample count, the surface integrator, and a scene of named materials and Prop / Light
// entities whose shapes are built-in shapes or triangle-mesh JSON files.  Each part is handed
// to the matching su_* entry point, so a take builds exactly the scene those calls would.

// Reads a whole file; false if it cannot be opened.
bool read_text(std::string const& path, std::string& out) {
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        return false;
    }
    out.clear();
    char buf[1 << 16];
    for (size_t n; (n = std::fread(buf, 1, sizeof(buf), f)) > 0;) {
        out.append(buf, n);
    }
    std::fclose(f);
    return true;
}

bool file_exists(std::string const& path) {
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (f) {
        std::fclose(f);
    }
    return f != nullptr;
}

std::string directory_of(std::string const& path) {
    size_t const slash = path.find_last_of('/');
    return slash == std::string::npos ? std::string() : path.substr(0, slash + 1);
}

// A file named in a take or scene: under the mounted folders (last mounted first), then
// beside the file that names it, then as given.
std::string resolve(std::string const& name, std::string const& base) {
    if (!name.empty() && name[0] == '/') {
        return name;
    }
    for (auto m = engine->mounts.rbegin(); m != engine->mounts.rend(); ++m) {
        std::string dir = *m;
        if (!dir.empty() && dir.back() != '/') {
            dir += '/';
        }
        if (file_exists(dir + name)) {
            return dir + name;
        }
    }
    if (!base.empty() && file_exists(base + name)) {
        return base + name;
    }
    return name;
}

bool read_vec3(spb::json::Value const* v, double out[3]) {
    if (!v || !v->is_array() || v->array.size() < 3) {
        return false;
    }
    for (int k = 0; k < 3; ++k) {
        out[k] = v->array[k].number;
    }
    return true;
}

// An image file (PNG or EXR) as a new image; Null (with a logged reason) if it cannot be read.
uint32_t load_image_file(std::string const& path) {
    spb::image_io::Pixels px;
    std::string           error;
    if (!spb::image_io::read_image(path, px, error)) {
        log(SU_LOG_ERROR, "texture: " + error);
        return Null;
    }
    Image img;
    img.dims[0]       = px.width;
    img.dims[1]       = px.height;
    img.dims[2]       = 1;
    img.channels      = px.channels;
    img.pixels        = std::move(px.values);
    img.encoded_bytes = px.encoded_bytes;
    engine->images.push_back(std::move(img));
    return uint32_t(engine->images.size() - 1);
}

// A texture description's image ({"id": image} or {"file": name}, read_texture_description,
// material_provider.cpp:895-946) and its uv scale; false if it names none.
bool texture_image(spb::json::Value const& v, uint32_t& image, float scale[2]) {
    if (!v.is_object()) {
        return false;
    }
    spb::json::Value const* id   = v.find("id");
    spb::json::Value const* file = v.find("file");
    if (id && id->is_number()) {
        image = uint32_t(id->number);
    } else if (file && file->is_string()) {
        image = load_image_file(resolve(file->string, ""));
    } else {
        return false;
    }
    if (spb::json::Value const* sc = v.find("scale")) {
        if (sc->is_array() && sc->array.size() >= 2) {
            scale[0] = float(sc->array[0].number);
            scale[1] = float(sc->array[1].number);
        } else if (sc->is_number()) {
            scale[0] = scale[1] = float(sc->number);
        }
    }
    return true;
}

// Row-major object-to-world matrix of a "transformation" object, as json::read_transformation
// (json.cpp:252-296) reads it: 16 numbers, or position / scale / rotation (Euler degrees, the
// basis Rz * Rx * Ry of json.cpp:216-227 with the rotation matrices of matrix3x3.inl:61-104)
// / look_at and up (basis rows: -cross(dir, up), up, dir); rows 0-2 are the basis rows times
// the scale, row 3 the position (compose, matrix4x4.inl:27-34).
bool transformation_matrix(spb::json::Value const& v, float m[16]) {
    if (v.is_array()) {
        if (v.array.size() != 16) {
            return false;
        }
        for (int i = 0; i < 16; ++i) {
            m[i] = float(v.array[i].number);
        }
        return true;
    }
    if (!v.is_object()) {
        return false;
    }
    double pos[3] = {0, 0, 0}, scale[3] = {1, 1, 1}, rot[3] = {0, 0, 0}, up[3] = {0, 1, 0}, at[3] = {0, 0, 1};
    read_vec3(v.find("position"), pos);
    read_vec3(v.find("scale"), scale);
    read_vec3(v.find("rotation"), rot);
    read_vec3(v.find("up"), up);
    bool const look = read_vec3(v.find("look_at"), at);
    double b[3][3];
    if (look) {
        double d[3] = {at[0] - pos[0], at[1] - pos[1], at[2] - pos[2]};
        double const l = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        for (double& x : d) {
            x /= l;
        }
        double const right[3] = {-(d[1] * up[2] - d[2] * up[1]), -(d[2] * up[0] - d[0] * up[2]),
                                 -(d[0] * up[1] - d[1] * up[0])};
        for (int k = 0; k < 3; ++k) {
            b[0][k] = right[k];
            b[1][k] = up[k];
            b[2][k] = d[k];
        }
    } else {
        double const d2r = 3.14159265358979323846 / 180.0;
        double const cx = std::cos(rot[0] * d2r), sx = std::sin(rot[0] * d2r);
        double const cy = std::cos(rot[1] * d2r), sy = std::sin(rot[1] * d2r);
        double const cz = std::cos(rot[2] * d2r), sz = std::sin(rot[2] * d2r);
        double const rx[3][3] = {{1, 0, 0}, {0, cx, -sx}, {0, sx, cx}};
        double const ry[3][3] = {{cy, 0, sy}, {0, 1, 0}, {-sy, 0, cy}};
        double const rz[3][3] = {{cz, -sz, 0}, {sz, cz, 0}, {0, 0, 1}};
        double zx[3][3];
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) {
                zx[i][j] = rz[i][0] * rx[0][j] + rz[i][1] * rx[1][j] + rz[i][2] * rx[2][j];
            }
        }
        for (int i = 0; i < 3; ++i) {
            for (int j = 0; j < 3; ++j) {
                b[i][j] = zx[i][0] * ry[0][j] + zx[i][1] * ry[1][j] + zx[i][2] * ry[2][j];
            }
        }
    }
    // The rotation is kept as a quaternion (quaternion::create, quaternion.inl:12-35) and
    // turned back into a basis (create_matrix3x3, quaternion.inl:64-86); for the look_at basis,
    // whose up is not made orthogonal to the direction, this round trip changes the matrix.
    float r[3][3];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            r[i][j] = float(b[i][j]);
        }
    }
    float q[4];  // x, y, z, w
    float t;
    if (r[2][2] < 0.f) {
        if (r[0][0] > r[1][1]) {
            t = 1.f + r[0][0] - r[1][1] - r[2][2];
            float const v[4] = {t, r[0][1] + r[1][0], r[2][0] + r[0][2], r[2][1] - r[1][2]};
            std::copy(v, v + 4, q);
        } else {
            t = 1.f - r[0][0] + r[1][1] - r[2][2];
            float const v[4] = {r[0][1] + r[1][0], t, r[1][2] + r[2][1], r[0][2] - r[2][0]};
            std::copy(v, v + 4, q);
        }
    } else {
        if (r[0][0] < -r[1][1]) {
            t = 1.f - r[0][0] - r[1][1] + r[2][2];
            float const v[4] = {r[2][0] + r[0][2], r[1][2] + r[2][1], t, r[1][0] - r[0][1]};
            std::copy(v, v + 4, q);
        } else {
            t = 1.f + r[0][0] + r[1][1] + r[2][2];
            float const v[4] = {r[2][1] - r[1][2], r[0][2] - r[2][0], r[1][0] - r[0][1], t};
            std::copy(v, v + 4, q);
        }
    }
    float const f = 0.5f / std::sqrt(t);
    float const x = f * q[0], y = f * q[1], z = f * q[2], w = f * q[3];
    float const basis[3][3] = {{1.f - (2.f * y * y + 2.f * z * z), 2.f * x * y - 2.f * z * w, 2.f * x * z + 2.f * y * w},
                               {2.f * x * y + 2.f * z * w, 1.f - (2.f * x * x + 2.f * z * z), 2.f * y * z - 2.f * x * w},
                               {2.f * x * z - 2.f * y * w, 2.f * y * z + 2.f * x * w, 1.f - (2.f * x * x + 2.f * y * y)}};
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            m[4 * i + j] = float(basis[i][j] * scale[i]);
        }
        m[4 * i + 3] = 0.f;
        m[12 + i]    = float(pos[i]);
    }
    m[15] = 1.f;
    return true;
}

// A triangle-mesh JSON file ({"geometry": {"parts", "vertices": {"positions", "normals"},
// "indices"}}, triangle_mesh_provider.cpp) through su_create_triangle_mesh_async.
uint32_t load_mesh_file(std::string const& path) {
    std::string text;
    spb::json::Value root;
    if (!read_text(path, text) || !spb::json::parse(text.c_str(), root)) {
        log(SU_LOG_ERROR, "su_load_take: cannot read mesh file " + path);
        return Null;
    }
    spb::json::Value const* g = root.find("geometry");
    spb::json::Value const* verts = g ? g->find("vertices") : nullptr;
    spb::json::Value const* pos = verts ? verts->find("positions") : nullptr;
    spb::json::Value const* nrm = verts ? verts->find("normals") : nullptr;
    spb::json::Value const* idx = g ? g->find("indices") : nullptr;
    if (!pos || !pos->is_array() || !nrm || !nrm->is_array() || !idx || !idx->is_array() ||
        pos->array.size() % 3 || nrm->array.size() != pos->array.size() || idx->array.size() % 3) {
        log(SU_LOG_ERROR, "su_load_take: mesh file " + path + " needs positions, normals and triangle indices");
        return Null;
    }
    std::string const topology = spb::json::string_or(g->find("primitive_topology"), "triangle_list");
    if (topology != "triangle_list") {
        log(SU_LOG_ERROR, "su_load_take: " + path + ": only triangle_list topology is supported");
        return Null;
    }
    std::vector<float> p(pos->array.size()), n(nrm->array.size());
    for (size_t i = 0; i < p.size(); ++i) {
        p[i] = float(pos->array[i].number);
        n[i] = float(nrm->array[i].number);
    }
    // "texture_coordinates_0": two per vertex (triangle_json_handler.cpp:189-199)
    std::vector<float>      uv;
    spb::json::Value const* tc = verts->find("texture_coordinates_0");
    if (tc && tc->is_array() && tc->array.size() == 2 * (p.size() / 3)) {
        uv.resize(tc->array.size());
        for (size_t i = 0; i < uv.size(); ++i) {
            uv[i] = float(tc->array[i].number);
        }
    }
    std::vector<uint32_t> ind(idx->array.size());
    for (size_t i = 0; i < ind.size(); ++i) {
        ind[i] = uint32_t(idx->array[i].number);
    }
    std::vector<uint32_t> parts;
    if (spb::json::Value const* pv = g->find("parts"); pv && pv->is_array()) {
        for (auto const& part : pv->array) {
            parts.push_back(uint32_t(spb::json::number_or(part.find("start_index"), 0)));
            parts.push_back(uint32_t(spb::json::number_or(part.find("num_indices"), 0)));
            parts.push_back(uint32_t(spb::json::number_or(part.find("material_index"), 0)));
        }
    }
    return su_create_triangle_mesh_async(uint32_t(ind.size() / 3), uint32_t(p.size() / 3), 3, p.data(), 3, n.data(),
                                         0, nullptr, uv.empty() ? 0 : 2, uv.empty() ? nullptr : uv.data(), ind.data(),
                                         uint32_t(parts.size() / 3), parts.empty() ? nullptr : parts.data());
}

// Built-in shape names (sprout.h's SU_SHAPE_* ids).
uint32_t builtin_shape(std::string const& type) {
    static std::map<std::string, uint32_t> const ids = {
        {"Canopy", 0}, {"Cube", 1}, {"Disk", 2}, {"Distant_sphere", 3}, {"Infinite_sphere", 4},
        {"Plane", 5}, {"Rectangle", 6}, {"Sphere", 7}};
    auto const it = ids.find(type);
    return it == ids.end() ? Null : it->second;
}

int32_t load_scene(std::string const& path) {
    std::string text;
    spb::json::Value root;
    if (!read_text(path, text) || !spb::json::parse(text.c_str(), root)) {
        log(SU_LOG_ERROR, "su_load_take: cannot read scene " + path);
        return -2;
    }
    std::string const base = directory_of(path);
    std::map<std::string, uint32_t> materials;
    if (spb::json::Value const* mv = root.find("materials"); mv && mv->is_array()) {
        for (auto const& m : mv->array) {
            std::string const name = spb::json::string_or(m.find("name"), "");
            uint32_t const id = su_create_material(spb::json::dump(m).c_str());
            if (id == Null) {
                log(SU_LOG_ERROR, "su_load_take: material \"" + name + "\" not supported");
                return -2;
            }
            materials[name] = id;
        }
    }
    std::map<std::string, uint32_t> meshes;
    spb::json::Value const* ev = root.find("entities");
    if (!ev || !ev->is_array()) {
        log(SU_LOG_ERROR, "su_load_take: scene " + path + " has no entities");
        return -2;
    }
    for (auto const& e : ev->array) {
        std::string const type = spb::json::string_or(e.find("type"), "");
        if (type != "Prop" && type != "Light") {
            log(SU_LOG_WARNING, "su_load_take: entity type \"" + type + "\" skipped");
            continue;
        }
        spb::json::Value const* sv = e.find("shape");
        uint32_t shape = Null;
        if (sv && sv->find("file")) {
            std::string const file = resolve(spb::json::string_or(sv->find("file"), ""), base);
            auto const it = meshes.find(file);
            shape = it != meshes.end() ? it->second : (meshes[file] = load_mesh_file(file));
        } else if (sv) {
            shape = builtin_shape(spb::json::string_or(sv->find("type"), ""));
        }
        if (shape == Null) {
            log(SU_LOG_ERROR, "su_load_take: entity shape not supported");
            return -2;
        }
        std::vector<uint32_t> mats;
        if (spb::json::Value const* names = e.find("materials"); names && names->is_array()) {
            for (auto const& n : names->array) {
                auto const it = materials.find(n.string);
                if (it == materials.end()) {
                    log(SU_LOG_ERROR, "su_load_take: unknown material \"" + n.string + "\"");
                    return -2;
                }
                mats.push_back(it->second);
            }
        }
        uint32_t const prop = su_create_prop(shape, uint32_t(mats.size()), mats.data());
        if (prop == Null) {
            return -2;
        }
        if (spb::json::Value const* tv = e.find("transformation")) {
            float m[16];
            if (!transformation_matrix(*tv, m) || su_entity_set_transformation(prop, m) != 0) {
                log(SU_LOG_ERROR, "su_load_take: bad transformation");
                return -2;
            }
        }
        if (type == "Light" && su_create_light(prop) != 0) {
            return -2;
        }
    }
    return 0;
}

// A 3-D image in the reference's SUB format (image::encoding::sub::Reader::read,
// sub_image_reader.cpp:35-224): "SUB\0", a uint64 header length, a JSON header (image
// description: dimensions, Byte1 or Float1; pixels and, for sparse images, a topology bitfield
// as offsets into the binary part), then the binary part.  A topology marks the stored voxels
// (32-bit words, bit i at the word's bit 31 - i % 32), whose values follow in order; the others
// are 0.  Bytes become value / 255.  Returns the new image's id, or Null.
uint32_t load_sub_image(std::string const& path) {
    std::string data;
    if (!read_text(path, data) || data.size() < 12 || data.compare(0, 3, "SUB") != 0) {
        log(SU_LOG_ERROR, "cannot read SUB image " + path);
        return Null;
    }
    uint64_t header = 0;
    std::memcpy(&header, data.data() + 4, sizeof(header));
    spb::json::Value root;
    if (12 + header > data.size() || !spb::json::parse(data.substr(12, header).c_str(), root)) {
        log(SU_LOG_ERROR, "bad SUB header in " + path);
        return Null;
    }
    uint64_t const           start = 12 + header;
    spb::json::Value const* image  = root.find("image");
    spb::json::Value const* desc   = image ? image->find("description") : nullptr;
    spb::json::Value const* dims   = desc ? desc->find("dimensions") : nullptr;
    std::string const       type   = desc ? spb::json::string_or(desc->find("type"), "") : "";
    spb::json::Value const* pixels = image ? image->find("pixels") : nullptr;
    spb::json::Value const* pbin   = pixels ? pixels->find("binary") : nullptr;
    if (!dims || !dims->is_array() || dims->array.size() != 3 || !pbin || (type != "Byte1" && type != "Float1")) {
        log(SU_LOG_ERROR, "SUB image " + path + ": need dimensions, a Byte1 or Float1 type and pixels");
        return Null;
    }
    Image img;
    uint64_t voxels = 1;
    for (int k = 0; k < 3; ++k) {
        img.dims[k] = uint32_t(dims->array[k].number);
        voxels *= img.dims[k];
    }
    img.channels = 1;
    img.pixels.assign(voxels, 0.f);
    uint64_t const bytes  = type == "Byte1" ? 1 : 4;
    uint64_t       cursor = start + uint64_t(spb::json::number_or(pbin->find("offset"), 0.0));
    auto const     value  = [&](uint64_t at, float& v) {
        if (at + bytes > data.size()) {
            return false;
        }
        if (bytes == 1) {
            v = float(uint8_t(data[at])) * (1.f / 255.f);
        } else {
            std::memcpy(&v, data.data() + at, 4);
        }
        return true;
    };
    spb::json::Value const* topo = image->find("topology");
    spb::json::Value const* tbin = topo ? topo->find("binary") : nullptr;
    if (tbin) {
        uint64_t const words = (voxels + 31) / 32;
        uint64_t const field = start + uint64_t(spb::json::number_or(tbin->find("offset"), 0.0));
        if (field + 4 * words > data.size()) {
            log(SU_LOG_ERROR, "SUB image " + path + ": truncated topology");
            return Null;
        }
        for (uint64_t i = 0; i < voxels; ++i) {
            uint32_t word;
            std::memcpy(&word, data.data() + field + 4 * (i >> 5), 4);
            if (word & (0x80000000u >> (i % 32))) {
                if (!value(cursor, img.pixels[i])) {
                    log(SU_LOG_ERROR, "SUB image " + path + ": truncated pixels");
                    return Null;
                }
                cursor += bytes;
            }
        }
    } else {
        for (uint64_t i = 0; i < voxels; ++i, cursor += bytes) {
            if (!value(cursor, img.pixels[i])) {
                log(SU_LOG_ERROR, "SUB image " + path + ": truncated pixels");
                return Null;
            }
        }
    }
    engine->images.push_back(std::move(img));
    return uint32_t(engine->images.size() - 1);
}

// An 8-bit RGB PNG (the reference's default exporter, encoding::png::Writer, writes this from
// the postprocessed frame): one IHDR, the rows (filter byte 0 each) as a zlib stream of stored
// deflate blocks in one IDAT, IEND; CRC-32 per chunk, Adler-32 over the rows.
bool write_png(std::string const& path, uint32_t w, uint32_t h, uint8_t const* rgb) {
    static uint32_t const* const crc_table = [] {
        static uint32_t t[256];
        for (uint32_t n = 0; n < 256; ++n) {
            uint32_t c = n;
            for (int k = 0; k < 8; ++k) {
                c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            }
            t[n] = c;
        }
        return t;
    }();
    auto const be32 = [](std::string& out, uint32_t v) {
        for (int k = 3; k >= 0; --k) {
            out += char((v >> (8 * k)) & 0xFF);
        }
    };
    auto const chunk = [&](std::string& out, char const* type, std::string const& data) {
        be32(out, uint32_t(data.size()));
        std::string const body = std::string(type, 4) + data;
        uint32_t          crc  = 0xFFFFFFFFu;
        for (unsigned char const c : body) {
            crc = crc_table[(crc ^ c) & 0xFF] ^ (crc >> 8);
        }
        out += body;
        be32(out, crc ^ 0xFFFFFFFFu);
    };
    std::string raw;
    raw.reserve(size_t(h) * (3 * size_t(w) + 1));
    for (uint32_t y = 0; y < h; ++y) {
        raw += char(0);
        raw.append(reinterpret_cast<char const*>(rgb) + size_t(y) * 3 * w, 3 * size_t(w));
    }
    std::string z = "\x78\x01";
    for (size_t at = 0; at < raw.size() || at == 0; at += 65535) {
        size_t const n = std::min<size_t>(65535, raw.size() - at);
        z += char(at + n >= raw.size() ? 1 : 0);
        z += char(n & 0xFF);
        z += char(n >> 8);
        z += char(~n & 0xFF);
        z += char((~n >> 8) & 0xFF);
        z.append(raw, at, n);
        if (raw.empty()) {
            break;
        }
    }
    uint32_t a = 1, b = 0;
    for (unsigned char const c : raw) {
        a = (a + c) % 65521;
        b = (b + a) % 65521;
    }
    be32(z, (b << 16) | a);
    std::string ihdr;
    be32(ihdr, w);
    be32(ihdr, h);
    ihdr += std::string("\x08\x02\x00\x00\x00", 5);  // 8 bits, RGB, deflate, no filter, no interlace
    std::string png = "\x89PNG\r\n\x1a\n";
    chunk(png, "IHDR", ihdr);
    chunk(png, "IDAT", z);
    chunk(png, "IEND", "");
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        return false;
    }
    bool const ok = std::fwrite(png.data(), 1, png.size(), f) == png.size();
    return std::fclose(f) == 0 && ok;
}

// su_load_take: a take given as JSON text or as a file name.
// A take's tonemapper object (load_tonemapper, take_loader.cpp:864-903).
bool read_tonemapper(spb::json::Value const& v, spb::post::Tonemapper& t) {
    if (!v.is_object() || v.object.empty()) {
        return false;
    }
    auto const& [name, p] = v.object[0];
    auto const  num       = [&](char const* key, float fallback) {
        return float(spb::json::number_or(p.find(key), fallback));
    };
    t             = spb::post::Tonemapper();
    t.auto_expose = spb::json::bool_or(p.find("auto_expose"), false);
    t.exposure    = num("exposure", 0.f);
    if (name == "Linear") {
        t.kind = spb::post::Tonemapper::Kind::Linear;
    } else if (name == "ACES") {
        t.kind = spb::post::Tonemapper::Kind::Aces;
    } else if (name == "Generic") {
        t.kind     = spb::post::Tonemapper::Kind::Generic;
        t.contrast = num("contrast", t.contrast);
        t.shoulder = num("shoulder", t.shoulder);
        t.mid_in   = num("mid_in", t.mid_in);
        t.mid_out  = num("mid_out", t.mid_out);
        t.hdr_max  = num("hdr_max", t.hdr_max);
    } else if (name == "Piecewise") {
        t.kind              = spb::post::Tonemapper::Kind::Piecewise;
        t.toe_strength      = num("toe_strength", t.toe_strength);
        t.toe_length        = num("toe_length", t.toe_length);
        t.shoulder_strength = num("shoulder_strength", t.shoulder_strength);
        t.shoulder_length   = num("shoulder_length", t.shoulder_length);
        t.shoulder_angle    = num("shoulder_angle", t.shoulder_angle);
    } else {
        return false;
    }
    return true;
}

int32_t load_take(std::string const& string) {
    size_t const first = string.find_first_not_of(" \t\r\n");
    bool const   is_json = first != std::string::npos && string[first] == '{';
    std::string  text, base;
    if (is_json) {
        text = string;
    } else {
        std::string const path = resolve(string, "");
        if (!read_text(path, text)) {
            log(SU_LOG_ERROR, "su_load_take: cannot read " + string);
            return -2;
        }
        base = directory_of(path);
    }
    spb::json::Value take;
    if (!spb::json::parse(text.c_str(), take) || !take.is_object()) {
        log(SU_LOG_ERROR, "su_load_take: take JSON parse error");
        return -2;
    }
    if (spb::json::Value const* cam = take.find("camera")) {
        if (su_create_camera(spb::json::dump(*cam).c_str()) == Null) {
            return -2;
        }
        spb::json::Value const* persp = cam->find("Perspective");
        if (spb::json::Value const* tv = persp ? persp->find("transformation") : nullptr) {
            float m[16];
            if (!transformation_matrix(*tv, m) || su_entity_set_transformation(engine->camera_entity, m) != 0) {
                log(SU_LOG_ERROR, "su_load_take: bad camera transformation");
                return -2;
            }
        }
        // The sensor filter here is Gaussian, radius 1, alpha 1.8 (the C API's); other filters
        // (the take default is radius 2) are drawn with it.
        spb::json::Value const* sensor = persp ? persp->find("sensor") : nullptr;
        spb::json::Value const* filter = sensor ? sensor->find("filter") : nullptr;
        spb::json::Value const* gauss  = filter ? filter->find("Gaussian") : nullptr;
        if (!gauss || spb::json::number_or(gauss->find("radius"), 2.0) != 1.0 ||
            spb::json::number_or(gauss->find("alpha"), 1.8) != 1.8) {
            log(SU_LOG_WARNING, "su_load_take: the sensor filter is drawn as Gaussian (radius 1, alpha 1.8)");
        }
    }
    engine->sampler_golden = false;  // a take without a sampler samples randomly (take_loader.cpp:150-157)
    if (spb::json::Value const* sampler = take.find("sampler"); sampler && sampler->is_object() &&
                                                                !sampler->object.empty()) {
        su_create_sampler(uint32_t(spb::json::number_or(sampler->object[0].second.find("samples_per_pixel"), 1.0)));
        // "Golden_ratio" (and su_create_sampler) sample batch frames with golden ratio
        // sequences; "Random" (and the reference's "RD", whose sequence this renderer does not
        // have) with independent random numbers
        engine->sampler_golden = sampler->object[0].first == "Golden_ratio";
    }
    if (spb::json::Value const* integrator = take.find("integrator")) {
        su_create_integrators(spb::json::dump(*integrator).c_str());
    }
    // "post": the postprocessors in order (Loader::load_postprocessors, take_loader.cpp:817-862);
    // without it the Linear tonemapper (set_default_postprocessor, :965-978).
    engine->pipeline.assign(1, spb::post::Tonemapper());
    if (spb::json::Value const* post = take.find("post"); post && post->is_array()) {
        engine->pipeline.clear();
        for (auto const& pp : post->array) {
            if (!pp.is_object() || pp.object.empty()) {
                continue;
            }
            spb::json::Value const* tm = pp.find("tonemapper");
            spb::post::Tonemapper   t;
            if (!tm || !read_tonemapper(*tm, t)) {
                log(SU_LOG_WARNING, "su_load_take: postprocessor \"" + pp.object[0].first + "\" is not supported; skipped");
                continue;
            }
            engine->pipeline.push_back(t);
        }
    }
    // "export": {"Image": {"format": "PNG" | "EXR" | "RGBE"}} (load_exporters, take_loader.cpp:907-951);
    // without it the PNG writer (set_default_exporter, :980-994).
    engine->exporters.assign(1, "PNG");
    if (spb::json::Value const* ex = take.find("export"); ex && ex->is_object()) {
        engine->exporters.clear();
        for (auto const& [name, value] : ex->object) {
            if (name == "Image") {
                engine->exporters.push_back(spb::json::string_or(value.find("format"), "PNG"));
            } else {
                log(SU_LOG_WARNING, "su_load_take: exporter \"" + name + "\" is not supported; skipped");
            }
        }
    }
    if (spb::json::Value const* scene = take.find("scene"); scene && scene->is_string()) {
        return load_scene(resolve(scene->string, base));
    }
    return 0;
}

}  // namespace

extern "C" {

SU_LIBRARY_API char const* su_platform_revision(void) {
    return "sprout_b200 (sm_100a wavefront path tracer)";
}

SU_LIBRARY_API int32_t su_init(bool progressive) {
    if (engine) {
        return -1;
    }
    engine = new Engine(progressive);
    return 0;
}

SU_LIBRARY_API int32_t su_release(void) {
    delete engine;
    engine = nullptr;
    return 0;
}

SU_LIBRARY_API int32_t su_mount(char const* folder) {
    if (!engine) {
        return -1;
    }
    if (folder) {
        engine->mounts.emplace_back(folder);
    }
    return 0;
}

SU_LIBRARY_API int32_t su_clear(void) {
    if (!engine) {
        return -1;
    }
    engine->entities.clear();
    engine->meshes.clear();
    engine->materials.clear();
    engine->material_grids.clear();
    engine->material_maps.clear();
    engine->images.clear();
    engine->camera_entity = Null;
    engine->frame_started = false;
    engine->scene_dirty   = true;
    return 0;
}

SU_LIBRARY_API int32_t su_load_take(char const* string) {
    if (!engine) {
        return -1;
    }
    return load_take(string ? string : "");
}

SU_LIBRARY_API int32_t su_create_defaults(void) {
    if (!engine) {
        return -1;
    }
    // take_loader.cpp:965-978: with ACEScg the default pipeline is the Linear tonemapper
    // (exposure 0), which maps the AP1 film to linear sRGB (tonemapping/linear.cpp:10-27).
    engine->pipeline.assign(1, spb::post::Tonemapper());
    if (!engine->have_integrator) {
        engine->settings        = spb::render::Settings();
        engine->have_integrator = true;
    }
    return 0;
}

SU_LIBRARY_API uint32_t su_create_camera_perspective(uint32_t width, uint32_t height, float fov) {
    if (!engine) {
        return Null;
    }
    if (width == 0 || height == 0 || !(fov > 0.f)) {
        log(SU_LOG_ERROR, "su_create_camera_perspective: invalid resolution or fov");
        return Null;
    }
    Entity e;
    e.camera = true;
    engine->entities.push_back(e);
    engine->camera_entity = uint32_t(engine->entities.size() - 1);
    engine->scene_dirty   = true;
    engine->width         = width;
    engine->height        = height;
    engine->fov           = fov;
    return engine->camera_entity;
}

SU_LIBRARY_API uint32_t su_create_camera(char const* string) {
    if (!engine) {
        return Null;
    }
    spb::json::Value root;
    if (!spb::json::parse(string, root)) {
        log(SU_LOG_ERROR, "su_create_camera: JSON parse error");
        return Null;
    }
    spb::json::Value const* persp = root.find("Perspective");
    if (!persp) {
        log(SU_LOG_ERROR, "su_create_camera: only Perspective cameras are supported");
        return Null;
    }
    double fov_deg = 60.0;
    if (auto const* params = persp->find("parameters")) {
        fov_deg = spb::json::number_or(params->find("fov"), fov_deg);
    }
    uint32_t w = 0;
    uint32_t h = 0;
    if (auto const* sensor = persp->find("sensor")) {
        if (auto const* res = sensor->find("resolution"); res && res->is_array() && res->array.size() == 2) {
            w = uint32_t(res->array[0].number);
            h = uint32_t(res->array[1].number);
        }
    }
    if (w == 0 || h == 0) {
        log(SU_LOG_ERROR, "su_create_camera: missing sensor resolution");
        return Null;
    }
    return su_create_camera_perspective(w, h, float(fov_deg * 3.14159265358979323846 / 180.0));
}

SU_LIBRARY_API int32_t su_camera_set_resolution(uint32_t width, uint32_t height) {
    if (!engine) {
        return -1;
    }
    if (engine->camera_entity == Null) {
        return -2;
    }
    engine->width         = width;
    engine->height        = height;
    engine->frame_started = false;
    engine->camera_dirty  = true;
    return 0;
}

SU_LIBRARY_API int32_t su_create_sampler(uint32_t num_samples) {
    if (!engine) {
        return -1;
    }
    engine->spp = std::max(1u, num_samples);
    return 0;
}

SU_LIBRARY_API int32_t su_create_integrators(char const* string) {
    if (!engine) {
        return -1;
    }
    spb::json::Value root;
    if (!spb::json::parse(string, root)) {
        log(SU_LOG_ERROR, "su_create_integrators: JSON parse error");
        return 0;
    }
    // take_loader.cpp:617-738 defaults: min_bounces 4, max_bounces 8
    spb::render::Settings s;
    if (auto const* surface = root.find("surface")) {
        spb::json::Value const* pt = surface->find("PTMIS");
        if (!pt) {
            log(SU_LOG_WARNING, "su_create_integrators: only PTMIS is implemented; using PTMIS");
            pt = surface->object.empty() ? nullptr : &surface->object.front().second;
        }
        if (pt) {
            s.min_bounces = uint32_t(spb::json::number_or(pt->find("min_bounces"), s.min_bounces));
            s.max_bounces = uint32_t(spb::json::number_or(pt->find("max_bounces"), s.max_bounces));
            // "light_sampling": {"strategy": "Single" | "Adaptive", "splitting_threshold": t}
            // (load_light_sampling, take_loader.cpp:995-1015; the threshold is used as t^4,
            // Tree::set_splitting_threshold, light_tree.cpp:341-343)
            if (spb::json::Value const* ls = pt->find("light_sampling"); ls && ls->is_object()) {
                std::string const strategy = spb::json::string_or(ls->find("strategy"), "");
                if (strategy == "Single") {
                    s.light_split = false;
                } else if (strategy == "Adaptive") {
                    s.light_split = true;
                }
                if (spb::json::Value const* st = ls->find("splitting_threshold"); st && !st->is_string()) {
                    float const t     = float(spb::json::number_or(st, 0.08));
                    s.split_threshold = t * t * t * t;
                }
            }
            // "spectral": hero-wavelength spectral transport (this renderer's extension; scenes of
            // participating media, emitters and the environment)
            s.spectral = spb::json::bool_or(pt->find("spectral"), false);
            // "seed": the sample streams' seed (this renderer's extension, default 0), for
            // statistically independent renders of one scene
            s.seed = uint32_t(spb::json::number_or(pt->find("seed"), s.seed));
            // "wave_paths", "trace_blocks_per_sm": fixed launch shapes instead of the autotuner's
            // (this renderer's extension)
            s.wave_paths          = uint32_t(spb::json::number_or(pt->find("wave_paths"), 0.0));
            s.trace_blocks_per_sm = uint32_t(spb::json::number_or(pt->find("trace_blocks_per_sm"), 0.0));
            s.wave_paths          = s.wave_paths ? std::clamp(s.wave_paths, 1u << 16, 1u << 24) : 0u;
            // "cuda_graphs": false launches every wave's kernels one by one
            s.cuda_graphs = spb::json::bool_or(pt->find("cuda_graphs"), true);
            // "instancing": true keeps one tree per mesh under a top-level tree over the props,
            // false flattens every prop into one world-space tree; absent or "auto": two
            // levels when flattening would multiply the distinct meshes' triangles by more
            // than four and exceed a million (this renderer's extension)
            engine->instancing = -1;
            if (spb::json::Value const* inst = pt->find("instancing"); inst && !inst->is_string()) {
                engine->instancing = spb::json::bool_or(inst, false) ? 1 : 0;
            }
            // "guiding": true, or an object of the Settings guide fields (this renderer's
            // extension; the reference ignores the key)
            if (spb::json::Value const* g = pt->find("guiding")) {
                s.guiding = g->is_object() || spb::json::bool_or(g, false);
                if (g->is_object()) {
                    s.guide_fraction = float(spb::json::number_or(g->find("fraction"), s.guide_fraction));
                    s.metal_fraction = float(spb::json::number_or(g->find("metal_fraction"), s.metal_fraction));
                    s.guide_batch    = uint32_t(spb::json::number_or(g->find("batch"), s.guide_batch));
                    s.guide_steps    = uint32_t(spb::json::number_or(g->find("steps"), s.guide_steps));
                    s.guide_lr       = float(spb::json::number_or(g->find("learning_rate"), s.guide_lr));
                    s.record_depth   = uint32_t(spb::json::number_or(g->find("record_depth"), s.record_depth));
                    s.guide_seed     = uint32_t(spb::json::number_or(g->find("seed"), s.guide_seed));
                    s.guide_pass_spp = uint32_t(spb::json::number_or(g->find("pass_spp"), s.guide_pass_spp));
                    s.guide_train_spp = uint32_t(spb::json::number_or(g->find("train_spp"), s.guide_train_spp));
                    s.guide_depth     = uint32_t(spb::json::number_or(g->find("depth"), s.guide_depth));
                }
                s.guide_fraction = std::clamp(s.guide_fraction, 0.f, 0.95f);
                s.metal_fraction = s.metal_fraction < 0.f ? -1.f : std::min(s.metal_fraction, 0.95f);
                s.record_depth   = std::clamp(s.record_depth, 1u, 8u);
                s.guide_batch    = std::clamp(s.guide_batch, 128u, 1u << 22);
            }
        }
    }
    if (s.max_bounces > 60) {
        log(SU_LOG_WARNING, "su_create_integrators: max_bounces clamped to 60");
        s.max_bounces = 60;
    }
    engine->settings        = s;
    engine->have_integrator = true;
    engine->scene_dirty     = true;
    return 0;
}

SU_LIBRARY_API uint32_t su_create_image(uint32_t pixel_type, uint32_t num_channels, uint32_t width,
                                        uint32_t height, uint32_t depth, uint32_t num_elements,
                                        uint32_t stride, char const* data) {
    // capi.cpp:329-344 and image_provider.cpp:90-170: Byte (unorm) or Float pixels, 1 to 4
    // channels, pixels stride bytes apart (0: packed); ids count from 0 in creation order.
    if (!engine) {
        return Null;
    }
    uint32_t const bytes = pixel_type == 0 ? 1u : (pixel_type == 2 ? 4u : 0u);
    if (bytes == 0 || num_channels < 1 || num_channels > 4 || width == 0 || height == 0 || !data ||
        num_elements > 1) {
        log(SU_LOG_ERROR, "su_create_image: unsupported pixel type, channel count or size");
        return Null;
    }
    Image img;
    img.dims[0]  = width;
    img.dims[1]  = height;
    img.dims[2]  = std::max(depth, 1u);
    img.channels = num_channels;
    size_t const pixels = size_t(width) * height * img.dims[2];
    size_t const step   = stride ? stride : size_t(bytes) * num_channels;
    img.pixels.resize(pixels * num_channels);
    for (size_t i = 0; i < pixels; ++i) {
        char const* src = data + i * step;
        for (uint32_t c = 0; c < num_channels; ++c) {
            float v;
            if (bytes == 1) {
                v = float(uint8_t(src[c])) * (1.f / 255.f);
            } else {
                std::memcpy(&v, src + 4 * c, 4);
            }
            img.pixels[i * num_channels + c] = v;
        }
    }
    img.encoded_bytes = bytes == 1;
    engine->images.push_back(std::move(img));
    engine->scene_dirty = true;
    return uint32_t(engine->images.size() - 1);
}

SU_LIBRARY_API uint32_t su_create_material(char const* string) {
    if (!engine) {
        return Null;
    }
    spb::json::Value root;
    if (!spb::json::parse(string, root)) {
        log(SU_LOG_ERROR, "su_create_material: JSON parse error");
        return Null;
    }
    spb::json::Value const* rendering = root.find("rendering");
    if (!rendering || !rendering->is_object() || rendering->object.empty()) {
        log(SU_LOG_ERROR, "su_create_material: missing \"rendering\"");
        return Null;
    }
    std::string const&      type = rendering->object.front().first;
    spb::json::Value const& desc = rendering->object.front().second;

    Material      m{};
    Grid_ref      grid;
    Material_maps maps;
    m.two_sided = spb::json::bool_or(desc.find("two_sided"), false) ? 1u : 0u;
    if (type == "Light") {
        // material_provider.cpp:298-364: "emission" is a radiance, default 10
        V3 emission{10.f, 10.f, 10.f};
        emission   = srgb_to_ap1(emission);
        read_color(desc.find("emission"), emission);
        m.type     = spb::shading::Type_light;
        m.emission = emission;
    } else if (type == "Substitute") {
        // material_provider.cpp:483-760 defaults: color 0.5, roughness 0.8, metallic 0, ior 1.46
        V3 color = srgb_to_ap1(V3{0.5f, 0.5f, 0.5f});
        read_color(desc.find("color"), color);
        float const roughness = float(spb::json::number_or(desc.find("roughness"), 0.8));
        float const metallic  = float(spb::json::number_or(desc.find("metallic"), 0.0));
        float const ior       = float(spb::json::number_or(desc.find("ior"), 1.46));
        float const r         = std::max(roughness, spb::shading::Min_roughness);
        float const f0d       = ((1.f - ior) / (1.f + ior)) * ((1.f - ior) / (1.f + ior));
        m.type     = spb::shading::Type_substitute;
        m.metallic = metallic;
        m.alpha    = r * r;
        m.albedo   = V3{(1.f - metallic) * color.x, (1.f - metallic) * color.y,
                      (1.f - metallic) * color.z};
        m.f0       = V3{f0d + metallic * (color.x - f0d), f0d + metallic * (color.y - f0d),
                  f0d + metallic * (color.z - f0d)};
        V3 emission{0.f, 0.f, 0.f};
        if (read_color(desc.find("emission"), emission) &&
            (emission.x > 0.f || emission.y > 0.f || emission.z > 0.f)) {
            log(SU_LOG_WARNING, "su_create_material: Substitute emission is ignored by this renderer");
        }
        m.color = color;
        m.f0d   = f0d;
        // Texture maps (load_substitute, material_provider.cpp:483-600): "color" and
        // "roughness" as texture descriptions (with an optional constant "value"), "surface"
        // (roughness and metallic), or a "textures" array with a "usage" per entry.
        auto const bad_image = [&](uint32_t image) {
            return image >= engine->images.size() || engine->images[image].dims[2] != 1;
        };
        if (spb::json::Value const* c = desc.find("color"); c && c->is_object()) {
            if (texture_image(*c, maps.color, maps.color_scale) && bad_image(maps.color)) {
                log(SU_LOG_ERROR, "su_create_material: colour texture names no 2-D image");
                return Null;
            }
        }
        if (spb::json::Value const* rv = desc.find("roughness"); rv && rv->is_object()) {
            float const value = float(spb::json::number_or(rv->find("value"), 0.8));
            float const rr    = std::max(value, spb::shading::Min_roughness);
            m.alpha           = rr * rr;
            if (texture_image(*rv, maps.surface, maps.surface_scale)) {
                maps.surface_usage = 1;
            }
        }
        if (spb::json::Value const* sv = desc.find("surface"); sv && sv->is_object()) {
            if (texture_image(*sv, maps.surface, maps.surface_scale)) {
                maps.surface_usage = 2;
            }
        }
        if (spb::json::Value const* tv = desc.find("textures"); tv && tv->is_array()) {
            for (auto const& t : tv->array) {
                std::string const usage = spb::json::string_or(t.find("usage"), "");
                uint32_t          image = Null;
                float             scale[2] = {1.f, 1.f};
                if ((usage != "Color" && usage != "Surface" && usage != "Roughness") ||
                    !texture_image(t, image, scale)) {
                    log(SU_LOG_WARNING, "su_create_material: texture usage \"" + usage + "\" is not supported");
                    continue;
                }
                if (usage == "Color") {
                    maps.color = image;
                    std::copy(scale, scale + 2, maps.color_scale);
                } else {
                    maps.surface       = image;
                    maps.surface_usage = usage == "Surface" ? 2 : 1;
                    std::copy(scale, scale + 2, maps.surface_scale);
                }
            }
        }
        if ((maps.color != Null && bad_image(maps.color)) || (maps.surface != Null && bad_image(maps.surface))) {
            log(SU_LOG_ERROR, "su_create_material: texture names no 2-D image");
            return Null;
        }
        if (spb::json::Value const* sampler = desc.find("sampler")) {
            // read_sampler_settings, material_provider.cpp:866-892
            if (spb::json::Value const* f = sampler->find("filter"); f && f->is_string()) {
                maps.nearest = f->string == "Nearest";
            }
            spb::json::Value const* a = sampler->find("address");
            if (a && a->is_array() && !a->array.empty()) {
                a = &a->array[0];
            }
            if (a && a->is_string()) {
                maps.clamp = a->string == "Clamp";
            }
        }
    } else if (type == "Volumetric") {
        // material_provider.cpp:767-849 (homogeneous case): colour 0.5 by default, attenuation
        // and subsurface colours default to it, distance 1, anisotropy clamped to +-0.999;
        // coefficients from attenuation() (collision_coefficients.inl:50-71).
        if (spb::json::Value const* density = desc.find("density")) {
            // "density": {"id": image} or {"file": a SUB image} (read_texture_description,
            // material_provider.cpp:895-946); files resolve under the su_mount folders.
            spb::json::Value const* id   = density->is_object() ? density->find("id") : nullptr;
            spb::json::Value const* file = density->is_object() ? density->find("file") : nullptr;
            uint32_t const image = id && id->is_number() ? uint32_t(id->number)
                                   : (file && file->is_string() ? load_sub_image(resolve(file->string, ""))
                                                                : Null);
            // one channel, or two: density and emission scale (Grid_emission with a
            // two-channel density, volumetric_grid.cpp:80-127)
            if (image >= engine->images.size() || engine->images[image].channels > 2 ||
                engine->images[image].dims[2] < 1) {
                log(SU_LOG_ERROR, "su_create_material: density must name a one- or two-channel image id");
                return Null;
            }
            grid.image = image;
        }
        if (spb::json::Value const* temperature = desc.find("temperature")) {
            // "temperature": a one-channel image of the density's dimensions, looked up through
            // a black-body table scaled by the emission (Grid_emission, material_provider.cpp:823-830)
            spb::json::Value const* id   = temperature->is_object() ? temperature->find("id") : nullptr;
            spb::json::Value const* file = temperature->is_object() ? temperature->find("file") : nullptr;
            uint32_t const image = id && id->is_number() ? uint32_t(id->number)
                                   : (file && file->is_string() ? load_sub_image(resolve(file->string, ""))
                                                                : Null);
            if (grid.image == Null || image >= engine->images.size() || engine->images[image].channels != 1 ||
                !std::equal(engine->images[image].dims, engine->images[image].dims + 3,
                            engine->images[grid.image].dims)) {
                log(SU_LOG_ERROR, "su_create_material: temperature must name a one-channel image of the "
                                  "density's dimensions");
                return Null;
            }
            grid.temperature = image;
        }
        if (spb::json::Value const* color = desc.find("color"); color && color->is_object() && grid.image == Null) {
            // "color": {"id": image} or {"file": ...} without a density: an RGBA grid whose colour
            // sets the coefficients and whose alpha scales them (Grid_color,
            // material_provider.cpp:834-840, volumetric_grid.cpp:336-395)
            spb::json::Value const* id   = color->find("id");
            spb::json::Value const* file = color->find("file");
            uint32_t const image = id && id->is_number() ? uint32_t(id->number)
                                   : (file && file->is_string() ? load_sub_image(resolve(file->string, ""))
                                                                : Null);
            if (image >= engine->images.size() || engine->images[image].channels != 4) {
                log(SU_LOG_ERROR, "su_create_material: a colour grid must name a four-channel image");
                return Null;
            }
            if (engine->images[image].encoded_bytes) {
                grid.color = image;
            } else {
                // the reference reads 3-D colour only from four-channel byte images (sRGB and
                // alpha, Texture::at_4, texture.cpp:320-338); any other image is not a texture
                // there (texture_provider.cpp:17-116), and the material is homogeneous
                log(SU_LOG_WARNING, "su_create_material: a colour grid takes a four-channel byte image; "
                                    "rendering the homogeneous medium, as the reference does");
            }
        }
        // "emission" (material_provider.cpp:805-806): the emitted radiance per unit absorption
        // (Material::collision_coefficients_emission, material.cpp:87-89); with a density grid
        // the material is a Grid_emission (material_provider.cpp:823-830), whose absorption
        // scales with the density and whose emission does not (volumetric_grid.cpp:110-127).
        V3 emission{0.f, 0.f, 0.f};
        if (read_color(desc.find("emission"), emission) &&
            (emission.x > 0.f || emission.y > 0.f || emission.z > 0.f)) {
            m.emission = emission;
        }
        if (spb::json::Value const* sampler = desc.find("sampler")) {
            // read_sampler_settings, material_provider.cpp:866-892; 3-D lookups use address_u
            if (spb::json::Value const* f = sampler->find("filter"); f && f->is_string()) {
                grid.nearest = f->string == "Nearest";
            }
            spb::json::Value const* a = sampler->find("address");
            if (a && a->is_array() && !a->array.empty()) {
                a = &a->array[0];
            }
            if (a && a->is_string()) {
                grid.repeat = a->string == "Repeat";
            }
        }
        V3 color = srgb_to_ap1(V3{0.5f, 0.5f, 0.5f});
        read_color(desc.find("color"), color);
        V3 ac = color;
        V3 ssc = color;
        read_color(desc.find("attenuation_color"), ac);
        read_color(desc.find("subsurface_color"), ssc);
        float const distance = float(spb::json::number_or(desc.find("attenuation_distance"), 1.0));
        float const g = std::clamp(float(spb::json::number_or(desc.find("anisotropy"), 0.0)), -0.999f,
                                   0.999f);
        m.type = spb::shading::Type_volume;
        m.g    = g;
        spb::shading::attenuation(ac, ssc, distance, g, m.mu_a, m.mu_s);
        grid.distance = distance;
    } else {
        log(SU_LOG_ERROR, "su_create_material: unsupported material type " + type);
        return Null;
    }
    engine->materials.push_back(m);
    engine->material_grids.push_back(grid);
    engine->material_maps.push_back(maps);
    engine->scene_dirty = true;
    return uint32_t(engine->materials.size() - 1);
}

SU_LIBRARY_API uint32_t su_create_material_from_file(char const* filename) {
    if (!engine) {
        return Null;
    }
    // A material file holds the same JSON su_create_material takes ({"rendering": {...}},
    // material_provider.cpp:115-146); it is found under the mounted folders, then as given.
    std::string text;
    if (!filename || !read_text(resolve(filename, ""), text)) {
        log(SU_LOG_ERROR, std::string("su_create_material_from_file: cannot read ") + (filename ? filename : "(null)"));
        return Null;
    }
    return su_create_material(text.c_str());
}

SU_LIBRARY_API uint32_t su_create_triangle_mesh_async(
    uint32_t num_triangles, uint32_t num_vertices, uint32_t positions_stride,
    float const* positions, uint32_t normals_stride, float const* normals, uint32_t /*tangents_stride*/,
    float const* /*tangents*/, uint32_t uvs_stride, float const* uvs, uint32_t const* indices,
    uint32_t num_parts, uint32_t const* parts) {
    if (!engine) {
        return Null;
    }
    // triangle_mesh_provider.cpp:176-247: positions and normals are required
    if (!positions || !normals || num_triangles == 0 || num_vertices == 0 ||
        positions_stride < 3 || normals_stride < 3) {
        log(SU_LOG_ERROR, "Mesh does not contain vertex positions or normals.");
        return Null;
    }
    Mesh mesh;
    mesh.positions.resize(3 * size_t(num_vertices));
    mesh.normals.resize(3 * size_t(num_vertices));
    for (uint32_t v = 0; v < num_vertices; ++v) {
        for (int k = 0; k < 3; ++k) {
            mesh.positions[3 * v + k] = positions[size_t(v) * positions_stride + k];
            mesh.normals[3 * v + k]   = normals[size_t(v) * normals_stride + k];
        }
    }
    // texture coordinates (optional; zero without them)
    mesh.uvs.assign(2 * size_t(num_vertices), 0.f);
    if (uvs && uvs_stride >= 2) {
        for (uint32_t v = 0; v < num_vertices; ++v) {
            mesh.uvs[2 * v]     = uvs[size_t(v) * uvs_stride];
            mesh.uvs[2 * v + 1] = uvs[size_t(v) * uvs_stride + 1];
        }
    }
    mesh.indices.resize(3 * size_t(num_triangles));
    for (uint32_t t = 0; t < num_triangles; ++t) {
        for (int k = 0; k < 3; ++k) {
            uint32_t const i = indices ? indices[3 * size_t(t) + k] : 3 * t + uint32_t(k);
            if (i >= num_vertices) {
                log(SU_LOG_ERROR, "su_create_triangle_mesh_async: index out of range");
                return Null;
            }
            mesh.indices[3 * size_t(t) + k] = i;
        }
    }
    mesh.part_of.assign(num_triangles, 0);
    if (parts && num_parts > 0) {
        mesh.part_slot.resize(num_parts);
        for (uint32_t p = 0; p < num_parts; ++p) {
            uint32_t const start = parts[3 * p] / 3;
            uint32_t const end   = std::min(num_triangles, (parts[3 * p] + parts[3 * p + 1]) / 3);
            for (uint32_t t = start; t < end; ++t) {
                mesh.part_of[t] = p;
            }
            mesh.part_slot[p] = parts[3 * p + 2];
        }
    } else {
        mesh.part_slot.assign(1, 0);
    }
    engine->meshes.push_back(std::move(mesh));
    engine->frame_started = false;
    engine->scene_dirty   = true;
    return First_mesh_id + uint32_t(engine->meshes.size() - 1);
}

SU_LIBRARY_API uint32_t su_create_triangle_mesh_from_file(char const* filename) {
    if (!engine) {
        return Null;
    }
    // A triangle-mesh JSON file (the format scene files name), under the mounted folders first.
    if (!filename) {
        log(SU_LOG_ERROR, "su_create_triangle_mesh_from_file: no file name");
        return Null;
    }
    return load_mesh_file(resolve(filename, ""));
}

SU_LIBRARY_API uint32_t su_create_prop(uint32_t shape, uint32_t num_materials,
                                       uint32_t const* materials) {
    if (!engine) {
        return Null;
    }
    bool const builtin = shape == Shape_cube || shape == Shape_disk || shape == Shape_rectangle ||
                         shape == Shape_sphere;
    if (builtin && engine->builtin[shape].indices.empty()) {
        engine->builtin[shape] = make_builtin(shape);
    }
    if (!builtin && shape != Shape_infinite_sphere &&
        (shape < First_mesh_id || shape - First_mesh_id >= engine->meshes.size())) {
        log(SU_LOG_ERROR, "su_create_prop: shape not supported by this renderer (triangle meshes, "
                          "Cube, Disk, Rectangle, Sphere and Infinite_sphere are)");
        return Null;
    }
    Entity e;
    e.shape = shape;
    for (uint32_t i = 0; i < num_materials; ++i) {
        e.materials.push_back(materials ? materials[i] : Null);
    }
    engine->entities.push_back(e);
    engine->frame_started = false;
    engine->scene_dirty   = true;
    return uint32_t(engine->entities.size() - 1);
}

SU_LIBRARY_API int32_t su_create_light(uint32_t entity) {
    if (!engine) {
        return -1;
    }
    if (entity >= engine->entities.size() || engine->entities[entity].camera) {
        return -2;
    }
    engine->entities[entity].light = true;
    engine->frame_started          = false;
    return 0;
}

SU_LIBRARY_API uint32_t su_camera_entity(void) {
    if (!engine) {
        return Null;
    }
    return engine->camera_entity;
}

SU_LIBRARY_API int32_t su_camera_sensor_dimensions(int32_t* dimensions) {
    if (!engine) {
        return -1;
    }
    if (engine->camera_entity == Null || !dimensions) {
        return -2;
    }
    dimensions[0] = int32_t(engine->width);
    dimensions[1] = int32_t(engine->height);
    return 0;
}

SU_LIBRARY_API int32_t su_entity_allocate_frames(uint32_t entity) {
    if (!engine) {
        return -1;
    }
    (void)entity;
    log(SU_LOG_ERROR, "su_entity_allocate_frames: animation is not supported by this renderer");
    return -2;
}

SU_LIBRARY_API int32_t su_entity_transformation(uint32_t entity, float* trafo) {
    if (!engine) {
        return -1;
    }
    if (entity >= engine->entities.size() || !trafo) {
        return -2;
    }
    std::memcpy(trafo, engine->entities[entity].trafo, sizeof(float) * 16);
    return 0;
}

SU_LIBRARY_API int32_t su_entity_set_transformation(uint32_t entity, float const* trafo) {
    if (!engine) {
        return -1;
    }
    if (entity >= engine->entities.size() || !trafo) {
        return -2;
    }
    std::memcpy(engine->entities[entity].trafo, trafo, sizeof(float) * 16);
    engine->frame_started = false;
    // moving the camera re-applies the camera only; moving a prop rebuilds the scene
    (entity == engine->camera_entity ? engine->camera_dirty : engine->scene_dirty) = true;
    return 0;
}

SU_LIBRARY_API int32_t su_entity_set_transformation_frame(uint32_t entity, uint32_t frame,
                                                          float const* trafo) {
    if (!engine) {
        return -1;
    }
    (void)entity;
    (void)frame;
    (void)trafo;
    log(SU_LOG_ERROR, "su_entity_set_transformation_frame: animation is not supported");
    return -2;
}

SU_LIBRARY_API int32_t su_start_render_frame(uint32_t frame) {
    if (!engine) {
        return -1;
    }
    (void)frame;
    if (!ready()) {
        return -2;
    }
    // The scene is flattened, its BVH built and uploaded only when something changed; a moved
    // camera or a new resolution only re-applies the camera.
    if (engine->scene_dirty) {
        if (int32_t const s = compile_scene()) {
            return s;
        }
        engine->scene_dirty  = false;
        engine->camera_dirty = false;
    } else if (engine->camera_dirty) {
        if (int32_t const s = apply_camera()) {
            return s;
        }
        engine->camera_dirty = false;
    }
    if (engine->renderer.start_frame()) {
        log(SU_LOG_ERROR, engine->renderer.error());
        return -2;
    }
    engine->frame_started = true;
    engine->iteration     = 0;
    return 0;
}

SU_LIBRARY_API int32_t su_set_expected_iterations(uint32_t iterations) {
    if (!engine) {
        return -1;
    }
    if (!ready()) {
        return -2;
    }
    (void)iterations;  // only steers ray differentials in the reference; no effect here
    return 0;
}

SU_LIBRARY_API int32_t su_render_iteration(void) {
    if (!engine) {
        return -1;
    }
    if (!ready() || !engine->frame_started) {
        return -2;
    }
    if (int32_t const s = render_samples(engine->iteration, 1)) {
        return s;
    }
    ++engine->iteration;
    return 0;
}

SU_LIBRARY_API int32_t su_render_frame(uint32_t frame) {
    if (!engine) {
        return -1;
    }
    if (int32_t const s = su_start_render_frame(frame)) {
        return s;
    }
    if (int32_t const s = render_samples(0, engine->spp)) {
        return s;
    }
    engine->iteration = engine->spp;
    return 0;
}

SU_LIBRARY_API int32_t su_render(void) {
    // render frame 0, then export it (capi.cpp:565-580)
    if (int32_t const s = su_render_frame(0)) {
        return s;
    }
    return su_export_frame(0);
}

// The reference's default exporter (take_loader.cpp set_default_exporter): the postprocessed
// frame as an 8-bit sRGB PNG named output_<frame, 6 digits>.png in the working directory.
SU_LIBRARY_API int32_t su_export_frame(uint32_t frame) {
    if (!engine) {
        return -1;
    }
    if (su_postprocess() != 0 && engine->target.empty()) {  // the current film, resolved
        log(SU_LOG_WARNING, "su_export_frame: no rendered frame to export");
        return 0;
    }
    std::vector<uint8_t> rgb(size_t(engine->width) * engine->height * 3);
    if (su_copy_framebuffer(SU_UINT8, engine->width, engine->height, 3, rgb.data()) != 0) {
        return 0;
    }
    // Image_sequence("output_", writer) per exporter (take_loader.cpp:907-951): PNG of the
    // 8-bit sRGB framebuffer, EXR (half) and RGBE of the postprocessed linear frame.
    for (std::string const& format : engine->exporters) {
        char name[40];
        bool ok = false;
        if (format == "EXR") {
            std::snprintf(name, sizeof(name), "output_%06u.exr", frame);
            ok = spb::post::write_exr(name, engine->width, engine->height, engine->target.data(), false);
        } else if (format == "RGBE") {
            std::snprintf(name, sizeof(name), "output_%06u.hdr", frame);
            ok = spb::post::write_rgbe(name, engine->width, engine->height, engine->target.data());
        } else {
            std::snprintf(name, sizeof(name), "output_%06u.png", frame);
            ok = write_png(name, engine->width, engine->height, rgb.data());
        }
        if (!ok) {
            log(SU_LOG_ERROR, std::string("su_export_frame: cannot write ") + name);
        }
    }
    return 0;
}

SU_LIBRARY_API int32_t su_postprocess(void) {
    if (!engine) {
        return -1;
    }
    if (!ready() || !engine->frame_started) {
        return -2;
    }
    engine->target.resize(4 * size_t(engine->width) * engine->height);
    if (engine->renderer.resolve(engine->target.data())) {
        log(SU_LOG_ERROR, engine->renderer.error());
        return -2;
    }
    // The postprocessor pipeline (Pipeline::apply, postprocessor_pipeline.cpp:69-102).
    for (spb::post::Tonemapper const& t : engine->pipeline) {
        spb::post::apply(t, engine->target.data(), engine->target.size() / 4);
    }
    return 0;
}

SU_LIBRARY_API int32_t su_copy_framebuffer(uint32_t type, uint32_t width, uint32_t height,
                                           uint32_t num_channels, uint8_t* destination) {
    if (!engine) {
        return -1;
    }
    if (!destination || engine->target.empty()) {
        return -2;
    }
    uint32_t const w = std::min(width, engine->width);
    uint32_t const h = std::min(height, engine->height);
    if (SU_UINT8 == type && 3 == num_channels) {
        // linear -> gamma sRGB, rounded to bytes (capi.cpp:667-700)
        for (uint32_t y = 0; y < h; ++y) {
            for (uint32_t x = 0; x < w; ++x) {
                size_t const i = size_t(y) * engine->width + x;
                for (int c = 0; c < 3; ++c) {
                    float       v = std::max(engine->target[4 * i + c], 0.f);
                    v             = v <= 0.0031308f ? 12.92f * v
                                                    : 1.055f * std::pow(v, 1.f / 2.4f) - 0.055f;
                    float const b = std::min(std::max(v, 0.f), 1.f) * 255.f + 0.5f;
                    destination[3 * i + c] = uint8_t(b);
                }
            }
        }
        return 0;
    }
    if (SU_FLOAT32 == type && 4 == num_channels) {
        size_t const len = std::min(size_t(width) * height, size_t(engine->width) * engine->height);
        std::memcpy(destination, engine->target.data(), len * 4 * sizeof(float));
        return 0;
    }
    return -2;
}

SPB_API int32_t spb_render_views(uint32_t count, spb_view const* views, uint32_t samples_per_pixel,
                                 float* rgba) {
    if (!engine) {
        return SPB_ERROR_STATE;
    }
    if (!views || !rgba || count == 0 || count > spb::render::Max_views || samples_per_pixel == 0) {
        return SPB_ERROR_ARGUMENT;
    }
    if (!ready()) {
        return SPB_ERROR_STATE;
    }
    std::vector<spb::render::Camera_desc> cams(count);
    for (uint32_t v = 0; v < count; ++v) {
        cams[v].width  = views[v].width;
        cams[v].height = views[v].height;
        cams[v].fov    = views[v].fov;
        decompose(views[v].transformation, cams[v].rotation, cams[v].position);
    }
    // the scene (if it changed) and the engine's settings; its camera entity comes back with
    // its next frame
    if (engine->scene_dirty) {
        if (compile_scene() != 0) {
            return SPB_ERROR_STATE;
        }
        engine->scene_dirty = false;
    } else if (apply_camera() != 0) {
        return SPB_ERROR_STATE;
    }
    engine->camera_dirty  = true;
    engine->frame_started = false;
    if (int32_t const s = engine->renderer.set_views(cams)) {
        log(SU_LOG_ERROR, engine->renderer.error());
        return s;
    }
    if (render_samples(0, samples_per_pixel) != 0) {
        return SPB_ERROR_CUDA;
    }
    if (int32_t const s = engine->renderer.resolve(rgba)) {
        log(SU_LOG_ERROR, engine->renderer.error());
        return s;
    }
    return SPB_OK;
}

SPB_API int32_t spb_render_last_stats(spb_render_stats* out) {
    if (!engine || !out) {
        return SPB_ERROR_ARGUMENT;
    }
    spb::render::Stats const& st = engine->renderer.stats();
    out->paths          = st.paths;
    out->extension_rays = st.extension_rays;
    out->shadow_rays    = st.shadow_rays;
    out->device_seconds = st.seconds;
    out->overflow       = st.overflow;
    out->guide_vertices          = st.guide_vertices;
    out->guide_inference_seconds = st.guide_inference_seconds;
    out->guide_training_samples  = st.guide_training_samples;
    out->guide_training_seconds  = st.guide_training_seconds;
    out->wave_paths              = st.wave_paths;
    out->trace_blocks_per_sm     = st.trace_blocks_per_sm;
    out->graph_waves             = st.graph_waves;
    out->instances               = st.instances;
    out->tracking_capped         = st.tracking_capped;
    out->device_triangles        = st.device_triangles;
    return SPB_OK;
}

SU_LIBRARY_API int32_t su_register_log(Post post) {
    if (!post) {
        return -1;
    }
    log_post = post;
    return 0;
}

SU_LIBRARY_API int32_t su_register_progress(Progress_start start, Progress_tick tick) {
    if (!engine) {
        return -1;
    }
    progress_start = start;
    progress_tick  = tick;
    return 0;
}

}  // extern "C"
